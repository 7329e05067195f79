// Test stand-in for LAMMPS's Comm: rank, rank count, ghost cutoff and the
// reverse communication of a fix (the harness implements it across its
// thread ranks).
#ifndef STUB_COMM_H
#define STUB_COMM_H
#include <vector>
namespace LAMMPS_NS {
class Fix;
class LAMMPS;
class Comm {
 public:
  LAMMPS *lmp = nullptr;
  int me = 0, nprocs = 1;
  double cutghostuser = 0.0;
  // where each ghost of this rank lives: owner rank and the owner's local index
  std::vector<int> ghost_rank, ghost_index;
  double get_comm_cutoff() const { return cutghostuser; }
  void reverse_comm(Fix *fix);
};
}  // namespace LAMMPS_NS
#endif
