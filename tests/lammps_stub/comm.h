// Test stand-in for LAMMPS's Comm (one rank).
#ifndef STUB_COMM_H
#define STUB_COMM_H
namespace LAMMPS_NS {
class Comm {
 public:
  int me = 0, nprocs = 1;
};
}  // namespace LAMMPS_NS
#endif
