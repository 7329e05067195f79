// Test stand-in for LAMMPS's Compute base (per-atom output members).
#ifndef STUB_COMPUTE_H
#define STUB_COMPUTE_H
#include "group.h"
#include "pointers.h"
namespace LAMMPS_NS {
class Compute : protected Pointers {
 public:
  char *id = nullptr, *style = nullptr;
  int igroup = 0, groupbit = 0;
  int peratom_flag = 0, size_peratom_cols = 0;
  double *vector_atom = nullptr;
  double **array_atom = nullptr;
  bigint invoked_peratom = -1;
  Compute(LAMMPS *lmp, int, char **arg) : Pointers(lmp), id(arg[0]), style(arg[2]) {
    igroup = group->find(arg[1]);
    groupbit = igroup >= 0 ? group->bitmask[igroup] : 0;
  }
  ~Compute() override = default;
  virtual void init() = 0;
  virtual void compute_peratom() {}
  virtual double memory_usage() { return 0.0; }
};
}  // namespace LAMMPS_NS
#endif
