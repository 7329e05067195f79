// Test stand-in for LAMMPS's Atom (per-atom arrays of the local atoms).
#ifndef STUB_ATOM_H
#define STUB_ATOM_H
#include "lmptype.h"
namespace LAMMPS_NS {
class Atom {
 public:
  double **x = nullptr, **f = nullptr;
  int *mask = nullptr;
  int *type = nullptr;
  imageint *image = nullptr;
  int nlocal = 0, nghost = 0, nmax = 0;
};
}  // namespace LAMMPS_NS
#endif
