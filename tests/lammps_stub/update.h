// Test stand-in for LAMMPS's Update (current timestep).
#ifndef STUB_UPDATE_H
#define STUB_UPDATE_H
#include "lmptype.h"
namespace LAMMPS_NS {
class Update {
 public:
  bigint ntimestep = 0;
};
}  // namespace LAMMPS_NS
#endif
