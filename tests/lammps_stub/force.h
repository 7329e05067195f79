// Test stand-in for LAMMPS's Force (unit constants; metal units).
#ifndef STUB_FORCE_H
#define STUB_FORCE_H
namespace LAMMPS_NS {
class Force {
 public:
  double boltz = 8.617343e-5;
};
}  // namespace LAMMPS_NS
#endif
