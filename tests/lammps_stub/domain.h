// Test stand-in for LAMMPS's Domain (orthogonal box).
#ifndef STUB_DOMAIN_H
#define STUB_DOMAIN_H
namespace LAMMPS_NS {
class Domain {
 public:
  double boxlo[3] = {0, 0, 0}, boxhi[3] = {1, 1, 1};
  double sublo[3] = {0, 0, 0}, subhi[3] = {1, 1, 1};   // this rank's subdomain
  int xperiodic = 1, yperiodic = 1, zperiodic = 1;
  int triclinic = 0;
};
}  // namespace LAMMPS_NS
#endif
