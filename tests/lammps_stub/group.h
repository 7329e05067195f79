// Test stand-in for LAMMPS's Group (name -> bitmask table, 32 slots).
#ifndef STUB_GROUP_H
#define STUB_GROUP_H
#include <cstring>
namespace LAMMPS_NS {
class Group {
 public:
  int ngroup = 0;
  char *names[32] = {};
  int bitmask[32] = {};
  int find(const char *name) const {
    for (int g = 0; g < ngroup; ++g)
      if (names[g] && std::strcmp(names[g], name) == 0) return g;
    return -1;
  }
};
}  // namespace LAMMPS_NS
#endif
