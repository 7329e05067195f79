// Test stand-in for LAMMPS's Modify (fix lookup by ID).
#ifndef STUB_MODIFY_H
#define STUB_MODIFY_H
#include <string>
#include <vector>
#include "fix.h"
namespace LAMMPS_NS {
class Modify {
 public:
  std::vector<Fix *> fixes;
  Fix *get_fix_by_id(const std::string &id) const {
    for (Fix *f : fixes)
      if (f && id == f->id) return f;
    return nullptr;
  }
};
}  // namespace LAMMPS_NS
#endif
