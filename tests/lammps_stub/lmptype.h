// Test stand-in for LAMMPS's lmptype.h: only what the metad-b200 shim uses.
#ifndef STUB_LMPTYPE_H
#define STUB_LMPTYPE_H
#include <cstdint>
namespace LAMMPS_NS {
typedef int64_t bigint;
typedef int tagint;
typedef int imageint;
}  // namespace LAMMPS_NS
#endif
