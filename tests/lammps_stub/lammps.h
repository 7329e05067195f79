// Test stand-in for LAMMPS's top-level class: owns the sub-objects the shim reads.
#ifndef STUB_LAMMPS_H
#define STUB_LAMMPS_H
#include "mpi.h"
namespace LAMMPS_NS {
class Memory;
class Error;
class Atom;
class Update;
class Domain;
class Force;
class Modify;
class Group;
class Comm;
class LAMMPS {
 public:
  Memory *memory;
  Error *error;
  Atom *atom;
  Update *update;
  Domain *domain;
  Force *force;
  Modify *modify;
  Group *group;
  Comm *comm;
  MPI_Comm world = 0;
  LAMMPS();
  ~LAMMPS();
};
}  // namespace LAMMPS_NS
#endif
