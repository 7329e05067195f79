// Test stand-in for LAMMPS's Pointers base (references to the LAMMPS members).
#ifndef STUB_POINTERS_H
#define STUB_POINTERS_H
#include "lammps.h"
#include "lmptype.h"
namespace LAMMPS_NS {
class Pointers {
 public:
  explicit Pointers(LAMMPS *ptr) :
      lmp(ptr), memory(ptr->memory), error(ptr->error), atom(ptr->atom), update(ptr->update),
      domain(ptr->domain), force(ptr->force), modify(ptr->modify), group(ptr->group), comm(ptr->comm),
      world(ptr->world) {}
  virtual ~Pointers() = default;

 protected:
  LAMMPS *lmp;
  Memory *&memory;
  Error *&error;
  Atom *&atom;
  Update *&update;
  Domain *&domain;
  Force *&force;
  Modify *&modify;
  Group *&group;
  Comm *&comm;
  MPI_Comm &world;
};
}  // namespace LAMMPS_NS
#endif
