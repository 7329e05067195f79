// compute_metad_atom_b200.cpp -- see compute_metad_atom_b200.h.
#include "compute_metad_atom_b200.h"

#include <cstring>

#include "atom.h"
#include "error.h"
#include "fix.h"
#include "memory.h"
#include "modify.h"
#include "update.h"

using namespace LAMMPS_NS;

ComputeMetadAtomB200::ComputeMetadAtomB200(LAMMPS *lmp, int narg, char **arg) : Compute(lmp, narg, arg)
{
  if (narg < 5) error->all(FLERR, "compute metad/atom needs a fix ID and at least one <CAL>.<prop>");
  id_fix_ = arg[3];
  for (int i = 4; i < narg; ++i) requests_.emplace_back(arg[i]);
  peratom_flag = 1;
  size_peratom_cols = requests_.size() == 1 ? 0 : (int) requests_.size();
}

ComputeMetadAtomB200::~ComputeMetadAtomB200()
{
  memory->destroy(vector_atom);
  memory->destroy(array_atom);
}

void ComputeMetadAtomB200::init()
{
  Fix *f = modify->get_fix_by_id(id_fix_);
  if (!f) error->all(FLERR, "compute metad/atom: fix " + id_fix_ + " does not exist");
  if (std::strcmp(f->style, "metad") != 0) error->all(FLERR, "compute metad/atom: fix " + id_fix_ + " is not a metad fix");
}

void ComputeMetadAtomB200::compute_peratom()
{
  invoked_peratom = update->ntimestep;
  if (atom->nmax > nmax_) {
    nmax_ = atom->nmax;
    if (requests_.size() == 1) {
      memory->destroy(vector_atom);
      memory->create(vector_atom, nmax_, "metad/atom:vector_atom");
    } else {
      memory->destroy(array_atom);
      memory->create(array_atom, nmax_, (int) requests_.size(), "metad/atom:array_atom");
    }
  }
  Fix *f = modify->get_fix_by_id(id_fix_);
  if (!f) error->all(FLERR, "compute metad/atom: fix " + id_fix_ + " does not exist");
  const int nlocal = atom->nlocal;
  for (size_t m = 0; m < requests_.size(); ++m) {
    int dim = 0;
    const std::string key = "colvar_peratom:" + requests_[m];
    const double *src = static_cast<const double *>(f->extract(key.c_str(), dim));
    if (!src) error->all(FLERR, "compute metad/atom: fix " + id_fix_ + " has no per-atom " + requests_[m]);
    for (int i = 0; i < nlocal; ++i) {
      const double v = (atom->mask[i] & groupbit) ? src[i] : 0.0;
      if (requests_.size() == 1) vector_atom[i] = v;
      else array_atom[i][m] = v;
    }
  }
}

double ComputeMetadAtomB200::memory_usage()
{
  return (double) nmax_ * (double) requests_.size() * sizeof(double);
}
