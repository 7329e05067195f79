// fix_metad_b200.cpp -- see fix_metad_b200.h.
#include "fix_metad_b200.h"

#include <cstring>
#include <string>

#include "atom.h"
#include "comm.h"
#include "domain.h"
#include "error.h"
#include "force.h"
#include "group.h"
#include "update.h"

using namespace LAMMPS_NS;
using namespace FixConst;

FixMetadB200::FixMetadB200(LAMMPS *lmp, int narg, char **arg) : Fix(lmp, narg, arg)
{
  if (comm->nprocs > 1)
    error->all(FLERR, "fix metad (libmetad_b200): one MPI rank per GPU with all atoms local is required");
  // the group table resolves `CAL ... <group>` keywords to mask bits
  std::vector<const char *> names;
  std::vector<int> bits;
  for (int g = 0; g < group->ngroup; ++g)
    if (group->names[g]) {
      names.push_back(group->names[g]);
      bits.push_back(group->bitmask[g]);
    }
  mtd_options opt;
  mtd_options_default(&opt);
  opt.boltz = force->boltz;
  opt.n_groups = (int) names.size();
  opt.group_names = names.data();
  opt.group_bits = bits.data();
  // the tokens after the style name, as the reference parses them (fix_crystallize.cu:32-302)
  const mtd_status s = mtd_create(narg - 3, arg + 3, &opt, &ctx_);
  if (s != MTD_OK) error->all(FLERR, std::string("fix metad: ") + mtd_last_error(ctx_));
  needs_types_ = mtd_needs_types(ctx_) != 0;
  scalar_flag = 1;
  vector_flag = 1;
  size_vector = mtd_cv_dim(ctx_);
  global_freq = 1;
  extscalar = 0;
  extvector = 0;
  energy_global_flag = 1;
  virial_global_flag = 1;
  thermo_energy = 1;
  thermo_virial = 1;
}

FixMetadB200::~FixMetadB200()
{
  mtd_destroy(ctx_);
}

int FixMetadB200::setmask()
{
  return POST_FORCE | MIN_POST_FORCE;
}

void FixMetadB200::check(mtd_status s)
{
  if (s != MTD_OK) error->all(FLERR, std::string("fix metad: ") + mtd_last_error(ctx_));
}

void FixMetadB200::set_box()
{
  if (domain->triclinic) error->all(FLERR, "fix metad (libmetad_b200): orthogonal boxes only");
  const int periodic[3] = {domain->xperiodic, domain->yperiodic, domain->zperiodic};
  check(mtd_set_box(ctx_, domain->boxlo, domain->boxhi, periodic));
}

void FixMetadB200::init()
{
  set_box();
  check(mtd_init(ctx_));
}

void FixMetadB200::setup(int vflag)
{
  post_force(vflag);
}

void FixMetadB200::min_setup(int vflag)
{
  post_force(vflag);
}

void FixMetadB200::post_force(int vflag)
{
  v_init(vflag);
  set_box();   // the box may change between steps (NPT)
  double vir[6] = {0, 0, 0, 0, 0, 0};
  const int n = atom->nlocal;
  if (needs_types_) check(mtd_set_types(ctx_, n, atom->type));   // types follow LAMMPS's atom sorting
  check(mtd_post_force(ctx_, (int64_t) update->ntimestep, n, n ? &atom->x[0][0] : nullptr, atom->mask,
                       atom->image, n ? &atom->f[0][0] : nullptr, vflag_global ? vir : nullptr));
  if (vflag_global)
    for (int k = 0; k < 6; ++k) virial[k] = vir[k];
}

void FixMetadB200::min_post_force(int vflag)
{
  post_force(vflag);
}

double FixMetadB200::compute_scalar()
{
  return mtd_compute_scalar(ctx_);
}

double FixMetadB200::compute_vector(int k)
{
  return mtd_compute_vector(ctx_, k);
}

// "colvar_peratom:<CAL>.<prop>" (the reference's keys, fix_crystallize.cu:592-613):
// a per-atom array owned by the fix, valid until the next extract.
void *FixMetadB200::extract(const char *name, int &dim)
{
  if (!name || std::strncmp(name, "colvar_peratom:", 15) != 0) return nullptr;
  dim = 1;
  peratom_.assign(atom->nlocal, 0.0);
  if (mtd_extract_peratom(ctx_, name, peratom_.data(), atom->nlocal) != MTD_OK) return nullptr;
  return peratom_.data();
}
