// fix_metad_b200.cpp -- see fix_metad_b200.h.
#include "fix_metad_b200.h"

#include <mpi.h>

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

namespace {
// The library's per-step exchange: this rank's totals, summed over the ranks in place.
int allreduce_world(double *buf, int count, void *user)
{
  MPI_Comm *world = static_cast<MPI_Comm *>(user);
  return MPI_Allreduce(MPI_IN_PLACE, buf, count, MPI_DOUBLE, MPI_SUM, *world) == MPI_SUCCESS ? 0 : 1;
}
}  // namespace

FixMetadB200::FixMetadB200(LAMMPS *lmp, int narg, char **arg) : Fix(lmp, narg, arg)
{
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
  if (comm->nprocs > 1) {
    // several ranks: owned atoms are the centres, ghosts the neighbours; the
    // ghost rows of the bias force go back to their owners by reverse comm
    check(mtd_set_domain(ctx_, atom->nlocal, comm->me, allreduce_world, &world));
    multi_ = true;
    comm_reverse = 3;
  }
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
  if (multi_) {   // this rank's subdomain and its ghost shell; the ghosts carry the periodic images
    const double g = mtd_ghost_cutoff(ctx_);
    const double lo[3] = {domain->sublo[0] - g, domain->sublo[1] - g, domain->sublo[2] - g};
    const double hi[3] = {domain->subhi[0] + g, domain->subhi[1] + g, domain->subhi[2] + g};
    const int open[3] = {0, 0, 0};
    check(mtd_set_box(ctx_, lo, hi, open));
    return;
  }
  const int periodic[3] = {domain->xperiodic, domain->yperiodic, domain->zperiodic};
  check(mtd_set_box(ctx_, domain->boxlo, domain->boxhi, periodic));
}

void FixMetadB200::init()
{
  if (multi_ && comm->get_comm_cutoff() < mtd_ghost_cutoff(ctx_))
    error->all(FLERR, "fix metad (libmetad_b200): ghost atoms are needed within " +
                          std::to_string(mtd_ghost_cutoff(ctx_)) + " (comm_modify cutoff)");
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
  if (multi_) {
    const int nlocal = atom->nlocal, nall = nlocal + atom->nghost;
    check(mtd_set_nlocal(ctx_, nlocal));
    if (needs_types_) check(mtd_set_types(ctx_, nall, atom->type));
    fbuf_.assign((size_t) nall * 3, 0.0);
    check(mtd_post_force(ctx_, (int64_t) update->ntimestep, nall, nall ? &atom->x[0][0] : nullptr, atom->mask,
                         nullptr, fbuf_.data(), vflag_global ? vir : nullptr));
    comm->reverse_comm(this);   // ghost rows summed into their owners' rows of fbuf_
    for (int i = 0; i < nlocal; ++i)
      for (int d = 0; d < 3; ++d) atom->f[i][d] += fbuf_[3 * (size_t) i + d];
    if (vflag_global)
      for (int k = 0; k < 6; ++k) virial[k] = vir[k];
    return;
  }
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

int FixMetadB200::pack_reverse_comm(int n, int first, double *buf)
{
  int m = 0;
  for (int i = first; i < first + n; ++i)
    for (int d = 0; d < 3; ++d) buf[m++] = fbuf_[3 * (size_t) i + d];
  return m;
}

void FixMetadB200::unpack_reverse_comm(int n, int *list, double *buf)
{
  int m = 0;
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) fbuf_[3 * (size_t) list[i] + d] += buf[m++];
}

// "colvar_peratom:<CAL>.<prop>" (the reference's keys, fix_crystallize.cu:592-613):
// a per-atom array owned by the fix, valid until the next extract (rows of
// the local atoms first; with several ranks the ghost rows follow).
void *FixMetadB200::extract(const char *name, int &dim)
{
  if (!name || std::strncmp(name, "colvar_peratom:", 15) != 0) return nullptr;
  dim = 1;
  const int n = atom->nlocal + (multi_ ? atom->nghost : 0);
  peratom_.assign(n, 0.0);
  if (mtd_extract_peratom(ctx_, name, peratom_.data(), n) != MTD_OK) return nullptr;
  return peratom_.data();
}
