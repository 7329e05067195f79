// Drives the LAMMPS shim (fix metad + compute metad/atom of metad-toy_b200/lammps)
// through the stand-in LAMMPS classes the way LAMMPS's integrator would: load
// the plugin, create the fix and the compute from input-deck tokens, init,
// then per step set x, zero f and call post_force with the virial flag.
//
//   harness <in.bin> <tokens.txt> <out.bin>
//   in.bin:   int n, int steps, double lo[3], double hi[3], int periodic[3],
//             double x[steps][n][3], int mask[n]
//   tokens:   the fix tokens after "metad", one per line; then a line "--"
//             and the compute metad/atom requests (<CAL>.<prop>), one per line
//   out.bin:  per step: double bias, cv[size_vector], virial[6], f[n][3];
//             then the compute's per-atom values of the last step [n][ncols]
//
// Several ranks (domain decomposition), one host thread per rank, each with
// its own LAMMPS instance; MPI_Allreduce and Comm::reverse_comm are served
// across the threads:
//
//   harness --ranks R <rank_0.bin> .. <rank_R-1.bin> <tokens.txt> <out_prefix>
//   rank_r.bin: int steps, double ghost_cutoff; per step: int nlocal, nghost,
//               double sublo[3], subhi[3], double x[nall][3], int mask[nall],
//               int type[nall], int ghost_rank[nghost], int ghost_index[nghost]
//   out_prefix.r: per step: double bias, cv[size_vector], virial[6], f[nlocal][3]
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "atom.h"
#include "comm.h"
#include "compute.h"
#include "domain.h"
#include "error.h"
#include "fix.h"
#include "force.h"
#include "group.h"
#include "lammps.h"
#include "lammpsplugin.h"
#include "memory.h"
#include "modify.h"
#include "update.h"

using namespace LAMMPS_NS;

LAMMPS::LAMMPS() :
    memory(new Memory), error(new Error), atom(new Atom), update(new Update), domain(new Domain),
    force(new Force), modify(new Modify), group(new Group), comm(new Comm) {
  comm->lmp = this;
}
LAMMPS::~LAMMPS() {
  delete memory; delete error; delete atom; delete update; delete domain;
  delete force; delete modify; delete group; delete comm;
}

extern "C" void lammpsplugin_init(void *lmp, void *handle, void *regfunc);

static std::map<std::string, lammpsplugin_factory2 *> g_factories;
static void regfunc(lammpsplugin_t *p, void *) { g_factories[std::string(p->style) + "/" + p->name] = p->creator.v2; }

// ------------------------------------------------------------------ thread ranks
namespace {
struct Ranks {
  int n = 1;
  std::mutex mu;
  std::condition_variable cv;
  int arrived = 0;
  long gen = 0;
  bool broken = false;
  std::vector<std::vector<double>> slot;             // one buffer per rank
  std::vector<std::vector<int>> route_rank, route_index;
  // all ranks meet here; false when a rank failed or the wait ran out
  bool wait() {
    std::unique_lock<std::mutex> lk(mu);
    if (broken) return false;
    const long g = gen;
    if (++arrived == n) {
      arrived = 0;
      ++gen;
      cv.notify_all();
      return true;
    }
    if (!cv.wait_for(lk, std::chrono::seconds(120), [&] { return gen != g || broken; }) || broken) {
      broken = true;
      cv.notify_all();
      return false;
    }
    return true;
  }
  void abort() {
    std::lock_guard<std::mutex> lk(mu);
    broken = true;
    cv.notify_all();
  }
};
Ranks g_ranks;
thread_local int t_rank = 0;
}  // namespace

// Sum in rank order: every rank receives the same bits.
int MPI_Allreduce(const void *send, void *recv, int count, MPI_Datatype, MPI_Op, MPI_Comm) {
  double *r = static_cast<double *>(recv);
  const double *s = send == MPI_IN_PLACE ? r : static_cast<const double *>(send);
  g_ranks.slot[t_rank].assign(s, s + count);
  if (!g_ranks.wait()) return 1;
  for (int t = 0; t < count; ++t) {
    double acc = g_ranks.slot[0][t];
    for (int q = 1; q < g_ranks.n; ++q) acc += g_ranks.slot[q][t];
    r[t] = acc;
  }
  return g_ranks.wait() ? MPI_SUCCESS : 1;
}

// Every ghost row of every rank, packed by the fix, is unpacked on the rank
// that owns the atom, at the owner's local index (source rank order, ghost order).
void LAMMPS_NS::Comm::reverse_comm(Fix *fix) {
  Atom *a = lmp->atom;
  const int w = fix->comm_reverse, ng = a->nghost;
  g_ranks.slot[me].assign((size_t) ng * w, 0.0);
  if (ng) fix->pack_reverse_comm(ng, a->nlocal, g_ranks.slot[me].data());
  g_ranks.route_rank[me] = ghost_rank;
  g_ranks.route_index[me] = ghost_index;
  if (!g_ranks.wait()) throw std::runtime_error("reverse_comm: a rank failed");
  std::vector<int> list;
  std::vector<double> buf;
  for (int src = 0; src < nprocs; ++src)
    for (size_t g = 0; g < g_ranks.route_rank[src].size(); ++g)
      if (g_ranks.route_rank[src][g] == me) {
        list.push_back(g_ranks.route_index[src][g]);
        buf.insert(buf.end(), g_ranks.slot[src].begin() + (long) g * w, g_ranks.slot[src].begin() + (long) (g + 1) * w);
      }
  if (!g_ranks.wait()) throw std::runtime_error("reverse_comm: a rank failed");
  if (!list.empty()) fix->unpack_reverse_comm((int) list.size(), list.data(), buf.data());
}

namespace {
struct RankStep {
  int nlocal = 0, nghost = 0;
  double sublo[3], subhi[3];
  std::vector<double> x;
  std::vector<int> mask, type, grank, gindex;
};

void run_rank(int r, int nranks, const std::string &in_path, const std::vector<std::string> &fixtok,
              const std::string &out_path, std::string *err) {
  t_rank = r;
  try {
    std::ifstream in(in_path, std::ios::binary);
    int steps = 0;
    double gc = 0.0;
    in.read((char *) &steps, 4);
    in.read((char *) &gc, 8);
    std::vector<RankStep> st(steps);
    int nmax = 1;
    for (RankStep &s : st) {
      in.read((char *) &s.nlocal, 4);
      in.read((char *) &s.nghost, 4);
      in.read((char *) s.sublo, 24);
      in.read((char *) s.subhi, 24);
      const int nall = s.nlocal + s.nghost;
      nmax = std::max(nmax, nall);
      s.x.resize((size_t) nall * 3);
      s.mask.resize(nall);
      s.type.resize(nall);
      s.grank.resize(s.nghost);
      s.gindex.resize(s.nghost);
      in.read((char *) s.x.data(), (std::streamsize) s.x.size() * 8);
      in.read((char *) s.mask.data(), (std::streamsize) nall * 4);
      in.read((char *) s.type.data(), (std::streamsize) nall * 4);
      in.read((char *) s.grank.data(), (std::streamsize) s.nghost * 4);
      in.read((char *) s.gindex.data(), (std::streamsize) s.nghost * 4);
    }
    if (!in) throw std::runtime_error("short rank input " + in_path);

    LAMMPS lmp;
    static char all[] = "all";
    lmp.group->ngroup = 1;
    lmp.group->names[0] = all;
    lmp.group->bitmask[0] = 1;
    lmp.comm->me = r;
    lmp.comm->nprocs = nranks;
    lmp.comm->cutghostuser = gc;
    lmp.memory->create(lmp.atom->x, nmax, 3, "x");
    lmp.memory->create(lmp.atom->f, nmax, 3, "f");
    lmp.atom->nmax = nmax;
    auto load = [&](RankStep &s) {
      for (int d = 0; d < 3; ++d) {
        lmp.domain->sublo[d] = s.sublo[d];
        lmp.domain->subhi[d] = s.subhi[d];
      }
      lmp.atom->nlocal = s.nlocal;
      lmp.atom->nghost = s.nghost;
      lmp.atom->mask = s.mask.data();
      lmp.atom->type = s.type.data();
      for (int i = 0; i < s.nlocal + s.nghost; ++i)
        for (int d = 0; d < 3; ++d) {
          lmp.atom->x[i][d] = s.x[(size_t) i * 3 + d];
          lmp.atom->f[i][d] = 0.0;
        }
      lmp.comm->ghost_rank = s.grank;
      lmp.comm->ghost_index = s.gindex;
    };
    if (!st.empty()) load(st[0]);
    std::vector<std::string> fargs = {"mtd", "all", "metad"};
    fargs.insert(fargs.end(), fixtok.begin(), fixtok.end());
    std::vector<char *> fv;
    for (auto &s : fargs) fv.push_back(&s[0]);
    std::unique_ptr<Fix> fix((Fix *) g_factories.at("fix/metad")(&lmp, (int) fv.size(), fv.data()));
    fix->init();
    std::ofstream out(out_path, std::ios::binary);
    for (int s = 0; s < steps; ++s) {
      load(st[s]);
      lmp.update->ntimestep = s;
      fix->post_force(1);
      const double bias = fix->compute_scalar();
      out.write((const char *) &bias, 8);
      for (int k = 0; k < fix->size_vector; ++k) {
        const double v = fix->compute_vector(k);
        out.write((const char *) &v, 8);
      }
      out.write((const char *) fix->virial, 48);
      out.write((const char *) &lmp.atom->f[0][0], (std::streamsize) st[s].nlocal * 24);
    }
    fix.reset();
    lmp.memory->destroy(lmp.atom->x);
    lmp.memory->destroy(lmp.atom->f);
  } catch (const std::exception &e) {
    *err = e.what();
    g_ranks.abort();
  }
}

int run_ranks(int argc, char **argv) {
  const int R = std::atoi(argv[2]);
  if (R < 1 || argc != 5 + R) {
    std::fprintf(stderr, "usage: harness --ranks R rank_0.bin .. rank_R-1.bin tokens.txt out_prefix\n");
    return 2;
  }
  std::ifstream tf(argv[3 + R]);
  std::vector<std::string> fixtok;
  std::string line;
  while (std::getline(tf, line))
    if (!line.empty()) fixtok.push_back(line);
  g_ranks.n = R;
  g_ranks.slot.resize(R);
  g_ranks.route_rank.resize(R);
  g_ranks.route_index.resize(R);
  std::vector<std::string> errs(R);
  std::vector<std::thread> th;
  for (int r = 0; r < R; ++r)
    th.emplace_back(run_rank, r, R, std::string(argv[3 + r]), std::cref(fixtok),
                    std::string(argv[4 + R]) + "." + std::to_string(r), &errs[r]);
  for (auto &t : th) t.join();
  int rc = 0;
  for (int r = 0; r < R; ++r)
    if (!errs[r].empty()) {
      std::fprintf(stderr, "harness rank %d: %s\n", r, errs[r].c_str());
      rc = 1;
    }
  return rc;
}
}  // namespace

int main(int argc, char **argv) {
  if (argc >= 3 && std::strcmp(argv[1], "--ranks") == 0) {
    lammpsplugin_init(nullptr, nullptr, (void *) &regfunc);
    return run_ranks(argc, argv);
  }
  if (argc != 4) {
    std::fprintf(stderr, "usage: harness in.bin tokens.txt out.bin\n");
    return 2;
  }
  try {
    std::ifstream in(argv[1], std::ios::binary);
    int n = 0, steps = 0, periodic[3];
    double lo[3], hi[3];
    in.read((char *) &n, 4);
    in.read((char *) &steps, 4);
    in.read((char *) lo, 24);
    in.read((char *) hi, 24);
    in.read((char *) periodic, 12);
    std::vector<double> xs((size_t) steps * n * 3);
    in.read((char *) xs.data(), (std::streamsize) (xs.size() * 8));
    std::vector<int> mask(n);
    in.read((char *) mask.data(), (std::streamsize) n * 4);
    std::ifstream tf(argv[2]);
    std::vector<std::string> fixtok, req;
    std::string line;
    bool comp = false;
    while (std::getline(tf, line)) {
      if (line == "--") { comp = true; continue; }
      if (!line.empty()) (comp ? req : fixtok).push_back(line);
    }

    LAMMPS lmp;
    static char all[] = "all", half[] = "half";
    lmp.group->ngroup = 2;
    lmp.group->names[0] = all;
    lmp.group->bitmask[0] = 1;
    lmp.group->names[1] = half;
    lmp.group->bitmask[1] = 2;
    for (int d = 0; d < 3; ++d) {
      lmp.domain->boxlo[d] = lo[d];
      lmp.domain->boxhi[d] = hi[d];
    }
    lmp.domain->xperiodic = periodic[0];
    lmp.domain->yperiodic = periodic[1];
    lmp.domain->zperiodic = periodic[2];
    lmp.memory->create(lmp.atom->x, n, 3, "x");
    lmp.memory->create(lmp.atom->f, n, 3, "f");
    lmp.atom->mask = mask.data();
    lmp.atom->nlocal = n;
    lmp.atom->nmax = n;

    lammpsplugin_init(&lmp, nullptr, (void *) &regfunc);
    std::vector<std::string> fargs = {"mtd", "all", "metad"};
    fargs.insert(fargs.end(), fixtok.begin(), fixtok.end());
    std::vector<char *> fv;
    for (auto &s : fargs) fv.push_back(&s[0]);
    std::unique_ptr<Fix> fix((Fix *) g_factories.at("fix/metad")(&lmp, (int) fv.size(), fv.data()));
    lmp.modify->fixes.push_back(fix.get());
    std::unique_ptr<Compute> cmp;
    std::vector<std::string> cargs = {"pa", "all", "metad/atom", "mtd"};
    cargs.insert(cargs.end(), req.begin(), req.end());
    std::vector<char *> cv;
    for (auto &s : cargs) cv.push_back(&s[0]);
    if (!req.empty()) cmp.reset((Compute *) g_factories.at("compute/metad/atom")(&lmp, (int) cv.size(), cv.data()));
    if (!(fix->setmask() & FixConst::POST_FORCE)) throw std::runtime_error("fix does not ask for post_force");
    fix->init();
    if (cmp) cmp->init();

    std::ofstream out(argv[3], std::ios::binary);
    for (int s = 0; s < steps; ++s) {
      for (int i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d) {
          lmp.atom->x[i][d] = xs[((size_t) s * n + i) * 3 + d];
          lmp.atom->f[i][d] = 0.0;
        }
      lmp.update->ntimestep = s;
      fix->post_force(1);
      const double bias = fix->compute_scalar();
      out.write((const char *) &bias, 8);
      for (int k = 0; k < fix->size_vector; ++k) {
        const double v = fix->compute_vector(k);
        out.write((const char *) &v, 8);
      }
      out.write((const char *) fix->virial, 48);
      out.write((const char *) &lmp.atom->f[0][0], (std::streamsize) n * 24);
    }
    if (cmp) {
      cmp->compute_peratom();
      for (int i = 0; i < n; ++i) {
        if (req.size() == 1) out.write((const char *) &cmp->vector_atom[i], 8);
        else out.write((const char *) cmp->array_atom[i], (std::streamsize) req.size() * 8);
      }
    }
    cmp.reset();
    fix.reset();
    lmp.memory->destroy(lmp.atom->x);
    lmp.memory->destroy(lmp.atom->f);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "harness: %s\n", e.what());
    return 1;
  }
  return 0;
}
