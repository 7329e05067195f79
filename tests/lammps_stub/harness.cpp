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
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <string>
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
    force(new Force), modify(new Modify), group(new Group), comm(new Comm) {}
LAMMPS::~LAMMPS() {
  delete memory; delete error; delete atom; delete update; delete domain;
  delete force; delete modify; delete group; delete comm;
}

extern "C" void lammpsplugin_init(void *lmp, void *handle, void *regfunc);

static std::map<std::string, lammpsplugin_factory2 *> g_factories;
static void regfunc(lammpsplugin_t *p, void *) { g_factories[std::string(p->style) + "/" + p->name] = p->creator.v2; }

int main(int argc, char **argv) {
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
