// Test stand-in for LAMMPS's Fix base: the members and virtuals the shim uses.
#ifndef STUB_FIX_H
#define STUB_FIX_H
#include "group.h"
#include "pointers.h"
namespace LAMMPS_NS {
namespace FixConst {
enum { POST_FORCE = 1 << 11, MIN_POST_FORCE = 1 << 19 };
}
class Fix : protected Pointers {
 public:
  char *id = nullptr, *style = nullptr;
  int igroup = 0, groupbit = 0;
  int scalar_flag = 0, vector_flag = 0, size_vector = 0, global_freq = 0;
  int extscalar = 0, extvector = 0;
  int energy_global_flag = 0, virial_global_flag = 0, thermo_energy = 0, thermo_virial = 0;
  int vflag_global = 0;
  int comm_reverse = 0;
  double virial[6] = {0, 0, 0, 0, 0, 0};
  Fix(LAMMPS *lmp, int, char **arg) : Pointers(lmp), id(arg[0]), style(arg[2]) {
    igroup = group->find(arg[1]);
    groupbit = igroup >= 0 ? group->bitmask[igroup] : 0;
  }
  ~Fix() override = default;
  virtual int setmask() = 0;
  virtual void init() {}
  virtual void setup(int) {}
  virtual void min_setup(int) {}
  virtual void post_force(int) {}
  virtual void min_post_force(int) {}
  virtual double compute_scalar() { return 0.0; }
  virtual double compute_vector(int) { return 0.0; }
  virtual void *extract(const char *, int &) { return nullptr; }
  virtual int pack_reverse_comm(int, int, double *) { return 0; }
  virtual void unpack_reverse_comm(int, int *, double *) {}

 protected:
  void v_init(int vflag) {
    vflag_global = (vflag && thermo_virial) ? 1 : 0;
    for (double &v : virial) v = 0.0;
  }
};
}  // namespace LAMMPS_NS
#endif
