// fix_metad_b200.h -- LAMMPS `fix ID group metad ...` on top of libmetad_b200.so.
//
// Drop-in for Metad-toy's FixMetadynamics (src/core/fix_crystallize.cu:32-613,
// include/core/fix_crystallize.h:136-192): same style name, same argument
// grammar (passed to mtd_create verbatim), same thermo scalar (bias energy)
// and vector (the CVs), the same `colvar_peratom:<CAL>.<prop>` extract keys,
// energy and virial contributions.  Compiled with the plugin against LAMMPS's
// headers; everything it computes is done by the library.  On several MPI
// ranks each rank's context takes its local atoms as centres and its ghosts
// as neighbours, sums its totals with MPI_Allreduce, and the ghost rows of
// the bias force return to their owners through reverse communication.
#ifndef LMP_FIX_METAD_B200_H
#define LMP_FIX_METAD_B200_H

#include <vector>

#include "fix.h"
#include "metad_b200.h"

namespace LAMMPS_NS {

class FixMetadB200 : public Fix {
 public:
  FixMetadB200(class LAMMPS *, int, char **);
  ~FixMetadB200() override;
  int setmask() override;
  void init() override;
  void setup(int) override;
  void min_setup(int) override;
  void post_force(int) override;
  void min_post_force(int) override;
  double compute_scalar() override;
  double compute_vector(int) override;
  void *extract(const char *, int &) override;
  int pack_reverse_comm(int, int, double *) override;
  void unpack_reverse_comm(int, int *, double *) override;

 private:
  mtd_ctx *ctx_ = nullptr;
  bool needs_types_ = false;   // a STRU_FACTOR Chemical CAL reads atom->type every step
  bool multi_ = false;         // more than one MPI rank: domain decomposition
  std::vector<double> peratom_;
  std::vector<double> fbuf_;   // bias force of local and ghost rows (several ranks)
  void set_box();
  void check(mtd_status s);
};

}  // namespace LAMMPS_NS

#endif
