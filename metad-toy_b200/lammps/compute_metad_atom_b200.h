// compute_metad_atom_b200.h -- LAMMPS `compute ID group metad/atom <fix_id>
// <CAL.prop> ...`: per-atom CV data of a `fix metad` for dumps.  Same syntax
// and output layout as Metad-toy's ComputeMetaDToy
// (src/core/compute_MetaDToy.cu:22-153): one request -> vector_atom, several
// -> array_atom with one column per request; atoms outside the group get 0.
#ifndef LMP_COMPUTE_METAD_ATOM_B200_H
#define LMP_COMPUTE_METAD_ATOM_B200_H

#include <string>
#include <vector>

#include "compute.h"

namespace LAMMPS_NS {

class ComputeMetadAtomB200 : public Compute {
 public:
  ComputeMetadAtomB200(class LAMMPS *, int, char **);
  ~ComputeMetadAtomB200() override;
  void init() override;
  void compute_peratom() override;
  double memory_usage() override;

 private:
  std::string id_fix_;
  std::vector<std::string> requests_;
  int nmax_ = 0;
};

}  // namespace LAMMPS_NS

#endif
