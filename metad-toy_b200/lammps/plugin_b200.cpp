// plugin_b200.cpp -- registers `fix metad` and `compute metad/atom` backed by
// libmetad_b200.so, under the style names of Metad-toy's plugin
// (lammpsplugin_init, src/core/fix_crystallize.cu:632-654), so input decks
// load this plugin instead and run unchanged.
#include "lammpsplugin.h"

#include "compute_metad_atom_b200.h"
#include "fix_metad_b200.h"
#include "version.h"

using namespace LAMMPS_NS;

static Fix *fix_metad_b200(LAMMPS *lmp, int narg, char **arg)
{
  return new FixMetadB200(lmp, narg, arg);
}

static Compute *compute_metad_atom_b200(LAMMPS *lmp, int narg, char **arg)
{
  return new ComputeMetadAtomB200(lmp, narg, arg);
}

extern "C" void lammpsplugin_init(void *lmp, void *handle, void *regfunc)
{
  lammpsplugin_t plugin;
  lammpsplugin_regfunc register_plugin = (lammpsplugin_regfunc) regfunc;
  plugin.version = LAMMPS_VERSION;
  plugin.style = "fix";
  plugin.name = "metad";
  plugin.info = "metadynamics on libmetad_b200 (sm_100a)";
  plugin.author = "metad-b200";
  plugin.creator.v2 = (lammpsplugin_factory2 *) &fix_metad_b200;
  plugin.handle = handle;
  (*register_plugin)(&plugin, lmp);
  plugin.style = "compute";
  plugin.name = "metad/atom";
  plugin.info = "per-atom CV data of fix metad (libmetad_b200)";
  plugin.creator.v2 = (lammpsplugin_factory2 *) &compute_metad_atom_b200;
  (*register_plugin)(&plugin, lmp);
}
