// args.h -- the `fix metad` argument grammar, parsed into a plain configuration.
//
// Grammar and defaults follow FixMetadynamics::FixMetadynamics
// (src/core/fix_crystallize.cu:32-302) and the per-CV sub-parsers it calls:
// SwitchFunction::create (include/utils/zqc_switch_function.h:81-161),
// Steinhardt::create (src/cvs/CVs_Steinhardt.cu:33-161) and
// Stru_factor::create (src/cvs/CVs_Strufactor.cu:34-237).
#pragma once

#include <map>
#include <string>
#include <vector>

#include "common.cuh"

namespace mtd {

enum CalKind { CAL_STEINH_Q = 0, CAL_STEINH_L = 1, CAL_STRU_FACTOR = 2, CAL_STRU_FACTOR_K = 3 };

struct CalDef {
    std::string name;
    CalKind kind = CAL_STEINH_Q;
    std::string group = "all";
    int groupbit = 1;
    // STEINH (Steinhardt::create defaults, src/cvs/CVs_Steinhardt.cu:57-60)
    int l = 6;
    double cutoff_r = 4.0;
    int cutoff_natoms = 12;
    double cutoff_eps = 1e-6;
    int block = 128;
    SwParams sw_r{SW_LINE, 0, 0, 0, 0, 0};    // default_step() is LINE (switch.h:215-218)
    SwParams sw_cv{SW_LINE, 0, 0, 0, 0, 0};
    // STRU_FACTOR (src/cvs/CVs_Strufactor.cu:49-57); q_factor has no default there
    double q_factor = -1.0;
    bool has_q_factor = false;
    bool sf_use_sw = false;
    SwParams sf_sw{SW_RATIONAL, 1.25, 0.0, 20.0, 6, 12};
    // STRU_FACTOR Chemical: pair terms weighted by w(type_i) w(type_j), w from
    // Chem_map (type weight) pairs, else exp(-(type - Chem_ctarget)^2 / (2 Chem_sigma^2)), w(0) = 0
    // (StruFactorRequest defaults, include/CVsets/CV_Stru_factor.h:28-33)
    bool chem = false;
    bool wchem = false;           // WEIGHT_CHEM: the same pair sum with the taper alone as pair term (q_factor 0)
    double chem_ctarget = 0.0, chem_sigma = 1.0;
    std::vector<std::pair<int, double>> chem_map;
    // STRU_FACTOR_K (k-vector S(k), no reference counterpart)
    int nk = 96;
    double kmag = 0.0;
    unsigned long long seed = 1;
    std::vector<double> kvecs;   // nk * 3, filled at parse time
};

struct SymbolDef {
    std::string name;    // e.g. v1
    std::string cal;     // e.g. Q6
    std::string func;    // e.g. AVE, SW_FUNC, MEAN_SOLID, NSOLID, FRAC, COUNT
    std::string sub;     // switching-function name after the second dot, may be empty
};

struct DimDef {
    bool set = false;
    double lo = 0.0, hi = 1.0;
    int nbins = 100;
    std::string expr;
};

struct Config {
    double sigma = 0.05, height0 = 0.1, biasf = 10.0, temp = 300.0;   // fix_crystallize.cu:68-72
    int pace = 100;
    int cv_dim = 1;
    bool cv_dim_set = false;
    std::string rec_file;
    int rec_pace = 0;
    int hill_type = 0;
    bool restart = false;
    bool wt = false;
    // hill-list bias (no grid): CV_dim 4, or any CV_dim with NN_BIAS 1
    bool nn = false;              // NN_BIAS 1: learned bias checked against, and falling back to, the exact hill sum
    double nn_tol = 1e-3;         // NN_TOL: max |V_theta - V_exact| on validation points
    int nn_refit = 1000;          // NN_REFIT: new hills between fits
    int nn_iters = 2000;          // NN_ITERS: Adam steps per fit
    bool hill_list() const { return nn || cv_dim > 3; }
    // neighbour lists kept across steps (extensions, no reference keyword: the
    // reference reads LAMMPS's skin lists, src/cvs/CVs_Steinhardt.cu:135-147)
    double neigh_skin = 0.0;      // NEIGH_SKIN: candidates within cutoff + skin; 0 = exact lists rebuilt every step
    int neigh_every = 0;          // NEIGH_EVERY: rebuild at least every k steps (0: only when an atom moved > skin/2)
    std::map<std::string, SwParams> sws;
    std::map<std::string, CalDef> cals;     // std::map: alphabetical order, as cal_registry
    std::vector<SymbolDef> symbols;
    std::vector<DimDef> dims;
};

struct GroupTable {
    std::vector<std::string> names;
    std::vector<int> bits;
    int find(const std::string &name) const;
};

// Returns an empty string on success, else the error message.
std::string parse_fix_args(int narg, const char *const *arg, const GroupTable &groups, Config &cfg);

// Host inverse of a switching function at eps (switch.h:339-367); -1 when undefined.
double sw_invert_for_eps(const SwParams &p, double eps);

// Deterministic k-vectors of length kmag with directions uniform on the sphere
// (Marsaglia 1972) from a SplitMix64 stream seeded with `seed`.
std::vector<double> make_kvectors(int nk, double kmag, unsigned long long seed);

}  // namespace mtd
