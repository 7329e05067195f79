// args.cpp -- `fix metad` argument parser (see args.h for the reference lines).
#include "args.h"

#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <sstream>

namespace mtd {

int GroupTable::find(const std::string &name) const {
    for (size_t i = 0; i < names.size(); ++i)
        if (names[i] == name) return bits[i];
    return -1;
}

namespace {

struct Cursor {
    int narg;
    const char *const *arg;
    std::string err;
    bool fail(const std::string &m) {
        if (err.empty()) err = m;
        return false;
    }
};

// Strict numbers like LAMMPS utils::numeric / utils::inumeric.
bool to_double(const char *s, double &v) {
    if (!s || !*s) return false;
    char *end = nullptr;
    errno = 0;
    v = std::strtod(s, &end);
    return errno == 0 && end && *end == '\0';
}
bool to_int(const char *s, int &v) {
    if (!s || !*s) return false;
    char *end = nullptr;
    errno = 0;
    long t = std::strtol(s, &end, 10);
    if (errno != 0 || !end || *end != '\0' || t < -2147483647L || t > 2147483647L) return false;
    v = (int)t;
    return true;
}

bool need_double(Cursor &c, int i, double &v, const char *what) {
    if (i >= c.narg) return c.fail(std::string("Error: '") + what + "' requires a numeric value");
    if (!to_double(c.arg[i], v)) return c.fail(std::string("Error: '") + what + "' expects a number, got '" + c.arg[i] + "'");
    return true;
}
bool need_int(Cursor &c, int i, int &v, const char *what) {
    if (i >= c.narg) return c.fail(std::string("Error: '") + what + "' requires an integer");
    if (!to_int(c.arg[i], v)) return c.fail(std::string("Error: '") + what + "' expects an integer, got '" + c.arg[i] + "'");
    return true;
}

// SwitchFunction::create: `SW_FUNC TYPE [r_0 x] [d_0 x] [alpha x] [n i] [m i]`,
// i points at TYPE on entry and past the options on exit (switch.h:81-161).
bool parse_switch(Cursor &c, int &i, SwParams &p) {
    if (i >= c.narg) return c.fail("Error: SW_FUNC command requires a type (LINE, STEP, FERMI, TANH, RATIONAL).");
    std::string t = c.arg[i];
    p = SwParams{SW_RATIONAL, 1.25, 0.0, 20.0, 6, 12};
    if (t == "STEP") { p.type = SW_STEP; p.r0 = 1.0; }
    else if (t == "FERMI") { p.type = SW_FERMI; p.r0 = 1.0; p.alpha = 20.0; }
    else if (t == "TANH") { p.type = SW_TANH; p.r0 = 1.0; p.alpha = 20.0; }
    else if (t == "RATIONAL") { p.type = SW_RATIONAL; p.r0 = 1.25; p.d0 = 0.0; p.n = 6; p.m = 12; }
    else if (t == "LINE") { p.type = SW_LINE; }
    else return c.fail("Error: Unknown SW_func type. Choose from FERMI, TANH, RATIONAL.");
    int k = i + 1;
    while (k < c.narg) {
        if (!std::strcmp(c.arg[k], "r_0")) { if (!need_double(c, k + 1, p.r0, "r_0")) return false; k += 2; }
        else if (!std::strcmp(c.arg[k], "d_0")) { if (!need_double(c, k + 1, p.d0, "d_0")) return false; k += 2; }
        else if (!std::strcmp(c.arg[k], "alpha")) { if (!need_double(c, k + 1, p.alpha, "alpha")) return false; k += 2; }
        else if (!std::strcmp(c.arg[k], "n")) { if (!need_int(c, k + 1, p.n, "n")) return false; k += 2; }
        else if (!std::strcmp(c.arg[k], "m")) { if (!need_int(c, k + 1, p.m, "m")) return false; k += 2; }
        else break;
    }
    i = k;
    return true;
}

bool lookup_sw(Cursor &c, const Config &cfg, const char *name, SwParams &out) {
    auto it = cfg.sws.find(name);
    if (it == cfg.sws.end())
        return c.fail(std::string("Error: SwitchFunction named ") + name + " not found in registry!");
    out = it->second;
    return true;
}

// Steinhardt::create: `STEINH {Q|L} l group [options]` (CVs_Steinhardt.cu:33-161).
bool parse_steinh(Cursor &c, int &i, const GroupTable &groups, Config &cfg, CalDef &d) {
    if (i + 3 >= c.narg) return c.fail("Error: STEINH command requires \"STEINH <Q/L> <4/6/8/12> <group> \".");
    std::string qtype = c.arg[i + 1];
    int l = 0;
    if (!need_int(c, i + 2, l, "STEINH order")) return false;
    d.group = c.arg[i + 3];
    d.groupbit = groups.find(d.group);
    if (d.groupbit < 0) return c.fail("Error: Steinhardt group name " + d.group + " not found.");
    if (l != 3 && l != 4 && l != 6 && l != 8 && l != 12)
        return c.fail("Error: Steinhardt order L must be 3, 4, 6, 8, or 12.");
    if (qtype != "Q" && qtype != "L") return c.fail("Error: Steinhardt type must be 'Q' (local) or 'L' (global).");
    d.kind = (qtype == "Q") ? CAL_STEINH_Q : CAL_STEINH_L;
    d.l = l;
    int k = i + 4;
    while (k < c.narg) {
        if (!std::strcmp(c.arg[k], "cutoff_r")) { if (!need_double(c, k + 1, d.cutoff_r, "cutoff_r")) return false; k += 2; }
        else if (!std::strcmp(c.arg[k], "cutoff_Natoms")) { if (!need_int(c, k + 1, d.cutoff_natoms, "cutoff_Natoms")) return false; k += 2; }
        else if (!std::strcmp(c.arg[k], "cutoff_eps")) { if (!need_double(c, k + 1, d.cutoff_eps, "cutoff_eps")) return false; k += 2; }
        else if (!std::strcmp(c.arg[k], "d_block_size")) {
            if (!need_int(c, k + 1, d.block, "d_block_size")) return false;
            if (d.block <= 0) return c.fail("Error: 'd_block_size' must be > 0");
            k += 2;
        } else if (!std::strcmp(c.arg[k], "SW_FUNC_r")) {
            if (k + 1 >= c.narg) return c.fail("Error: 'SW_FUNC_r' keyword requires a value");
            if (!lookup_sw(c, cfg, c.arg[k + 1], d.sw_r)) return false;
            k += 2;
        } else if (!std::strcmp(c.arg[k], "SW_FUNC_cv")) {
            if (k + 1 >= c.narg) return c.fail("Error: 'SW_FUNC_cv' keyword requires a value");
            if (!lookup_sw(c, cfg, c.arg[k + 1], d.sw_cv)) return false;
            k += 2;
        } else break;
    }
    if (l == 8 || l == 12)   // accepted by the check, no CV class behind it (CVs_Steinhardt.cu:163-187)
        return c.fail("Metad-toy Error: Unknown or unregistered object type 'STEINH' (order 8/12 has no implementation).");
    if (d.kind == CAL_STEINH_L && d.sw_r.type != SW_STEP) {
        double rc = sw_invert_for_eps(d.sw_r, d.cutoff_eps);   // CVs_Steinhardt.cu:120-125
        if (!(rc > 0.0)) return c.fail("Error: invalid neighbor cutoff derived from SW_FUNC_r (use STEP, FERMI, TANH or RATIONAL).");
        d.cutoff_r = rc;
    }
    if (!(d.cutoff_r > 0.0)) return c.fail("Error: invalid neighbor cutoff.");
    if (d.kind == CAL_STEINH_Q && d.cutoff_natoms < 1) return c.fail("Error: 'cutoff_Natoms' must be >= 1");
    i = k;
    return true;
}

// Stru_factor::create: `STRU_FACTOR group [cutoff_r x] [q_factor x] [d_block_size n] [SW_func TYPE ...]
// [Chemical] [Chem_ctarget c] [Chem_sigma s] [Chem_map (t w) ...]`; with wchem, Weighted_chem_pair::create
// (src/cvs/CV_Weighted_Chemical_Pair_Order.cu:33-210): `WEIGHT_CHEM group [cutoff_r x] [d_block_size n]
// [SW_func ...] [Chem_map ...] [Chem_ctarget c] [Chem_sigma s]`, always type-weighted, no q_factor.
bool parse_sf(Cursor &c, int &i, const GroupTable &groups, CalDef &d, bool wchem) {
    if (i + 1 >= c.narg)
        return c.fail(wchem ? "Error: CHEM_PAIR command requires at least \"CHEM_PAIR <group> \"."
                            : "Error: STRU_FACTOR command requires at least \"STRU_FACTOR <group> \".");
    d.kind = CAL_STRU_FACTOR;
    if (wchem) {
        d.wchem = true;
        d.chem = true;
        d.q_factor = 0.0;
        d.has_q_factor = true;
    }
    d.group = c.arg[i + 1];
    d.groupbit = groups.find(d.group);
    if (d.groupbit < 0) return c.fail("Error: group name " + d.group + " not found.");
    d.cutoff_r = 8.0;
    int k = i + 2;
    while (k < c.narg) {
        if (!std::strcmp(c.arg[k], "cutoff_r")) { if (!need_double(c, k + 1, d.cutoff_r, "cutoff_r")) return false; k += 2; }
        else if (!wchem && !std::strcmp(c.arg[k], "q_factor")) {
            if (!need_double(c, k + 1, d.q_factor, "q_factor")) return false;
            if (d.q_factor <= 0) return c.fail("Error: 'q_factor' must be > 0");
            d.has_q_factor = true;
            k += 2;
        } else if (!std::strcmp(c.arg[k], "d_block_size")) {
            if (!need_int(c, k + 1, d.block, "d_block_size")) return false;
            if (d.block <= 0) return c.fail("Error: 'd_block_size' must be > 0");
            k += 2;
        } else if (!std::strcmp(c.arg[k], "SW_func")) {
            if (k + 1 >= c.narg) return c.fail("Error: 'SW_func' keyword requires a type (FERMI, TANH, RATIONAL)");
            std::string t = c.arg[k + 1];
            if (t != "FERMI" && t != "TANH" && t != "RATIONAL")
                return c.fail("Error: Unknown SW_func type. Choose from FERMI, TANH, RATIONAL.");
            int kk = k + 1;
            if (!parse_switch(c, kk, d.sf_sw)) return false;
            d.sf_use_sw = true;
            k = kk;
        } else if (!wchem && !std::strcmp(c.arg[k], "Chemical")) {
            d.chem = true;
            k += 1;
        } else if (!std::strcmp(c.arg[k], "Chem_ctarget")) {
            if (k + 1 >= c.narg) return c.fail("Error: 'Chem_ctarget' keyword requires a number");
            if (!need_double(c, k + 1, d.chem_ctarget, "Chem_ctarget")) return false;
            k += 2;
        } else if (!std::strcmp(c.arg[k], "Chem_sigma")) {
            if (k + 1 >= c.narg) return c.fail("Error: 'sigma' keyword requires a number");
            if (!need_double(c, k + 1, d.chem_sigma, "Chem_sigma")) return false;
            k += 2;
        } else if (!std::strcmp(c.arg[k], "Chem_map")) {
            // (type weight) pairs: one token "(1,0.5)" / "(1 0.5)", or two tokens "(1" "0.5)"
            k += 1;
            while (k < c.narg && c.arg[k][0] == '(') {
                std::string a = c.arg[k];
                std::string type_s, w_s;
                if (a.size() >= 2 && a.back() == ')') {
                    const std::string body = a.substr(1, a.size() - 2);
                    const size_t sep = body.find_first_of(" ,");
                    if (sep == std::string::npos) return c.fail("Error: Chem_map pairs must be formatted as (type weight)");
                    type_s = body.substr(0, sep);
                    w_s = body.substr(sep + 1);
                } else {
                    if (k + 1 >= c.narg) return c.fail("Error: Invalid Chem_map format near " + a);
                    const std::string b = c.arg[k + 1];
                    if (b.empty() || b.back() != ')') return c.fail("Error: Chem_map pairs must be formatted as (type weight)");
                    type_s = a.substr(1);
                    w_s = b.substr(0, b.size() - 1);
                    k += 1;
                }
                char *e1 = nullptr, *e2 = nullptr;
                const long t = std::strtol(type_s.c_str(), &e1, 10);
                const double w = std::strtod(w_s.c_str(), &e2);
                if (e1 == type_s.c_str() || e2 == w_s.c_str() || t < 0)
                    return c.fail("Error: Chem_map pairs must be formatted as (type weight)");
                d.chem_map.emplace_back((int)t, w);
                k += 1;
            }
        } else break;
    }
    if (!d.has_q_factor) return c.fail("Error: STRU_FACTOR requires 'q_factor' (it has no default).");
    if (d.chem && !(d.chem_sigma > 0.0)) return c.fail("Error: STRU_FACTOR 'Chem_sigma' must be > 0.");
    i = k;
    return true;
}

// STRU_FACTOR_K group [nk N] [kmag k] [seed s] -- k-vector S(k) (no reference counterpart).
bool parse_sk(Cursor &c, int &i, const GroupTable &groups, CalDef &d) {
    if (i + 1 >= c.narg) return c.fail("Error: STRU_FACTOR_K requires a group.");
    d.kind = CAL_STRU_FACTOR_K;
    d.group = c.arg[i + 1];
    d.groupbit = groups.find(d.group);
    if (d.groupbit < 0) return c.fail("Error: group name " + d.group + " not found.");
    int k = i + 2;
    while (k < c.narg) {
        if (!std::strcmp(c.arg[k], "nk")) { if (!need_int(c, k + 1, d.nk, "nk")) return false; k += 2; }
        else if (!std::strcmp(c.arg[k], "kmag")) { if (!need_double(c, k + 1, d.kmag, "kmag")) return false; k += 2; }
        else if (!std::strcmp(c.arg[k], "seed")) {
            int s = 0;
            if (!need_int(c, k + 1, s, "seed")) return false;
            d.seed = (unsigned long long)(unsigned)s;
            k += 2;
        } else break;
    }
    if (d.nk < 1 || d.nk > 1024) return c.fail("Error: STRU_FACTOR_K 'nk' must be in [1, 1024].");
    if (!(d.kmag > 0)) return c.fail("Error: STRU_FACTOR_K requires 'kmag' > 0.");
    d.kvecs = make_kvectors(d.nk, d.kmag, d.seed);
    i = k;
    return true;
}

// A SYMBOL's function against its CAL kind: set_CV_calculate of each CV
// (src/cvs/CVs_Steinhardt.cu:709-737, src/cvs/CVs_Steinhardt_Local.cu:600-645,
// src/cvs/CVs_Strufactor.cu:616-624).  STEINH L binds `.sw` as its CV switch.
std::string resolve_symbol(Config &cfg, const SymbolDef &s) {
    CalDef &d = cfg.cals[s.cal];
    bool ok = false;
    if (d.kind == CAL_STEINH_Q) ok = (s.func == "AVE" || s.func == "SW_FUNC");
    else if (d.kind == CAL_STEINH_L)
        ok = (s.func == "MEAN_SOLID" || s.func == "AVE" || s.func == "NSOLID" || s.func == "SW_FUNC" || s.func == "FRAC");
    else if (d.kind == CAL_STRU_FACTOR) ok = (s.func == "AVE" || s.func == "COUNT");
    else ok = (s.func == "AVE");
    if (!ok) return "Error: We can't find the func " + s.func + " for CAL " + s.cal + ".";
    if (d.kind == CAL_STEINH_Q && s.func == "SW_FUNC") {
        if (s.sub.empty() || !cfg.sws.count(s.sub))
            return "Switching function " + s.sub + " used in SYMBOL but not defined in CAL!";
    }
    if (d.kind == CAL_STEINH_L && !s.sub.empty()) {
        if (!cfg.sws.count(s.sub)) return "Switching function " + s.sub + " used in SYMBOL but not defined in CAL!";
        d.sw_cv = cfg.sws[s.sub];
    }
    if (d.kind == CAL_STRU_FACTOR && s.func == "COUNT" && !d.sf_use_sw)
        return d.wchem ? "Error: WEIGHT_CHEM COUNT needs 'SW_func' on the CAL."
                       : "Error: STRU_FACTOR COUNT needs 'SW_func' on the CAL.";
    return "";
}

}  // namespace

double sw_invert_for_eps(const SwParams &p, double eps) {
    switch (p.type) {
    case SW_STEP: return p.r0;
    case SW_FERMI: return p.r0 - std::log(1.0 / eps - 1.0) / p.alpha;
    case SW_TANH: return p.r0 + std::atanh(2.0 * eps - 1.0) / p.alpha;
    case SW_RATIONAL:
        if (p.n == 6 && p.m == 12) return std::pow(1.0 / eps - 1.0, 1.0 / 6.0) * p.r0 + p.d0;
        if (p.n == 4 && p.m == 8) return std::pow(1.0 / eps - 1.0, 1.0 / 4.0) * p.r0 + p.d0;
        if (2 * p.n == p.m) return std::pow(1.0 / eps - 1.0, 1.0 / p.n) * p.r0 + p.d0;
        {
            double lo = 0.0, hi = 1.0;
            while (sw_f<double>(p, hi) > eps) { hi *= 2.0; if (hi > 1e8) break; }
            for (int it = 0; it < 100; it++) {
                double mid = 0.5 * (lo + hi);
                if (sw_f<double>(p, mid) > eps) lo = mid; else hi = mid;
            }
            return 0.5 * (lo + hi);
        }
    default: return -1.0;
    }
}

std::vector<double> make_kvectors(int nk, double kmag, unsigned long long seed) {
    unsigned long long s = seed;
    auto next = [&s]() {   // SplitMix64
        s += 0x9E3779B97F4A7C15ULL;
        unsigned long long z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        return z ^ (z >> 31);
    };
    auto uni = [&]() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0; };
    std::vector<double> k(3 * (size_t)nk);
    for (int q = 0; q < nk; ++q) {
        double a, b, r2;
        do { a = uni(); b = uni(); r2 = a * a + b * b; } while (r2 >= 1.0 || r2 == 0.0);
        double t = 2.0 * std::sqrt(1.0 - r2);
        k[3 * q + 0] = kmag * a * t;
        k[3 * q + 1] = kmag * b * t;
        k[3 * q + 2] = kmag * (1.0 - 2.0 * r2);
    }
    return k;
}

std::string parse_fix_args(int narg, const char *const *arg, const GroupTable &groups, Config &cfg) {
    Cursor c{narg, arg, ""};
    int i = 0;
    while (i < narg) {
        const char *kw = arg[i];
        if (!std::strcmp(kw, "GAUSSIAN")) {
            if (i + 3 >= narg) return "Error: GAUSSIAN command requires 3 arguments: sigma, height, biasf.";
            if (!need_double(c, i + 1, cfg.sigma, "GAUSSIAN sigma") || !need_double(c, i + 2, cfg.height0, "GAUSSIAN height") ||
                !need_double(c, i + 3, cfg.biasf, "GAUSSIAN biasf"))
                return c.err;
            i += 4;
        } else if (!std::strcmp(kw, "PACE")) {
            if (i + 1 >= narg) return "Error: PACE command requires 1 argument: integer timesteps.";
            if (!need_int(c, i + 1, cfg.pace, "PACE")) return c.err;
            if (cfg.pace < 0) return "Error: PACE must be >= 0.";
            i += 2;
        } else if (!std::strcmp(kw, "RECORD")) {
            if (i + 1 >= narg) return "Error: RECORD command requires 1 argument: integer timesteps.";
            int k = i + 1;
            while (k < narg) {
                if (!std::strcmp(arg[k], "FILE_NAME")) {
                    if (k + 1 >= narg) return "Error: 'FILE_NAME' keyword requires a value";
                    cfg.rec_file = arg[k + 1];
                    k += 2;
                } else if (!std::strcmp(arg[k], "REC_PACE")) {
                    if (!need_int(c, k + 1, cfg.rec_pace, "REC_PACE")) return c.err;
                    k += 2;
                } else break;
            }
            i = k;
        } else if (!std::strcmp(kw, "CV_dim")) {
            if (i + 1 >= narg) return "Error: CV_dim command requires 1 argument.";
            if (!need_int(c, i + 1, cfg.cv_dim, "CV_dim")) return c.err;
            if (cfg.cv_dim < 1) return "Error: CV_dim must be >= 1.";
            cfg.cv_dim_set = true;
            cfg.dims.assign(cfg.cv_dim, DimDef{});
            i += 2;
        } else if (!std::strcmp(kw, "TEMP")) {
            if (i + 1 >= narg) return "Error: TEMP command requires 1 argument: target temperature.";
            if (!need_double(c, i + 1, cfg.temp, "TEMP")) return c.err;
            i += 2;
        } else if (!std::strcmp(kw, "CAL")) {
            if (i + 3 >= narg || std::strcmp(arg[i + 1], "NAME")) return "Error: CAL requires NAME keyword.";
            std::string name = arg[i + 2];
            std::string type = arg[i + 3];
            i += 3;
            if (type == "SW_FUNC") {
                if (cfg.sws.count(name)) return "Error: CAL name '" + name + "' is duplicated.";
                int k = i + 1;
                SwParams p;
                if (!parse_switch(c, k, p)) return c.err;
                cfg.sws[name] = p;
                i = k;
            } else {
                if (cfg.cals.count(name)) return "Error: CAL name '" + name + "' is duplicated.";
                CalDef d;
                d.name = name;
                bool ok;
                if (type == "STEINH") ok = parse_steinh(c, i, groups, cfg, d);
                else if (type == "STRU_FACTOR") ok = parse_sf(c, i, groups, d, false);
                else if (type == "WEIGHT_CHEM" || type == "CHEM_PAIR") ok = parse_sf(c, i, groups, d, true);
                else if (type == "STRU_FACTOR_K") ok = parse_sk(c, i, groups, d);
                else
                    return "Metad-toy Error: Unknown or unregistered object type '" + type + "' specified in CAL '" + name +
                           "'. Please register it in CVFactory or check your input script.";
                if (!ok) return c.err;
                cfg.cals[name] = d;
            }
        } else if (!std::strcmp(kw, "SYMBOL") || !std::strcmp(kw, "SIMBOL")) {
            if (i + 2 >= narg) return "Error: SYMBOL command requires 2 arguments: SYMBOL <symbol_name> <cv_method>.";
            SymbolDef s;
            s.name = arg[i + 1];
            std::string target = arg[i + 2];
            size_t dot = target.find('.');
            if (dot == std::string::npos) { s.cal = target; s.func = "value"; }
            else {
                s.cal = target.substr(0, dot);
                std::string rest = target.substr(dot + 1);
                size_t d2 = rest.find('.');
                s.func = rest.substr(0, d2);
                if (d2 != std::string::npos) s.sub = rest.substr(d2 + 1);
            }
            if (!cfg.cals.count(s.cal)) return "Error: SYMBOL " + s.name + " refers to unknown CAL '" + s.cal + "'.";
            for (auto &o : cfg.symbols)
                if (o.name == s.name) return "Error: SYMBOL '" + s.name + "' is duplicated.";
            if ((int)cfg.symbols.size() >= kMaxSymbols) return "Error: too many SYMBOL entries.";
            std::string e = resolve_symbol(cfg, s);   // set_CV_calculate at add_symbol time (DimSet.cu:28-52)
            if (!e.empty()) return e;
            cfg.symbols.push_back(s);
            i += 3;
        } else if (!std::strcmp(kw, "DIM")) {
            if (i + 5 >= narg) return "Error: DIM command requires 5 arguments: index, lower, upper, bins, cv_expr.";
            if (!cfg.cv_dim_set) return "Error: CV_dim must be given before DIM.";
            int idx = 0, nb = 0;
            double lo = 0, hi = 0;
            if (!need_int(c, i + 1, idx, "DIM index") || !need_double(c, i + 2, lo, "DIM lower") ||
                !need_double(c, i + 3, hi, "DIM upper") || !need_int(c, i + 4, nb, "DIM bins"))
                return c.err;
            idx -= 1;
            if (idx < 0 || idx >= cfg.cv_dim) return "Error: DIM index out of range or unsupported dimension.";
            if (!(hi > lo)) return "Error: DIM upper bound must exceed the lower bound.";
            if (nb < 4) return "Error: DIM needs at least 4 bins (Catmull-Rom stencil).";
            cfg.dims[idx] = DimDef{true, lo, hi, nb, arg[i + 5]};
            i += 6;
        } else if (!std::strcmp(kw, "Gaussian_Hill_type")) {
            if (!need_int(c, i + 1, cfg.hill_type, "Gaussian_Hill_type")) return c.err;
            cfg.hill_type = cfg.hill_type != 0;
            i += 2;
        } else if (!std::strcmp(kw, "METAD_RESTART")) {
            int v = 0;
            if (!need_int(c, i + 1, v, "METAD_RESTART")) return c.err;
            cfg.restart = v != 0;
            i += 2;
        } else if (!std::strcmp(kw, "NN_BIAS")) {   // extension: learned bias for CV_dim >= 3
            int v = 0;
            if (!need_int(c, i + 1, v, "NN_BIAS")) return c.err;
            cfg.nn = v != 0;
            i += 2;
        } else if (!std::strcmp(kw, "NN_TOL")) {
            if (!need_double(c, i + 1, cfg.nn_tol, "NN_TOL")) return c.err;
            if (!(cfg.nn_tol > 0)) return "Error: NN_TOL must be > 0.";
            i += 2;
        } else if (!std::strcmp(kw, "NN_REFIT")) {
            if (!need_int(c, i + 1, cfg.nn_refit, "NN_REFIT")) return c.err;
            if (cfg.nn_refit < 1) return "Error: NN_REFIT must be >= 1.";
            i += 2;
        } else if (!std::strcmp(kw, "NN_ITERS")) {
            if (!need_int(c, i + 1, cfg.nn_iters, "NN_ITERS")) return c.err;
            if (cfg.nn_iters < 1) return "Error: NN_ITERS must be >= 1.";
            i += 2;
        } else if (!std::strcmp(kw, "WT")) {
            int v = 0;
            if (!need_int(c, i + 1, v, "WT")) return c.err;
            cfg.wt = v != 0;
            i += 2;
        } else if (!std::strcmp(kw, "NEIGH_SKIN")) {   // extension: neighbour lists kept across steps
            if (!need_double(c, i + 1, cfg.neigh_skin, "NEIGH_SKIN")) return c.err;
            if (!(cfg.neigh_skin >= 0.0)) return "Error: NEIGH_SKIN must be >= 0.";
            i += 2;
        } else if (!std::strcmp(kw, "NEIGH_EVERY")) {
            if (!need_int(c, i + 1, cfg.neigh_every, "NEIGH_EVERY")) return c.err;
            if (cfg.neigh_every < 0) return "Error: NEIGH_EVERY must be >= 0.";
            i += 2;
        } else {
            return std::string("Error: Unknown keyword in fix metadynamics command: ") + kw;
        }
    }
    if (cfg.cv_dim > 4) return "Only 1D-3D are supported for optimized grid (4D with the hill-list bias).";
    if (!cfg.cv_dim_set) cfg.dims.assign(cfg.cv_dim, DimDef{});
    for (int d = 0; d < cfg.cv_dim; ++d)
        if (!cfg.dims[d].set) {
            std::ostringstream o;
            o << "Error: CV_dim is set to " << cfg.cv_dim << ", but DIM " << d + 1 << " is missing.";
            return o.str();
        }
    if (!(cfg.sigma > 0)) return "Error: GAUSSIAN sigma must be > 0.";
    return "";
}

}  // namespace mtd
