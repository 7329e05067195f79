"""The C ABI without a GPU: the library loads, exports every entry point that
include/metad_b200.h declares, and its host logic (the `fix metad` grammar and
the DIM expression compiler) behaves like the reference's."""
import os
import re

import pytest

import mtd
import oracle as O

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "metad_b200.h")

C1 = ["GAUSSIAN", "0.01", "0.005", "10", "PACE", "10",
      "CAL", "NAME", "Q6", "STEINH", "Q", "6", "all", "cutoff_r", "3.9", "cutoff_Natoms", "18",
      "SYMBOL", "v1", "Q6.AVE", "CV_dim", "1", "DIM", "1", "0", "1", "1000", "v1", "WT", "0"]
C2 = ["GAUSSIAN", "0.01", "0.005", "9", "PACE", "10", "TEMP", "300",
      "CAL", "NAME", "ST", "SW_FUNC", "STEP", "r_0", "3.9",
      "CAL", "NAME", "Q4", "STEINH", "L", "4", "all", "cutoff_r", "3.9", "cutoff_Natoms", "18", "SW_FUNC_r", "ST",
      "CAL", "NAME", "Q6", "STEINH", "L", "6", "all", "cutoff_r", "3.9", "cutoff_Natoms", "18", "SW_FUNC_r", "ST",
      "SYMBOL", "v1", "Q4.MEAN_SOLID", "SYMBOL", "v2", "Q6.MEAN_SOLID",
      "CV_dim", "2", "DIM", "1", "0", "1", "200", "v1", "DIM", "2", "0", "1", "200", "v2", "WT", "1"]


def test_library_exports_every_declared_symbol():
    decl = set(re.findall(r"\b(mtd_[a-z_0-9]+)\s*\(", open(HEADER).read()))
    L = mtd.lib()
    missing = [s for s in sorted(decl) if not hasattr(L, s)]
    assert not missing, missing
    assert decl == set(mtd.EXPORTS)
    assert L.mtd_abi_version() == 1


def test_reference_configs_parse():
    assert mtd.parse_args(C1) == ""
    assert mtd.parse_args(C2) == ""
    # the README's SIMBOL spelling is accepted as an alias of SYMBOL
    assert mtd.parse_args([t if t != "SYMBOL" else "SIMBOL" for t in C1]) == ""
    # the reference decks (test/in.test-steinhardt:104-112, in.test-structurefactor:95-103)
    deck1 = ["GAUSSIAN", "0.01", "0.05", "10.0", "PACE", "50", "RECORD", "FILE_NAME", "rec.log", "REC_PACE", "1",
             "CAL", "NAME", "Q6", "STEINH", "Q", "6", "metad_group", "cutoff_r", "3.8", "cutoff_Natoms", "18",
             "SYMBOL", "v1", "Q6.AVE", "CV_dim", "1", "DIM", "1", "0", "1", "10000", "v1", "METAD_RESTART", "1", "WT", "0"]
    deck2 = ["GAUSSIAN", "0.01", "0.01", "10.0", "PACE", "50", "RECORD", "FILE_NAME", "rec.log", "REC_PACE", "1",
             "CAL", "NAME", "SF", "STRU_FACTOR", "metad_group", "cutoff_r", "6", "q_factor", "2.8",
             "SYMBOL", "v1", "SF.AVE", "CV_dim", "1", "DIM", "1", "1.0", "4.0", "30000", "v1", "METAD_RESTART", "1", "WT", "0"]
    g = {"all": 1, "metad_group": 2}
    assert mtd.parse_args(deck1, groups=g) == ""
    assert mtd.parse_args(deck2, groups=g) == ""
    # STRU_FACTOR Chemical with both Chem_map spellings (CVs_Strufactor.cu:125-183)
    chem = deck2[:20] + ["Chemical", "Chem_ctarget", "2", "Chem_sigma", "0.5", "Chem_map", "(1,0.5)", "(3", "0.2)"] + \
        deck2[20:]
    assert mtd.parse_args(chem, groups=g) == ""
    # WEIGHT_CHEM as the user manual writes it (docs/manuals/User_Manual.zh.md:156)
    wchem = ["GAUSSIAN", "0.01", "0.01", "10.0", "PACE", "50", "CAL", "NAME", "CP", "WEIGHT_CHEM", "metad_group",
             "cutoff_r", "3", "Chem_map", "(1,0.1)", "(2,3.0)", "SYMBOL", "v1", "CP.AVE", "CV_dim", "1",
             "DIM", "1", "0", "10", "1000", "v1"]
    assert mtd.parse_args(wchem, groups=g) == ""


@pytest.mark.parametrize("args,needle", [
    (["FOO"], "Unknown keyword"),
    (C1[:-2] + ["WT"], "WT"),
    (["CAL", "NAME", "Q6", "STEINH", "X", "6", "all"], "type must be"),
    (["CAL", "NAME", "Q6", "STEINH", "Q", "5", "all"], "order L"),
    (["CAL", "NAME", "Q6", "STEINH", "Q", "8", "all"], "unregistered"),
    (["CAL", "NAME", "Q6", "STEINH", "Q", "6", "nogroup"], "group name"),
    (["CAL", "NAME", "Q6", "STEINH", "L", "6", "all", "SYMBOL", "v1", "Q6.AVE", "CV_dim", "1",
      "DIM", "1", "0", "1", "100", "v1"], "invalid neighbor cutoff"),
    (["CAL", "NAME", "S", "STRU_FACTOR", "all", "SYMBOL", "v1", "S.AVE"], "q_factor"),
    (["CAL", "NAME", "Z", "MYSTERY_CV", "all"], "Unknown or unregistered"),
    (["CAL", "NAME", "Q6", "STEINH", "Q", "6", "all", "CAL", "NAME", "Q6", "STEINH", "Q", "6", "all"], "duplicated"),
    (C1[:17] + ["SYMBOL", "v1", "Q6.LOC_AVE"], "find the func"),
    (C1[:17] + ["SYMBOL", "v1", "Q6.SW_FUNC.nosw"], "not defined"),
    (C1[:17] + ["SYMBOL", "v1", "Q6.AVE", "DIM", "1", "0", "1", "10", "v1"], "CV_dim must be given"),
    (C1[:17] + ["SYMBOL", "v1", "Q6.AVE", "CV_dim", "5"], "1D-3D"),
    (C1[:17] + ["SYMBOL", "v1", "Q6.AVE", "CV_dim", "4"], "DIM 1 is missing"),
    (C1[:17] + ["SYMBOL", "v1", "Q6.AVE", "NN_TOL", "0"], "NN_TOL must be > 0"),
    (C1[:17] + ["SYMBOL", "v1", "Q6.AVE", "CV_dim", "2", "DIM", "1", "0", "1", "10", "v1"], "DIM 2 is missing"),
    (C1[:17] + ["SYMBOL", "v1", "Q6.AVE", "CV_dim", "1", "DIM", "1", "0", "1", "10", "v1+w"], "unknown symbol"),
    (C1[:17] + ["SYMBOL", "v1", "Q6.AVE", "CV_dim", "1", "DIM", "1", "0", "1", "10", "(v1"], "expected ')'"),
    (["CAL", "NAME", "S", "STRU_FACTOR", "all", "q_factor", "2.8", "Chemical", "Chem_sigma", "0"], "Chem_sigma"),
    (["CAL", "NAME", "S", "STRU_FACTOR", "all", "q_factor", "2.8", "Chemical", "Chem_map", "(2"],
     "Invalid Chem_map format"),
    (["CAL", "NAME", "S", "STRU_FACTOR", "all", "q_factor", "2.8", "Chemical", "Chem_map", "(2;1)"],
     "(type weight)"),
    (["PACE", "ten"], "expects an integer"),
    (["GAUSSIAN", "0.01", "x", "10"], "expects a number"),
])
def test_parse_errors(args, needle):
    msg = mtd.parse_args(args)
    assert needle in msg, msg


@pytest.mark.parametrize("expr,vals", [
    ("v1", {"v1": 0.3}),
    ("(v1+v2)/2", {"v1": 0.3, "v2": 0.7}),
    ("v1*v2 - v1^3", {"v1": 0.31, "v2": 0.72}),
    ("sqrt(v1^2+v2^2)*2 - exp(-v2)", {"v1": 0.3, "v2": 0.4}),
    ("-v1^2 + 2^-1*v2", {"v1": 1.3, "v2": 0.4}),
    ("log(v1)+sin(v2)*cos(v1)-tanh(v1*v2)+abs(v2-1)", {"v1": 0.8, "v2": 0.35}),
    ("pow(v1, 2.5) + pi*v2 + e", {"v1": 0.8, "v2": 0.35}),
])
def test_expression_compiler_matches_oracle(expr, vals):
    v, g = mtd.eval_expression(expr, vals)
    vo, go = O.eval_expr(expr, vals)
    assert abs(v - vo) < 1e-14 * max(1.0, abs(vo))
    for k in vals:
        assert abs(g[k] - go[k]) < 1e-13 * max(1.0, abs(go[k]))


def test_library_refuses_to_run_without_build(tmp_path, monkeypatch):
    monkeypatch.setattr(mtd, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(mtd, "_lib", None)
    with pytest.raises(ImportError):
        mtd.lib()
