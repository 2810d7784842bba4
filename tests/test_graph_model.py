"""Bit-exact parity of graph construction, edge indexing and clamping.

The product's graph model (the C++ CausalFactorGraph behind the C ABI) is
compared with the FP64 oracle's restatement and, where it was built here,
with the reference's own graph model compiled from its sources.
"""

import numpy as np
import pytest

import oracle as O
from fastlbp_b200 import CausalFactorGraph, FlbpError, workloads

KEYS = ["type", "head", "p", "q", "clamped", "mask0", "mask1", "nvars", "vars_off", "vars"]


def same_graph(a, b):
    fa, fb = a.factor_info(), b.factor_info()
    for k in KEYS:
        assert np.array_equal(fa[k], fb[k]), k
    assert np.array_equal(a.var_labels(), b.var_labels())
    for side in (0, 1):
        for x, y in zip(a.neighbors(bool(side)), b.neighbors(bool(side))):
            assert np.array_equal(x, y)


def triple(fl, tmp_path):
    path = str(tmp_path / "g.causal_fg")
    fl.write(path)
    prod = CausalFactorGraph.read_file(path)
    orc = O.OracleGraph.from_file(path)
    ref = O.RefGraph.from_file(path) if O.ref_lib() is not None else None
    return prod, orc, ref


@pytest.mark.parametrize("seed", [0, 1])
def test_read_and_construct_config0(seed, tmp_path):
    fl = workloads.config0(seed)
    prod, orc, ref = triple(fl, tmp_path)
    same_graph(prod, orc)
    if ref is not None:
        same_graph(orc, ref)
    same_graph(CausalFactorGraph.from_factors(fl), orc)
    c, o = prod.construct(), orc.construct()
    assert np.array_equal(c["factor_offsets"], o["row_ptr_vf"])
    assert np.array_equal(c["slot_var"], o["col_ind_vf"])
    assert np.array_equal(c["factor_head"], o["head"])
    assert np.array_equal(c["row_ptr_fv"], o["row_ptr_fv"])
    assert np.array_equal(c["col_ind_fv"], o["col_ind_fv"])


def test_clamping_all_cases(tmp_path):
    """Head clamps, double clamps (mask product), AND/OR body clamps that
    remove or resolve the rule, singleton clamps; then the fl_wrapper rebuild."""
    fl = workloads.config0(2)
    prod, orc, ref = triple(fl, tmp_path)
    graphs = [g for g in (prod, orc, ref) if g is not None]
    labels = orc.var_labels()
    rng = np.random.default_rng(0)
    idx = rng.choice(labels.size, 120, replace=False)
    for n, i in enumerate(idx):
        for g in graphs:
            g.clamp(int(i), n % 2)
    for i in idx[:10]:  # clamp again with the other value: head masks multiply to (0,0)
        for g in graphs:
            g.clamp(int(i), 1)
    for g in graphs[1:]:
        same_graph(graphs[0], g)
    rebuilt = [g.rebuild() for g in graphs]
    for g in rebuilt[1:]:
        same_graph(rebuilt[0], g)
    info = rebuilt[0].factor_info()
    assert (info["clamped"] == 1).any()
    assert ((info["mask0"] == 0) & (info["mask1"] == 0)).any()


def test_reader_grammar_variants():
    text = "\n".join([
        "5",
        "",
        "1",
        "*0.75",          # p without ';'
        "2",
        "2 3",
        "",
        "4",
        "+;0.25",         # only q
        "1",
        "1",
        "",
        "5",
        "*0.5;0.125",
        "0",
        "",               # empty body line
        "",
        "6",
        "# comment line after the head line",
        "+",
        "2",
        "5 4",
        "",
        "2",
        "I",
        "0.875",
        "# trailing comment",
        "",
    ])
    prod = CausalFactorGraph.from_text(text)
    orc = O.OracleGraph.from_text(text)
    same_graph(prod, orc)
    info = prod.factor_info()
    assert info["p"][0] == 0.75 and info["q"][0] == 0.0
    assert info["p"][1] == 1.0 and info["q"][1] == 0.25
    assert info["p"][2] == 0.5 and info["q"][2] == 0.125
    # variable 3 never heads a factor: the reader appends Singleton(0.5)
    assert info["type"][-1] == 0 and info["head"][-1] == 3 and info["p"][-1] == 0.5


def test_reader_errors_are_reported_not_fatal(tmp_path):
    with pytest.raises(FlbpError):
        CausalFactorGraph.read_file(str(tmp_path / "missing.causal_fg"))
    with pytest.raises(FlbpError, match="Unreachable"):
        CausalFactorGraph.from_text("1\n\n3\nX\n0.5\n")
    g = CausalFactorGraph.from_factors(workloads.config0(0))
    with pytest.raises(FlbpError):
        g.clamp(g.nrVars() + 5, 1)
    with pytest.raises(FlbpError):
        g.clamp(0, 2)
