"""Evidence sets on one graph (flbp_sets_*) against the reference's loop.

FastLBP's alarm-ranking wrappers clamp the factor graph for a label set,
rebuild it and build a new CausalBP for every set (fl_wrapper.cu:29-45,
bingo_wrapper.cu:25-77). An engine of evidence sets holds the graph's
layout once and every set's messages, priors and beliefs; each set stops by
the tolerance rule on its own. Set k must give what its own engine gives:
the incremental-clamp engine (flbp_clamp_vars on a new engine, which the
clamp tests pin to the rebuilt graph) run with the same pass form, bit for
bit in FP32 and to 1e-12 in FP64, with the same sweep count and stop
reason; and the FP64 oracle on the clamped and rebuilt graph, to 1e-9
(FP64) / 1e-5 (FP32). Covered: AND/OR bodies clamped both ways, clamped
heads, variables and factors of every size class, sets without clamps,
sets that reach the sweep limit, damping, a second run from init(), and the
errors of malformed sets and of single-graph calls.
"""

import numpy as np
import pytest

import oracle as O
from fastlbp_b200 import CausalFactorGraph, Engine, FlbpError, SetsEngine, workloads
from test_engine_gpu import _large_item_graph

pytestmark = pytest.mark.gpu


def _bingo():
    return workloads.bingo_graph(600, 900, 40, workloads.uniform_int(2, 4), workloads.uniform_int(1, 6), 11,
                                 n_layers=6, back_frac=0.10, p_lo=0.6, p_hi=0.97, input_prior=0.8, n_alarms=30)


def _label_sets(fl, n_sets, seed, extra=()):
    """Label clamp maps: set 0 empty, then growing random sets over the graph's labels."""
    g = CausalFactorGraph.from_factors(fl)
    labels = g.var_labels()
    rng = np.random.default_rng(seed)
    out = [{}]
    for k in range(1, n_sets):
        n = int(rng.integers(1, 40))
        pick = rng.choice(labels, size=min(n, labels.size), replace=False).tolist()
        if k % 3 == 0:
            pick += list(extra)
        out.append({int(lab): int(rng.integers(0, 2)) for lab in pick})
    return out


def _own_engine(g, arrays, clamps, prec, damping):
    eng = Engine(arrays, precision=prec, damping=damping)
    eng.set_tuning(1, 1)  # the sets engine runs the direct form 1 of both passes
    items = sorted(clamps.items())
    if items:
        eng.clamp([g.findVar(lab) for lab, _ in items], [x for _, x in items])
    return eng


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("kind,damping", [("bingo", 0.0), ("large", 0.0), ("bingo", 0.1)])
def test_sets_equal_own_engines(kind, damping, prec):
    if kind == "bingo":
        fl, extra = _bingo(), ()
    else:
        fl = _large_item_graph(4)
        hub = 1200 + 30  # the 2100-entry variable, a big-tile variable, an input, a large factor's head
        extra = (hub, hub + 1 + 2100, 7, 1201)
    sets = _label_sets(fl, 9, seed=21, extra=extra)
    g = CausalFactorGraph.from_factors(fl)
    arrays = g.graph_arrays()
    tol, maxiter = 1e-6, 70
    want_b, want_s, want_r = [], [], []
    for cl in sets:
        e = _own_engine(g, arrays, cl, prec, damping)
        e.init()
        info = e.run_tol(tol, maxiter, 1e9)
        want_b.append(e.beliefs())
        want_s.append(info["sweeps"])
        want_r.append(info["reason"])
        e.close()
    se = SetsEngine(arrays, [{g.findVar(lab): x for lab, x in cl.items()} for cl in sets], precision=prec,
                    damping=damping)
    for rep in range(2):  # a second run from init() repeats the first
        se.init()
        sweeps, reasons = se.run_sets_tol(tol, maxiter)
        got = se.beliefs()
        assert sweeps.tolist() == want_s
        assert reasons.tolist() == want_r
        for k in range(len(sets)):
            assert np.array_equal(np.isnan(got[k]), np.isnan(want_b[k])), k
            ok = ~np.isnan(want_b[k])
            if prec == 32:
                assert np.array_equal(got[k][ok], want_b[k][ok]), k
            else:
                assert np.max(np.abs(got[k][ok] - want_b[k][ok])) <= 1e-12, k
    assert max(want_s) > min(want_s)  # sets really stop at different sweeps
    se.close()


@pytest.mark.parametrize("prec,tol", [(64, 1e-9), (32, 1e-5)])
def test_sets_match_oracle(prec, tol):
    """Each set against the FP64 oracle on its clamped and rebuilt graph:
    a fixed number of sweeps (a negative tolerance: every sweep counts as a
    move, so each set runs to the limit), then the
    tolerance loop's sweep count (FP32 rounding may move the last residual
    across tol by one sweep) and beliefs."""
    fl = _bingo()
    sets = _label_sets(fl, 6, seed=33)
    g = CausalFactorGraph.from_factors(fl)
    se = SetsEngine(g.graph_arrays(), [{g.findVar(lab): x for lab, x in cl.items()} for cl in sets], precision=prec)
    se.init()
    sweeps0, reasons0 = se.run_sets_tol(-1.0, 30)
    assert sweeps0.tolist() == [30] * len(sets) and set(reasons0.tolist()) == {2}
    fixed = se.beliefs()
    se.init()
    sweeps, _ = se.run_sets_tol(1e-6, 400)
    conv = se.beliefs()
    for k, cl in enumerate(sets):
        og = O.OracleGraph.from_factors(fl)
        og.clamp_labels(cl)
        og = og.rebuild()
        ref = O.OracleBP(og)
        ref.init()
        ref.run_fixed(1e-9, 30, 1)
        want = ref.beliefs()
        assert np.array_equal(np.isnan(want), np.isnan(fixed[k])), k
        ok = ~np.isnan(want)
        assert np.max(np.abs(fixed[k][ok] - want[ok])) <= tol, k
        ref = O.OracleBP(og)  # a new one: the reference's sweep count runs on across run calls
        ref.init()
        ref.run(1e-6, 400, 1e9)
        assert abs(int(sweeps[k]) - ref.iters) <= (0 if prec == 64 else 1), k
        assert np.max(np.abs(conv[k][ok] - ref.beliefs()[ok])) <= max(tol, 1e-6), k


def test_sets_errors():
    fl = _bingo()
    g = CausalFactorGraph.from_factors(fl)
    a = g.graph_arrays()
    with pytest.raises(FlbpError):
        SetsEngine(a, [{3: 1}, {5: 2}])  # a value other than 0/1
    with pytest.raises(FlbpError):
        SetsEngine(a, [{int(a["n_vars"]): 0}])  # out of range
    with pytest.raises(FlbpError):
        SetsEngine(a, [])
    se = SetsEngine(a, [{3: 1}, {3: 0}])  # the same variable, each value in its own set
    se.init()
    with pytest.raises(FlbpError):
        se.run_tol(1e-6, 10, 1e9)
    with pytest.raises(FlbpError):
        se.run_fixed(3)
    with pytest.raises(FlbpError):
        se.clamp([4], [1])
    sweeps, reasons = se.run_sets_tol(1e-6, 200)
    assert sweeps.shape == (2,) and reasons.tolist() == [0, 0]
    se.close()
