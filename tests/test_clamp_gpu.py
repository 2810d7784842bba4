"""Incremental evidence (flbp_clamp_vars) against FastLBP's own sequence:
clamp the factor graph (CausalFactorGraph::clamp on every neighbouring
factor, csrc/ext/causal_factor.cpp:63-100), rebuild it and build a new
engine, as fl_wrapper.cu:29-45 and bingo_wrapper.cu do after every label.

Both runs start from init(); beliefs agree to 1e-9 (FP64) / 1e-5 (FP32)
after a fixed number of sweeps, and tolerance runs stop after the same
number of sweeps. Covered: AND bodies clamped to 0 (the reference "kills"
the factor: p := q, empty body) and to 1 (the variable leaves the body), OR
bodies alike, clamped heads of AND/OR factors and singletons, variables of
the sliced-ELL, big-tile and block-cooperative size classes, damping, and
clamps given in two batches.
"""

import numpy as np
import pytest

from fastlbp_b200 import CausalFactorGraph, Engine, FlbpError, workloads
from test_engine_gpu import _large_item_graph

pytestmark = pytest.mark.gpu


def _bingo():
    return workloads.bingo_graph(600, 900, 40, workloads.uniform_int(2, 4), workloads.uniform_int(1, 6), 11,
                                 n_layers=6, back_frac=0.10, p_lo=0.6, p_hi=0.97, input_prior=0.8, n_alarms=30)


def _clamps(fl, n, seed, extra=()):
    """n clamps on random labels of the graph (heads and bodies alike), plus `extra`."""
    g = CausalFactorGraph.from_factors(fl)
    labels = g.var_labels()
    rng = np.random.default_rng(seed)
    pick = rng.choice(labels, size=min(n, labels.size), replace=False).tolist() + list(extra)
    return {int(lab): int(rng.integers(0, 2)) for lab in pick}


def _rebuilt(fl, clamps):
    g = CausalFactorGraph.from_factors(fl)
    g.clamp_labels(clamps)
    return g.rebuild().graph_arrays()


def _incremental(fl, clamps, batches=1, **kw):
    g = CausalFactorGraph.from_factors(fl)
    eng = Engine(g.graph_arrays(), **kw)
    items = sorted(clamps.items())
    for part in np.array_split(np.arange(len(items)), batches):
        eng.clamp([g.findVar(items[i][0]) for i in part], [items[i][1] for i in part])
    return eng


@pytest.mark.parametrize("prec,tol", [(64, 1e-9), (32, 1e-5)])
@pytest.mark.parametrize("kind", ["bingo", "large"])
def test_clamp_matches_rebuilt_graph(kind, prec, tol):
    if kind == "bingo":
        fl, n = _bingo(), 60
        extra = ()
    else:
        fl, n = _large_item_graph(4), 80
        hub = 1200 + 30  # after 1,200 inputs and 30 large factors: the 2100-entry variable
        extra = (hub, hub + 1 + 2100, 7, 1201)  # the hub, the big-tile variable, an input, a large factor's head
    clamps = _clamps(fl, n, seed=5, extra=extra)
    ref = Engine(_rebuilt(fl, clamps), precision=prec)
    ref.init()
    ref.run_fixed(30)
    eng = _incremental(fl, clamps, batches=2, precision=prec)
    eng.init()
    eng.run_fixed(30)
    want, got = ref.beliefs(), eng.beliefs()
    assert want.shape == got.shape
    assert np.array_equal(np.isnan(want), np.isnan(got))
    ok = ~np.isnan(want)
    assert np.max(np.abs(got[ok] - want[ok])) <= tol
    # the tolerance loop stops after the same number of sweeps
    ref.init()
    a = ref.run_tol(1e-6, 400, 1e9)
    eng.init()
    b = eng.run_tol(1e-6, 400, 1e9)
    assert a["sweeps"] == b["sweeps"]
    assert np.max(np.abs(eng.beliefs()[ok] - ref.beliefs()[ok])) <= max(tol, 1e-6)


def test_clamp_with_damping():
    fl = _bingo()
    clamps = _clamps(fl, 40, seed=6)
    ref = Engine(_rebuilt(fl, clamps), precision=32, damping=0.1)
    ref.init()
    ref.run_fixed(40)
    eng = _incremental(fl, clamps, precision=32, damping=0.1)
    eng.init()
    eng.run_fixed(40)
    assert np.max(np.abs(eng.beliefs() - ref.beliefs())) <= 1e-5


def test_label_loop_matches_new_engine_per_label():
    """The alarm-ranking loop: one clamp after another, a tolerance run after
    each. A new engine per label (the reference's loop) starts its sweep count
    and its previous beliefs afresh; so does an engine after a clamp, so the
    two agree at every label even when maxiter is small."""
    fl = _bingo()
    g = CausalFactorGraph.from_factors(fl)
    labels = sorted(_clamps(fl, 12, seed=9).items())
    eng = Engine(g.graph_arrays(), precision=32)
    done = {}
    for lab, val in labels:
        done[lab] = val
        ref = Engine(_rebuilt(fl, done), precision=32)
        ref.init()
        a = ref.run_tol(1e-6, 40, 1e9)
        eng.clamp([g.findVar(lab)], [val])
        eng.init()
        b = eng.run_tol(1e-6, 40, 1e9)
        assert a["sweeps"] == b["sweeps"]
        assert np.max(np.abs(eng.beliefs() - ref.beliefs())) <= 1e-5
        ref.close()


def test_clamp_rejects_conflicts():
    fl = _bingo()
    eng = Engine(CausalFactorGraph.from_factors(fl).graph_arrays(), precision=32)
    eng.clamp([3], [1])
    eng.clamp([3], [1])  # the same value again: nothing changes
    with pytest.raises(FlbpError):
        eng.clamp([3], [0])
    with pytest.raises(FlbpError):
        eng.clamp([5, 5], [0, 1])
    with pytest.raises(FlbpError):
        eng.clamp([eng.n_vars], [0])
    with pytest.raises(FlbpError):
        eng.clamp([4], [2])


def test_gradient_after_clamps_matches_rebuilt_graph():
    """Gradients through unrolled sweeps on an engine with incremental clamps
    equal those of the rebuilt graph at every factor whose (p, q) the clamp
    rewrite leaves as it is (a killed factor's p becomes q there)."""
    fl = _bingo()
    clamps = _clamps(fl, 30, seed=12)
    g = CausalFactorGraph.from_factors(fl)
    a0 = g.graph_arrays()
    a1 = _rebuilt(fl, clamps)
    ref = Engine(a1, precision=64)
    eng = _incremental(fl, clamps, precision=64)
    T, K = 15, 4
    b_ref = ref.adjoint_forward(T, K)
    b_eng = eng.adjoint_forward(T, K)
    ok = ~np.isnan(b_ref)  # conflicting clamps leave NaN beliefs in both
    assert np.array_equal(ok, ~np.isnan(b_eng))
    assert np.max(np.abs(b_ref[ok] - b_eng[ok])) <= 1e-9
    clamped = {g.findVar(lab) for lab in clamps}
    rng = np.random.default_rng(13)
    pool = set(rng.choice(eng.n_vars, 60, replace=False).tolist()) - clamped
    labelled = np.array(sorted(v for v in pool if ok[v]))
    grad = np.zeros(eng.n_vars)
    grad[labelled] = rng.standard_normal(labelled.size)
    gp_ref, _ = ref.adjoint_backward(grad)
    gp_eng, _ = eng.adjoint_backward(grad)
    same = (np.asarray(a0["factor_p"]) == np.asarray(a1["factor_p"])) & \
           (np.asarray(a0["factor_q"]) == np.asarray(a1["factor_q"]))
    assert same.sum() > 0.9 * same.size
    scale = max(np.max(np.abs(gp_ref[same])), 1e-300)
    assert scale > 0
    assert np.max(np.abs(gp_eng[same] - gp_ref[same])) <= 1e-8 * scale


@pytest.mark.parametrize("prec,tol", [(64, 1e-9), (32, 1e-5)])
def test_clamp_matches_oracle(prec, tol):
    """The incremental clamp against the FP64 oracle run on the clamped and
    rebuilt graph (CausalFactorGraph::clamp on every neighbouring factor, then
    a new graph from its factors, as fl_wrapper.cu:29-45 does): beliefs after
    a fixed run, and the tolerance loop's sweep count and beliefs."""
    import oracle as O

    fl = _bingo()
    clamps = _clamps(fl, 60, seed=12)
    og = O.OracleGraph.from_factors(fl)
    og.clamp_labels(clamps)
    og = og.rebuild()
    eng = _incremental(fl, clamps, batches=3, precision=prec)
    ref = O.OracleBP(og)
    ref.init()
    ref.run_fixed(1e-9, 30, 1)
    eng.init()
    eng.run_fixed(30)
    want, got = ref.beliefs(), eng.beliefs()
    assert np.array_equal(np.isnan(want), np.isnan(got))
    ok = ~np.isnan(want)
    assert np.max(np.abs(got[ok] - want[ok])) <= tol
    ref = O.OracleBP(og)  # a new one: the reference's sweep count runs on across run calls
    ref.init()
    ref.run(1e-6, 400, 1e9)
    eng.init()
    info = eng.run_tol(1e-6, 400, 1e9)
    # FP32 rounding may move the last residual across tol by one sweep
    assert abs(info["sweeps"] - ref.iters) <= (0 if prec == 64 else 1)
    assert np.max(np.abs(eng.beliefs()[ok] - ref.beliefs()[ok])) <= max(tol, 1e-6)
