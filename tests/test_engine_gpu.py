"""GPU parity of the CUDA engine against the FP64 oracle and exact marginals.

Tolerances: FP64 engine within 1e-9 of the oracle (log-odds vs probability
arithmetic differ only by rounding); FP32 engine within 1e-5 absolute on
beliefs, the target of the FP32 log-domain design.
"""

import numpy as np
import pytest

import brute
import oracle as O
import trees
from fastlbp_b200 import CausalFactorGraph, Engine, workloads

pytestmark = pytest.mark.gpu

TOL = {64: 1e-9, 32: 1e-5}


def _pair(fl, clamps=None):
    g = CausalFactorGraph.from_factors(fl)
    og = O.OracleGraph.from_factors(fl)
    if clamps:
        g.clamp_labels(clamps)
        og.clamp_labels(clamps)
        g, og = g.rebuild(), og.rebuild()
    return g, og


@pytest.mark.parametrize("prec", [64, 32])
def test_trees_exact_marginals(prec):
    checked = 0
    for seed in range(120):
        fl = trees.random_tree(seed, n_factors=5)
        labels = sorted(set(fl.head.tolist()) | set(fl.body.tolist()))
        rng = np.random.default_rng(seed + 7)
        cl = {int(l): int(rng.integers(0, 2)) for l in labels if rng.random() < 0.2}
        with np.errstate(all="ignore"):
            ex = brute.marginals(labels, trees.as_brute_factors(fl, cl))
        if not np.all(np.isfinite(ex)):
            continue  # contradictory evidence
        g, _ = _pair(fl, cl)
        eng = Engine.from_graph(g, precision=prec)
        eng.init()
        eng.run_tol(1e-13 if prec == 64 else 1e-7, 2000, 100.0)
        b = eng.beliefs()
        pos = {l: i for i, l in enumerate(labels)}
        want = np.array([ex[pos[int(l)]] for l in g.var_labels()])
        assert np.max(np.abs(b - want)) <= (1e-9 if prec == 64 else 2e-5), seed
        checked += 1
    assert checked > 80


@pytest.mark.parametrize("prec", [64, 32])
def test_config0_tolerance_run(prec):
    fl = workloads.config0(0)
    g, og = _pair(fl)
    bp = O.OracleBP(og)
    bp.init()
    bp.run(1e-6, 1000, 100.0)
    eng = Engine.from_graph(g, precision=prec)
    eng.init()
    info = eng.run_tol(1e-6, 1000, 100.0)
    assert np.max(np.abs(eng.beliefs() - bp.beliefs())) <= TOL[prec]
    if prec == 64:
        assert info["sweeps"] == bp.iters
    else:
        assert abs(info["sweeps"] - bp.iters) <= 2


@pytest.mark.parametrize("prec", [64, 32])
def test_config0_clamped_fixed_sweeps(prec):
    fl = workloads.config0(0)
    cl = {int(a): int(i % 2) for i, a in enumerate(fl.alarms)}
    g, og = _pair(fl, cl)
    bp = O.OracleBP(og)
    bp.init()
    bp.run_fixed(1e-6, 500, 1)
    eng = Engine.from_graph(g, precision=prec)
    eng.init()
    info = eng.run_fixed(500)
    assert info["sweeps"] == 500
    assert np.max(np.abs(eng.lowpass() - bp.lowpass())) <= TOL[prec]
    assert np.max(np.abs(eng.beliefs() - bp.beliefs())) <= TOL[prec]


@pytest.mark.parametrize("prec", [64, 32])
def test_damped_sweeps(prec):
    fl = workloads.config1(seed=5, scale=0.002)
    g, og = _pair(fl)
    bp = O.OracleBP(og, damping=0.1)
    bp.init()
    bp.run_fixed(1e-6, 200, 1)
    eng = Engine.from_graph(g, precision=prec, damping=0.1)
    eng.init()
    eng.run_fixed(200)
    assert np.max(np.abs(eng.beliefs() - bp.beliefs())) <= TOL[prec]


@pytest.mark.parametrize("prec", [64, 32])
def test_lowpass_run(prec):
    fl = workloads.config0(3)
    cl = {int(a): int(i % 2) for i, a in enumerate(fl.alarms)}
    g, og = _pair(fl, cl)
    bp = O.OracleBP(og)
    bp.init()
    frac, reason, sweeps = bp.run_lowpass(1e-6, 50, 120, 20)
    eng = Engine.from_graph(g, precision=prec)
    eng.init()
    info = eng.run_lowpass(1e-6, 50, 120, 20)
    if prec == 64:
        assert (info["reason"], info["sweeps"]) == (reason, sweeps)
        assert abs(info["frac"] - frac) <= 1e-12
    assert np.max(np.abs(eng.lowpass() - bp.lowpass())) <= TOL[prec] * (1 if prec == 64 else 2)


@pytest.mark.parametrize("prec", [64, 32])
def test_messages_each_sweep(prec):
    fl = workloads.config0(1)
    cl = {int(a): int(i % 2) for i, a in enumerate(fl.alarms[:8])}
    g, og = _pair(fl, cl)
    bp = O.OracleBP(og)
    bp.init()
    eng = Engine.from_graph(g, precision=prec)
    eng.init()
    for _ in range(6):
        bp.sweep()
        eng.sweep(1)
        fv0, fv1, vf0, vf1 = bp.messages()
        m0, m1 = eng.fv_messages()
        assert np.max(np.abs(m1 - fv1 / (fv0 + fv1))) <= (1e-12 if prec == 64 else 2e-6)
        n0, n1 = eng.vf_messages()
        assert np.max(np.abs(n1 - vf1 / (vf0 + vf1))) <= (1e-12 if prec == 64 else 2e-6)


@pytest.mark.parametrize("prec", [64, 32])
def test_high_fanin_fault_localisation(prec):
    fl, cl = workloads.config2(seed=4, scale=0.01)
    g, og = _pair(fl, cl)
    eng = Engine.from_graph(g, precision=prec)
    assert eng.stats()["warp_factors"] > 0
    bp = O.OracleBP(og)
    bp.init()
    bp.run_fixed(1e-6, 100, 1)
    eng.init()
    eng.run_fixed(100)
    assert np.max(np.abs(eng.beliefs() - bp.beliefs())) <= TOL[prec]


def test_repeat_runs_continue_iteration_count():
    fl = workloads.config0(2)
    g, og = _pair(fl)
    bp = O.OracleBP(og)
    bp.init()
    bp.run_fixed(1e-6, 7, 1)
    bp.run(1e-6, 1000, 100.0)
    eng = Engine.from_graph(g, precision=64)
    eng.init()
    eng.run_fixed(7)
    info = eng.run_tol(1e-6, 1000, 100.0)
    assert info["total_sweeps"] == bp.iters
    assert np.max(np.abs(eng.beliefs() - bp.beliefs())) <= 1e-9


def _large_item_graph(seed):
    """Factors of every large-item size class (bodies of 17 to 1000 slots, on
    both sides of the 32/64/128/256 register splits and of the tile limit)
    and variables with more entries than a tile holds."""
    rng = np.random.default_rng(seed)
    n_in = 1200
    kind, head, off, body, p, q = [], [], [0], [], [], []

    def add(k, h, b, pp, qq):
        kind.append(k)
        head.append(h)
        body.extend(int(x) for x in b)
        off.append(len(body))
        p.append(pp)
        q.append(qq)

    for v in range(n_in):  # input priors
        add(workloads.SINGLETON, v, [], float(rng.uniform(0.05, 0.95)), 0.0)
    nxt = n_in
    for size in (17, 20, 33, 40, 64, 65, 100, 128, 129, 200, 255, 256, 257, 300, 1000):
        for k in (workloads.AND, workloads.OR):
            b = rng.choice(n_in, size=size, replace=False)
            qq = 0.0 if rng.random() < 0.5 else float(rng.uniform(0.0, 0.1))
            add(k, nxt, b, float(rng.uniform(0.6, 0.99)), qq)
            nxt += 1
    hub = nxt  # a variable in the bodies of 2100 rules: more entries than a tile holds
    add(workloads.SINGLETON, hub, [], 0.7, 0.0)
    nxt += 1
    for i in range(2100):
        add(workloads.AND, nxt, [hub, int(rng.integers(n_in))], float(rng.uniform(0.6, 0.99)), 0.0)
        nxt += 1
    mid = nxt  # and one with a few hundred entries (a big-tile variable)
    add(workloads.SINGLETON, mid, [], 0.4, 0.0)
    nxt += 1
    for i in range(300):
        add(workloads.OR, nxt, [mid, int(rng.integers(n_in)), int(rng.integers(n_in))], 1.0, 0.0)
        nxt += 1
    k, h, o, b, pp, qq = workloads._append_auto_singletons(
        np.array(kind, np.int32), np.array(head, np.int64), np.array(off, np.int64), np.array(body, np.int64),
        workloads._quant(np.array(p)), workloads._quant(np.array(q)))
    return workloads.FactorList(k, h, o, b, pp, qq)


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("damping", [0.0, 0.15])
def test_large_items(prec, damping):
    fl = _large_item_graph(11)
    clamps = {1200 + 3: 1, 1200 + 7: 0, 5: 1}  # clamp two big factors' heads and one input
    g, og = _pair(fl, clamps)
    eng = Engine.from_graph(g, precision=prec, damping=damping)
    st = eng.stats()
    assert st["huge_factors"] > 0 and st["huge_vars"] > 0 and st["big_factor_tiles"] > 0 and st["big_var_tiles"] > 0
    bp = O.OracleBP(og, damping=damping)
    bp.init()
    bp.run_fixed(1e-6, 40, 1)
    eng.init()
    eng.run_fixed(40)
    assert np.max(np.abs(eng.beliefs() - bp.beliefs())) <= TOL[prec]


def test_many_tiles_per_block():
    """A graph with at least 8 factor tiles per block of the staged factor
    pass (1.4 M factors, each block walking the list of tiles dealt to it
    by cost): FP32 damped sweeps within the FP32 tolerance of the FP64
    oracle, and a second run split over two run calls bit-equal to the
    first."""
    fl = workloads.config1(seed=7, scale=0.6)
    g, og = _pair(fl)
    eng = Engine.from_graph(g, precision=32, damping=0.1)
    eng.set_tuning(0, 0)  # the staged forms
    st = eng.stats()
    assert st["factor_tiles"] >= 8 * eng.tuning()["factor_blocks"]
    bp = O.OracleBP(og, damping=0.1)
    bp.init()
    bp.run_fixed(1e-6, 10, 1)
    eng.init()
    eng.run_fixed(10)
    b1, bo = eng.beliefs(), bp.beliefs()
    assert np.array_equal(np.isnan(b1), np.isnan(bo))
    assert np.nanmax(np.abs(b1 - bo)) <= TOL[32]
    eng.init()
    eng.run_fixed(4)
    eng.run_fixed(6)
    assert np.array_equal(eng.beliefs(), b1, equal_nan=True)


def test_fault_localisation_statement_ranking():
    """cfg2 shape at reduced size: tolerance run (tol 1e-6, maxiter 500) in
    FP32 against the FP64 oracle. Beliefs within the FP32 tolerance, and the
    ranking of the statements (the input tuples) by belief agrees: Spearman
    correlation >= 0.999, and every pair of statements whose oracle beliefs
    differ by more than twice the tolerance is ordered the same way."""
    from scipy.stats import spearmanr

    fl, cl = workloads.config2(seed=6, scale=0.02)
    g, og = _pair(fl, cl)
    eng = Engine.from_graph(g, precision=32)
    eng.init()
    info = eng.run_tol(1e-6, 500, 1e9)
    bp = O.OracleBP(og)
    bp.init()
    bp.run(1e-6, 500, 1e9)
    b, bo = eng.beliefs(), bp.beliefs()
    assert np.max(np.abs(b - bo)) <= TOL[32]
    assert abs(info["sweeps"] - bp.iters) <= 2
    labels = g.var_labels()
    stm = np.nonzero(labels < fl.info["n_inputs"])[0]
    assert stm.size > 20
    assert spearmanr(b[stm], bo[stm]).statistic >= 0.999
    d_o = bo[stm][:, None] - bo[stm][None, :]
    d_e = b[stm][:, None] - b[stm][None, :]
    sure = np.abs(d_o) > 2 * TOL[32]
    assert np.all(np.sign(d_e[sure]) == np.sign(d_o[sure]))


def test_reset_counts_gives_a_new_engines_run():
    """run_tol's maxiter counts every sweep since construction (the
    reference's _iters), so a second tolerance run on the same engine can
    stop at the limit; flbp_reset_counts gives the engine a new engine's
    sweep count and beliefs, and the next init() + run_tol repeats a new
    engine's run bit for bit."""
    fl = workloads.config0(2)
    g, _ = _pair(fl)
    a = g.graph_arrays()
    fresh = Engine(a, precision=32)
    fresh.init()
    want = fresh.run_tol(1e-6, 60, 1e9)
    b_want = fresh.beliefs()
    eng = Engine(a, precision=32)
    for _ in range(3):
        eng.init()
        eng.run_tol(1e-6, 60, 1e9)
    eng.init()
    capped = eng.run_tol(1e-6, 60, 1e9)
    assert capped["sweeps"] < want["sweeps"]  # the limit counts the earlier runs' sweeps too
    eng.reset_counts()
    eng.init()
    got = eng.run_tol(1e-6, 60, 1e9)
    assert got["sweeps"] == want["sweeps"] and got["reason"] == want["reason"]
    assert np.array_equal(eng.beliefs(), b_want)
