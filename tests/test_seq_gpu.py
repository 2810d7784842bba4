"""Sequential schedules (updates=SEQFIX / TOPO) of the CUDA engine against the
FP64 oracle's restatement of the reference (buildFixedUpdateSeq /
buildTopoUpdateSeq, the conflict-free batches of putUpdateSeqToKernelFused,
csrc/ext/causal_bp.cu:186-304, 583-722, and the batch kernels of
csrc/kernel/causal_bp_seq.cu).

Tolerances as for PARALL: FP64 within 1e-9 of the oracle, FP32 within 1e-5
absolute on beliefs. SEQFIX orders come from std::mt19937(42), the order of
the reference's first CausalBP of a thread.
"""

import numpy as np
import pytest

import brute
import oracle as O
import trees
from fastlbp_b200 import BatchEngine, CausalFactorGraph, Engine, FlbpError, update_seq, workloads
from fastlbp_b200 import _native as N
from test_engine_gpu import TOL, _large_item_graph, _pair

pytestmark = pytest.mark.gpu


def _oracle(og, updates, damping=0.0):
    bp = O.OracleBP(og, damping=damping)
    n = bp.set_schedule(updates, 42)
    bp.init()
    return bp, n


def _clamped_cfg0(seed):
    fl = workloads.config0(seed)
    cl = {int(a): int(i % 2) for i, a in enumerate(fl.alarms)}
    return _pair(fl, cl)


@pytest.mark.parametrize("kernel", [1, 2, 3])
@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("updates,sweeps", [("SEQFIX", 60), ("TOPO", 20)])
def test_fixed_sweeps(updates, sweeps, prec, kernel):
    """kernel 1: two launches per batch; 2: the sweep on one cluster; 3: as 1
    with programmatic dependent launch."""
    g, og = _clamped_cfg0(0)
    bp, nb = _oracle(og, updates)
    bp.run_fixed(1e-6, sweeps, 1)
    eng = Engine.from_graph(g, precision=prec, updates=updates)
    assert eng.update_info() == (True, nb)
    eng.set_seq_kernel(kernel)
    eng.init()
    info = eng.run_fixed(sweeps)
    assert info["sweeps"] == sweeps
    assert info["launches"] == sweeps * (1 if kernel == 2 else 1 + 2 * nb) + 1
    assert np.max(np.abs(eng.beliefs() - bp.beliefs())) <= TOL[prec]
    assert np.max(np.abs(eng.lowpass() - bp.lowpass())) <= TOL[prec]


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("kernel", [0, 3])
def test_tolerance_run(prec, kernel):
    g, og = _pair(workloads.config0(1))
    bp, _ = _oracle(og, "SEQFIX")
    bp.run(1e-6, 1000, 100.0)
    eng = Engine.from_graph(g, precision=prec, updates="SEQFIX")
    eng.set_seq_kernel(kernel)
    eng.init()
    info = eng.run_tol(1e-6, 1000, 100.0)
    assert np.max(np.abs(eng.beliefs() - bp.beliefs())) <= TOL[prec]
    if prec == 64:
        assert info["sweeps"] == bp.iters
    else:
        assert abs(info["sweeps"] - bp.iters) <= 2


def test_lowpass_run():
    g, og = _clamped_cfg0(3)
    bp, _ = _oracle(og, "SEQFIX")
    frac, reason, sweeps = bp.run_lowpass(1e-6, 20, 60, 10)
    eng = Engine.from_graph(g, precision=64, updates="SEQFIX")
    eng.init()
    info = eng.run_lowpass(1e-6, 20, 60, 10)
    assert (info["reason"], info["sweeps"]) == (reason, sweeps)
    assert abs(info["frac"] - frac) <= 1e-12
    assert np.max(np.abs(eng.lowpass() - bp.lowpass())) <= 1e-9


@pytest.mark.parametrize("prec", [64, 32])
@pytest.mark.parametrize("damping", [0.0, 0.15])
def test_large_items(prec, damping):
    """Factors with bodies of 17 to 1000 slots (the warp forms on both sides
    of 256 body slots), a variable in 2100 factors, clamped heads; both
    launch forms give the same bits."""
    fl = _large_item_graph(11)
    clamps = {1200 + 3: 1, 1200 + 7: 0, 5: 1}
    g, og = _pair(fl, clamps)
    bp, _ = _oracle(og, "SEQFIX", damping)
    bp.run_fixed(1e-6, 15, 1)
    eng = Engine.from_graph(g, precision=prec, damping=damping, updates="SEQFIX")
    out = []
    for kernel in (1, 2, 3):
        eng.set_seq_kernel(kernel)
        eng.init()
        eng.run_fixed(15)
        out.append(eng.beliefs())
    assert np.max(np.abs(out[0] - bp.beliefs())) <= TOL[prec]
    assert np.array_equal(out[0], out[1]) and np.array_equal(out[0], out[2])


def test_trees_exact_marginals():
    """On trees the sequential schedule also converges to the exact marginals."""
    checked = 0
    for seed in range(40):
        fl = trees.random_tree(seed, n_factors=5)
        labels = sorted(set(fl.head.tolist()) | set(fl.body.tolist()))
        rng = np.random.default_rng(seed + 7)
        cl = {int(l): int(rng.integers(0, 2)) for l in labels if rng.random() < 0.2}
        with np.errstate(all="ignore"):
            ex = brute.marginals(labels, trees.as_brute_factors(fl, cl))
        if not np.all(np.isfinite(ex)):
            continue  # contradictory evidence
        g, _ = _pair(fl, cl)
        eng = Engine.from_graph(g, precision=64, updates="SEQFIX", seed=seed)
        eng.init()
        eng.run_tol(1e-13, 2000, 100.0)
        pos = {l: i for i, l in enumerate(labels)}
        want = np.array([ex[pos[int(l)]] for l in g.var_labels()])
        assert np.max(np.abs(eng.beliefs() - want)) <= 1e-9, seed
        checked += 1
    assert checked > 25


def test_back_to_parall_and_messages():
    g, og = _clamped_cfg0(0)
    a = g.graph_arrays()
    eng = Engine(a, precision=64, updates="SEQFIX")
    eng.init()
    eng.run_fixed(5)
    bp, _ = _oracle(og, "SEQFIX")
    bp.run_fixed(1e-6, 5, 1)
    m0, m1 = eng.fv_messages()
    o0, o1, _, _ = bp.messages()
    assert np.max(np.abs(m1 - o1 / (o0 + o1))) <= 1e-9
    eng.set_update_seq(None)
    assert eng.update_info() == (False, 1)
    ref = Engine(a, precision=64)
    for x in (eng, ref):
        x.init()
        x.run_fixed(30)
    assert np.array_equal(eng.beliefs(), ref.beliefs())


def test_unsupported_combinations():
    fl = workloads.config0(0)
    g = CausalFactorGraph.from_factors(fl)
    a = g.graph_arrays()
    eng = Engine(a, precision=32, updates="TOPO")
    with pytest.raises(FlbpError):
        eng.clamp([3], [1])
    with pytest.raises(FlbpError):
        eng.adjoint_forward(5, 5)
    with pytest.raises(FlbpError):
        eng.set_update_seq(np.arange(eng.n_slots - 1))  # not every slot
    bad = np.arange(eng.n_slots)
    bad[1] = 0
    with pytest.raises(FlbpError):
        eng.set_update_seq(bad)  # a slot twice
    eng.init()
    eng.run_fixed(3)  # the failed calls left the schedule in place
    eng2 = Engine(a, precision=32)
    eng2.clamp([3], [1])
    with pytest.raises(FlbpError):
        eng2.set_update_seq(update_seq(a, "SEQFIX"))
    be = BatchEngine([a, a], precision=32)
    seq = np.arange(2 * eng.n_slots, dtype=np.int64)
    rc = N.lib().flbp_set_update_seq(be._h, seq.ctypes.data, seq.size)
    assert rc == 4  # FLBP_ERR_STATE
