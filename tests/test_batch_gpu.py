"""Batched solves (flbp_batch_*) against one engine per graph.

A batch holds several independent graphs of uneven size (Bingo-style, with
clamps, and one with factors and variables of every large-item class). Each
graph stops by the tolerance rule on its own and is then frozen, so its
sweep count and stop reason must equal those of the same graph solved alone
with run_tol from init(), and so must its beliefs: bit for bit in FP32, where
every factor and variable is evaluated by the same arithmetic in either
layout, and to within 1e-12 in FP64, where the two layouts were seen to
differ in the last bit of a few values. Some graphs are given a sweep limit
they reach before converging.
"""

import numpy as np
import pytest

import oracle as O
from fastlbp_b200 import BatchEngine, CausalFactorGraph, Engine, workloads
from test_engine_gpu import _large_item_graph

pytestmark = pytest.mark.gpu


def _graphs():
    out = []
    for i, nt in enumerate([400, 2500, 900, 6000, 150, 1800]):
        fl = workloads.bingo_graph(nt, int(1.5 * nt), max(10, nt // 20), workloads.uniform_int(2, 4),
                                   workloads.uniform_int(1, 6), 100 + i, n_layers=8, back_frac=0.10, p_lo=0.85,
                                   p_hi=0.99, input_prior=0.99, n_alarms=20)
        g = CausalFactorGraph.from_factors(fl)
        g.clamp_labels({int(a): int(k % 2) for k, a in enumerate(fl.alarms[: 1 + i * 3])})
        out.append(g.rebuild().graph_arrays())
    big = CausalFactorGraph.from_factors(_large_item_graph(5))
    out.insert(3, big.graph_arrays())
    return out


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("damping", [0.0, 0.1])
def test_batch_equals_separate_solves(prec, damping):
    graphs = _graphs()
    tol, maxiter = 1e-6, 60
    want_b, want_s, want_r = [], [], []
    for a in graphs:
        e = Engine(a, precision=prec, damping=damping)
        e.init()
        info = e.run_tol(tol, maxiter, 1e9)
        want_b.append(e.beliefs())
        want_s.append(info["sweeps"])
        want_r.append(info["reason"])
        e.close()
    be = BatchEngine(graphs, precision=prec, damping=damping)
    be.init()
    sweeps, reasons = be.run_batch_tol(tol, maxiter)
    allb = be.beliefs()
    assert sweeps.tolist() == want_s
    assert reasons.tolist() == want_r
    for g in range(len(graphs)):
        got = be.beliefs_of(g, allb)
        if prec == 32:
            assert np.array_equal(got, want_b[g]), g
        else:
            assert np.max(np.abs(got - want_b[g])) <= 1e-12, g
    assert max(want_s) > min(want_s)  # graphs really stop at different sweeps
    # run again from init: same results (the per-graph state is reset per call)
    be.init()
    sweeps2, _ = be.run_batch_tol(tol, maxiter)
    assert sweeps2.tolist() == want_s
    be.close()


def test_batch_graph_matches_oracle():
    graphs = _graphs()
    be = BatchEngine(graphs, precision=64)
    be.init()
    sweeps, _ = be.run_batch_tol(1e-6, 1000)
    fl = workloads.bingo_graph(900, 1350, 45, workloads.uniform_int(2, 4), workloads.uniform_int(1, 6), 102,
                               n_layers=8, back_frac=0.10, p_lo=0.85, p_hi=0.99, input_prior=0.99, n_alarms=20)
    og = O.OracleGraph.from_factors(fl)
    og.clamp_labels({int(a): int(k % 2) for k, a in enumerate(fl.alarms[:7])})
    og = og.rebuild()
    bp = O.OracleBP(og)
    bp.init()
    bp.run(1e-6, 1000, 1e9)
    assert sweeps[2] == bp.iters
    assert np.max(np.abs(be.beliefs_of(2) - bp.beliefs())) <= 1e-9
