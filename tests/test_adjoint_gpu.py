"""Gradients through unrolled sweeps (flbp_adjoint_*): the adjoint kernels
against a dense PyTorch unrolled-BP reference (autograd, float64) and
against central finite differences of the engine's own forward pass.

Loss: binary cross-entropy of the beliefs of labelled variables after T
sweeps; gradient with respect to every factor's p (rule firing
probabilities, input priors). Tolerances: FP64 adjoint against the torch
reference 1e-7 relative (both exact up to rounding), against central
differences (eps 1e-6) 1e-4 relative; the FP32 engine's adjoint (FP32
states, FP64 derivative arithmetic) against the FP64 one 2e-3 relative.
"""

import numpy as np
import pytest
import torch

import torch_bp
from fastlbp_b200 import CausalFactorGraph, Engine, workloads
from fastlbp_b200.autograd import unrolled_beliefs
from test_engine_gpu import _large_item_graph

pytestmark = pytest.mark.gpu


def _graph(kind):
    if kind == "bingo":
        fl = workloads.bingo_graph(300, 450, 20, workloads.uniform_int(2, 4), workloads.uniform_int(1, 6), 9,
                                   n_layers=6, back_frac=0.10, p_lo=0.6, p_hi=0.95, input_prior=0.8, n_alarms=30)
    else:
        fl = _large_item_graph(3)
    return CausalFactorGraph.from_factors(fl).graph_arrays()


def _labels(arrays, seed=0, n=40):
    rng = np.random.default_rng(seed)
    V = int(arrays["n_vars"])
    idx = np.sort(rng.choice(V, size=min(n, V), replace=False))
    return idx, (rng.random(idx.size) < 0.3).astype(np.float64)


def _bce(b, idx, y):
    bb = b[idx]
    return -(y * torch.log(bb) + (1 - y) * torch.log(1 - bb)).sum()


@pytest.mark.parametrize("kind", ["bingo", "large"])
def test_adjoint_matches_torch_reference(kind):
    a = _graph(kind)
    T, K = 12, 5
    idx, y = _labels(a)
    yt = torch.as_tensor(y)
    p = torch.tensor(np.asarray(a["factor_p"], np.float64), requires_grad=True)
    loss = _bce(torch_bp.unrolled(a, p, T), idx, yt)
    loss.backward()
    want = p.grad.numpy()
    eng = Engine(a, precision=64)
    pe = torch.tensor(np.asarray(a["factor_p"], np.float64), requires_grad=True)
    b = unrolled_beliefs(pe, eng, a["factor_q"], T, K)
    _bce(b, idx, yt).backward()
    got = pe.grad.numpy()
    assert np.max(np.abs(got - want)) <= 1e-7 * max(1.0, np.max(np.abs(want)))
    assert np.max(np.abs(want)) > 0


def test_adjoint_matches_central_differences():
    a = _graph("bingo")
    T, K, eps = 20, 4, 1e-6
    idx, y = _labels(a, seed=1)
    eng = Engine(a, precision=64)
    p0, q0 = np.asarray(a["factor_p"], np.float64).copy(), np.asarray(a["factor_q"], np.float64)

    def loss(p):
        eng.set_factor_probs(p, q0)
        b = eng.adjoint_forward(T, K)
        return float(_bce(torch.as_tensor(b), idx, torch.as_tensor(y)))

    eng.set_factor_probs(p0, q0)
    b = torch.as_tensor(eng.adjoint_forward(T, K), dtype=torch.float64).requires_grad_(True)
    _bce(b, idx, torch.as_tensor(y)).backward()
    gp, _ = eng.adjoint_backward(b.grad.numpy())
    rng = np.random.default_rng(2)
    cand = np.nonzero((p0 > 1e-3) & (p0 < 1 - 1e-3))[0]
    sample = rng.choice(cand, size=min(60, cand.size), replace=False)
    scale = np.max(np.abs(gp))
    for I in sample:
        pp, pm = p0.copy(), p0.copy()
        pp[I] += eps
        pm[I] -= eps
        fd = (loss(pp) - loss(pm)) / (2 * eps)
        assert abs(fd - gp[I]) <= 1e-4 * max(abs(gp[I]), 1e-3 * scale), (I, fd, gp[I])


def test_fp32_adjoint_close_to_fp64():
    a = _graph("large")
    T, K = 15, 5
    idx, y = _labels(a, seed=3)
    grads = {}
    for prec in (64, 32):
        eng = Engine(a, precision=prec)
        p = torch.tensor(np.asarray(a["factor_p"], np.float64), requires_grad=True)
        _bce(unrolled_beliefs(p, eng, a["factor_q"], T, K), idx, torch.as_tensor(y)).backward()
        grads[prec] = p.grad.numpy()
    g64, g32 = grads[64], grads[32]
    assert np.linalg.norm(g32 - g64) <= 2e-3 * np.linalg.norm(g64)
