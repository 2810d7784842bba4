"""Gradients through unrolled sweeps (flbp_adjoint_*): the adjoint kernels
against a dense PyTorch unrolled-BP reference (autograd, float64) and
against central finite differences of the engine's own forward pass.

Loss: binary cross-entropy of the beliefs of labelled variables after T
sweeps; gradient with respect to every factor's p (rule firing
probabilities, input priors). Tolerances: FP64 adjoint against the torch
reference 1e-7 relative (both exact up to rounding), against central
differences (eps 1e-6) 1e-4 relative, also on a graph with clamped AND and
OR heads; the FP32 engine's adjoint (FP32
states and derivative arithmetic) against the FP64 one 2e-3 relative (L2).
The device-buffer entry points give the host-buffer results bit for bit,
and a batch engine's gradient is its graphs' gradients side by side.
"""

import numpy as np
import pytest
import torch

import torch_bp
from fastlbp_b200 import BatchEngine, CausalFactorGraph, Engine, workloads
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


def test_device_entry_points_match_host():
    a = _graph("large")
    T, K = 10, 3
    idx, y = _labels(a, seed=4)
    eng = Engine(a, precision=32)
    b_host = eng.adjoint_forward(T, K)
    bd = torch.empty(eng.n_vars, dtype=torch.float64, device="cuda")
    eng.beliefs_device(bd)
    assert np.array_equal(bd.cpu().numpy(), b_host)
    g = np.zeros(eng.n_vars)
    g[idx] = np.random.default_rng(5).standard_normal(idx.size)
    gp_h, gq_h = eng.adjoint_backward(g)
    gp = torch.empty(eng.n_factors, dtype=torch.float64, device="cuda")
    gq = torch.empty_like(gp)
    eng.adjoint_backward_device(torch.as_tensor(g, device="cuda"), gp, gq)
    assert np.array_equal(gp.cpu().numpy(), gp_h) and np.array_equal(gq.cpu().numpy(), gq_h)
    assert np.max(np.abs(gp_h)) > 0
    gp_only, none = eng.adjoint_backward(g, want_q=False)  # dL/dq not accumulated: dL/dp unchanged
    assert none is None and np.array_equal(gp_only, gp_h)
    # the autograd bridge on CUDA tensors against the host path (labels on
    # variables whose beliefs are not exactly 0 or 1, where the loss is finite)
    keep = (b_host[idx] > 0) & (b_host[idx] < 1)
    yt, it = torch.as_tensor(y[keep]), torch.as_tensor(idx[keep])
    p = torch.tensor(np.asarray(a["factor_p"], np.float64), requires_grad=True)
    _bce(unrolled_beliefs(p, eng, a["factor_q"], T, K), it, yt).backward()
    pd = torch.tensor(np.asarray(a["factor_p"], np.float64), device="cuda", requires_grad=True)
    _bce(unrolled_beliefs(pd, eng, a["factor_q"], T, K), it.cuda(), yt.cuda()).backward()
    want, got = p.grad.numpy(), pd.grad.cpu().numpy()
    assert np.max(np.abs(got - want)) <= 1e-12 * np.max(np.abs(want))


def test_batch_gradient_is_per_graph_gradients():
    graphs = [_graph("bingo"), _graph("large")]
    T, K = 12, 4
    labels = [_labels(a, seed=6 + k) for k, a in enumerate(graphs)]
    want_p, want_q = [], []
    for a, (idx, y) in zip(graphs, labels):
        e = Engine(a, precision=64)
        b = e.adjoint_forward(T, K)
        g = np.zeros(e.n_vars)
        g[idx] = -y / b[idx] + (1 - y) / (1 - b[idx])
        gp, gq = e.adjoint_backward(g)
        want_p.append(gp)
        want_q.append(gq)
        e.close()
    be = BatchEngine(graphs, precision=64)
    b = be.adjoint_forward(T, K)
    g = np.zeros(be.n_vars)
    for k, (idx, y) in enumerate(labels):
        j = be.var_off[k] + idx
        g[j] = -y / b[j] + (1 - y) / (1 - b[j])
    gp, gq = be.adjoint_backward(g)
    wp, wq = np.concatenate(want_p), np.concatenate(want_q)
    assert np.max(np.abs(gp - wp)) <= 1e-9 * np.max(np.abs(wp))
    assert np.max(np.abs(gq - wq)) <= 1e-9 * max(np.max(np.abs(wq)), 1e-300)


@pytest.mark.parametrize("prec", [32, 64])
def test_checkpointed_forward_is_the_plain_run(prec):
    """adjoint_forward leaves the engine exactly where T plain sweeps do, and
    a second backward (segment buffers reused) repeats the first."""
    a = _graph("large")
    T, K = 13, 4
    eng = Engine(a, precision=prec)
    b_ck = eng.adjoint_forward(T, K)
    eng.sweep(3)
    b_more = eng.compute_beliefs()
    ref = Engine(a, precision=prec)
    ref.init()
    ref.run_fixed(T)
    assert np.array_equal(b_ck, ref.beliefs())
    ref.sweep(3)
    assert np.array_equal(b_more, ref.compute_beliefs())
    idx, y = _labels(a, seed=8)
    g = np.zeros(eng.n_vars)
    g[idx] = y - 0.5
    eng.adjoint_forward(T, K)
    g1 = eng.adjoint_backward(g)
    g2 = eng.adjoint_backward(g)
    assert np.array_equal(g1[0], g2[0]) and np.array_equal(g1[1], g2[1])


def test_adjoint_on_clamped_graph_matches_central_differences():
    """Head-clamped AND and OR factors (a clamped graph, rebuilt): the
    adjoint against central differences (eps 1e-6) of the FP64 engine."""
    fl = workloads.bingo_graph(300, 450, 20, workloads.uniform_int(2, 4), workloads.uniform_int(1, 6), 9,
                               n_layers=6, back_frac=0.10, p_lo=0.6, p_hi=0.95, input_prior=0.8, n_alarms=30)
    g = CausalFactorGraph.from_factors(fl)
    labels = g.var_labels()
    rng = np.random.default_rng(21)
    g.clamp_labels({int(l): int(rng.integers(0, 2)) for l in rng.choice(labels, 25, replace=False)})
    a = g.rebuild().graph_arrays()
    assert np.asarray(a["factor_head_clamped"]).any()
    T, K, eps = 12, 4, 1e-6
    eng = Engine(a, precision=64)
    p0, q0 = np.asarray(a["factor_p"], np.float64).copy(), np.asarray(a["factor_q"], np.float64)
    b0 = eng.adjoint_forward(T, K)
    idx = np.array([i for i in rng.choice(eng.n_vars, 50, replace=False) if 0 < b0[i] < 1])
    y = (rng.random(idx.size) < 0.3).astype(np.float64)

    def loss(p):
        eng.set_factor_probs(p, q0)
        return float(_bce(torch.as_tensor(eng.adjoint_forward(T, K)), idx, torch.as_tensor(y)))

    eng.set_factor_probs(p0, q0)
    b = torch.as_tensor(eng.adjoint_forward(T, K), dtype=torch.float64).requires_grad_(True)
    _bce(b, idx, torch.as_tensor(y)).backward()
    gp, _ = eng.adjoint_backward(b.grad.numpy())
    cand = np.nonzero((p0 > 1e-3) & (p0 < 1 - 1e-3))[0]
    sample = rng.choice(cand, size=min(60, cand.size), replace=False)
    scale = np.max(np.abs(gp))
    assert scale > 0
    for I in sample:
        pp, pm = p0.copy(), p0.copy()
        pp[I] += eps
        pm[I] -= eps
        fd = (loss(pp) - loss(pm)) / (2 * eps)
        assert abs(fd - gp[I]) <= 1e-4 * max(abs(gp[I]), 1e-3 * scale), (I, fd, gp[I])


def test_shared_rule_gradient_matches_central_differences():
    """Three copies of one graph, each with its own labels, share every
    factor's p (the same rules analysed under different evidence). The
    shared gradient - the adjoint's per-factor gradients of a BatchEngine
    summed into their rules (fastlbp_b200.shard.shared_gradient, the
    reduction a multi-GPU learning step all-reduces) - against central
    differences of the summed loss, each rule moved in every copy at once
    (expand_shared)."""
    from fastlbp_b200.shard import expand_shared, shared_gradient

    a = _graph("bingo")
    T, K, eps = 20, 4, 1e-6
    copies = 3
    labels = [_labels(a, seed=20 + c) for c in range(copies)]
    be = BatchEngine([a] * copies, precision=64)
    F0 = len(a["factor_p"])
    rule_of = torch.as_tensor(np.tile(np.arange(F0), copies))
    p_rules = torch.as_tensor(np.asarray(a["factor_p"], np.float64))
    q_all = np.tile(np.asarray(a["factor_q"], np.float64), copies)
    base = torch.as_tensor(np.tile(np.asarray(a["factor_p"], np.float64), copies))

    def loss_and_grad(pr):
        be.set_factor_probs(expand_shared(pr, rule_of, base).numpy(), q_all)
        b = be.adjoint_forward(T, K)
        total, g = 0.0, np.zeros(be.n_vars)
        for c, (idx, y) in enumerate(labels):
            j = be.var_off[c] + idx
            total += float(_bce(torch.as_tensor(b), torch.as_tensor(j), torch.as_tensor(y)))
            g[j] += -y / b[j] + (1 - y) / (1 - b[j])
        return total, g

    _, g = loss_and_grad(p_rules)
    gp, _ = be.adjoint_backward(g, want_q=False)
    shared = shared_gradient(torch.as_tensor(gp), rule_of, F0).numpy()
    per_copy = gp.reshape(copies, F0)
    assert np.max(np.abs(shared - per_copy.sum(0))) <= 1e-12 * np.max(np.abs(shared))
    rng = np.random.default_rng(7)
    p0 = p_rules.numpy()
    cand = np.nonzero((p0 > 1e-3) & (p0 < 1 - 1e-3))[0]
    scale = np.max(np.abs(shared))
    for r in rng.choice(cand, size=min(25, cand.size), replace=False):
        pp, pm = p_rules.clone(), p_rules.clone()
        pp[r] += eps
        pm[r] -= eps
        fd = (loss_and_grad(pp)[0] - loss_and_grad(pm)[0]) / (2 * eps)
        assert abs(fd - shared[r]) <= 1e-4 * max(abs(shared[r]), 1e-3 * scale), (r, fd, shared[r])


@pytest.mark.parametrize("prec", [32, 64])
def test_device_factor_probs_match_host(prec):
    """flbp_set_factor_probs_device against flbp_set_factor_probs with the
    same new p and q: beliefs after a fixed run (FP64 1e-12; FP32 1e-6, the
    folded priors' logarithms being the device's), gradients (1e-9
    relative), an out-of-range value rejected with the engine unchanged,
    and a sequential schedule set afterwards built on the new values."""
    from fastlbp_b200 import FlbpError

    a = _graph("large")
    rng = np.random.default_rng(17)
    p = np.clip(np.asarray(a["factor_p"], np.float64) * rng.uniform(0.9, 1.0, len(a["factor_p"])), 0.0, 1.0)
    q = np.asarray(a["factor_q"], np.float64)
    host, dev = Engine(a, precision=prec), Engine(a, precision=prec)
    host.set_factor_probs(p, q)
    pd, qd = torch.as_tensor(p, device="cuda"), torch.as_tensor(q, device="cuda")
    torch.cuda.synchronize()
    dev.set_factor_probs_device(pd, qd)
    tol = 1e-12 if prec == 64 else 1e-6
    T, K = 12, 4
    bh, bd = host.adjoint_forward(T, K), dev.adjoint_forward(T, K)
    assert np.max(np.abs(bh - bd)) <= tol
    idx, _ = _labels(a, seed=8)
    g = np.zeros(host.n_vars)
    g[idx] = rng.standard_normal(idx.size)
    gh, gd = host.adjoint_backward(g)[0], dev.adjoint_backward(g)[0]
    if prec == 64:
        assert np.max(np.abs(gh - gd)) <= 1e-9 * np.max(np.abs(gh))
    else:
        assert np.linalg.norm(gh - gd) <= 1e-4 * np.linalg.norm(gh)
    bad = pd.clone()
    bad[5] = 1.5
    torch.cuda.synchronize()
    with pytest.raises(FlbpError):
        dev.set_factor_probs_device(bad, qd)
    assert np.array_equal(dev.adjoint_forward(T, K), bd)
    # a sequential schedule set afterwards reads the new values on the host
    from fastlbp_b200 import update_seq

    seq = update_seq(a, "SEQFIX", 42)
    host.set_update_seq(seq)
    dev.set_update_seq(seq)
    for e in (host, dev):
        e.init()
        e.run_fixed(5)
    assert np.max(np.abs(host.beliefs() - dev.beliefs())) <= tol
    host.close()
    dev.close()
