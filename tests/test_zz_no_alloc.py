"""The allocation-free entry point, flbp_run_fixed_device_noalloc.

It exists for callers that may not allocate GPU memory at solve time
(serving loops with a no-allocation policy, processes whose GPU memory
belongs to another allocator): the graph and the belief
output are device arrays the caller owns, and the messages live in the
library's fixed 4 MiB scratch array. This file runs last so that a failure
here does not hide the other tests; it passes alone or after them.

Checks: two calls in a row, on different graphs and settings, each agree
with the regular engine (flbp_engine_create + flbp_run_fixed) within the
FP32 tolerance of the other tests, and the second call leaves the device's
free memory unchanged; the solve agrees with the FP64 oracle on a clamped
graph and with the engine on a head clamped both ways.
"""

import ctypes as C

import numpy as np
import pytest

from fastlbp_b200 import CausalFactorGraph, Engine, _native, workloads

pytestmark = pytest.mark.gpu

TOL32 = 1e-5


def device_graph(g, torch):
    """Upload a graph's reference-order arrays as int32/float32 device tensors."""
    a = g.graph_arrays()
    c = g.construct()
    off = a["factor_offsets"]
    slot_var = a["slot_var"]
    state = np.zeros(off.size - 1, np.uint8)
    cl = a["factor_head_clamped"] == 1
    m0, m1 = a["factor_mask0"], a["factor_mask1"]
    state[cl & (m0 == 0) & (m1 == 1)] = 1
    state[cl & (m0 == 1) & (m1 == 0)] = 2
    state[cl & (m0 == 0) & (m1 == 0)] = 3
    var_slots = np.argsort(slot_var, kind="stable")
    host = dict(factor_offsets=off.astype(np.int32), slot_var=slot_var.astype(np.int32),
                factor_head=a["factor_head"].astype(np.int32), factor_type=a["factor_type"].astype(np.int32),
                factor_head_state=state, factor_p=a["factor_p"].astype(np.float32),
                factor_q=a["factor_q"].astype(np.float32), var_offsets=c["row_ptr_fv"].astype(np.int32),
                var_slots=var_slots.astype(np.int32))
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in host.items()}
    d = _native.DeviceGraph()
    d.n_vars, d.n_factors, d.n_slots = int(a["n_vars"]), int(off.size - 1), int(off[-1])
    for k, t in dev.items():
        setattr(d, k, t.data_ptr())
    return d, dev, a


def solve_noalloc(d, sweeps, damping, torch):
    out = torch.zeros(d.n_vars, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    rc = _native.lib().flbp_run_fixed_device_noalloc(C.byref(d), sweeps, damping, C.c_void_p(out.data_ptr()),
                                                     C.c_void_p(stream.cuda_stream))
    assert rc == 0, _native.last_error()
    torch.cuda.synchronize()
    return out.cpu().numpy()


def solve_engine(arrays, sweeps, damping):
    eng = Engine(arrays, precision=32, damping=damping)
    eng.init()
    eng.run_fixed(sweeps)
    b = eng.beliefs()
    eng.close()
    return b


def test_two_calls_match_the_engine_and_allocate_nothing():
    torch = pytest.importorskip("torch")
    fl = workloads.config0(0)
    clamps = {int(x): i % 2 for i, x in enumerate(fl.alarms)}
    g1 = CausalFactorGraph.from_factors(fl)
    g1.clamp_labels(clamps)
    g1 = g1.rebuild()
    g2 = CausalFactorGraph.from_factors(workloads.config0(5))
    d1, keep1, a1 = device_graph(g1, torch)
    d2, keep2, a2 = device_graph(g2, torch)
    assert d1.n_slots <= _native.NOALLOC_MAX_SLOTS and d2.n_slots <= _native.NOALLOC_MAX_SLOTS
    want1 = solve_engine(a1, 150, 0.1)
    want2 = solve_engine(a2, 80, 0.0)
    torch.cuda.synchronize()

    got1 = solve_noalloc(d1, 150, 0.1, torch)  # first call on the device also does the scratch set-up
    free_before, _ = torch.cuda.mem_get_info()
    got2 = solve_noalloc(d2, 80, 0.0, torch)
    free_after, _ = torch.cuda.mem_get_info()

    assert np.max(np.abs(got1 - want1)) <= TOL32
    assert np.max(np.abs(got2 - want2)) <= TOL32
    assert free_after == free_before


def test_oversized_graph_is_rejected():
    d = _native.DeviceGraph()
    d.n_vars, d.n_factors, d.n_slots = 1, 1, _native.NOALLOC_MAX_SLOTS + 1
    out = C.c_double()
    rc = _native.lib().flbp_run_fixed_device_noalloc(C.byref(d), 1, 0.0, C.c_void_p(C.addressof(out)), None)
    assert rc == 5
    assert b"at most" in _native.lib().flbp_last_error()


def test_against_the_oracle_and_a_doubly_clamped_head():
    """The allocation-free solve against the FP64 oracle on a clamped graph
    (1e-5), and against the engine on a graph whose head is clamped both
    ways (head mask (0,0), state 3): the reference's head fallback gives
    (0, 1) there and its body messages are NaN (0/0); NaN patterns and the
    finite beliefs must agree."""
    torch = pytest.importorskip("torch")
    import oracle as O

    fl = workloads.config0(3)
    clamps = {int(x): (i + 1) % 2 for i, x in enumerate(fl.alarms)}
    g = CausalFactorGraph.from_factors(fl)
    g.clamp_labels(clamps)
    g = g.rebuild()
    og = O.OracleGraph.from_factors(fl)
    og.clamp_labels(clamps)
    og = og.rebuild()
    d, keep, _ = device_graph(g, torch)
    got = solve_noalloc(d, 60, 0.0, torch)
    ref = O.OracleBP(og)
    ref.init()
    ref.run_fixed(1e-9, 60, 1)
    want = ref.beliefs()
    assert np.array_equal(np.isnan(got), np.isnan(want))
    ok = ~np.isnan(want)
    assert np.max(np.abs(got[ok] - want[ok])) <= TOL32

    g2 = CausalFactorGraph.from_factors(fl)
    head = g2.findVar(int(fl.alarms[0]))
    g2.clamp(head, 0)
    g2.clamp(head, 1)
    g2 = g2.rebuild()
    info = g2.factor_info()
    assert ((info["mask0"] == 0) & (info["mask1"] == 0)).any()
    d2, keep2, a2 = device_graph(g2, torch)
    got2 = solve_noalloc(d2, 4, 0.0, torch)
    want2 = solve_engine(a2, 4, 0.0)
    assert np.array_equal(np.isnan(got2), np.isnan(want2))
    ok2 = ~np.isnan(want2)
    assert ok2.any() and np.max(np.abs(got2[ok2] - want2[ok2])) <= TOL32
