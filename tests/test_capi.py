"""The C-ABI library: it loads, exports every entry point declared in
include/fastlbp_b200.h, and rejects malformed graphs with an error code and
message instead of exiting (validation runs before any CUDA call, so these
tests need no GPU)."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from fastlbp_b200 import Engine, FlbpError, _native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    text = open(os.path.join(ROOT, "include", "fastlbp_b200.h")).read()
    return sorted(set(re.findall(r"\b(flbp_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _native.lib()
    names = declared()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_native.EXPORTED)


def test_version_string():
    assert b"sm_100a" in _native.lib().flbp_version()


def good():
    # factor 0: AND head x1 (slot 1) body x0; factor 1: singleton x0; factor 2: singleton x1
    return dict(n_vars=2, factor_offsets=np.array([0, 2, 3, 4]), slot_var=np.array([0, 1, 0, 1]),
                factor_head=np.array([1, 2, 3]), factor_type=np.array([1, 0, 0], np.int32),
                factor_p=np.array([0.9, 0.5, 0.5]), factor_q=np.array([0.0, 0.0, 0.0]))


@pytest.mark.parametrize("mutate,msg", [
    (lambda a: a.update(factor_p=np.array([1.5, 0.5, 0.5])), "probabilities"),
    (lambda a: a.update(factor_q=np.array([np.nan, 0.0, 0.0])), "probabilities"),
    (lambda a: a.update(factor_type=np.array([7, 0, 0], np.int32)), "unknown factor type"),
    (lambda a: a.update(slot_var=np.array([0, 5, 0, 1])), "slot_var out of range"),
    (lambda a: a.update(factor_head=np.array([3, 2, 3])), "factor_head"),
    (lambda a: a.update(factor_offsets=np.array([0, 3, 2, 4])), "monotone"),
    (lambda a: a.update(factor_offsets=np.array([0, 1, 3, 4]), factor_head=np.array([0, 1, 3])), "singleton"),
    (lambda a: a.update(factor_head_clamped=np.array([1, 0, 0], np.int32), factor_mask0=np.array([0.5, 1, 1.0]),
                        factor_mask1=np.array([1.0, 1, 1])), "head_mask"),
])
def test_invalid_graphs_are_rejected(mutate, msg):
    a = good()
    mutate(a)
    with pytest.raises(FlbpError, match=msg) as ei:
        Engine(a)
    assert ei.value.code == 1


def test_invalid_options_are_rejected():
    with pytest.raises(FlbpError, match="precision"):
        Engine(good(), precision=16)
    with pytest.raises(FlbpError, match="damping"):
        Engine(good(), damping=1.0)


def test_size_limits_are_checked():
    desc = _native.GraphDesc()
    desc.n_vars = 1 << 33
    desc.n_factors = 0
    desc.n_slots = 0
    opts = _native.EngineOpts(32, -1, 0.0, None)
    h = C.c_void_p()
    rc = _native.lib().flbp_engine_create(C.byref(desc), C.byref(opts), C.byref(h))
    assert rc == 5 and b"2^32" in _native.lib().flbp_last_error()
