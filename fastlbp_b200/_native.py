"""ctypes bindings of the C ABI in include/fastlbp_b200.h.

Loading fails loudly when libfastlbp_b200.so has not been built: there is no
CPU fallback anywhere in the package.
"""

from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfastlbp_b200.so")

FLBP_OK = 0
ERRORS = {1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "invalid state", 5: "limit exceeded",
          6: "device wait timed out"}

_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_vp = C.c_void_p


class _F64OrNull:
    """A C-contiguous float64 array, or None for a NULL pointer."""

    @classmethod
    def from_param(cls, obj):
        return None if obj is None else _f64p.from_param(obj)


class GraphDesc(C.Structure):
    _fields_ = [("n_vars", C.c_int64), ("n_factors", C.c_int64), ("n_slots", C.c_int64),
                ("factor_offsets", _vp), ("slot_var", _vp), ("factor_head", _vp), ("factor_type", _vp),
                ("factor_p", _vp), ("factor_q", _vp), ("factor_head_clamped", _vp), ("factor_mask0", _vp),
                ("factor_mask1", _vp)]


class EngineOpts(C.Structure):
    _fields_ = [("precision", C.c_int32), ("device", C.c_int32), ("damping", C.c_double), ("stream", _vp)]


class DeviceGraph(C.Structure):
    """flbp_device_graph: a graph in device memory for the allocation-free solve."""
    _fields_ = [("n_vars", C.c_int32), ("n_factors", C.c_int32), ("n_slots", C.c_int32),
                ("factor_offsets", _vp), ("slot_var", _vp), ("factor_head", _vp), ("factor_type", _vp),
                ("factor_head_state", _vp), ("factor_p", _vp), ("factor_q", _vp), ("var_offsets", _vp),
                ("var_slots", _vp)]


NOALLOC_MAX_SLOTS = 1 << 19


class Tuning(C.Structure):
    """flbp_tuning: form of each sweep pass (0 staged, 1/2 direct) and the blocks it launches."""
    _fields_ = [("factor_form", C.c_int32), ("var_form", C.c_int32), ("factor_blocks", C.c_int32),
                ("var_blocks", C.c_int32)]


class RunInfo(C.Structure):
    _fields_ = [("sweeps", C.c_int64), ("total_sweeps", C.c_int64), ("maxdiff", C.c_double), ("frac", C.c_double),
                ("reason", C.c_int32), ("status", C.c_int32), ("launches", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class FlbpError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s (%d): %s" % (ERRORS.get(code, "error"), code, msg))
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("libfastlbp_b200.so is not built; run `python -m fastlbp_b200.build` "
                          "(or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    L.flbp_last_error.restype = C.c_char_p
    L.flbp_version.restype = C.c_char_p
    P = C.POINTER
    sig = {
        "flbp_engine_create": [P(GraphDesc), P(EngineOpts), P(_vp)],
        "flbp_engine_destroy": [_vp],
        "flbp_init": [_vp],
        "flbp_run_tol": [_vp, C.c_double, C.c_int64, C.c_double, P(RunInfo)],
        "flbp_run_fixed": [_vp, C.c_int64, P(RunInfo)],
        "flbp_run_lowpass": [_vp, C.c_double, C.c_int64, C.c_int64, C.c_int64, C.c_double, P(RunInfo)],
        "flbp_sweep": [_vp, C.c_int64],
        "flbp_get_beliefs": [_vp, _f64p, C.c_int64],
        "flbp_get_lowpass": [_vp, _f64p, C.c_int64],
        "flbp_compute_beliefs": [_vp, _f64p, C.c_int64],
        "flbp_get_fv_messages": [_vp, _f64p, _f64p, C.c_int64],
        "flbp_get_vf_messages": [_vp, _f64p, _f64p, C.c_int64],
        "flbp_engine_stats": [_vp, _i64p, C.c_int64],
        "flbp_last_run_ms": [_vp, P(C.c_double)],
        "flbp_set_kernel_timing": [_vp, C.c_int32],
        "flbp_kernel_times": [_vp, _f64p, _i64p],
        "flbp_fg_read_file": [C.c_char_p, P(_vp)],
        "flbp_fg_read_string": [C.c_char_p, P(_vp)],
        "flbp_fg_from_factors": [C.c_int64, _i32p, _i64p, _i64p, _i64p, _f64p, _f64p, P(_vp)],
        "flbp_fg_destroy": [_vp],
        "flbp_fg_clamp": [_vp, C.c_int64, C.c_int64],
        "flbp_fg_rebuild": [_vp, P(_vp)],
        "flbp_fg_sizes": [_vp, _i64p],
        "flbp_fg_var_labels": [_vp, _i64p, C.c_int64],
        "flbp_fg_factors": [_vp, _i32p, _i64p, _f64p, _f64p, _i32p, _f64p, _f64p, _i64p, _i64p],
        "flbp_fg_neighbors": [_vp, C.c_int32, _i64p, _i64p, _i64p, _i64p],
        "flbp_fg_construct": [_vp, _i64p, _i64p, _i64p, _i64p, _i64p],
        "flbp_engine_create_from_fg": [_vp, P(EngineOpts), P(_vp)],
        "flbp_run_fixed_device_noalloc": [P(DeviceGraph), C.c_int64, C.c_double, _vp, _vp],
        "flbp_batch_create": [P(GraphDesc), C.c_int64, P(EngineOpts), P(_vp)],
        "flbp_batch_info": [_vp, P(C.c_int64), _i64p],
        "flbp_batch_run_tol": [_vp, C.c_double, C.c_int64, C.c_double, _i64p, _i32p, P(RunInfo)],
        "flbp_adjoint_forward": [_vp, C.c_int64, C.c_int64, _F64OrNull, C.c_int64],
        "flbp_adjoint_backward": [_vp, _f64p, _F64OrNull, _F64OrNull],
        "flbp_adjoint_backward_device": [_vp, _vp, _vp, _vp],
        "flbp_get_beliefs_device": [_vp, _vp, C.c_int64],
        "flbp_clamp_vars": [_vp, C.c_int64, _i64p, _i32p],
        "flbp_layout_digest": [P(GraphDesc), _vp, _vp, C.c_uint32, C.c_int32, P(C.c_uint64)],
        "flbp_set_factor_probs": [_vp, _f64p, _f64p],
        "flbp_set_factor_probs_device": [_vp, _vp, _vp],
        "flbp_update_seq": [P(GraphDesc), C.c_int32, _vp, _i64p],
        "flbp_shuffled_factors": [C.c_int64, C.c_uint32, _i32p],
        "flbp_seq_batches": [P(GraphDesc), _i64p, C.c_int64, _vp, P(C.c_int64)],
        "flbp_set_update_seq": [_vp, _vp, C.c_int64],
        "flbp_update_info": [_vp, P(C.c_int32), P(C.c_int64)],
        "flbp_set_seq_kernel": [_vp, C.c_int32],
        "flbp_set_tuning": [_vp, P(Tuning)],
        "flbp_get_tuning": [_vp, P(Tuning)],
        "flbp_autotune": [_vp, C.c_int32, C.c_int64, C.c_double, C.c_int32, P(Tuning)],
        "flbp_set_layout_builder": [C.c_int32],
        "flbp_engine_layout_digest": [_vp, P(C.c_uint64), P(C.c_int32)],
        "flbp_sets_create": [P(GraphDesc), C.c_int64, _i64p, _vp, _vp, P(EngineOpts), P(_vp)],
        "flbp_sets_run_tol": [_vp, C.c_double, C.c_int64, C.c_double, _i64p, _i32p, P(RunInfo)],
        "flbp_sets_info": [_vp, P(C.c_int64), P(C.c_int64)],
        "flbp_reset_counts": [_vp],
    }
    for name, args in sig.items():
        f = getattr(L, name)
        f.argtypes = args
        f.restype = C.c_int
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != FLBP_OK:
        raise FlbpError(rc, lib().flbp_last_error().decode())


def last_error() -> str:
    return lib().flbp_last_error().decode()


EXPORTED = ["flbp_last_error", "flbp_version", "flbp_engine_create", "flbp_engine_destroy", "flbp_init",
            "flbp_run_tol", "flbp_run_fixed", "flbp_run_lowpass", "flbp_sweep", "flbp_get_beliefs",
            "flbp_get_lowpass", "flbp_compute_beliefs", "flbp_get_fv_messages", "flbp_get_vf_messages",
            "flbp_engine_stats", "flbp_last_run_ms", "flbp_set_kernel_timing", "flbp_kernel_times", "flbp_fg_read_file", "flbp_fg_read_string",
            "flbp_fg_from_factors", "flbp_fg_destroy", "flbp_fg_clamp", "flbp_fg_rebuild", "flbp_fg_sizes",
            "flbp_fg_var_labels", "flbp_fg_factors", "flbp_fg_neighbors", "flbp_fg_construct",
            "flbp_engine_create_from_fg", "flbp_run_fixed_device_noalloc", "flbp_batch_create", "flbp_batch_info",
            "flbp_batch_run_tol", "flbp_adjoint_forward", "flbp_adjoint_backward", "flbp_set_factor_probs", "flbp_set_factor_probs_device",
            "flbp_adjoint_backward_device", "flbp_get_beliefs_device", "flbp_clamp_vars", "flbp_layout_digest",
            "flbp_update_seq", "flbp_shuffled_factors", "flbp_seq_batches", "flbp_set_update_seq", "flbp_update_info",
            "flbp_set_seq_kernel", "flbp_set_tuning", "flbp_get_tuning", "flbp_autotune", "flbp_set_layout_builder",
            "flbp_engine_layout_digest", "flbp_sets_create", "flbp_sets_run_tol", "flbp_sets_info", "flbp_reset_counts"]
