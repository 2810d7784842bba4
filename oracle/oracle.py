"""ctypes front-end of the FP64 oracle (liboracle.so) and of the reference's
own graph model (_ref/libref_graph.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
the CPU-baseline leg of bench.py, always as the checker. The product package
(fastlbp_b200) never imports this module.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_GRAPH_PATH = os.path.join(HERE, "_ref", "libref_graph.so")
REF_BP_PATH = os.path.join(HERE, "_ref", "ref_bp")

_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_vp = C.c_void_p


def build(ref: bool = True) -> None:
    """Compile the oracle (and, when the reference sources are present, _ref)."""
    subprocess.run(["make", "-C", HERE, "oracle"] + (["ref"] if ref else []), check=True,
                   stdout=subprocess.DEVNULL)


_lib = None
_ref = None


def _graph_api(lib, pre):
    f = lambda n: getattr(lib, pre + n)
    f("free").argtypes = [_vp]
    f("clamp").argtypes = [_vp, C.c_int64, C.c_int64]
    f("rebuild").argtypes = [_vp]
    f("rebuild").restype = _vp
    for n in ("nr_vars", "nr_factors", "nr_edges"):
        f(n).argtypes = [_vp]
        f(n).restype = C.c_int64
    f("vars").argtypes = [_vp, _i64p]
    f("factor_info").argtypes = [_vp, _i32p, _i64p, _f64p, _f64p, _i32p, _f64p, _f64p, _i64p]
    f("factor_vars").argtypes = [_vp, _i64p, _i64p]
    f("neighbors").argtypes = [_vp, C.c_int, _i64p, _i64p, _i64p, _i64p]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(ref=False)
        L = C.CDLL(LIB_PATH)
        _graph_api(L, "orc_")
        L.orc_last_error.restype = C.c_char_p
        L.orc_read_file.argtypes = [C.c_char_p]
        L.orc_read_file.restype = _vp
        L.orc_read_string.argtypes = [C.c_char_p]
        L.orc_read_string.restype = _vp
        L.orc_from_factors.argtypes = [C.c_int64, _i32p, _i64p, _i64p, _i64p, _f64p, _f64p]
        L.orc_from_factors.restype = _vp
        L.orc_clamp.restype = C.c_int
        L.orc_nr_slots.argtypes = [_vp]
        L.orc_nr_slots.restype = C.c_int64
        L.orc_construct.argtypes = [_vp, _i64p, _i64p, _i64p, _i64p, _i64p, _i64p, _f64p, _i64p]
        L.orc_bp_create.argtypes = [_vp, C.c_double, C.c_int, C.c_int]
        L.orc_bp_create.restype = _vp
        for n in ("orc_bp_free", "orc_bp_init", "orc_bp_sweep"):
            getattr(L, n).argtypes = [_vp]
        for n in ("orc_bp_nr_vars", "orc_bp_nr_slots", "orc_bp_iters"):
            getattr(L, n).argtypes = [_vp]
            getattr(L, n).restype = C.c_int64
        L.orc_bp_set_threads.argtypes = [_vp, C.c_int]
        L.orc_bp_run_tol.argtypes = [_vp, C.c_double, C.c_int64, C.c_double]
        L.orc_bp_run_tol.restype = C.c_double
        L.orc_bp_run_fixed.argtypes = [_vp, C.c_double, C.c_int64, C.c_int64]
        L.orc_bp_run_fixed.restype = C.c_double
        L.orc_bp_run_lowpass.argtypes = [_vp, C.c_double, C.c_int64, C.c_int64, C.c_int64, C.c_double,
                                         C.POINTER(C.c_int32), C.POINTER(C.c_int64)]
        L.orc_bp_run_lowpass.restype = C.c_double
        L.orc_bp_beliefs.argtypes = [_vp, _f64p]
        L.orc_bp_lowpass.argtypes = [_vp, _f64p]
        L.orc_bp_lowpass.restype = C.c_int
        L.orc_bp_current_beliefs.argtypes = [_vp, _f64p]
        L.orc_bp_messages.argtypes = [_vp, _f64p, _f64p, _f64p, _f64p]
        L.orc_bp_set_vf.argtypes = [_vp, _f64p, _f64p]
        L.orc_bp_set_schedule.argtypes = [_vp, C.c_int, C.c_uint32]
        L.orc_bp_set_schedule.restype = C.c_int64
        L.orc_bp_schedule.argtypes = [_vp, _i64p, _i64p]
        L.orc_bp_set_mode.argtypes = [_vp, C.c_int]
        L.orc_bp_set_mode.restype = C.c_int
        L.orc_bp_underflow.argtypes = [_vp, np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")]
        L.orc_bp_underflow.restype = C.c_int64
        _lib = L
    return _lib


def ref_lib():
    """The reference's own graph model, or None when it was not built here."""
    global _ref
    if _ref is None and os.path.exists(REF_GRAPH_PATH):
        L = C.CDLL(REF_GRAPH_PATH)
        _graph_api(L, "ref_")
        L.ref_read_file.argtypes = [C.c_char_p]
        L.ref_read_file.restype = _vp
        _ref = L
    return _ref


class _GraphBase:
    _pre = "orc_"

    def __init__(self, handle, L):
        if not handle:
            raise RuntimeError("graph construction failed: %s" % _lib.orc_last_error().decode())
        self.h = handle
        self.L = L

    def _f(self, n):
        return getattr(self.L, self._pre + n)

    def __del__(self):
        if getattr(self, "h", None):
            self._f("free")(self.h)
            self.h = None

    def nr_vars(self):
        return int(self._f("nr_vars")(self.h))

    def nr_factors(self):
        return int(self._f("nr_factors")(self.h))

    def nr_edges(self):
        return int(self._f("nr_edges")(self.h))

    def clamp(self, i, x):
        self._f("clamp")(self.h, int(i), int(x))

    def rebuild(self):
        return type(self)(self._f("rebuild")(self.h), self.L)

    def var_labels(self):
        out = np.zeros(self.nr_vars(), np.int64)
        self._f("vars")(self.h, out)
        return out

    def factor_info(self) -> Dict[str, np.ndarray]:
        F = self.nr_factors()
        d = dict(type=np.zeros(F, np.int32), head=np.zeros(F, np.int64), p=np.zeros(F), q=np.zeros(F),
                 clamped=np.zeros(F, np.int32), mask0=np.zeros(F), mask1=np.zeros(F),
                 nvars=np.zeros(F, np.int64))
        self._f("factor_info")(self.h, d["type"], d["head"], d["p"], d["q"], d["clamped"], d["mask0"],
                               d["mask1"], d["nvars"])
        off = np.zeros(F + 1, np.int64)
        labels = np.zeros(int(d["nvars"].sum()), np.int64)
        self._f("factor_vars")(self.h, off, labels)
        d["vars_off"], d["vars"] = off, labels
        return d

    def neighbors(self, factor_side: bool):
        n = self.nr_factors() if factor_side else self.nr_vars()
        E = self.nr_edges()
        off = np.zeros(n + 1, np.int64)
        node, it, du = (np.zeros(E, np.int64) for _ in range(3))
        self._f("neighbors")(self.h, 1 if factor_side else 0, off, node, it, du)
        return off, node, it, du

    def clamp_labels(self, clamps: Dict[int, int]):
        """fl_wrapper's clamp loop: for each (label, value) in ascending label
        order, clamp every variable with that label (examples/fl_wrapper.cu:29-43)."""
        labels = self.var_labels()
        pos = {int(l): i for i, l in enumerate(labels)}
        for lab in sorted(clamps):
            if lab in pos:
                self.clamp(pos[lab], clamps[lab])


class OracleGraph(_GraphBase):
    _pre = "orc_"

    @classmethod
    def from_file(cls, path):
        L = lib()
        return cls(L.orc_read_file(path.encode()), L)

    @classmethod
    def from_text(cls, text):
        L = lib()
        return cls(L.orc_read_string(text.encode()), L)

    @classmethod
    def from_factors(cls, fl):
        L = lib()
        return cls(L.orc_from_factors(fl.n, np.ascontiguousarray(fl.kind, np.int32),
                                      np.ascontiguousarray(fl.head, np.int64),
                                      np.ascontiguousarray(fl.body_off, np.int64),
                                      np.ascontiguousarray(fl.body, np.int64),
                                      np.ascontiguousarray(fl.p, np.float64),
                                      np.ascontiguousarray(fl.q, np.float64)), L)

    def nr_slots(self):
        return int(self.L.orc_nr_slots(self.h))

    def construct(self) -> Dict[str, np.ndarray]:
        F, V, E = self.nr_factors(), self.nr_vars(), self.nr_slots()
        d = dict(row_ptr_vf=np.zeros(F + 1, np.int64), col_ind_vf=np.zeros(E, np.int64),
                 row_ptr_fv=np.zeros(V + 1, np.int64), col_ind_fv=np.zeros(E, np.int64),
                 head=np.zeros(F, np.int64), rec_i=np.zeros(6 * E, np.int64), rec_r=np.zeros(4 * E),
                 vf_i=np.zeros(3 * E, np.int64))
        self.L.orc_construct(self.h, d["row_ptr_vf"], d["col_ind_vf"], d["row_ptr_fv"], d["col_ind_fv"],
                             d["head"], d["rec_i"], d["rec_r"], d["vf_i"])
        d["rec_i"] = d["rec_i"].reshape(E, 6)
        d["rec_r"] = d["rec_r"].reshape(E, 4)
        d["vf_i"] = d["vf_i"].reshape(E, 3)
        return d


class RefGraph(_GraphBase):
    """The reference's own CausalFactorGraph (compiled from its sources)."""
    _pre = "ref_"

    @classmethod
    def from_file(cls, path):
        L = ref_lib()
        if L is None:
            raise RuntimeError("reference graph tool not built")
        return cls(L.ref_read_file(path.encode()), L)


class OracleBP:
    """FP64 CausalBP restatement over an OracleGraph: updates=PARALL, or after
    set_schedule() the sequential SEQFIX / TOPO schedules.

    arith: "reference" (the reference's probability-space arithmetic, which
    underflows to exact zeros beyond log-odds of about +-745), "lodds" (the
    same PARALL recurrence in FP64 log-odds: no underflow) or "track" (the
    reference's arithmetic, marking every belief that depends on an
    underflow; see underflow()). `logdomain` is the reference's own property
    of that name (messages initialised to (0, 0))."""

    ARITH = {"reference": 0, "lodds": 1, "track": 2}

    def __init__(self, g: OracleGraph, damping: float = 0.0, threads: int = 1, logdomain: bool = False,
                 arith: str = "reference"):
        self.L = lib()
        self.h = self.L.orc_bp_create(g.h, float(damping), int(threads), 1 if logdomain else 0)
        self.V = int(self.L.orc_bp_nr_vars(self.h))
        self.E = int(self.L.orc_bp_nr_slots(self.h))
        if self.L.orc_bp_set_mode(self.h, self.ARITH[arith]) != 0:
            raise ValueError("unknown arithmetic mode " + arith)
        self.arith = arith

    def underflow(self):
        """(per-variable flags: the belief depends on an underflow, number of
        underflow events since init()) of a "track" run."""
        t = np.zeros(self.V, np.uint8)
        n = int(self.L.orc_bp_underflow(self.h, t))
        if n < 0:
            raise RuntimeError("underflow tracking needs arith='track'")
        return t.astype(bool), n

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_bp_free(self.h)
            self.h = None

    def set_threads(self, n):
        self.L.orc_bp_set_threads(self.h, int(n))

    def init(self):
        self.L.orc_bp_init(self.h)

    def sweep(self):
        self.L.orc_bp_sweep(self.h)

    @property
    def iters(self):
        return int(self.L.orc_bp_iters(self.h))

    def run(self, tol=1e-9, maxiter=10000, maxtime=10.0):
        return self.L.orc_bp_run_tol(self.h, tol, maxiter, maxtime)

    def run_fixed(self, tol, max_iters, hist=1):
        return self.L.orc_bp_run_fixed(self.h, tol, max_iters, hist)

    def run_lowpass(self, tol, min_iters, max_iters, hist, maxtime=1e9):
        r, s = C.c_int32(), C.c_int64()
        frac = self.L.orc_bp_run_lowpass(self.h, tol, min_iters, max_iters, hist, maxtime, C.byref(r), C.byref(s))
        return frac, int(r.value), int(s.value)

    def beliefs(self):
        out = np.zeros(self.V)
        self.L.orc_bp_beliefs(self.h, out)
        return out

    def lowpass(self) -> Optional[np.ndarray]:
        out = np.zeros(self.V)
        return out if self.L.orc_bp_lowpass(self.h, out) == 0 else None

    def current_beliefs(self):
        out = np.zeros(self.V)
        self.L.orc_bp_current_beliefs(self.h, out)
        return out

    def messages(self):
        a = [np.zeros(self.E) for _ in range(4)]
        self.L.orc_bp_messages(self.h, *a)
        return a  # fv0, fv1 (variable-major), vf0, vf1 (factor-major)

    def set_schedule(self, updates: str, seed: int = 42) -> int:
        """Switch to updates="SEQFIX" (factor order shuffled by std::mt19937(seed),
        as the reference's first CausalBP of a thread) or "TOPO"; returns the
        number of batches."""
        kind = {"SEQFIX": 1, "TOPO": 2}[updates]
        n = int(self.L.orc_bp_set_schedule(self.h, kind, int(seed)))
        self.n_batches = n
        return n

    def schedule(self):
        """(update sequence as factor-major slots, batch of every slot)."""
        seq = np.zeros(self.E, np.int64)
        batch = np.zeros(self.E, np.int64)
        self.L.orc_bp_schedule(self.h, seq, batch)
        return seq, batch

    def set_vf(self, vf0, vf1):
        self.L.orc_bp_set_vf(self.h, np.ascontiguousarray(vf0, np.float64), np.ascontiguousarray(vf1, np.float64))
