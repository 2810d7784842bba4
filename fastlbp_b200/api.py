"""Python mirror of the drop-in API, over the C ABI.

Names and argument meanings follow FastLBP's C++ classes
(include/ext/causal_fg.h, include/ext/causal_bp.h, include/lbp/properties.h):
``CausalFactorGraph.ReadFromFile / clamp / nrVars ...``, ``CausalBP(fg, opts)``,
``init()``, the three ``run`` forms, ``newBelief`` and ``belief``. Errors raise
``FlbpError`` instead of exiting the process.
"""

from __future__ import annotations

import ctypes as C
from typing import Dict, Optional, Sequence, Tuple

import numpy as np

from . import _native as N
from ._native import check, lib

_CLEANUP = {}


class PropertySet(dict):
    """String-keyed parameters (include/lbp/properties.h:21-59)."""

    def set(self, key, val):
        self[key] = val
        return self

    def hasKey(self, key):  # noqa: N802 (reference name)
        return key in self

    def getStringAs(self, typ, key):  # noqa: N802
        v = self[key]
        if isinstance(v, typ) and not (typ is int and isinstance(v, bool)):
            return v
        print("get properties error")
        return typ()


class CausalFactorGraph:
    """A causal factor graph held by the library (include/ext/causal_fg.h)."""

    def __init__(self, handle=None):
        self._h = handle

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                lib().flbp_fg_destroy(h)
            except Exception:
                pass
            self._h = None

    # construction ---------------------------------------------------------
    @classmethod
    def read_file(cls, path: str) -> "CausalFactorGraph":
        h = C.c_void_p()
        check(lib().flbp_fg_read_file(path.encode(), C.byref(h)))
        return cls(h)

    def ReadFromFile(self, path: str) -> None:  # noqa: N802
        other = CausalFactorGraph.read_file(path)
        self._h, other._h = other._h, None

    @classmethod
    def from_text(cls, text: str) -> "CausalFactorGraph":
        h = C.c_void_p()
        check(lib().flbp_fg_read_string(text.encode(), C.byref(h)))
        return cls(h)

    @classmethod
    def from_factors(cls, fl) -> "CausalFactorGraph":
        """From a ``workloads.FactorList`` (CausalFactorGraph(std::vector<CausalFactor>))."""
        h = C.c_void_p()
        check(lib().flbp_fg_from_factors(
            fl.n, np.ascontiguousarray(fl.kind, np.int32), np.ascontiguousarray(fl.head, np.int64),
            np.ascontiguousarray(fl.body_off, np.int64), np.ascontiguousarray(fl.body, np.int64),
            np.ascontiguousarray(fl.p, np.float64), np.ascontiguousarray(fl.q, np.float64), C.byref(h)))
        return cls(h)

    def rebuild(self) -> "CausalFactorGraph":
        """CausalFactorGraph(fg.factors()): the topology after clamps (fl_wrapper.cu:45)."""
        h = C.c_void_p()
        check(lib().flbp_fg_rebuild(self._h, C.byref(h)))
        return CausalFactorGraph(h)

    # queries --------------------------------------------------------------
    def _sizes(self):
        c = np.zeros(4, np.int64)
        check(lib().flbp_fg_sizes(self._h, c))
        return c

    def nrVars(self):  # noqa: N802
        return int(self._sizes()[0])

    def nrFactors(self):  # noqa: N802
        return int(self._sizes()[1])

    def nrEdges(self):  # noqa: N802
        return int(self._sizes()[2])

    def nrSlots(self):  # noqa: N802
        return int(self._sizes()[3])

    def var_labels(self) -> np.ndarray:
        out = np.zeros(self.nrVars(), np.int64)
        check(lib().flbp_fg_var_labels(self._h, out, out.size))
        return out

    def findVar(self, label: int) -> int:  # noqa: N802
        labels = self.var_labels()
        i = int(np.searchsorted(labels, label))
        return i if i < labels.size and labels[i] == label else labels.size

    def factor_info(self) -> Dict[str, np.ndarray]:
        F, S = self.nrFactors(), self.nrSlots()
        d = dict(type=np.zeros(F, np.int32), head=np.zeros(F, np.int64), p=np.zeros(F), q=np.zeros(F),
                 clamped=np.zeros(F, np.int32), mask0=np.zeros(F), mask1=np.zeros(F),
                 vars_off=np.zeros(F + 1, np.int64), vars=np.zeros(S, np.int64))
        check(lib().flbp_fg_factors(self._h, d["type"], d["head"], d["p"], d["q"], d["clamped"], d["mask0"],
                                    d["mask1"], d["vars_off"], d["vars"]))
        d["nvars"] = np.diff(d["vars_off"])
        return d

    def neighbors(self, factor_side: bool):
        n = self.nrFactors() if factor_side else self.nrVars()
        E = self.nrEdges()
        off = np.zeros(n + 1, np.int64)
        node, it, du = (np.zeros(E, np.int64) for _ in range(3))
        check(lib().flbp_fg_neighbors(self._h, 1 if factor_side else 0, off, node, it, du))
        return off, node, it, du

    def construct(self) -> Dict[str, np.ndarray]:
        """Reference-order arrays of CausalBP::construct() (causal_bp.cu:310-407)."""
        F, V, S = self.nrFactors(), self.nrVars(), self.nrSlots()
        d = dict(factor_offsets=np.zeros(F + 1, np.int64), slot_var=np.zeros(S, np.int64),
                 factor_head=np.zeros(F, np.int64), row_ptr_fv=np.zeros(V + 1, np.int64),
                 col_ind_fv=np.zeros(S, np.int64))
        check(lib().flbp_fg_construct(self._h, d["factor_offsets"], d["slot_var"], d["factor_head"],
                                      d["row_ptr_fv"], d["col_ind_fv"]))
        return d

    def graph_arrays(self) -> Dict[str, np.ndarray]:
        """Everything flbp_engine_create() takes, as numpy arrays."""
        c = self.construct()
        f = self.factor_info()
        return dict(n_vars=self.nrVars(), factor_offsets=c["factor_offsets"], slot_var=c["slot_var"],
                    factor_head=c["factor_head"], factor_type=f["type"], factor_p=f["p"], factor_q=f["q"],
                    factor_head_clamped=f["clamped"], factor_mask0=f["mask0"], factor_mask1=f["mask1"])

    # evidence -------------------------------------------------------------
    def clamp(self, i: int, x: int) -> None:
        check(lib().flbp_fg_clamp(self._h, int(i), int(x)))

    def clamp_labels(self, clamps: Dict[int, int]) -> None:
        """fl_wrapper's loop: each (label, value) in ascending label order (fl_wrapper.cu:29-43)."""
        labels = self.var_labels()
        for lab in sorted(clamps):
            i = int(np.searchsorted(labels, lab))
            if i < labels.size and labels[i] == lab:
                self.clamp(i, clamps[lab])


def set_layout_builder(mode: str) -> None:
    """Where new engines build their layout: "auto" (GPU from 2^18 edge slots),
    "host" or "device" (flbp_set_layout_builder; process-wide)."""
    check(lib().flbp_set_layout_builder({"auto": 0, "host": 1, "device": 2}[mode]))


def layout_digest(arrays: Dict[str, np.ndarray], threads: int = 0, graph_of=None) -> int:
    """Digest of the device layout built for reference-order graph arrays
    (flbp_layout_digest; host only). graph_of: optional (factor_graph,
    var_graph, n_graphs) of a batch."""
    keep = []
    desc = _desc_from_arrays(arrays, keep)
    out = C.c_uint64()
    if graph_of is None:
        check(lib().flbp_layout_digest(C.byref(desc), None, None, 0, int(threads), C.byref(out)))
    else:
        fg = np.ascontiguousarray(graph_of[0], np.uint32)
        vg = np.ascontiguousarray(graph_of[1], np.uint32)
        check(lib().flbp_layout_digest(C.byref(desc), fg.ctypes.data_as(C.c_void_p), vg.ctypes.data_as(C.c_void_p),
                                       int(graph_of[2]), int(threads), C.byref(out)))
    return int(out.value)


UPDATES = {"PARALL": 0, "SEQFIX": 1, "TOPO": 2}


def update_seq(arrays: Dict[str, np.ndarray], updates: str = "SEQFIX", seed: int = 42,
               factor_order=None) -> np.ndarray:
    """The update sequence of a sequential schedule as factor-major slots
    (flbp_update_seq). SEQFIX takes the factors in `factor_order`, by default
    0..F-1 shuffled by std::mt19937(seed) as the reference's first CausalBP of
    a thread does (csrc/ext/causal_bp.cu:116, 186-201); TOPO ranks edges by a
    breadth-first order (:203-304)."""
    if updates not in ("SEQFIX", "TOPO"):
        raise ValueError("updates must be SEQFIX or TOPO")
    keep = []
    desc = _desc_from_arrays(arrays, keep)
    seq = np.zeros(max(1, desc.n_slots), np.int64)
    order = None
    if updates == "SEQFIX":
        if factor_order is None:
            order = np.zeros(max(1, desc.n_factors), np.int32)
            check(lib().flbp_shuffled_factors(int(desc.n_factors), int(seed) & 0xffffffff, order))
        else:
            order = np.ascontiguousarray(factor_order, np.int32)
            if order.size != desc.n_factors:
                raise ValueError("factor_order must list every factor once")
    check(lib().flbp_update_seq(C.byref(desc), UPDATES[updates],
                                None if order is None else order.ctypes.data_as(C.c_void_p), seq))
    return seq[:desc.n_slots]


def seq_batches(arrays: Dict[str, np.ndarray], seq) -> Tuple[np.ndarray, int]:
    """(batch of every factor-major slot, number of batches) of an update
    sequence (flbp_seq_batches; host only)."""
    keep = []
    desc = _desc_from_arrays(arrays, keep)
    sq = np.ascontiguousarray(seq, np.int64)
    out = np.zeros(max(1, desc.n_slots), np.int64)
    nb = C.c_int64()
    check(lib().flbp_seq_batches(C.byref(desc), sq, sq.size, out.ctypes.data_as(C.c_void_p), C.byref(nb)))
    return out[:desc.n_slots], int(nb.value)


def _check_device_tensor(t, n: int, name: str) -> None:
    import torch

    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()
            and t.numel() == n):
        raise ValueError("%s must be a contiguous float64 CUDA tensor of %d elements" % (name, n))


def _desc_from_arrays(a: Dict[str, np.ndarray], keep: list) -> N.GraphDesc:
    def ptr(name, dt):
        v = a.get(name)
        if v is None:
            return None
        arr = np.ascontiguousarray(v, dt)
        keep.append(arr)
        return arr.ctypes.data

    off = np.ascontiguousarray(a["factor_offsets"], np.int64)
    keep.append(off)
    d = N.GraphDesc()
    d.n_vars = int(a["n_vars"])
    d.n_factors = off.size - 1
    d.n_slots = int(off[-1]) if off.size else 0
    d.factor_offsets = off.ctypes.data
    d.slot_var = ptr("slot_var", np.int64)
    d.factor_head = ptr("factor_head", np.int64)
    d.factor_type = ptr("factor_type", np.int32)
    d.factor_p = ptr("factor_p", np.float64)
    d.factor_q = ptr("factor_q", np.float64)
    d.factor_head_clamped = ptr("factor_head_clamped", np.int32)
    d.factor_mask0 = ptr("factor_mask0", np.float64)
    d.factor_mask1 = ptr("factor_mask1", np.float64)
    return d


class Engine:
    """The C-ABI engine over reference-order graph arrays (flbp_engine_*)."""

    def __init__(self, arrays: Dict[str, np.ndarray], precision: int = 32, damping: float = 0.0,
                 stream: Optional[int] = None, device: int = -1, updates: str = "PARALL", seed: int = 42):
        """updates: "PARALL" (default), or "SEQFIX" / "TOPO" to run the
        reference's sequential schedule (update_seq(arrays, updates, seed))."""
        if updates not in UPDATES:
            raise ValueError("updates must be one of PARALL, SEQFIX, TOPO")
        keep = []
        desc = _desc_from_arrays(arrays, keep)
        opts = N.EngineOpts(int(precision), int(device), float(damping), stream)
        h = C.c_void_p()
        check(lib().flbp_engine_create(C.byref(desc), C.byref(opts), C.byref(h)))
        self._h = h
        self.n_vars = int(desc.n_vars)
        self.n_slots = int(desc.n_slots)
        self.n_factors = int(desc.n_factors)
        self.info = None
        if updates != "PARALL":
            self.set_update_seq(update_seq(arrays, updates, seed))

    def set_update_seq(self, seq) -> None:
        """Run the sweeps in the conflict-free batches of an update sequence
        (None: PARALL again); messages return to the init() state."""
        if seq is None:
            check(lib().flbp_set_update_seq(self._h, None, 0))
            return
        sq = np.ascontiguousarray(seq, np.int64)
        check(lib().flbp_set_update_seq(self._h, sq.ctypes.data_as(C.c_void_p), sq.size))

    def set_seq_kernel(self, kind: int) -> None:
        """Sequential sweeps: 0 choose, 1 two launches per batch, 2 one cluster
        per sweep, 3 as 1 with programmatic dependent launch
        (flbp_set_seq_kernel)."""
        check(lib().flbp_set_seq_kernel(self._h, int(kind)))

    def update_info(self) -> Tuple[bool, int]:
        """(runs a sequential schedule, batches per sweep)."""
        a, b = C.c_int32(), C.c_int64()
        check(lib().flbp_update_info(self._h, C.byref(a), C.byref(b)))
        return bool(a.value), int(b.value)

    @classmethod
    def from_graph(cls, fg: CausalFactorGraph, **kw) -> "Engine":
        return cls(fg.graph_arrays(), **kw)

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            lib().flbp_engine_destroy(h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except (AttributeError, TypeError, ImportError):  # interpreter shutdown: modules already torn down
            pass

    def init(self):
        check(lib().flbp_init(self._h))

    def reset_counts(self):
        """Sweep count and beliefs back to a new engine's (flbp_reset_counts):
        init() + run_tol then gives what a newly built engine gives."""
        check(lib().flbp_reset_counts(self._h))

    def sweep(self, n: int = 1):
        check(lib().flbp_sweep(self._h, int(n)))

    def _info(self):
        self.info = N.RunInfo()
        return C.byref(self.info)

    def run_tol(self, tol=1e-9, maxiter=10000, maxtime=10.0):
        check(lib().flbp_run_tol(self._h, float(tol), int(maxiter), float(maxtime), self._info()))
        return self.info.as_dict()

    def run_fixed(self, sweeps: int):
        check(lib().flbp_run_fixed(self._h, int(sweeps), self._info()))
        return self.info.as_dict()

    def run_lowpass(self, tol, min_iters, max_iters, hist, maxtime=1e9):
        check(lib().flbp_run_lowpass(self._h, float(tol), int(min_iters), int(max_iters), int(hist),
                                     float(maxtime), self._info()))
        return self.info.as_dict()

    def beliefs(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        """Beliefs P(x_i = 1) of the last run, in variable order; into `out`
        (a C-contiguous float64 array of n_vars elements, e.g. one buffer
        reused over many solves) when given."""
        if out is None:
            out = np.empty(self.n_vars)
        elif not (isinstance(out, np.ndarray) and out.dtype == np.float64 and out.flags.c_contiguous
                  and out.size == self.n_vars):
            raise FlbpError("out must be a C-contiguous float64 array of n_vars elements")
        check(lib().flbp_get_beliefs(self._h, out, out.size))
        return out

    def lowpass(self) -> np.ndarray:
        out = np.zeros(self.n_vars)
        check(lib().flbp_get_lowpass(self._h, out, out.size))
        return out

    def compute_beliefs(self) -> np.ndarray:
        out = np.zeros(self.n_vars)
        check(lib().flbp_compute_beliefs(self._h, out, out.size))
        return out

    def fv_messages(self):
        m0, m1 = np.zeros(self.n_slots), np.zeros(self.n_slots)
        check(lib().flbp_get_fv_messages(self._h, m0, m1, self.n_slots))
        return m0, m1

    def vf_messages(self):
        m0, m1 = np.zeros(self.n_slots), np.zeros(self.n_slots)
        check(lib().flbp_get_vf_messages(self._h, m0, m1, self.n_slots))
        return m0, m1

    def stats(self) -> Dict[str, int]:
        c = np.zeros(20, np.int64)
        check(lib().flbp_engine_stats(self._h, c, c.size))
        keys = ["vars", "factors", "slots", "active_factors", "active_slots", "warp_factors", "warp_vars", "bytes",
                "h2d_bytes", "launches", "huge_factors", "huge_vars", "big_factor_tiles", "big_var_tiles",
                "create_us_layout", "create_us_alloc", "create_us_upload", "create_us_rest", "factor_tiles",
                "var_tiles"]
        return dict(zip(keys, (int(x) for x in c)))

    # gradients through unrolled sweeps --------------------------------------
    def adjoint_forward(self, sweeps: int, every: int, fetch: bool = True) -> Optional[np.ndarray]:
        """init() and `sweeps` sweeps with checkpoints every `every`; the
        beliefs (None with fetch=False: they stay on the device, see
        beliefs_device)."""
        out = np.zeros(self.n_vars) if fetch else None
        check(lib().flbp_adjoint_forward(self._h, int(sweeps), int(every), out, self.n_vars))
        return out

    def beliefs_device(self, out) -> None:
        """Beliefs of the last run into `out`, a contiguous float64 CUDA tensor
        of n_vars elements on the engine's device."""
        _check_device_tensor(out, self.n_vars, "out")
        check(lib().flbp_get_beliefs_device(self._h, C.c_void_p(out.data_ptr()), self.n_vars))

    def adjoint_backward_device(self, grad_beliefs, grad_p, grad_q=None) -> None:
        """adjoint_backward on contiguous float64 CUDA tensors (grad_q may be
        None). Waits for the current torch stream before reading grad_beliefs."""
        import torch

        _check_device_tensor(grad_beliefs, self.n_vars, "grad_beliefs")
        _check_device_tensor(grad_p, self.n_factors, "grad_p")
        if grad_q is not None:
            _check_device_tensor(grad_q, self.n_factors, "grad_q")
        torch.cuda.current_stream(grad_beliefs.device).synchronize()
        check(lib().flbp_adjoint_backward_device(self._h, C.c_void_p(grad_beliefs.data_ptr()),
                                                 C.c_void_p(grad_p.data_ptr()),
                                                 None if grad_q is None else C.c_void_p(grad_q.data_ptr())))

    def adjoint_backward(self, grad_beliefs: np.ndarray, want_q: bool = True):
        """dL/dp and dL/dq of every factor (reference order) for dL/dbeliefs
        (dL/dq None, and not accumulated, with want_q=False)."""
        g = np.ascontiguousarray(grad_beliefs, np.float64)
        gp = np.zeros(self.n_factors)
        gq = np.zeros(self.n_factors) if want_q else None
        check(lib().flbp_adjoint_backward(self._h, g, gp, gq))
        return gp, gq

    def clamp(self, variables, values) -> None:
        """Clamp variables (graph order) to 0/1 in place (flbp_clamp_vars): the
        same solution as clamping the factor graph and building a new engine,
        without the rebuild; takes effect from the next init()/run."""
        v = np.ascontiguousarray(np.atleast_1d(variables), np.int64)
        x = np.ascontiguousarray(np.atleast_1d(values), np.int32)
        if v.shape != x.shape:
            raise ValueError("one value per clamped variable")
        check(lib().flbp_clamp_vars(self._h, v.size, v, x))

    def set_factor_probs(self, p: np.ndarray, q: np.ndarray) -> None:
        check(lib().flbp_set_factor_probs(self._h, np.ascontiguousarray(p, np.float64),
                                          np.ascontiguousarray(q, np.float64)))

    def set_factor_probs_device(self, p, q) -> None:
        """p, q: float64 CUDA tensors (reference factor order) that stay on the
        device (flbp_set_factor_probs_device); the caller's stream must have
        finished writing them."""
        for t in (p, q):
            if not (t.is_cuda and t.dtype.is_floating_point and t.element_size() == 8 and t.is_contiguous()
                    and t.numel() == self.n_factors):
                raise ValueError("p and q must be contiguous float64 CUDA tensors of n_factors values")
        check(lib().flbp_set_factor_probs_device(self._h, C.c_void_p(p.data_ptr()), C.c_void_p(q.data_ptr())))

    def set_kernel_timing(self, enable: bool) -> None:
        check(lib().flbp_set_kernel_timing(self._h, 1 if enable else 0))

    def kernel_times(self):
        """(factor-pass ms, variable-pass ms, factor launches, variable launches) in timing mode."""
        ms, n = np.zeros(2), np.zeros(2, np.int64)
        check(lib().flbp_kernel_times(self._h, ms, n))
        return float(ms[0]), float(ms[1]), int(n[0]), int(n[1])

    def set_tuning(self, factor_form: int, var_form: int) -> None:
        """Form of each sweep pass: 0 staged, 1 or 2 direct (flbp_set_tuning)."""
        t = N.Tuning(int(factor_form), int(var_form), 0, 0)
        check(lib().flbp_set_tuning(self._h, C.byref(t)))

    def autotune(self, sweeps: int = 200, tol: Optional[float] = None, reps: int = 3) -> Dict[str, int]:
        """Time the pass forms on this graph and keep the fastest (flbp_autotune):
        whole fixed-sweep runs, or whole tolerance runs when tol is given."""
        t = N.Tuning()
        check(lib().flbp_autotune(self._h, 0 if tol is None else 1, int(sweeps), float(tol or 0.0), int(reps),
                                  C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def autotune_batch(self, tol: float = 1e-6, maxiter: int = 500, reps: int = 2) -> Dict[str, int]:
        """autotune over whole batched tolerance runs (flbp_batch_run_tol)."""
        return self.autotune(maxiter, tol=tol, reps=reps)

    def layout_digest(self) -> Tuple[int, bool]:
        """(digest of the engine's device layout, built on the GPU) - flbp_engine_layout_digest."""
        d, on_dev = C.c_uint64(), C.c_int32()
        check(lib().flbp_engine_layout_digest(self._h, C.byref(d), C.byref(on_dev)))
        return int(d.value), bool(on_dev.value)

    def tuning(self) -> Dict[str, int]:
        t = N.Tuning()
        check(lib().flbp_get_tuning(self._h, C.byref(t)))
        return {k: getattr(t, k) for k, _ in t._fields_}

    def last_run_ms(self) -> float:
        v = C.c_double()
        check(lib().flbp_last_run_ms(self._h, C.byref(v)))
        return v.value


class BatchEngine(Engine):
    """Many independent graphs in one engine (flbp_batch_*): one sweep is one
    pass over all of them; each graph stops on its own tolerance rule and is
    frozen from then on. beliefs() covers all graphs in order;
    beliefs_of(g) is graph g's part."""

    def __init__(self, graphs: Sequence[Dict[str, np.ndarray]], precision: int = 32, damping: float = 0.0,
                 stream: Optional[int] = None, device: int = -1):
        keep = []
        descs = (N.GraphDesc * len(graphs))()
        for i, a in enumerate(graphs):
            descs[i] = _desc_from_arrays(a, keep)
        opts = N.EngineOpts(int(precision), int(device), float(damping), stream)
        h = C.c_void_p()
        check(lib().flbp_batch_create(descs, len(graphs), C.byref(opts), C.byref(h)))
        self._h = h
        self.n_graphs = len(graphs)
        self.var_off = np.zeros(self.n_graphs + 1, np.int64)
        ng = C.c_int64()
        check(lib().flbp_batch_info(h, C.byref(ng), self.var_off))
        self.n_vars = int(self.var_off[-1])
        self.n_slots = int(sum(int(d.n_slots) for d in descs))
        self.n_factors = int(sum(int(d.n_factors) for d in descs))
        self.info = None

    def run_batch_tol(self, tol=1e-6, maxiter=500, maxtime=1e9):
        """Per-graph sweeps and stop reasons (0 converged, 2 iteration/time limit)."""
        sweeps = np.zeros(self.n_graphs, np.int64)
        reasons = np.zeros(self.n_graphs, np.int32)
        check(lib().flbp_batch_run_tol(self._h, float(tol), int(maxiter), float(maxtime), sweeps, reasons,
                                       self._info()))
        return sweeps, reasons

    def beliefs_of(self, g: int, all_beliefs: Optional[np.ndarray] = None) -> np.ndarray:
        b = self.beliefs() if all_beliefs is None else all_beliefs
        return b[self.var_off[g]:self.var_off[g + 1]]


class SetsEngine(Engine):
    """Evidence sets on one graph (flbp_sets_*): the graph's layout once, per
    set its own clamps, messages and beliefs; every set stops on its own
    tolerance rule. beliefs() holds n_sets x n_vars values (set k in row k)."""

    def __init__(self, arrays: Dict[str, np.ndarray], sets: Sequence[Dict[int, int]], precision: int = 32,
                 damping: float = 0.0, stream: Optional[int] = None, device: int = -1):
        """sets: one {graph variable index: 0/1} clamp map per evidence set."""
        keep = []
        desc = _desc_from_arrays(arrays, keep)
        off = np.zeros(len(sets) + 1, np.int64)
        vs, vl = [], []
        for k, cl in enumerate(sets):
            for v, x in sorted(cl.items()):
                vs.append(int(v))
                vl.append(int(x))
            off[k + 1] = len(vs)
        vs_a, vl_a = np.array(vs, np.int64), np.array(vl, np.int32)
        opts = N.EngineOpts(int(precision), int(device), float(damping), stream)
        h = C.c_void_p()
        check(lib().flbp_sets_create(C.byref(desc), len(sets), off, vs_a.ctypes.data_as(C.c_void_p),
                                     vl_a.ctypes.data_as(C.c_void_p), C.byref(opts), C.byref(h)))
        self._h = h
        self.n_sets = len(sets)
        self.n_vars = int(desc.n_vars)
        self.n_slots = int(desc.n_slots)
        self.n_factors = int(desc.n_factors)
        self.info = None

    def run_sets_tol(self, tol=1e-6, maxiter=500, maxtime=1e9):
        """Per-set sweeps and stop reasons (0 converged, 2 iteration/time limit)."""
        sweeps = np.zeros(self.n_sets, np.int64)
        reasons = np.zeros(self.n_sets, np.int32)
        check(lib().flbp_sets_run_tol(self._h, float(tol), int(maxiter), float(maxtime), sweeps, reasons,
                                      self._info()))
        return sweeps, reasons

    def beliefs(self) -> np.ndarray:
        out = np.zeros(self.n_sets * self.n_vars)
        check(lib().flbp_get_beliefs(self._h, out, out.size))
        return out.reshape(self.n_sets, self.n_vars)


class CausalBP:
    """CausalBP(fg, opts) with the reference's run semantics (include/ext/causal_bp.h:167-193)."""

    def __init__(self, fg: CausalFactorGraph, opts: PropertySet):
        self.fg = fg
        get = lambda k, d: opts[k] if k in opts else d
        self.tol = float(get("tol", 1e-9))
        self.maxiter = int(get("maxiter", 10000))
        self.maxtime = float(get("maxtime", 10.0))
        self.updates = str(get("updates", "SEQFIX"))
        if self.updates not in UPDATES:
            self.updates = "SEQFIX"  # unknown names fall back to SEQFIX (csrc/ext/causal_bp.cu:173-178)
        prec = str(get("precision", "FP32")).upper()
        # SEQFIX shuffles the factors with std::mt19937("seed", 42 by default): the
        # order of the reference's first CausalBP of a thread
        self.engine = Engine.from_graph(fg, precision=64 if prec == "FP64" else 32,
                                        damping=float(get("damping", 0.0)), updates=self.updates,
                                        seed=int(get("seed", 42)))
        self._beliefs = np.zeros(self.engine.n_vars)
        self._lowpass = None
        self._iters = 0

    def init(self):
        self.engine.init()

    def run(self, *args):
        if len(args) == 0:  # run(): tolerance loop with the properties
            info = self.engine.run_tol(self.tol, self.maxiter, self.maxtime)
            self._beliefs = self.engine.beliefs()
            self._lowpass = self._beliefs.copy()
            self._iters = info["total_sweeps"]
            return None
        if len(args) == 3:  # run(tol, maxIters, histLength)
            info = self.engine.run_fixed(int(args[1]))
            self._beliefs = self.engine.beliefs()
            self._lowpass = self.engine.lowpass()
            self._iters = info["total_sweeps"]
            return 1.0
        if len(args) == 4:  # run(tol, minIters, maxIters, histLength)
            info = self.engine.run_lowpass(args[0], args[1], args[2], args[3], self.maxtime)
            self._beliefs = self.engine.beliefs()
            self._lowpass = self.engine.lowpass()
            self._iters = info["total_sweeps"]
            return info["frac"]
        raise TypeError("run() takes 0, 3 or 4 arguments")

    def newBelief(self, i: int) -> float:  # noqa: N802
        return float(self._lowpass[i])

    def belief(self, i: int):
        b = float(self._beliefs[i])
        return (1.0 - b, b)

    def beliefs(self) -> np.ndarray:
        return self._beliefs.copy()

    def lowpass_beliefs(self) -> np.ndarray:
        return None if self._lowpass is None else self._lowpass.copy()

    @property
    def iterations(self) -> int:
        return self._iters
