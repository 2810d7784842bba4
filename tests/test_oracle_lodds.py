"""The oracle's log-odds mode: the reference's PARALL recurrence (the nine
factor / clamp / direction cases of csrc/kernel/causal_bp_parall.cu:94-398,
the zero-count rules of :20-92, damping, the run loops) with every product
taken as a sum of logs, so that nothing underflows.

* On every PARALL golden case (beliefs made by FastLBP's own code) it agrees
  with the reference within 1e-10, with the same sweep counts: those graphs'
  messages never leave the double range, and then the two arithmetics are
  the same function.
* On the fault-localisation shape (OR fan-in up to 4096, clamped test
  outcomes), the reference's probability products underflow from sweep 4
  on. The reference-arithmetic oracle with underflow tracking marks every
  belief that depends on an underflow; until the first underflow both modes
  agree to rounding, and afterwards every belief on which they differ is a
  marked one. That is what the engine's log-odds arithmetic is checked
  against on that shape.
"""

import os

import numpy as np
import pytest

import oracle as O
from fastlbp_b200 import workloads
from test_golden_reference import CASES, load_case

PARALL = [c for c in CASES if load_case(c)[0].get("updates", "PARALL") == "PARALL"]


def _run(rec, text, arith):
    g = O.OracleGraph.from_text(text)
    g.clamp_labels({int(k): int(v) for k, v in rec["clamps"].items()})
    g = g.rebuild()
    bp = O.OracleBP(g, arith=arith)
    bp.init()
    mode = rec["mode"]
    if mode[0] == "fixed":
        bp.run_fixed(1e-6, int(mode[1]), 1)
        b = bp.lowpass()
    elif mode[0] == "tol":
        bp.run(float(mode[1]), int(mode[2]), 57600.0)
        b = bp.beliefs()
    else:
        bp.run_lowpass(float(mode[1]), int(mode[2]), int(mode[3]), int(mode[4]))
        b = bp.lowpass()
    return g, bp, b


@pytest.mark.parametrize("name", PARALL)
def test_lodds_matches_reference_binary(name):
    rec, text = load_case(name)
    g, bp, b = _run(rec, text, "lodds")
    ref = np.array([float(rec["beliefs"][str(lab)]) for lab in g.var_labels()])
    assert np.array_equal(np.isnan(b), np.isnan(ref))
    ok = ~np.isnan(ref)
    assert np.max(np.abs(b[ok] - ref[ok])) <= 1e-10
    if rec["mode"][0] == "tol" and rec.get("ref_sweeps") is not None:
        assert bp.iters == rec["ref_sweeps"]


@pytest.mark.parametrize("name", PARALL)
def test_tracking_changes_nothing(name):
    """Underflow tracking leaves the reference arithmetic's results bit for bit."""
    rec, text = load_case(name)
    _, _, a = _run(rec, text, "reference")
    _, bt, b = _run(rec, text, "track")
    assert np.array_equal(a, b, equal_nan=True)
    taint, events = bt.underflow()
    assert events == 0 and not taint.any()


def test_damping_and_lowpass_modes_agree():
    """A damped fixed run and a low-pass run on a clamped Bingo graph: both
    arithmetics agree to rounding (no message leaves the double range)."""
    fl = workloads.config0(2)
    cl = {int(a): i % 2 for i, a in enumerate(fl.alarms[:12])}
    g = O.OracleGraph.from_factors(fl)
    g.clamp_labels(cl)
    g = g.rebuild()
    for damping in (0.0, 0.3):
        out = {}
        for arith in ("reference", "lodds"):
            bp = O.OracleBP(g, damping=damping, arith=arith)
            bp.init()
            bp.run_fixed(1e-9, 80, 1)
            fixed = bp.beliefs()
            bp.init()
            frac, reason, sweeps = bp.run_lowpass(1e-6, 10, 200, 7)
            out[arith] = (fixed, bp.lowpass(), frac, reason, sweeps)
        r, lo = out["reference"], out["lodds"]
        assert np.max(np.abs(r[0] - lo[0])) <= 1e-12
        assert np.max(np.abs(r[1] - lo[1])) <= 1e-12
        assert r[2:] == lo[2:]


def test_fault_localisation_underflow_is_what_differs():
    """cfg2 shape at a quarter of its size: the reference's products
    underflow from sweep 4; before that the arithmetics agree to 1e-14, and
    at every sweep every belief on which they differ by more than 1e-9
    depends on an underflow."""
    fl, clamps = workloads.config2(2, scale=0.25)
    g = O.OracleGraph.from_factors(fl)
    g.clamp_labels(clamps)
    g = g.rebuild()
    threads = os.cpu_count() or 1
    lo = O.OracleBP(g, threads=threads, arith="lodds")
    tr = O.OracleBP(g, threads=threads, arith="track")
    lo.init()
    tr.init()
    first = None
    for t in range(1, 7):
        lo.sweep()
        tr.sweep()
        taint, events = tr.underflow()
        a, b = lo.current_beliefs(), tr.current_beliefs()
        differ = (np.abs(a - b) > 1e-9) | (np.isnan(a) != np.isnan(b))
        if events and first is None:
            first = t
        if first is None:
            assert np.nanmax(np.abs(a - b)) <= 1e-14 and not differ.any()
        assert not (differ & ~taint).any(), t
    assert first is not None and first >= 2  # there is an underflow, and not in the first sweep
    assert differ.any()  # and it changes beliefs
