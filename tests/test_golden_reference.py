"""The FP64 oracle against golden vectors produced by FastLBP's own GPU code.

tests/golden/make_golden.py ran the reference sources (compiled into
oracle/_ref/ref_bp, driven through the reference's public API the way
examples/fl_wrapper.cu does) on seeded graphs and stored the graph, clamps,
run mode and the reference's beliefs at 17 digits. The oracle restates the
same arithmetic in double precision on the CPU without FMA contraction, so
it agrees to ~1e-12 rather than bit for bit.
"""

import gzip
import json
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = json.load(open(os.path.join(GOLDEN, "index.json")))


def load_case(name):
    rec = json.load(open(os.path.join(GOLDEN, name + ".json")))
    with gzip.open(os.path.join(GOLDEN, name + ".causal_fg.gz"), "rt") as f:
        text = f.read()
    return rec, text


def oracle_run(rec, text):
    g = O.OracleGraph.from_text(text)
    g.clamp_labels({int(k): int(v) for k, v in rec["clamps"].items()})
    g = g.rebuild()
    bp = O.OracleBP(g)
    if rec.get("updates", "PARALL") != "PARALL":
        bp.set_schedule(rec["updates"], 42)
    bp.init()
    mode = rec["mode"]
    out = {}
    if mode[0] == "fixed":
        out["ret"] = bp.run_fixed(1e-6, int(mode[1]), 1)
        b = bp.lowpass()
    elif mode[0] == "tol":
        bp.run(float(mode[1]), int(mode[2]), 57600.0)
        out["sweeps"] = bp.iters
        b = bp.beliefs()
    else:
        frac, reason, sweeps = bp.run_lowpass(float(mode[1]), int(mode[2]), int(mode[3]), int(mode[4]))
        out["ret"] = frac
        b = bp.lowpass()
    out["beliefs"] = dict(zip(g.var_labels().tolist(), b.tolist()))
    return out


@pytest.mark.parametrize("name", CASES)
def test_oracle_matches_reference_binary(name):
    rec, text = load_case(name)
    got = oracle_run(rec, text)
    ref = {int(k): float(v) for k, v in rec["beliefs"].items()}
    assert set(ref) == set(got["beliefs"])
    err = max(abs(got["beliefs"][k] - ref[k]) for k in ref)
    assert err <= 1e-10, (name, err)
    if "sweeps" in got and rec.get("ref_sweeps") is not None:
        assert got["sweeps"] == rec["ref_sweeps"]
    if "ret" in got:
        assert abs(got["ret"] - rec["ref"]["ret"]) <= 1e-12


def test_golden_graphs_match_generator():
    """The committed graphs are exactly what the seeded generators produce."""
    from fastlbp_b200 import workloads as W

    rec, text = load_case("cfg0_s0_tol")
    assert text == W.config0(0).text()


@pytest.mark.gpu
@pytest.mark.parametrize("name", CASES)
def test_engine_matches_reference_binary(name):
    """The FP64 engine (PARALL or the case's sequential schedule) against the
    reference's own beliefs."""
    from fastlbp_b200 import CausalFactorGraph, Engine

    rec, text = load_case(name)
    g = CausalFactorGraph.from_text(text)
    g.clamp_labels({int(k): int(v) for k, v in rec["clamps"].items()})
    g = g.rebuild()
    eng = Engine.from_graph(g, precision=64, updates=rec.get("updates", "PARALL"), seed=42)
    eng.init()
    mode = rec["mode"]
    if mode[0] == "fixed":
        eng.run_fixed(int(mode[1]))
        b = eng.lowpass()
    elif mode[0] == "tol":
        info = eng.run_tol(float(mode[1]), int(mode[2]), 57600.0)
        if rec.get("ref_sweeps") is not None:
            assert info["total_sweeps"] == rec["ref_sweeps"]
        b = eng.beliefs()
    else:
        info = eng.run_lowpass(float(mode[1]), int(mode[2]), int(mode[3]), int(mode[4]))
        assert abs(info["frac"] - rec["ref"]["ret"]) <= 1e-12
        b = eng.lowpass()
    got = dict(zip(g.var_labels().tolist(), b.tolist()))
    ref = {int(k): float(v) for k, v in rec["beliefs"].items()}
    assert set(ref) == set(got)
    err = max(abs(got[k] - ref[k]) for k in ref)
    assert err <= 1e-9, (name, err)
