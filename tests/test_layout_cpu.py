"""The device layout is built on all host threads; it must not depend on
how many (flbp_layout_digest hashes every layout array and count). Graphs
large enough for the parallel paths (>= 32 k factors, slots and variables),
a batch of graphs (graph-major order), and the graph with every large-item
size class; each built with 1, 3 and all threads, twice."""

import numpy as np
import pytest

from fastlbp_b200 import CausalFactorGraph, workloads
from fastlbp_b200.api import layout_digest
from test_engine_gpu import _large_item_graph


def _arrays(fl, clamps=None):
    g = CausalFactorGraph.from_factors(fl)
    if clamps:
        g.clamp_labels(clamps)
        g = g.rebuild()
    return g.graph_arrays()


@pytest.mark.parametrize("name", ["cfg1_small", "cfg2_small", "large_items"])
def test_layout_independent_of_threads(name):
    if name == "cfg1_small":
        a = _arrays(workloads.config1(1, scale=0.05))
    elif name == "cfg2_small":
        fl, clamps = workloads.config2(2, scale=0.25)
        a = _arrays(fl, clamps)
    else:
        a = _arrays(_large_item_graph(2))
    digests = {layout_digest(a, t) for t in (1, 3, 0, 0)}
    assert len(digests) == 1


def test_batch_layout_independent_of_threads():
    parts = [_arrays(workloads.config1(s, scale=0.02)) for s in (3, 4, 5)]
    off = [0]
    slot_off, var_off = 0, 0
    sv, head, ty, p, q, fgr, vgr = [], [], [], [], [], [], []
    for k, a in enumerate(parts):
        F = a["factor_offsets"].size - 1
        off.extend((a["factor_offsets"][1:] + slot_off).tolist())
        sv.append(a["slot_var"] + var_off)
        head.append(a["factor_head"] + slot_off)
        ty.append(a["factor_type"])
        p.append(a["factor_p"])
        q.append(a["factor_q"])
        fgr.append(np.full(F, k, np.uint32))
        vgr.append(np.full(int(a["n_vars"]), k, np.uint32))
        slot_off += int(a["factor_offsets"][-1])
        var_off += int(a["n_vars"])
    u = {"n_vars": var_off, "factor_offsets": np.array(off, np.int64), "slot_var": np.concatenate(sv),
         "factor_head": np.concatenate(head), "factor_type": np.concatenate(ty), "factor_p": np.concatenate(p),
         "factor_q": np.concatenate(q)}
    gof = (np.concatenate(fgr), np.concatenate(vgr), len(parts))
    digests = {layout_digest(u, t, gof) for t in (1, 2, 0)}
    assert len(digests) == 1
    assert layout_digest(u, 0, gof) != layout_digest(u, 0)  # graph-major order differs from the single-graph one
