"""Host side of the sequential schedules (no GPU): the library's SEQFIX / TOPO
update sequences and conflict-free batches against the oracle's direct
restatement of buildFixedUpdateSeq, buildTopoUpdateSeq and
putUpdateSeqToKernelFused (csrc/ext/causal_bp.cu:186-304, 583-722), which
keeps the reference's std::set bookkeeping where the library uses stamps.
"""

import numpy as np
import pytest

import oracle as O
import trees
from fastlbp_b200 import CausalFactorGraph, FlbpError, seq_batches, update_seq, workloads
from test_engine_gpu import _large_item_graph


def _graphs():
    fl = workloads.config0(0)
    yield "cfg0", fl, {}
    fl1 = workloads.config0(1)
    yield "cfg0_clamped", fl1, {int(a): int(i % 2) for i, a in enumerate(fl1.alarms)}
    fl2, cl2 = workloads.config2(seed=4, scale=0.01)
    yield "cfg2_small_clamped", fl2, cl2
    yield "large_items", _large_item_graph(11), {1203: 1, 1207: 0, 5: 1}
    yield "tree", trees.random_tree(3, n_factors=6), {}


@pytest.mark.parametrize("case", list(_graphs()), ids=lambda c: c[0])
@pytest.mark.parametrize("updates", ["SEQFIX", "TOPO"])
def test_sequences_and_batches_match_oracle(case, updates):
    _, fl, cl = case
    g = CausalFactorGraph.from_factors(fl)
    og = O.OracleGraph.from_factors(fl)
    if cl:
        g.clamp_labels(cl)
        og.clamp_labels(cl)
        g, og = g.rebuild(), og.rebuild()
    a = g.graph_arrays()
    bp = O.OracleBP(og)
    nb = bp.set_schedule(updates, 42)
    oseq, obatch = bp.schedule()
    seq = update_seq(a, updates, 42)
    assert np.array_equal(seq, oseq)
    sb, n = seq_batches(a, seq)
    assert n == nb
    assert np.array_equal(sb, obatch)
    # batches are consecutive runs of the sequence, and within one no variable
    # receives two messages
    assert np.all(np.diff(sb[seq]) >= 0)
    var = np.asarray(a["slot_var"])
    key = sb[seq].astype(np.int64) * (var.max() + 1) + var[seq]
    assert np.unique(key).size == key.size


def test_seqfix_takes_a_given_factor_order():
    g = CausalFactorGraph.from_factors(workloads.config0(0))
    a = g.graph_arrays()
    off = np.asarray(a["factor_offsets"])
    F = off.size - 1
    order = np.arange(F)[::-1].copy()
    seq = update_seq(a, "SEQFIX", factor_order=order)
    want = np.concatenate([np.arange(off[I], off[I + 1]) for I in order])
    assert np.array_equal(seq, want)
    # the default order is std::shuffle with std::mt19937(seed); seeds differ
    assert not np.array_equal(update_seq(a, "SEQFIX", 42), update_seq(a, "SEQFIX", 7))


def test_malformed_sequences_are_rejected():
    g = CausalFactorGraph.from_factors(workloads.config0(0))
    a = g.graph_arrays()
    seq = update_seq(a, "TOPO")
    with pytest.raises(FlbpError):
        seq_batches(a, seq[:-1])
    bad = seq.copy()
    bad[0] = bad[1]
    with pytest.raises(FlbpError):
        seq_batches(a, bad)
    bad[0] = seq.size
    with pytest.raises(FlbpError):
        seq_batches(a, bad)
    F = np.asarray(a["factor_offsets"]).size - 1
    with pytest.raises(FlbpError):
        update_seq(a, "SEQFIX", factor_order=np.zeros(F, np.int32))


def test_schedule_entry_points_reject_bad_arguments():
    import ctypes as C

    from fastlbp_b200 import _native as N
    from fastlbp_b200.api import _desc_from_arrays

    g = CausalFactorGraph.from_factors(workloads.config0(0))
    a = g.graph_arrays()
    keep = []
    desc = _desc_from_arrays(a, keep)
    seq = np.zeros(desc.n_slots, np.int64)
    assert N.lib().flbp_update_seq(C.byref(desc), 7, None, seq) == 1      # unknown kind
    assert N.lib().flbp_update_seq(C.byref(desc), 1, None, seq) == 1      # SEQFIX without an order
    order = np.zeros(4, np.int32)
    assert N.lib().flbp_shuffled_factors(-1, 0, order) == 1
    assert N.lib().flbp_shuffled_factors(4, 0, order) == 0
    assert sorted(order.tolist()) == [0, 1, 2, 3]
    nb = C.c_int64()
    assert N.lib().flbp_seq_batches(None, seq, seq.size, None, C.byref(nb)) == 1
    # a factor listing a variable twice is refused (the batching assumes distinct variables)
    bad = dict(a)
    sv = np.asarray(a["slot_var"]).copy()
    off = np.asarray(a["factor_offsets"])
    I = int(np.nonzero(np.diff(off) >= 2)[0][0])
    sv[off[I] + 1] = sv[off[I]]
    bad["slot_var"] = sv
    with pytest.raises(FlbpError):
        update_seq(bad, "TOPO")


@pytest.mark.parametrize("seed", range(12))
def test_random_graphs_and_orders_match_oracle(seed):
    """Seeded random graphs (sizes, fan-ins, back edges, clamps) and SEQFIX
    seeds: the library's sequences and batches equal the oracle's."""
    rng = np.random.default_rng(1000 + seed)
    nt = int(rng.integers(20, 400))
    fl = workloads.bingo_graph(nt, int(nt * rng.uniform(1.0, 2.0)), max(3, nt // 15),
                               workloads.uniform_int(1, int(rng.integers(2, 7))),
                               workloads.uniform_int(1, int(rng.integers(2, 12))), int(rng.integers(1 << 30)),
                               n_layers=int(rng.integers(2, 9)), back_frac=float(rng.uniform(0.0, 0.3)),
                               n_alarms=max(2, nt // 20))
    g = CausalFactorGraph.from_factors(fl)
    og = O.OracleGraph.from_factors(fl)
    labels = g.var_labels()
    cl = {int(l): int(rng.integers(0, 2)) for l in rng.choice(labels, size=min(5, labels.size), replace=False)}
    g.clamp_labels(cl)
    og.clamp_labels(cl)
    g, og = g.rebuild(), og.rebuild()
    a = g.graph_arrays()
    for updates in ("SEQFIX", "TOPO"):
        s = int(rng.integers(1 << 31))
        bp = O.OracleBP(og)
        nb = bp.set_schedule(updates, s)
        oseq, obatch = bp.schedule()
        seq = update_seq(a, updates, s)
        assert np.array_equal(seq, oseq)
        sb, n = seq_batches(a, seq)
        assert n == nb and np.array_equal(sb, obatch)
