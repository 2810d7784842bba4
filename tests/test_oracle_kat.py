"""Known answers for the oracle that do not depend on the reference's
arithmetic: on tree-shaped graphs loopy BP converges to the exact marginals,
computed here by enumerating every joint state (tests/brute.py). Clamped
variables are conditioned on by indicator factors, which checks the
reference's clamp rewrite (causal_factor.cpp:63-100) as well."""

import numpy as np
import pytest

import brute
import oracle as O
import trees


@pytest.mark.parametrize("chunk", range(4))
def test_oracle_exact_on_trees(chunk):
    checked = 0
    for seed in range(chunk * 50, chunk * 50 + 50):
        fl = trees.random_tree(seed, n_factors=5)
        labels = sorted(set(fl.head.tolist()) | set(fl.body.tolist()))
        rng = np.random.default_rng(seed + 7)
        cl = {int(l): int(rng.integers(0, 2)) for l in labels if rng.random() < 0.2}
        with np.errstate(all="ignore"):
            ex = brute.marginals(labels, trees.as_brute_factors(fl, cl))
        if not np.all(np.isfinite(ex)):
            continue
        g = O.OracleGraph.from_factors(fl)
        g.clamp_labels(cl)
        g = g.rebuild()
        bp = O.OracleBP(g)
        bp.init()
        bp.run(1e-14, 2000, 100.0)
        pos = {l: i for i, l in enumerate(labels)}
        want = np.array([ex[pos[int(l)]] for l in g.var_labels()])
        assert np.max(np.abs(bp.beliefs() - want)) < 1e-9, seed
        checked += 1
    assert checked >= 30


def test_single_rule_closed_forms():
    """AND and OR heads with independent parents: P(h=1) = p*a*b + q*(1-a*b)
    for AND; P(h=0) = p*(1-a)(1-b) + q*(1 - (1-a)(1-b)) for OR."""
    from fastlbp_b200.workloads import FactorList

    a, b, p, q = 0.8, 0.6, 0.9, 0.05
    for kind in (1, 2):
        fl = FactorList(np.array([kind, 0, 0], np.int32), np.array([0, 1, 2], np.int64),
                        np.array([0, 2, 2, 2], np.int64), np.array([1, 2], np.int64), np.array([p, a, b]),
                        np.array([q, 0.0, 0.0]))
        g = O.OracleGraph.from_factors(fl)
        bp = O.OracleBP(g)
        bp.init()
        bp.run(1e-15, 100, 10.0)
        h = bp.beliefs()[0]
        if kind == 1:
            want = p * a * b + q * (1 - a * b)
        else:
            want = 1 - (p * (1 - a) * (1 - b) + q * (1 - (1 - a) * (1 - b)))
        assert abs(h - want) < 1e-14
