"""Random tree-shaped causal factor graphs for known-answer tests.

Each new factor joins exactly one existing variable with fresh ones, so the
factor graph stays a tree and loopy BP converges to the exact marginals.
"""

import numpy as np

from fastlbp_b200.workloads import FactorList


def random_tree(seed, n_factors=5, max_body=3, extreme=0.15, prior_frac=0.5, max_vars=12):
    rng = np.random.default_rng(seed)
    nxt = 0
    vars_ = [nxt]
    nxt += 1
    is_head = set()
    facs = []  # (kind, head, body, p, q)

    def prob():
        r = rng.random()
        if r < extreme:
            return float(rng.choice([0.0, 1.0]))
        return float(np.round(rng.uniform(0.02, 0.98) * 2 ** 20) / 2 ** 20)

    for _ in range(n_factors):
        if nxt >= max_vars:
            break
        a = int(rng.choice(vars_))
        kind = int(rng.choice([1, 2]))
        d = int(rng.integers(1, max_body + 1))
        d = min(d, max_vars - nxt)
        if d < 1:
            break
        if a not in is_head and rng.random() < 0.5:
            head, body = a, list(range(nxt, nxt + d))
            nxt += d
        else:
            head = nxt
            body = [a] + list(range(nxt + 1, nxt + d))
            nxt += d
        vars_ += [v for v in [head] + body if v not in vars_]
        is_head.add(head)
        facs.append((kind, head, body, prob(), prob()))
    # priors on some variables that head nothing; the rest get the reader's Singleton(0.5)
    for v in sorted(vars_):
        if v not in is_head:
            p = prob() if rng.random() < prior_frac else 0.5
            facs.append((0, v, [], p, 0.0))
    kind = np.array([f[0] for f in facs], np.int32)
    head = np.array([f[1] for f in facs], np.int64)
    body_off = np.concatenate([[0], np.cumsum([len(f[2]) for f in facs])]).astype(np.int64)
    body = np.array([b for f in facs for b in f[2]], np.int64)
    p = np.array([f[3] for f in facs])
    q = np.array([f[4] for f in facs])
    return FactorList(kind, head, body_off, body, p, q)


def as_brute_factors(fl, clamps=None):
    """(kind, head, body, p, q, mask) tuples plus indicator factors for clamps."""
    out = []
    for i in range(fl.n):
        b = fl.body[fl.body_off[i]:fl.body_off[i + 1]].tolist()
        out.append((int(fl.kind[i]), int(fl.head[i]), b, float(fl.p[i]), float(fl.q[i]), None))
    for lab, x in (clamps or {}).items():
        out.append((0, int(lab), [], float(x), 0.0, None))
    return out
