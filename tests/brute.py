"""Exact marginals of tiny causal factor graphs by enumerating all joint
states. On tree-shaped graphs loopy BP is exact, which gives known answers
that do not depend on the reference's arithmetic."""

import itertools

import numpy as np


def factor_value(kind, head_val, body_vals, p, q, mask=None):
    if kind == 0:
        v = p if head_val == 1 else 1.0 - p
    elif kind == 1:  # AND: P(h=1 | all body 1) = p, else q
        r = p if all(b == 1 for b in body_vals) else q
        v = r if head_val == 1 else 1.0 - r
    else:  # OR: P(h=0 | all body 0) = p, else q
        r = p if all(b == 0 for b in body_vals) else q
        v = r if head_val == 0 else 1.0 - r
    if mask is not None:
        v *= mask[head_val]
    return v


def marginals(labels, factors):
    """factors: list of (kind, head_label, body_labels, p, q, mask_or_None)."""
    pos = {l: i for i, l in enumerate(labels)}
    n = len(labels)
    z = 0.0
    m1 = np.zeros(n)
    for st in itertools.product((0, 1), repeat=n):
        w = 1.0
        for kind, h, body, p, q, mask in factors:
            w *= factor_value(kind, st[pos[h]], [st[pos[b]] for b in body], p, q, mask)
            if w == 0.0:
                break
        z += w
        if w:
            m1 += w * np.array(st)
    return m1 / z
