"""Seeded synthetic causal factor graphs (Bingo- and fault-localisation-shaped).

FastLBP ships no graphs, generators or benchmark data, so every workload here
is synthetic and seeded. A graph is a list of causal factors exactly as the
``.causal_fg`` reader produces them (csrc/ext/causal_fg.cpp:129-279):

* every derivation rule ``r`` gets its own rule variable, the head of a
  noisy-AND factor (``*p;q``) whose body is the rule's antecedent tuples;
* every derived tuple ``t`` gets one OR factor (``+``, p=1, q=0: a
  deterministic OR over its rule variables, which together realise a
  noisy-OR);
* input tuples get a singleton prior (``I p``);
* every variable that is never a head gets ``Singleton(0.5)``, appended in
  ascending label order - the reader's own rule (causal_fg.cpp:264-269) -
  so the array form and the file form describe the same factor list.

Probabilities are rounded to multiples of 2**-24 and written with enough
digits to be exact, so the text and array forms agree bit for bit.
"""

from __future__ import annotations

import dataclasses
import math
from typing import Callable, Dict, Optional

import numpy as np

SINGLETON, AND, OR = 0, 1, 2
_Q = float(2 ** 24)


def _quant(x: np.ndarray) -> np.ndarray:
    return np.round(np.asarray(x, dtype=np.float64) * _Q) / _Q


@dataclasses.dataclass
class FactorList:
    """Causal factors as parallel arrays; bodies are label lists in CSR form."""

    kind: np.ndarray      # int32, 0 singleton / 1 AND / 2 OR
    head: np.ndarray      # int64 head labels
    body_off: np.ndarray  # int64, n+1
    body: np.ndarray      # int64 body labels (unsorted, may repeat; the model dedups)
    p: np.ndarray         # float64 prob()
    q: np.ndarray         # float64 prob_default()
    alarms: Optional[np.ndarray] = None  # labels of designated alarm / test variables
    info: Optional[Dict] = None

    @property
    def n(self) -> int:
        return int(self.kind.shape[0])

    def text(self) -> str:
        """The ``.causal_fg`` text for this factor list."""
        out = [str(self.n)]
        bo = self.body_off
        for i in range(self.n):
            out.append("")
            out.append(str(int(self.head[i])))
            k = int(self.kind[i])
            if k == SINGLETON:
                out.append("I")
                out.append("%.30g" % self.p[i])
            else:
                out.append("%s%.30g;%.30g" % ("*" if k == AND else "+", self.p[i], self.q[i]))
                b = self.body[bo[i]:bo[i + 1]]
                out.append(str(len(b)))
                out.append(" ".join(str(int(x)) for x in b))
        return "\n".join(out) + "\n"

    def write(self, path: str) -> None:
        with open(path, "w") as f:
            f.write(self.text())

    def n_slots(self) -> int:
        """E = sum over factors of |vars(factor)| (deduplicated body plus head)."""
        tot = 0
        bo = self.body_off
        for i in range(self.n):
            b = self.body[bo[i]:bo[i + 1]]
            s = set(int(x) for x in b)
            s.add(int(self.head[i]))
            tot += len(s)
        return tot


def _append_auto_singletons(kind, head, body_off, body, p, q):
    used = np.unique(np.concatenate([head, body])) if body.size else np.unique(head)
    heads = np.unique(head)
    never = np.setdiff1d(used, heads, assume_unique=True)
    n_new = never.size
    kind = np.concatenate([kind, np.zeros(n_new, np.int32)])
    head = np.concatenate([head, never.astype(np.int64)])
    body_off = np.concatenate([body_off, np.full(n_new, body_off[-1], np.int64)])
    p = np.concatenate([p, np.full(n_new, 0.5)])
    q = np.concatenate([q, np.zeros(n_new)])
    return kind, head, body_off, body, p, q


def bingo_graph(
    n_tuples: int,
    n_rules: int,
    n_inputs: int,
    and_fanin: Callable[[np.random.Generator, int], np.ndarray],
    or_fanin: Callable[[np.random.Generator, int], np.ndarray],
    seed: int,
    n_layers: int = 8,
    back_frac: float = 0.10,
    p_lo: float = 0.85,
    p_hi: float = 0.99,
    input_prior: float = 0.99,
    n_alarms: int = 20,
) -> FactorList:
    """A layered derivation graph.

    Tuples 0..n_tuples-1 are ordered by layer (layer 0 = inputs). Rules are
    spread over derived tuples by drawing each consequent's OR fan-in from
    ``or_fanin`` until all ``n_rules`` rules are used; tuples left without a
    rule stay underived. A rule with consequent in layer L draws its
    antecedents uniformly from layers < L; with probability ``back_frac`` one
    antecedent comes from a layer >= L instead, which closes loops.
    """
    rng = np.random.default_rng(seed)
    n_inputs = max(1, min(n_inputs, n_tuples - 1))
    rest = n_tuples - n_inputs
    per = np.full(n_layers - 1, rest // (n_layers - 1), np.int64)
    per[: rest % (n_layers - 1)] += 1
    layer_start = np.concatenate([[0, n_inputs], n_inputs + np.cumsum(per)]).astype(np.int64)
    layer_of = np.searchsorted(layer_start, np.arange(n_tuples), side="right") - 1

    # OR fan-ins over derived candidates in random order until the rules run out.
    cand = rng.permutation(np.arange(n_inputs, n_tuples))
    fan = or_fanin(rng, cand.size).astype(np.int64)
    fan = np.maximum(fan, 1)
    csum = np.cumsum(fan)
    n_der = int(np.searchsorted(csum, n_rules, side="left")) + 1
    n_der = min(n_der, cand.size)
    fan = fan[:n_der].copy()
    fan[-1] -= int(csum[n_der - 1] - n_rules) if csum[n_der - 1] > n_rules else 0
    if fan.sum() < n_rules:  # not enough candidates: pile the rest onto the last tuple
        fan[-1] += n_rules - int(fan.sum())
    derived = np.sort(cand[:n_der])
    fan = fan[np.argsort(cand[:n_der], kind="stable")]
    cons = np.repeat(derived, fan)  # consequent of each rule, grouped by tuple label
    n_rules = cons.size

    # Antecedents.
    na = np.clip(and_fanin(rng, n_rules).astype(np.int64), 1, None)
    lo_limit = layer_start[layer_of[cons]]  # antecedents come from [0, lo_limit)
    a_off = np.concatenate([[0], np.cumsum(na)]).astype(np.int64)
    rule_of_slot = np.repeat(np.arange(n_rules), na)
    ante = (rng.random(a_off[-1]) * lo_limit[rule_of_slot]).astype(np.int64)
    back = rng.random(n_rules) < back_frac
    br = np.nonzero(back)[0]
    if br.size:
        lo = lo_limit[br]
        span = n_tuples - lo
        ante[a_off[br]] = lo + (rng.random(br.size) * span).astype(np.int64)
    p_rule = _quant(rng.uniform(p_lo, p_hi, n_rules))

    # Factor list: inputs, then per derived tuple its OR factor followed by its rules.
    rule_var = n_tuples + np.arange(n_rules, dtype=np.int64)
    n_or = derived.size
    kinds, heads, boffs, bodies, ps, qs = [], [], [], [], [], []
    # inputs
    kinds.append(np.zeros(n_inputs, np.int32))
    heads.append(np.arange(n_inputs, dtype=np.int64))
    boffs.append(np.zeros(n_inputs, np.int64))
    ps.append(np.full(n_inputs, _quant(np.array([input_prior]))[0]))
    qs.append(np.zeros(n_inputs))
    # interleave OR and AND factors: order key = (tuple group, 0 for OR / 1+r for AND)
    grp_start = np.concatenate([[0], np.cumsum(fan)]).astype(np.int64)
    n_f = n_or + n_rules
    f_kind = np.empty(n_f, np.int32)
    f_head = np.empty(n_f, np.int64)
    f_len = np.empty(n_f, np.int64)
    f_p = np.empty(n_f)
    f_q = np.zeros(n_f)
    or_pos = grp_start[:-1] + np.arange(n_or)  # position of each OR factor in the block
    is_or = np.zeros(n_f, bool)
    is_or[or_pos] = True
    and_pos = np.nonzero(~is_or)[0]
    f_kind[or_pos] = OR
    f_head[or_pos] = derived
    f_len[or_pos] = fan
    f_p[or_pos] = 1.0
    f_kind[and_pos] = AND
    f_head[and_pos] = rule_var
    f_len[and_pos] = na
    f_p[and_pos] = p_rule
    f_off = np.concatenate([[0], np.cumsum(f_len)]).astype(np.int64)
    f_body = np.empty(f_off[-1], np.int64)
    # OR bodies: the rule variables of the group
    or_slots = np.repeat(f_off[or_pos], fan) + (np.arange(n_rules) - np.repeat(grp_start[:-1], fan))
    f_body[or_slots] = rule_var
    and_slots = np.repeat(f_off[and_pos], na) + (np.arange(a_off[-1]) - np.repeat(a_off[:-1], na))
    f_body[and_slots] = ante
    kind = np.concatenate([kinds[0], f_kind])
    head = np.concatenate([heads[0], f_head])
    body_off = np.concatenate([[0], np.zeros(n_inputs, np.int64), f_off[1:]]).astype(np.int64)
    body = f_body
    p = np.concatenate([ps[0], f_p])
    q = np.concatenate([qs[0], f_q])
    kind, head, body_off, body, p, q = _append_auto_singletons(kind, head, body_off, body, p, q)

    last = derived[layer_of[derived] >= max(1, n_layers - 2)]
    pool = last if last.size >= n_alarms else derived
    alarms = np.sort(rng.choice(pool, size=min(n_alarms, pool.size), replace=False)) if pool.size else np.zeros(0, np.int64)
    info = dict(n_tuples=n_tuples, n_rules=n_rules, n_inputs=n_inputs, n_derived=int(n_or), n_layers=n_layers, seed=seed)
    return FactorList(kind, head, body_off, body, p, q, alarms=alarms.astype(np.int64), info=info)


# ----------------------------------------------------------------- fan-in laws

def uniform_int(lo: int, hi: int):
    return lambda rng, n: rng.integers(lo, hi + 1, size=n)


def geometric_clipped(p: float, cap: int):
    """1 + Geometric(p) failures before the first success, clipped at ``cap``."""
    return lambda rng, n: np.minimum(rng.geometric(p, size=n), cap)


def zipf_capped(alpha: float, cap: int):
    """Zipf(alpha) truncated to [1, cap] (values above cap are redrawn)."""
    def draw(rng, n):
        out = rng.zipf(alpha, size=n)
        bad = out > cap
        while bad.any():
            out[bad] = rng.zipf(alpha, size=int(bad.sum()))
            bad = out > cap
        return out
    return draw


def log_uniform_int(lo: int, hi: int):
    return lambda rng, n: np.clip(
        np.floor(np.exp(rng.uniform(math.log(lo), math.log(hi + 1), size=n))).astype(np.int64), lo, hi)


# -------------------------------------------------------------------- configs

def config0(seed: int = 0) -> FactorList:
    """Small Bingo-style graph: 2,000 tuples / 8 layers, 100 inputs at 0.99,
    3,000 rules with 2-4 antecedents, OR fan-in 1-6, 10 % back edges,
    p ~ U[0.85, 0.99], 20 alarms."""
    return bingo_graph(2000, 3000, 100, uniform_int(2, 4), uniform_int(1, 6), seed,
                       n_layers=8, back_frac=0.10, p_lo=0.85, p_hi=0.99, input_prior=0.99, n_alarms=20)


def config1(seed: int = 1, scale: float = 1.0) -> FactorList:
    """Large single graph: 1 M tuples, 10 k inputs at 0.99, 1.5 M AND rules with
    fan-in 1+Geom(0.6) clipped at 8, OR fan-in Zipf(2.0) capped at 256, 5 % back
    edges, p ~ U[0.8, 0.999]. ``scale`` shrinks it for tests."""
    nt = max(200, int(1_000_000 * scale))
    return bingo_graph(nt, int(1.5 * nt), max(10, int(10_000 * scale)), geometric_clipped(0.6, 8),
                       zipf_capped(2.0, 256), seed, n_layers=8, back_frac=0.05, p_lo=0.8, p_hi=0.999,
                       input_prior=0.99, n_alarms=200)


def config2(seed: int = 2, scale: float = 1.0):
    """Fault-localisation-shaped graph: 200 k tuples, 300 k rules, OR fan-in
    log-uniform 1-4,096, AND fan-in 2-6, p ~ U[0.5, 0.99]; 2 % of the tuples are
    test outcomes clamped to 1 (fail, 10 %) or 0. Returns (factors, clamps)."""
    nt = max(500, int(200_000 * scale))
    fl = bingo_graph(nt, int(1.5 * nt), max(10, nt // 20), uniform_int(2, 6), log_uniform_int(1, 4096), seed,
                     n_layers=6, back_frac=0.05, p_lo=0.5, p_hi=0.99, input_prior=0.99, n_alarms=0)
    rng = np.random.default_rng(seed + 1000)
    n_tests = max(1, int(0.02 * nt))
    derived = np.unique(fl.head[fl.kind == OR])
    others = np.setdiff1d(np.arange(nt), derived)
    if derived.size >= n_tests:
        tests = rng.choice(derived, n_tests, replace=False)
    else:
        tests = np.concatenate([derived, rng.choice(others, n_tests - derived.size, replace=False)])
    vals = (rng.random(tests.size) < 0.10).astype(np.int64)
    fl.alarms = np.sort(tests)
    return fl, dict(zip(tests.tolist(), vals.tolist()))


def config3_graph(index: int, seed: int = 3):
    """Graph ``index`` of the batched-serving set: config-0 laws, tuple count
    log-uniform in [1 k, 200 k], rules = 1.5 x tuples, 5 % inputs, and 1-50
    alarm clamps fixed to 0/1 uniformly. Returns (factors, clamps)."""
    rng = np.random.default_rng([seed, index])
    nt = int(math.exp(rng.uniform(math.log(1000), math.log(200_000))))
    fl = bingo_graph(nt, int(1.5 * nt), max(10, nt // 20), uniform_int(2, 4), uniform_int(1, 6),
                     int(rng.integers(1 << 31)), n_layers=8, back_frac=0.10, p_lo=0.85, p_hi=0.99,
                     input_prior=0.99, n_alarms=50)
    k = int(rng.integers(1, 51))
    al = fl.alarms[: min(k, fl.alarms.size)]
    vals = rng.integers(0, 2, size=al.size)
    return fl, dict(zip(al.tolist(), vals.tolist()))


def config4_graph(index: int, seed: int = 4, n_tuples: int = 50_000, n_labels: int = 200):
    """Graph ``index`` of the gradient set: config-0 laws at ``n_tuples``
    tuples (rules = 1.5 x tuples, 5 % inputs at 0.99, AND fan-in 2-4, OR
    fan-in 1-6, 10 % back edges, p ~ U[0.85, 0.99]) with ``n_labels``
    labelled alarm tuples, labels Bernoulli(0.3). Returns (factors, alarm
    labels, labels)."""
    rng = np.random.default_rng([seed, index])
    fl = bingo_graph(n_tuples, int(1.5 * n_tuples), max(10, n_tuples // 20), uniform_int(2, 4), uniform_int(1, 6),
                     int(rng.integers(1 << 31)), n_layers=8, back_frac=0.10, p_lo=0.85, p_hi=0.99,
                     input_prior=0.99, n_alarms=n_labels)
    y = (rng.random(fl.alarms.size) < 0.3).astype(np.float64)
    return fl, fl.alarms.copy(), y


def config3_sizes(n_graphs: int = 512, seed: int = 3) -> np.ndarray:
    return np.array([int(math.exp(np.random.default_rng([seed, i]).uniform(math.log(1000), math.log(200_000))))
                     for i in range(n_graphs)])


def from_text(text: str) -> FactorList:
    """Parse ``.causal_fg`` text into a FactorList in file order (no auto singletons)."""
    lines = text.split("\n")
    pos = 0

    def nxt():
        nonlocal pos
        s = lines[pos]
        pos += 1
        while pos < len(lines) and lines[pos].startswith("#"):
            pos += 1
        return s

    n = int(nxt())
    kind, head, boff, body, p, q = [], [], [0], [], [], []
    for _ in range(n):
        pos += 1
        head.append(int(nxt()))
        t = nxt()
        if t[0] == "I":
            kind.append(0)
            p.append(float(nxt()))
            q.append(0.0)
            boff.append(boff[-1])
        else:
            kind.append(1 if t[0] == "*" else 2)
            pv, qv = 1.0, 0.0
            if len(t) > 1:
                sp = t.find(";")
                if sp == -1 or sp > 1:
                    pv = float(t[1:sp] if sp != -1 else t[1:])
                if sp != -1 and sp + 1 != len(t):
                    qv = float(t[sp + 1:])
            p.append(pv)
            q.append(qv)
            bl = int(nxt())
            ids = [int(x) for x in nxt().split()[:bl]]
            body.extend(ids)
            boff.append(boff[-1] + len(ids))
    return FactorList(np.array(kind, np.int32), np.array(head, np.int64), np.array(boff, np.int64),
                      np.array(body, np.int64), np.array(p), np.array(q))
