"""The pass forms give the same bits.

Each sweep pass exists as the staged form (producer warp, bulk copies into
a shared-memory ring) and two direct-load forms (warps load their items
themselves; form 1 at most 64 registers, form 2 at most 40). They share the
arithmetic, so every run must give the same beliefs bit for bit, and the
same sweep counts, whatever the forms: fixed runs, tolerance runs and
low-pass runs, FP32 and FP64, with and without damping. The graphs hold
every item class: a clamped fault-localisation graph (huge OR factors) and
the large-item graph (big and huge factors and variables, clamped big
factors' heads), both with 100 more variables that only have a prior
(whole sliced-ELL groups of variables without entries).
"""

import numpy as np
import pytest

from fastlbp_b200 import CausalFactorGraph, Engine, workloads
from test_engine_gpu import _large_item_graph

pytestmark = pytest.mark.gpu

FORMS = [(1, 1), (2, 2), (1, 0), (0, 2)]


def _with_isolated(fl, n=100):
    """fl plus n variables whose only factor is their prior (singleton): the
    engine's variables without entries, which fill whole sliced-ELL groups
    (width 0) and take their beliefs from the priors alone."""
    top = int(max(fl.head.max(), fl.body.max() if fl.body.size else 0)) + 1
    rng = np.random.default_rng(5)
    return workloads.FactorList(
        np.concatenate([fl.kind, np.full(n, workloads.SINGLETON, fl.kind.dtype)]),
        np.concatenate([fl.head, np.arange(top, top + n, dtype=fl.head.dtype)]),
        np.concatenate([fl.body_off, np.full(n, fl.body_off[-1], fl.body_off.dtype)]), fl.body,
        np.concatenate([fl.p, rng.uniform(0.05, 0.95, n)]), np.concatenate([fl.q, np.zeros(n)]))


def _graphs():
    fl, cl = workloads.config2(seed=6, scale=0.02)
    g = CausalFactorGraph.from_factors(_with_isolated(fl))
    g.clamp_labels(cl)
    g2 = CausalFactorGraph.from_factors(_with_isolated(_large_item_graph(11)))
    g2.clamp_labels({1200 + 3: 1, 1200 + 7: 0, 5: 1})
    return {"fault_loc": g.rebuild().graph_arrays(), "large_items": g2.rebuild().graph_arrays()}


def _runs(a, prec, damping, forms):
    eng = Engine(a, precision=prec, damping=damping)
    eng.set_tuning(*forms)
    eng.init()
    eng.run_fixed(23)
    b_fixed = eng.beliefs()
    eng.init()
    info = eng.run_tol(1e-6, 200, 1e9)
    b_tol = eng.beliefs()
    eng.init()
    eng.run_lowpass(1e-6, 10, 120, 5)
    b_low = eng.lowpass()
    eng.close()
    return info["sweeps"], (b_fixed, b_tol, b_low)


@pytest.mark.parametrize("prec", [32, 64])
@pytest.mark.parametrize("damping", [0.0, 0.2])
def test_forms_bit_equal(prec, damping):
    for name, a in _graphs().items():
        s0, want = _runs(a, prec, damping, (0, 0))
        for forms in FORMS:
            s, got = _runs(a, prec, damping, forms)
            assert s == s0, (name, forms)
            for x, y in zip(got, want):
                assert np.array_equal(x, y, equal_nan=True), (name, forms)
