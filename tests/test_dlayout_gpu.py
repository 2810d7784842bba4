"""The layout built on the GPU (flbp_set_layout_builder "device") against the
host build, which the other tests check against the FP64 oracle.

For graphs covering every layout class (sliced-ELL factors and variables of
every width, large factors on both sides of the register and tile limits, a
variable with more entries than a tile holds, clamped heads with every mask,
singletons, factors reduced to their head, degree-0 variables), in FP32 and
FP64, with and without damping:
* the engine's device layout (every buffer the kernels read, copied back,
  and its counts) has the same digest from both builds;
* runs give bit-identical beliefs and sweep counts;
* a device-built engine builds its complete host layout when a call needs
  it (clamps, message export, gradients) and then behaves as a host-built one;
* malformed graphs give the same error code and message from both builds.
"""

import numpy as np
import pytest

from fastlbp_b200 import CausalFactorGraph, Engine, FlbpError, workloads
from fastlbp_b200.api import set_layout_builder
from test_engine_gpu import _large_item_graph

pytestmark = pytest.mark.gpu


def _graphs():
    out = {}
    fl = workloads.config0(3)
    g = CausalFactorGraph.from_factors(fl)
    g.clamp_labels({int(a): i % 2 for i, a in enumerate(fl.alarms)})
    out["cfg0_clamped"] = g.rebuild().graph_arrays()
    fl4 = workloads.config0(4)
    g2 = CausalFactorGraph.from_factors(fl4)
    h = g2.findVar(int(fl4.alarms[0]))
    g2.clamp(h, 0)
    g2.clamp(h, 1)  # head mask (0, 0)
    out["cfg0_double_clamp"] = g2.rebuild().graph_arrays()
    out["cfg1_small"] = CausalFactorGraph.from_factors(workloads.config1(1, scale=0.02)).graph_arrays()
    fl2, cl2 = workloads.config2(2, scale=0.05)
    g3 = CausalFactorGraph.from_factors(fl2)
    g3.clamp_labels(cl2)
    out["cfg2_clamped"] = g3.rebuild().graph_arrays()
    out["large_items"] = CausalFactorGraph.from_factors(_large_item_graph(3)).graph_arrays()
    # folded constants of extreme probabilities (0, 1, subnormal, next to 1): both builds take
    # their log-odds from the same code, so even these give the same bits
    a = dict(CausalFactorGraph.from_factors(workloads.config0(5)).graph_arrays())
    deg = np.diff(a["factor_offsets"])
    folded = np.flatnonzero((a["factor_type"] == workloads.SINGLETON) | (deg == 1))
    vals = [5e-324, 1e-300, 1e-17, 0.3, 0.5, 1 - 2.0 ** -53, 0.999999, 1e-8, 0.0, 1.0] + [0.9] * 20
    p = a["factor_p"].copy()
    p[folded] = np.resize(np.array(vals), folded.size)
    a["factor_p"] = p
    out["extreme_p"] = a
    return out


GRAPHS = _graphs()


def _engine(a, builder, **kw):
    set_layout_builder(builder)
    try:
        return Engine(a, **kw)
    finally:
        set_layout_builder("auto")


@pytest.mark.parametrize("name", sorted(GRAPHS))
@pytest.mark.parametrize("prec,damping", [(32, 0.0), (64, 0.0), (32, 0.15)])
def test_device_layout_equals_host_layout(name, prec, damping):
    a = GRAPHS[name]
    eh = _engine(a, "host", precision=prec, damping=damping)
    ed = _engine(a, "device", precision=prec, damping=damping)
    dh, on_h = eh.layout_digest()
    dd, on_d = ed.layout_digest()
    assert not on_h and on_d
    assert dh == dd
    for e in (eh, ed):
        e.init()
    ih = eh.run_tol(1e-6, 200, 1e9)
    id_ = ed.run_tol(1e-6, 200, 1e9)
    assert ih["sweeps"] == id_["sweeps"]
    assert np.array_equal(eh.beliefs(), ed.beliefs(), equal_nan=True)
    for e in (eh, ed):
        e.init()
        e.run_fixed(23)
    assert np.array_equal(eh.beliefs(), ed.beliefs(), equal_nan=True)
    eh.close()
    ed.close()


def test_device_built_engine_builds_its_host_layout_on_demand():
    """Clamps, message export and gradients need the complete host layout; a
    device-built engine builds it then, and its layout digest and results
    stay those of the host-built engine."""
    a = GRAPHS["cfg0_clamped"]
    eh = _engine(a, "host", precision=64)
    ed = _engine(a, "device", precision=64)
    digest = ed.layout_digest()[0]
    for e in (eh, ed):
        e.init()
        e.run_fixed(10)
    assert all(np.array_equal(x, y) for x, y in zip(eh.fv_messages(), ed.fv_messages()))
    assert ed.layout_digest()[0] == digest
    lab = np.nonzero(np.isfinite(eh.beliefs()))[0][:5]
    for e in (eh, ed):
        e.clamp(lab.tolist(), [1, 0, 1, 0, 1][: lab.size])
        e.init()
        e.run_fixed(30)
    assert np.array_equal(eh.beliefs(), ed.beliefs(), equal_nan=True)
    assert np.array_equal(eh.adjoint_forward(20, 5), ed.adjoint_forward(20, 5), equal_nan=True)


def _malformed(kind):
    a = {k: np.array(v, copy=True) if isinstance(v, np.ndarray) else v for k, v in GRAPHS["cfg0_clamped"].items()}
    if kind == "offsets":
        a["factor_offsets"][5] = a["factor_offsets"][7]
    elif kind == "slot_var":
        a["slot_var"][100] = int(a["n_vars"]) + 3
    elif kind == "type":
        a["factor_type"][40] = 7
    elif kind == "prob":
        a["factor_p"][41] = 1.5
    elif kind == "head":
        I = int(np.nonzero(np.diff(a["factor_offsets"]) > 1)[0][3])
        a["factor_head"][I] = a["factor_offsets"][I + 1]
    elif kind == "mask":
        I = int(np.nonzero(a["factor_head_clamped"])[0][0])
        a["factor_mask0"][I] = 0.5
    return a


@pytest.mark.parametrize("kind", ["offsets", "slot_var", "type", "prob", "head", "mask"])
def test_malformed_graphs_fail_alike(kind):
    a = _malformed(kind)
    errs = []
    for builder in ("host", "device"):
        with pytest.raises(FlbpError) as ex:
            _engine(a, builder, precision=32)
        errs.append((ex.value.code, str(ex.value)))
    assert errs[0] == errs[1]
