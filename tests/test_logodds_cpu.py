"""The folded constants' log-odds (csrc/logodds.h, det_logit / det_log).

The host layout build, the device layout build and the probability setters
all compute +-log(p / (1 - p)) of singletons and of factors reduced to their
head (causal_bp_parall.cu:110-117, :154-156), and must agree bit for bit, so
the logarithm is written out from correctly rounded double operations. This
test compiles the header on the host (g++, as the library's host code is
built) and checks it against a 60-digit decimal reference: det_log within
2 units in the last place over the whole double range (normal and subnormal
arguments), det_logit within 3e-16 relative to max(1, |log-odds|), and the
special values (0, 1, NaN, outside [0, 1]). The device side is the same
source; `test_dlayout_gpu.py` checks that both builds give the same bits.
"""

import math
import os
import shutil
import struct
import subprocess
from decimal import Decimal, getcontext

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

DRIVER = r"""
#include <cstdio>
#include <vector>
#include "logodds.h"
int main() {
    std::vector<double> x;
    double v;
    while (std::fread(&v, 8, 1, stdin) == 1) x.push_back(v);
    for (double a : x) {
        double r[2] = {flbp::det_log(a), flbp::det_logit(a)};
        std::fwrite(r, 8, 2, stdout);
    }
    return 0;
}
"""


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("logodds")
    src = d / "drv.cpp"
    src.write_text(DRIVER)
    exe = d / "drv"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(ROOT, "fastlbp_b200", "csrc"), str(src), "-o",
                    str(exe)], check=True)

    def run(xs):
        xs = np.ascontiguousarray(xs, dtype=np.float64)
        out = subprocess.run([str(exe)], input=xs.tobytes(), capture_output=True, check=True).stdout
        r = np.frombuffer(out, dtype=np.float64).reshape(-1, 2)
        return r[:, 0], r[:, 1]

    return run


def _ulp_err(got, x):
    getcontext().prec = 60
    ex = Decimal(float(x)).ln()
    return float(abs(Decimal(float(got)) - ex)) / math.ulp(float(ex))


def test_det_log_within_two_ulps(driver):
    rng = np.random.default_rng(5)
    xs = np.concatenate([
        rng.uniform(0.5, 2.0, 1500),                                       # around 1 (reduction boundaries)
        np.ldexp(rng.uniform(0.5, 1.0, 1500), rng.integers(-1021, 1024, 1500)),  # every binade
        np.ldexp(rng.uniform(0.5, 1.0, 300), rng.integers(-1074, -1022, 300)),   # subnormal
        [math.sqrt(2.0), np.nextafter(math.sqrt(2.0), 3), np.nextafter(1.0, 0), np.nextafter(1.0, 2), 2.0, 0.5,
         5e-324, np.finfo(np.float64).max],
    ])
    xs = xs[(xs > 0) & (xs != 1.0)]
    got, _ = driver(xs)
    worst = max(_ulp_err(g, x) for g, x in zip(got, xs))
    assert worst <= 2.0, worst
    g1, _ = driver(np.array([1.0]))
    assert g1[0] == 0.0


def test_det_logit_accuracy_and_specials(driver):
    getcontext().prec = 60
    rng = np.random.default_rng(6)
    ps = np.concatenate([rng.uniform(0, 1, 2000), 10.0 ** -rng.uniform(0, 300, 500),
                         1 - 10.0 ** -rng.uniform(1, 15.9, 500), [0.5, 0.25, 0.75, 1e-300, 5e-324, 1 - 2 ** -53]])
    ps = ps[(ps > 0) & (ps < 1)]
    _, got = driver(ps)
    worst = 0.0
    for g, p in zip(got, ps):
        ex = (Decimal(float(p)) / (1 - Decimal(float(p)))).ln()
        worst = max(worst, float(abs(Decimal(float(g)) - ex)) / max(1.0, abs(float(ex))))
    assert worst <= 3e-16, worst
    # close to the platform's log(p) - log1p(-p) as well
    ref = np.log(ps) - np.log1p(-ps)
    assert np.max(np.abs(got - ref) / np.maximum(1.0, np.abs(ref))) <= 1e-15
    sp = np.array([0.0, -0.0, 1.0, np.nan, -0.5, 1.5, np.inf])
    lg, lt = driver(sp)
    assert lt[0] == -np.inf and lt[1] == -np.inf and lt[2] == np.inf
    assert np.isnan(lt[3]) and np.isnan(lt[4]) and np.isnan(lt[5]) and np.isnan(lt[6])
    assert lg[0] == -np.inf and lg[2] == 0.0 and np.isnan(lg[3]) and np.isnan(lg[4]) and lg[6] == np.inf


def test_det_logit_is_antisymmetric_where_exact(driver):
    # p and 1 - p are both exact for dyadic p: log-odds of opposite sign and equal size
    ps = np.array([2.0 ** -k for k in range(1, 40)] + [3 / 8, 5 / 16, 7 / 64])
    _, a = driver(ps)
    _, b = driver(1 - ps)
    assert np.max(np.abs(a + b) / np.maximum(1, np.abs(a))) <= 4e-16
    assert struct.pack("<d", float(driver(np.array([0.5]))[1][0])) == struct.pack("<d", 0.0)
