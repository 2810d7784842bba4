"""FastLBP's own example drivers as drop-in clients of this library.

The CPU test compiles examples/fl_wrapper.cu, bingo_wrapper.cu, example_ext.cu
and example_ext_clamp.cu from the FastLBP sources (the directory named by the
FASTLBP_REF environment variable), unchanged, against this repository's
include/ and links them to libfastlbp_b200.so (bingo_wrapper also to NVML, as
FastLBP's own build does). Without FASTLBP_REF it checks the same four
programs as the build step made them (oracle/_ref/examples, by
`make -C oracle examples` from the unchanged sources): present, and linked
to libfastlbp_b200.so. Without either it is skipped.

The GPU test runs fl_wrapper built that way (oracle/_ref/examples, made by
`make -C oracle examples`) on a golden case whose beliefs FastLBP's own code
produced - the same graph, clamps and fixed 500 PARALL sweeps - and checks the
printed beliefs within the FP32 tolerance (1e-5 absolute).
"""

import concurrent.futures as cf
import gzip
import json
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_EXAMPLES = os.path.join(os.environ["FASTLBP_REF"], "examples") if os.environ.get("FASTLBP_REF") else ""
BUILT_EXAMPLES = os.path.join(ROOT, "oracle", "_ref", "examples")
EXAMPLES = ["fl_wrapper", "bingo_wrapper", "example_ext", "example_ext_clamp"]
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.mark.skipif(bool(REF_EXAMPLES) or not all(os.path.exists(os.path.join(BUILT_EXAMPLES, n)) for n in EXAMPLES)
                    or shutil.which("readelf") is None,
                    reason="FASTLBP_REF is set (the sources are compiled below) or the build step made no examples")
def test_built_examples_link_this_library():
    for name in EXAMPLES:
        r = subprocess.run(["readelf", "-d", os.path.join(BUILT_EXAMPLES, name)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert "[libfastlbp_b200.so]" in r.stdout, name


@pytest.mark.skipif(not REF_EXAMPLES or not os.path.isdir(REF_EXAMPLES) or shutil.which("nvcc") is None,
                    reason="FASTLBP_REF (FastLBP sources) or nvcc not available")
def test_reference_examples_compile_unchanged(tmp_path):
    lib = os.path.join(ROOT, "fastlbp_b200", "libfastlbp_b200.so")
    assert os.path.exists(lib)

    def compile_one(name):
        cmd = ["nvcc", "-std=c++17", "-O0", "-w", "-gencode", "arch=compute_100a,code=sm_100a",
               "-I" + os.path.join(ROOT, "include"), os.path.join(REF_EXAMPLES, name + ".cu"),
               "-L" + os.path.dirname(lib), "-lfastlbp_b200", "-L/usr/local/cuda/lib64/stubs", "-lnvidia-ml",
               "-o", str(tmp_path / name)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        return name, r.returncode, r.stderr[-2000:]

    with cf.ThreadPoolExecutor(4) as ex:
        for name, rc, err in ex.map(compile_one, EXAMPLES):
            assert rc == 0, (name, err)
            assert os.path.exists(tmp_path / name)


@pytest.mark.gpu
def test_fl_wrapper_reproduces_reference_beliefs(tmp_path):
    exe = os.path.join(ROOT, "oracle", "_ref", "examples", "fl_wrapper")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/examples/fl_wrapper not built (needs the FastLBP sources at build time)")
    name = "cfg0_s0_clamped_fixed500"
    rec = json.load(open(os.path.join(GOLDEN, name + ".json")))
    assert rec["mode"][0] == "fixed" and int(rec["mode"][1]) == 500  # fl_wrapper's own schedule
    graph = tmp_path / "g.causal_fg"
    with gzip.open(os.path.join(GOLDEN, name + ".causal_fg.gz"), "rt") as f:
        graph.write_text(f.read())
    obs = tmp_path / "obs.txt"
    obs.write_text("".join("%s %s\n" % (k, "true" if int(v) else "false") for k, v in rec["clamps"].items()))
    r = subprocess.run([exe, str(graph), str(obs)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    got = {}
    for line in r.stdout.splitlines():
        k, v = line.split()
        got[int(k)] = float(v)
    want = {int(k): float(v) for k, v in rec["beliefs"].items()}
    assert set(want) <= set(got)
    err = max(abs(got[k] - want[k]) for k in want)
    assert err <= 1e-5, err


@pytest.mark.gpu
def test_example_ext_clamp_runs_seqfix(tmp_path):
    """example_ext_clamp.cu asks for updates=SEQFIX and the low-pass run
    run(1e-6, 500, 1000, 100); built unchanged against this library it runs
    the sequential schedule with the factor order drawn from rnd_gen (seed
    42), and its yetToConverge fraction is the oracle's for that schedule."""
    import oracle as O
    from fastlbp_b200 import workloads as W

    exe = os.path.join(ROOT, "oracle", "_ref", "examples", "example_ext_clamp")
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/examples/example_ext_clamp not built (needs the FastLBP sources at build time)")
    fl = W.config0(2)
    graph = tmp_path / "g.causal_fg"
    fl.write(str(graph))
    r = subprocess.run([exe, str(graph)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    line = [x for x in r.stdout.splitlines() if x.startswith("yetToConverge:")]
    assert len(line) == 1, r.stdout[-2000:]
    got = float(line[0].split()[1])
    og = O.OracleGraph.from_factors(fl)
    bp = O.OracleBP(og)
    bp.set_schedule("SEQFIX", 42)
    bp.init()
    frac, _, _ = bp.run_lowpass(1e-6, 500, 1000, 100)
    assert abs(got - frac) <= 1e-5 * max(1.0, abs(frac)), (got, frac)
