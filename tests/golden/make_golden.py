"""Generate golden vectors by running FastLBP's own GPU CausalBP.

Runs oracle/_ref/ref_bp (the reference sources compiled by oracle/Makefile,
driven through the reference's public API the way examples/fl_wrapper.cu
does) on seeded graphs and stores, per case, the graph file (gzip), the
clamps, the update schedule, the run parameters and the reference's beliefs
at 17 significant digits. Needs a CUDA GPU; the outputs are committed under
tests/golden/.

    python tests/golden/make_golden.py --out tests/golden [--only REGEX]

With --only, just the matching cases are run and the existing index in --out
is extended.
"""

import argparse
import gzip
import json
import os
import re
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from fastlbp_b200 import workloads as W  # noqa: E402
import trees  # noqa: E402

REF_BP = os.path.join(ROOT, "oracle", "_ref", "ref_bp")


def cases():
    fl = W.config0(0)
    yield "cfg0_s0_tol", fl, {}, ["tol", "1e-6", "1000"]
    cl = {int(a): int(i % 2) for i, a in enumerate(fl.alarms)}
    yield "cfg0_s0_clamped_fixed500", fl, cl, ["fixed", "500"]
    fl1 = W.config0(1)
    cl1 = {int(a): int((i // 2) % 2) for i, a in enumerate(fl1.alarms)}
    yield "cfg0_s1_clamped_lowpass", fl1, cl1, ["lowpass", "1e-6", "50", "120", "20"]
    fl2, cl2 = W.config2(seed=4, scale=0.01)
    yield "cfg2_small_clamped_fixed100", fl2, cl2, ["fixed", "100"]
    fl3 = W.config1(seed=5, scale=0.002)
    yield "cfg1_small_fixed200", fl3, {}, ["fixed", "200"]
    for s in range(6):
        t = trees.random_tree(1000 + s, n_factors=6, extreme=0.2)
        import numpy as np
        rng = np.random.default_rng(s)
        labels = sorted(set(t.head.tolist()) | set(t.body.tolist()))
        clt = {int(l): int(rng.integers(0, 2)) for l in labels if rng.random() < 0.2}
        yield "tree_%d_fixed60" % s, t, clt, ["fixed", "60"]
    # sequential schedules (the SEQFIX order of the process's first CausalBP)
    yield "seqfix_cfg0_s0_fixed100", fl, {}, ["fixed", "100"], "SEQFIX"
    yield "seqfix_cfg0_s1_clamped_tol", fl1, cl1, ["tol", "1e-6", "1000"], "SEQFIX"
    yield "seqfix_cfg0_s1_clamped_lowpass", fl1, cl1, ["lowpass", "1e-6", "20", "60", "10"], "SEQFIX"
    yield "topo_cfg0_s0_clamped_fixed20", fl, cl, ["fixed", "20"], "TOPO"
    t = trees.random_tree(1003, n_factors=6, extreme=0.2)
    yield "seqfix_tree_3_fixed60", t, {}, ["fixed", "60"], "SEQFIX"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    ap.add_argument("--only", default=None, help="regex: run only the matching cases, extend the index")
    args = ap.parse_args()
    os.makedirs(args.out, exist_ok=True)
    tmp = tempfile.mkdtemp()
    index = []
    ipath = os.path.join(args.out, "index.json")
    if args.only and os.path.exists(ipath):
        index = json.load(open(ipath))
    for case in cases():
        name, fl, cl, mode = case[:4]
        updates = case[4] if len(case) > 4 else "PARALL"
        if args.only and not re.search(args.only, name):
            continue
        gpath = os.path.join(tmp, name + ".causal_fg")
        fl.write(gpath)
        cpath = os.path.join(tmp, name + ".clamps")
        with open(cpath, "w") as f:
            for k in sorted(cl):
                f.write("%d %d\n" % (k, cl[k]))
        opath = os.path.join(tmp, name + ".out")
        env = dict(os.environ, REF_BP_VERBOSE="1", REF_BP_UPDATES=updates)
        r = subprocess.run([REF_BP, gpath, cpath, opath] + mode, capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise SystemExit("ref_bp failed on %s: %s %s" % (name, r.stdout, r.stderr))
        meta = json.loads(r.stdout.strip().splitlines()[-1])
        m = re.search(r"converged in (\d+) passes|not converged after (\d+) passes", r.stderr)
        sweeps = int(m.group(1) or m.group(2)) if m else None
        beliefs = {}
        with open(opath) as f:
            for line in f:
                a, b = line.split()
                beliefs[a] = b
        with gzip.open(os.path.join(args.out, name + ".causal_fg.gz"), "wt") as f:
            f.write(fl.text())
        rec = dict(name=name, mode=mode, clamps={str(k): v for k, v in sorted(cl.items())}, ref=meta,
                   ref_sweeps=sweeps, beliefs=beliefs)
        if updates != "PARALL":
            rec["updates"] = updates
        with open(os.path.join(args.out, name + ".json"), "w") as f:
            json.dump(rec, f, indent=0)
        if name not in index:
            index.append(name)
        print(name, meta)
    with open(os.path.join(args.out, "index.json"), "w") as f:
        json.dump(index, f)


if __name__ == "__main__":
    main()
