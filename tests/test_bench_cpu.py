"""bench.py's multi-rank entry on CPU: `bench.py --gpus 2` without a launcher
starts two ranks itself (torch.distributed.run, one process per GPU; gloo
here, without GPUs), deals the batched-serving graphs to them by size and
prints one JSON line from rank 0 (--plan-only: the same partition and
gathering as the GPU runs, no GPU work)."""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _run(args, **env_extra):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    for k in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT"):
        env.pop(k, None)
    env.update(env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py")] + args, env=env, capture_output=True,
                          text=True, timeout=600, cwd=ROOT)


def test_gpus_flag_starts_that_many_ranks():
    r = _run(["--gpus", "2", "--plan-only", "--graphs", "40"])
    assert r.returncode == 0, r.stderr[-3000:]
    lines = [x for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    d = json.loads(lines[0])
    assert d["n_gpus"] == 2
    assert sorted(d["plan"]) == ["0", "1"]
    shares = [d["plan"][k]["graphs"] for k in ("0", "1")]
    assert sorted(shares[0] + shares[1]) == list(range(40))
    assert shares[0] and shares[1]
    loads = [d["plan"][k]["tuples"] for k in ("0", "1")]
    assert max(loads) - min(loads) <= 200_000  # within one graph of each other (largest graph <= 200 k tuples)


def test_single_rank_plan():
    r = _run(["--plan-only", "--graphs", "12"])
    assert r.returncode == 0, r.stderr[-3000:]
    d = json.loads([x for x in r.stdout.splitlines() if x.startswith("{")][0])
    assert d["n_gpus"] == 1 and d["plan"]["0"]["graphs"] == list(range(12))


@pytest.mark.parametrize("world", ["3"])
def test_rank_count_must_match_the_flag(world):
    """Launched by a launcher with a different number of ranks, bench.py refuses."""
    r = _run(["--gpus", "2", "--plan-only"], WORLD_SIZE=world, RANK="0", LOCAL_RANK="0")
    assert r.returncode != 0
    assert "ranks were started" in (r.stderr + r.stdout)
