"""Multi-rank host path on CPU: independent graphs dealt to two ranks with
the gloo backend (one process per rank, as one process per GPU), each rank
solving its own graphs with no per-sweep exchange and the results gathered
at the end. The solver here is the FP64 oracle, so the test runs without a
GPU; the partition and the gathering are the same code bench.py uses."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from fastlbp_b200 import workloads
from fastlbp_b200.shard import expand_shared, gather_results, partition, shared_gradient

N_GRAPHS = 10


def _sizes():
    return [60 + 37 * ((i * 7) % N_GRAPHS) for i in range(N_GRAPHS)]


def _solve(i):
    import oracle as O

    nt = _sizes()[i]
    fl = workloads.bingo_graph(nt, int(1.5 * nt), max(5, nt // 20), workloads.uniform_int(2, 4),
                               workloads.uniform_int(1, 6), 500 + i)
    og = O.OracleGraph.from_factors(fl)
    bp = O.OracleBP(og)
    bp.init()
    bp.run(1e-6, 300, 60.0)
    return bp.beliefs().tolist()


def _rank(rank, world, port, out_path):
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = partition(_sizes(), world)[rank]
    res = gather_results({i: _solve(i) for i in mine}, world)
    if rank == 0:
        np.save(out_path, np.array([np.array(res[i]) for i in range(N_GRAPHS)], dtype=object), allow_pickle=True)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_partition_covers_and_balances():
    w = _sizes()
    for world in (1, 2, 3, 8):
        parts = partition(w, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(w)))
        loads = [sum(w[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(w)
    assert partition(w, 2) == partition(list(w), 2)  # a pure function of the weights


def test_two_gloo_ranks_match_one_process(tmp_path):
    out = str(tmp_path / "res.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        if p.is_alive():
            p.kill()
            pytest.fail("gloo rank did not finish")
        assert p.exitcode == 0
    got = np.load(out, allow_pickle=True)
    for i in range(N_GRAPHS):
        assert np.array_equal(np.array(got[i]), np.array(_solve(i)))


N_RULES = 40


def _grad_of(i):
    """A graph's per-factor gradient and rule map (seeded stand-ins for the
    adjoint's output: this test covers the reduction, not the gradient)."""
    rng = np.random.default_rng(100 + i)
    nf = 50 + 7 * i
    rules = rng.integers(-1, N_RULES, nf)  # -1: a parameter of the factor's own
    return rng.standard_normal(nf), rules


def _grad_rank(rank, world, port, out_path):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = partition([50 + 7 * i for i in range(N_GRAPHS)], world)[rank]
    gp = torch.tensor(np.concatenate([_grad_of(i)[0] for i in mine]))
    rf = torch.tensor(np.concatenate([_grad_of(i)[1] for i in mine]))
    g = shared_gradient(gp, rf, N_RULES, world)
    allg = [torch.zeros(N_RULES, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(allg, g)
    if rank == 0:
        np.save(out_path, torch.stack(allg).numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_shared_rule_gradient_allreduce_two_gloo_ranks(tmp_path):
    """Two ranks, each with its share of the graphs, end with the same shared
    gradient, equal to summing every graph's gradient in one process."""
    import torch

    out = str(tmp_path / "g.npy")
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_grad_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=240)
        if p.is_alive():
            p.kill()
            pytest.fail("gloo rank did not finish")
        assert p.exitcode == 0
    got = np.load(out)
    want = np.zeros(N_RULES)
    for i in range(N_GRAPHS):
        gp, rf = _grad_of(i)
        np.add.at(want, rf[rf >= 0], gp[rf >= 0])
    assert np.array_equal(got[0], got[1])
    assert np.max(np.abs(got[0] - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))
    one = shared_gradient(torch.tensor(np.concatenate([_grad_of(i)[0] for i in range(N_GRAPHS)])),
                          torch.tensor(np.concatenate([_grad_of(i)[1] for i in range(N_GRAPHS)])), N_RULES)
    assert np.max(np.abs(one.numpy() - want)) <= 1e-12 * max(1.0, np.max(np.abs(want)))


def test_expand_shared():
    import torch

    rf = torch.tensor([2, -1, 0, 2, -1])
    p = expand_shared(torch.tensor([0.1, 0.2, 0.3], dtype=torch.float64), rf,
                      torch.tensor([0.9, 0.8, 0.7, 0.6, 0.5], dtype=torch.float64))
    assert p.tolist() == [0.3, 0.8, 0.1, 0.3, 0.5]


def test_rule_indices_out_of_range_are_rejected():
    """A rule index outside [-1, n_rules) raises ValueError on the host before
    any index_add_ (on a CUDA tensor that would be a device-side assert)."""
    import torch

    g = torch.ones(3, dtype=torch.float64)
    for bad in ([0, 3, -1], [0, -2, 1]):
        with pytest.raises(ValueError):
            shared_gradient(g, torch.tensor(bad), 3)
        with pytest.raises(ValueError):
            expand_shared(torch.zeros(3, dtype=torch.float64), torch.tensor(bad), g)
    assert shared_gradient(g, torch.tensor([0, 2, -1]), 3).tolist() == [1.0, 0.0, 1.0]
