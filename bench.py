#!/usr/bin/env python
"""Benchmark of the causal LBP sweep on the 1M-variable Bingo-style graph.

Workload (one "step"): init() + 200 synchronous (PARALL) sweeps with damping
0.1 in FP32 log-odds messages, then one belief evaluation, on the seeded
synthetic graph of 1,000,000 tuple variables (+1,500,000 rule variables,
2.32 M factors, 6.32 M edge slots): 10,000 inputs at 0.99, noisy-AND fan-in
1+Geom(0.6) clipped at 8, OR fan-in Zipf(2) capped at 256, 5 % back edges,
p ~ U[0.8, 0.999].

Metric: edge-message updates per second = 2 * E * sweeps / time, E = the
reference's edge-slot count (sum of |vars(factor)|).

  python bench.py [--gpus N --steps K --warmup W]            this engine
  python bench.py --impl reference [...]                       FastLBP's own code

`value` is device-resident throughput (graph already in HBM, CUDA events on
the engine stream, L2 flushed between steps); `e2e` goes through the C ABI
from host arrays: flbp_engine_create (host layout + H2D) + init + run +
belief D2H per step. Multi-GPU runs are replicas of the same graph on every
rank (a single graph does not shard); `value` sums all ranks' updates over
the slowest rank's time.
"""

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "edge msg updates/s"
UNIT = "updates/s"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--sweeps", type=int, default=200)
    ap.add_argument("--damping", type=float, default=0.1)
    ap.add_argument("--precision", type=int, default=32)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--scale", type=float, default=1.0, help="graph size factor (1.0 = the 1M-variable graph)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target length of the CPU baseline sample")
    ap.add_argument("--e2e-steps", type=int, default=4)
    ap.add_argument("--workload", default="single", choices=["single", "batch", "fl", "adjoint", "bingo", "seq"],
                    help="single: the 1M-variable graph (default); batch: many uneven graphs solved together; "
                         "fl: the fault-localisation graph with its statement ranking against the FP64 oracle; "
                         "adjoint: gradients through unrolled sweeps on 64 graphs of 50k tuples "
                         "(use --sweeps 100 --damping 0 --graphs 64); "
                         "bingo: re-solving after each label, rebuild against incremental clamps; "
                         "seq: the sequential SEQFIX / TOPO schedules against the reference's own")
    ap.add_argument("--graphs", type=int, default=512, help="batch / adjoint workloads: number of graphs")
    ap.add_argument("--every", type=int, default=10, help="adjoint workload: checkpoint interval")
    ap.add_argument("--fd-params", type=int, default=1000, help="adjoint workload: parameters checked by differences")
    ap.add_argument("--extras", default="batched,adjoint,sets",
                    help="sub-records of the default line: comma-separated subset of batched,adjoint,sets, or none")
    ap.add_argument("--forms", default="auto",
                    help="pass forms of the single-graph workload: auto (the autotuner) or F,V (0 staged, 1-2 direct)")
    ap.add_argument("--plan-only", action="store_true",
                    help="start the ranks, deal the batched graphs to them and print the plan; no GPU work")
    return ap.parse_args()


def maybe_spawn(args):
    """`--gpus N` with N > 1 and no launcher: run this script again under
    torch.distributed.run with N processes on this node, one per GPU (rank r
    on local device r). Under a launcher (WORLD_SIZE set) nothing happens."""
    if args.gpus <= 1 or "WORLD_SIZE" in os.environ:
        return
    import socket

    import torch

    if not args.plan_only and torch.cuda.device_count() < args.gpus:
        raise SystemExit("bench.py --gpus %d: only %d CUDA devices are visible" % (args.gpus, torch.cuda.device_count()))
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node=%d" % args.gpus,
           "--master-addr=127.0.0.1", "--master-port=%d" % port, os.path.abspath(__file__)] + sys.argv[1:]
    sys.stdout.flush()
    os.execv(sys.executable, cmd)


def dist_setup(args):
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus and not (world == 1 and args.gpus == 1):
        raise SystemExit("bench.py: %d ranks were started for --gpus %d" % (world, args.gpus))
    gpu = torch.cuda.is_available() and not args.plan_only
    if gpu:
        if torch.cuda.device_count() <= local:
            raise SystemExit("bench.py: rank %d has no CUDA device %d" % (rank, local))
        torch.cuda.set_device(local)
    if world > 1 and not dist.is_initialized():
        dist.init_process_group("nccl" if gpu else "gloo", timeout=datetime.timedelta(seconds=300))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_plan(args, rank, world):
    """--plan-only: every rank takes its share of the batched-serving graphs
    (dealt by size, as the batched sub-record and --workload batch do); rank
    0 prints the plan with the ranks' shares gathered. No GPU work."""
    from fastlbp_b200 import workloads
    from fastlbp_b200.shard import gather_results, partition

    sizes = workloads.config3_sizes(args.graphs)
    mine = partition(sizes, world)[rank]
    plan = gather_results({rank: {"graphs": mine, "tuples": int(sum(sizes[i] for i in mine))}}, world)
    t = allreduce_max(float(len(mine)), world)
    return {"plan": {str(r): plan[r] for r in sorted(plan)}, "n_gpus": world, "graphs": args.graphs,
            "max_graphs_per_rank": int(t)}


def graph_arrays(args):
    """Reference-order arrays of the workload graph (cached per seed/scale)."""
    from fastlbp_b200 import CausalFactorGraph, workloads

    cache = os.path.join(tempfile.gettempdir(), "fastlbp_b200_cfg1_s%d_x%g.npz" % (args.seed, args.scale))
    fl = workloads.config1(args.seed, scale=args.scale)
    if os.path.exists(cache):
        z = np.load(cache)
        return fl, {k: z[k] for k in z.files}
    g = CausalFactorGraph.from_factors(fl)
    a = g.graph_arrays()
    a["n_vars"] = np.int64(a["n_vars"])
    np.savez(cache, **a)
    return fl, a


def batch_graph_arrays(i):
    """Reference-order arrays of graph i of the batched-serving set (cached)."""
    from fastlbp_b200 import CausalFactorGraph, workloads

    cache = os.path.join(tempfile.gettempdir(), "fastlbp_b200_cfg3_s3_g%d.npz" % i)
    if os.path.exists(cache):
        z = np.load(cache)
        return {k: z[k] for k in z.files}
    fl, clamps = workloads.config3_graph(i)
    g = CausalFactorGraph.from_factors(fl)
    g.clamp_labels(clamps)
    a = g.rebuild().graph_arrays()
    a["n_vars"] = np.int64(a["n_vars"])
    np.savez(cache, **a)
    return a


def run_batch(args, rank, world, local):
    """Batched serving: uneven graphs (cfg-0 laws, 1 k-200 k tuple variables,
    1-50 clamps each), per-graph tolerance 1e-6 and at most 500 sweeps, FP32.
    One BatchEngine solve of this rank's graphs against the plain form - one
    engine per graph, solved one after another - on the same graphs; both
    give identical beliefs, which the line reports. Times are wall clock of
    whole solves (init + tolerance run, results on the device), max over
    ranks; graphs are dealt to ranks by size."""
    import torch

    from fastlbp_b200 import BatchEngine, Engine, workloads
    from fastlbp_b200.shard import partition

    tol, maxiter = 1e-6, 500
    sizes = workloads.config3_sizes(args.graphs)
    mine = partition(sizes, world)[rank]
    arrays = [batch_graph_arrays(i) for i in mine]
    Es = np.array([int(a["factor_offsets"][-1]) for a in arrays], np.float64)
    E = int(Es.sum())
    V = sum(int(a["n_vars"]) for a in arrays)
    be = BatchEngine(arrays, precision=32)
    plain = [Engine(a, precision=32) for a in arrays]
    for _ in range(max(1, args.warmup)):  # captures the sweep graphs of every engine
        be.init()
        be.run_batch_tol(tol, maxiter)
        for e in plain:
            e.reset_counts()  # a plain solve is a new engine's (maxiter counts from 0)
            e.init()
            e.run_tol(tol, maxiter, 1e9)
    torch.cuda.synchronize()
    tb, tp = [], []
    for _ in range(args.steps):
        barrier(world)
        t0 = time.perf_counter()
        be.init()
        sweeps, reasons = be.run_batch_tol(tol, maxiter)
        tb.append(time.perf_counter() - t0)
        barrier(world)
        t0 = time.perf_counter()
        psweeps = []
        for e in plain:
            e.reset_counts()
            e.init()
            psweeps.append(e.run_tol(tol, maxiter, 1e9)["sweeps"])
        tp.append(time.perf_counter() - t0)
    allb = be.beliefs()
    diff = max(float(np.max(np.abs(be.beliefs_of(k, allb) - e.beliefs()))) if e.n_vars else 0.0
               for k, e in enumerate(plain))
    t_b = allreduce_max(statistics.median(tb), world)
    t_p = allreduce_max(statistics.median(tp), world)
    n = args.graphs if world > 1 else len(mine)
    line = {"metric": "graphs/s (batched, per-graph tol 1e-6)", "value": n / t_b, "unit": "graphs/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "strong", "dtype": "f32", "data": "synthetic (seeded Bingo-style generator)",
            "config": {"workload": "%d uneven Bingo-style graphs, 1k-200k tuple vars, 1-50 clamps, tol 1e-6, "
                                   "maxiter 500, FP32" % args.graphs,
                       "vars_this_rank": V, "edge_slots_this_rank": E, "graphs_this_rank": len(mine)},
            "plain": {"value": n / t_p, "unit": "graphs/s", "form": "one engine per graph, solved in turn"},
            "batched_over_plain": t_p / t_b,
            "sweeps": {"min": int(sweeps.min()), "median": float(np.median(sweeps)), "max": int(sweeps.max()),
                       "converged": int((reasons == 0).sum()), "same_as_plain": bool(sweeps.tolist() == psweeps)},
            "max_belief_diff_batched_vs_plain": diff,
            "updates_per_s": {"batched": 2.0 * float(np.dot(sweeps, Es)) / t_b,
                              "plain": 2.0 * float(np.dot(sweeps, Es)) / t_p,
                              "note": "sum over graphs of 2 x edge slots x its own sweeps, per second"},
            "seconds": {"batched": t_b, "plain": t_p}}
    be.close()
    for e in plain:
        e.close()
    return line


def adjoint_graph_arrays(i):
    """Reference-order arrays of graph i of the gradient set, with the
    variable indices and labels of its labelled alarms (cached)."""
    from fastlbp_b200 import CausalFactorGraph, workloads

    cache = os.path.join(tempfile.gettempdir(), "fastlbp_b200_cfg4_s4_g%d.npz" % i)
    if os.path.exists(cache):
        z = np.load(cache)
        return {k: z[k] for k in z.files}
    fl, alarms, y = workloads.config4_graph(i)
    g = CausalFactorGraph.from_factors(fl)
    a = g.graph_arrays()
    a["n_vars"] = np.int64(a["n_vars"])
    a["label_vars"] = np.array([g.findVar(int(t)) for t in alarms], np.int64)
    a["labels"] = y
    np.savez(cache, **a)
    return a


def bce_and_grad(b, idx, y):
    """Binary cross-entropy of the beliefs b[idx] against labels y, and dL/db."""
    bb = np.clip(b[idx], 1e-300, 1.0 - 1e-16)
    loss = float(-(y * np.log(bb) + (1 - y) * np.log1p(-bb)).sum())
    g = np.zeros_like(b)
    np.add.at(g, idx, -y / bb + (1 - y) / (1 - bb))
    return loss, g


def run_adjoint(args, rank, world, local):
    """Gradient through unrolled sweeps: 64 graphs of 50 k tuples (config-0
    laws, ~75 k rules each), T = 100 sweeps from init(), checkpoints every
    10, FP32 messages; loss = binary cross-entropy of the beliefs of 200
    labelled alarms per graph (labels Bernoulli(0.3)); gradient with
    respect to every factor's p (rule firing probabilities and input
    priors). All graphs sit in one BatchEngine.

    Timed per step, device-resident (beliefs and gradients in CUDA tensors):
    a forward solve (init + T sweeps + beliefs) and a gradient (checkpointed
    forward + beliefs + the loss gradient in torch + the adjoint backward);
    the same two through the host-buffer calls (beliefs and gradients copied
    to numpy arrays). On rank 0, graph 0 alone is checked in FP64 against
    central differences (eps 1e-6) on sampled parameters, and the FP32
    gradient against the FP64 one."""
    import torch

    from fastlbp_b200 import BatchEngine
    from fastlbp_b200.shard import partition

    T, K, n_graphs = args.sweeps, args.every, args.graphs
    mine = partition(np.ones(n_graphs), world)[rank]
    arrays = [adjoint_graph_arrays(i) for i in mine]
    be = BatchEngine(arrays, precision=args.precision)
    idx = np.concatenate([be.var_off[k] + a["label_vars"] for k, a in enumerate(arrays)])
    y = np.concatenate([a["labels"] for a in arrays])
    E = int(sum(int(a["factor_offsets"][-1]) for a in arrays))
    dev = torch.device("cuda", local)
    idx_d = torch.as_tensor(idx, device=dev)
    y_d = torch.as_tensor(y, device=dev)
    b_d = torch.empty(be.n_vars, dtype=torch.float64, device=dev)
    gp_d = torch.empty(be.n_factors, dtype=torch.float64, device=dev)

    def forward_dev():
        be.init()
        be.run_fixed(T)
        be.beliefs_device(b_d)

    def gradient_dev():
        be.adjoint_forward(T, K, fetch=False)
        be.beliefs_device(b_d)
        bb = b_d[idx_d].clamp(1e-300, 1.0 - 1e-16)
        g = torch.zeros_like(b_d)
        g.index_put_((idx_d,), -y_d / bb + (1 - y_d) / (1 - bb), accumulate=True)
        be.adjoint_backward_device(g, gp_d)

    def forward_host():
        be.init()
        be.run_fixed(T)
        return be.beliefs()

    def gradient_host():
        b = be.adjoint_forward(T, K)
        loss, g = bce_and_grad(b, idx, y)
        gp, _ = be.adjoint_backward(g, want_q=False)
        return loss, gp

    def timed(fn):
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        out = fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0, out

    for _ in range(max(1, args.warmup)):
        forward_dev()
        gradient_dev()
        forward_host()
        gradient_host()
    torch.cuda.synchronize()
    tf, tg, tfh, tgh = [], [], [], []
    for _ in range(args.steps):
        tf.append(timed(forward_dev)[0])
        tg.append(timed(gradient_dev)[0])
        tfh.append(timed(forward_host)[0])
        t, (loss, gp_host) = timed(gradient_host)
        tgh.append(t)
    med = lambda xs: allreduce_max(statistics.median(xs), world)  # noqa: E731
    t_f, t_g, t_fh, t_gh = med(tf), med(tg), med(tfh), med(tgh)
    same = float(np.max(np.abs(gp_d.cpu().numpy() - gp_host))) if be.n_factors else 0.0
    line = {"metric": "adjoint time (gradient of the loss w.r.t. every p)", "value": t_g, "unit": "s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "scaling": "strong", "dtype": "f32" if args.precision == 32 else "f64",
            "data": "synthetic (seeded Bingo-style generator)",
            "config": {"workload": "%d graphs x 50k tuples (config-0 laws, 1.5 rules/tuple), T=%d sweeps from init, "
                                   "checkpoint every %d, BCE on 200 labelled alarms per graph" % (n_graphs, T, K),
                       "graphs_this_rank": len(mine), "vars_this_rank": be.n_vars,
                       "factors_this_rank": be.n_factors, "edge_slots_this_rank": E},
            "seconds": {"forward_solve": t_f, "gradient": t_g, "forward_solve_host_buffers": t_fh,
                        "gradient_host_buffers": t_gh},
            "gradient_over_forward": t_g / t_f,
            "gradient_over_forward_host_buffers": t_gh / t_fh,
            "forward_updates_per_s": 2.0 * E * T * world / t_f,
            "loss": loss,
            "device_vs_host_gradient_max_abs_diff": same}
    be.close()
    if rank == 0 and args.fd_params > 0:
        line["checks"] = adjoint_checks(arrays[0], T, K, args.fd_params)
    return line


def adjoint_checks(a, T, K, n_params):
    """Graph 0 alone: FP64 adjoint against central differences (eps 1e-6) on
    n_params sampled rule probabilities and input priors, and the FP32
    adjoint against the FP64 one."""
    from fastlbp_b200 import Engine

    idx, y = a["label_vars"], a["labels"]
    p0, q0 = np.asarray(a["factor_p"], np.float64).copy(), np.asarray(a["factor_q"], np.float64)
    grads = {}
    for prec in (64, 32):
        e = Engine(a, precision=prec)
        _, g = bce_and_grad(e.adjoint_forward(T, K), idx, y)
        grads[prec] = e.adjoint_backward(g)[0]
        if prec == 32:
            e.close()
        else:
            e64 = e
    g64, g32 = grads[64], grads[32]
    rng = np.random.default_rng(5)
    cand = np.nonzero((p0 > 1e-3) & (p0 < 1 - 1e-3))[0]
    sample = np.sort(rng.choice(cand, size=min(n_params, cand.size), replace=False))
    eps = 1e-6

    def loss(p):
        e64.set_factor_probs(p, q0)
        return bce_and_grad(e64.adjoint_forward(T, K), idx, y)[0]

    t0 = time.perf_counter()
    fd = np.zeros(sample.size)
    for j, I in enumerate(sample):
        pp, pm = p0.copy(), p0.copy()
        pp[I] += eps
        pm[I] -= eps
        fd[j] = (loss(pp) - loss(pm)) / (2 * eps)
    t_fd = time.perf_counter() - t0
    e64.close()
    ga = g64[sample]
    scale = float(np.max(np.abs(g64)))
    floor = 1e-3 * scale
    rel = np.abs(fd - ga) / np.maximum(np.abs(ga), floor)
    big = np.abs(ga) >= floor
    return {"fd": {"params": int(sample.size), "eps": eps, "within_1e-4": int((rel <= 1e-4).sum()),
                   "max_rel_err": float(rel.max()),
                   "max_rel_err_where_grad_ge_1e-3_max": float(rel[big].max()) if big.any() else None,
                   "params_with_grad_ge_1e-3_max": int(big.sum()), "seconds": t_fd,
                   "note": "relative error |fd - g| / max(|g|, 1e-3 max|g|), FP64 engine, graph 0"},
            "fp32_vs_fp64_rel_l2": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
            "grad_max_abs": scale}


def run_bingo(args, rank, world, local):
    """The alarm-ranking loop: after each label (an alarm clamped to its
    value) the graph is solved again (init + tolerance run, tol 1e-6, maxiter
    500, FP32, beliefs to the host). Graph: 50 k tuples with config-0 laws,
    its first 30 labelled alarms in turn. Three forms, each over the same
    label sequence: FastLBP's (clamp the factor graph, rebuild it, build a new
    engine: fl_wrapper.cu:29-45, bingo_wrapper.cu), incremental clamps on one
    engine (flbp_clamp_vars, same results), and incremental clamps with a
    warm start (no init: the previous solution is the starting point).
    Reported: labels/s of each and the largest belief difference to the
    first form."""
    if rank != 0:
        return None
    from fastlbp_b200 import CausalFactorGraph, Engine, workloads

    tol, maxiter, n_labels = 1e-6, 500, 30
    fl, alarms, y = workloads.config4_graph(0)
    labels = [(int(a), int(v)) for a, v in zip(alarms[:n_labels], y[:n_labels])]

    def rebuild_form():
        g = CausalFactorGraph.from_factors(fl)
        out = []
        t0 = time.perf_counter()
        for lab, val in labels:
            g.clamp(g.findVar(lab), val)
            e = Engine(g.rebuild().graph_arrays(), precision=32)
            e.init()
            info = e.run_tol(tol, maxiter, 1e9)
            out.append((info["sweeps"], e.beliefs()))
            e.close()
        return time.perf_counter() - t0, out

    def incremental_form(warm):
        g = CausalFactorGraph.from_factors(fl)
        idx = [g.findVar(lab) for lab, _ in labels]
        e = Engine(g.graph_arrays(), precision=32)
        out = []
        t0 = time.perf_counter()
        if warm:
            e.init()
        for i, (lab, val) in zip(idx, labels):
            e.clamp([i], [val])
            if not warm:
                e.init()
            info = e.run_tol(tol, maxiter, 1e9)
            out.append((info["sweeps"], e.beliefs()))
        dt = time.perf_counter() - t0
        e.close()
        return dt, out

    for _ in range(max(1, args.warmup)):
        incremental_form(False)
    t_r, ref = rebuild_form()
    t_i, inc = incremental_form(False)
    t_w, warm = incremental_form(True)
    diff = lambda a: max(float(np.max(np.abs(x[1] - r[1]))) for x, r in zip(a, ref))  # noqa: E731
    return {"metric": "labels/s (re-solve after each label)", "value": n_labels / t_i, "unit": "labels/s",
            "n_gpus": 1, "steps": 1, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
            "dtype": "f32", "data": "synthetic (seeded Bingo-style generator)",
            "config": {"workload": "50k-tuple Bingo-style graph (config-0 laws), %d labels in turn, tol 1e-6, "
                                   "maxiter 500, FP32, init + tolerance run after each label" % n_labels},
            "forms": {"rebuild": {"labels_per_s": n_labels / t_r, "sweeps": [s for s, _ in ref]},
                      "incremental": {"labels_per_s": n_labels / t_i, "sweeps": [s for s, _ in inc],
                                      "max_belief_diff_vs_rebuild": diff(inc)},
                      "incremental_warm": {"labels_per_s": n_labels / t_w, "sweeps": [s for s, _ in warm],
                                           "max_belief_diff_vs_rebuild": diff(warm)}},
            "incremental_over_rebuild": t_r / t_i}


def run_seq(args, rank, world, local):
    """The sequential schedules (updates=SEQFIX / TOPO): fixed sweeps from
    init() on Bingo-style graphs with config-1 laws, SEQFIX on 100 k tuples
    (50 sweeps), TOPO on 10 k tuples (5 sweeps; its batches hold about three
    edges each), each with the factor order of the first CausalBP of a
    thread. Ours: FP32 and FP64 engines timed with CUDA events around
    run_fixed (kernels only, the graph resident), with the engine's choice of
    launch form and with each form forced (two launches per batch; the whole
    sweep on one thread-block cluster). The reference's own code
    (oracle/_ref/ref_bp, REF_BP_UPDATES) runs the same schedule on the same
    graph in FP64, timed around its run(); its beliefs are compared with the
    FP64 engine's."""
    if rank != 0:
        return None
    import torch

    from fastlbp_b200 import CausalFactorGraph, Engine, workloads

    ref_bp = os.path.join(ROOT, "oracle", "_ref", "ref_bp")
    forms = {}
    for updates, scale, sweeps in (("SEQFIX", 0.1, 50), ("TOPO", 0.01, 5)):
        fl = workloads.config1(args.seed, scale=scale)
        g = CausalFactorGraph.from_factors(fl)
        a = g.graph_arrays()
        E = int(a["factor_offsets"][-1])
        rec = {"tuples": int(round(1_000_000 * scale)), "edge_slots": E, "sweeps": sweeps}
        b64 = None
        for prec in (32, 64):
            e = Engine(a, precision=prec, updates=updates)
            rec["batches"] = e.update_info()[1]
            # 0: the engine's choice, 1: two launches per batch, 2: one cluster per sweep,
            # 3: two launches per batch with programmatic dependent launch
            for kernel, tag in ((0, ""), (1, "_launches"), (2, "_cluster"), (3, "_pdl")):
                e.set_seq_kernel(kernel)
                ts = []
                for rep in range(max(1, args.warmup) + 2):
                    e.init()
                    info = e.run_fixed(sweeps)
                    if rep >= max(1, args.warmup):
                        ts.append(e.last_run_ms() / 1e3)
                rec["fp%d%s_updates_per_s" % (prec, tag)] = 2.0 * E * sweeps / statistics.median(ts)
                rec["fp%d%s_ms_per_sweep" % (prec, tag)] = statistics.median(ts) / sweeps * 1e3
                rec["fp%d%s_launches_per_sweep" % (prec, tag)] = info["launches"] / sweeps
            if prec == 64:
                e.set_seq_kernel(0)
                e.init()
                e.run_fixed(sweeps)
                b64 = dict(zip(g.var_labels().tolist(), e.lowpass().tolist()))
            e.close()
        if os.path.exists(ref_bp) and torch.cuda.is_available():
            path = os.path.join(tempfile.gettempdir(), "fastlbp_seq_%s_x%g.causal_fg" % (updates, scale))
            fl.write(path)
            out = path + ".out"
            r = subprocess.run([ref_bp, path, "-", out, "fixed", str(sweeps), "repeat", "2"], capture_output=True,
                               text=True, timeout=1200, env=dict(os.environ, REF_BP_UPDATES=updates))
            if r.returncode == 0:
                d = json.loads(r.stdout.strip().splitlines()[-1])
                t = d["run_event_all_s"][-1]
                rec["reference_updates_per_s"] = 2.0 * E * sweeps / t
                rec["reference_ms_per_sweep"] = t / sweeps * 1e3
                rec["reference_construct_s"] = d["construct_all_s"][-1]
                rec["fp32_over_reference"] = rec["fp32_updates_per_s"] / rec["reference_updates_per_s"]
                ref = {}
                with open(out) as f:
                    for line in f:
                        k, v = line.split()
                        ref[int(k)] = float(v)
                rec["fp64_max_belief_diff_vs_reference"] = max(abs(b64[k] - ref[k]) for k in ref)
            else:
                rec["reference_unavailable"] = (r.stderr or r.stdout)[-200:]
        forms[updates] = rec
    s0 = forms["SEQFIX"]
    return {"metric": METRIC, "value": s0["fp32_updates_per_s"], "unit": UNIT, "n_gpus": 1, "steps": 2,
            "warmup": args.warmup, "ms_per_step": s0["fp32_ms_per_sweep"] * s0["sweeps"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded Bingo-style generator)",
            "config": {"workload": "sequential schedules: SEQFIX on a 100k-tuple graph (50 sweeps), TOPO on a "
                                   "10k-tuple graph (5 sweeps), fixed sweeps from init, kernels only",
                       "l2": "inputs smaller than L2; every sweep rewrites all messages"},
            "forms": forms}


def run_fl(args, rank, world, local):
    """Fault-localisation graph (200 k tuples, OR fan-in log-uniform 1-4096,
    2 % of tuples clamped as test outcomes), tolerance run tol 1e-6, maxiter
    500, FP32, against the FP64 oracle (OpenMP on all host cores) run the same
    way: belief error, and the ranking of the statements (the input tuples)
    by belief - Spearman correlation and top-k overlap."""
    if rank != 0:
        return None
    import torch
    from scipy.stats import spearmanr

    from fastlbp_b200 import CausalFactorGraph, Engine, workloads

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    fl, clamps = workloads.config2(2, scale=args.scale)
    g = CausalFactorGraph.from_factors(fl)
    g.clamp_labels(clamps)
    g = g.rebuild()
    arr = g.graph_arrays()
    E = int(arr["factor_offsets"][-1])
    # The sweep count of a tolerance run continues across run calls, as the
    # reference's _iters does (it is reset only by construction), so every
    # solve gets a fresh engine; creation is outside the timed region.
    times = []
    for i in range(max(1, args.warmup) + args.steps):
        eng = Engine(arr, precision=args.precision)
        eng.init()
        info = eng.run_tol(1e-6, 500, 1e9)
        if i >= max(1, args.warmup):
            times.append(eng.last_run_ms())
            b = eng.beliefs()
            st = eng.stats()
        eng.close()
    og = O.OracleGraph.from_factors(fl)
    og.clamp_labels(clamps)
    og = og.rebuild()
    bp = O.OracleBP(og, threads=os.cpu_count() or 1)
    bp.init()
    t0 = time.perf_counter()
    bp.run(1e-6, 500, 1e9)
    t_cpu = time.perf_counter() - t0
    bo = bp.beliefs()
    # The same recurrence in FP64 log-odds (no underflow), and the reference
    # arithmetic once more with every belief marked that depends on a
    # probability product that underflowed to an exact zero.
    bl = O.OracleBP(og, threads=os.cpu_count() or 1, arith="lodds")
    bl.init()
    bl.run(1e-6, 500, 1e9)
    b_lo = bl.beliefs()
    bt = O.OracleBP(og, threads=os.cpu_count() or 1, arith="track")
    bt.init()
    bt.run(1e-6, 500, 1e9)
    tainted, n_uf = bt.underflow()
    off_ref = np.abs(b - bo) > 1e-5
    off_ref_nan = np.isnan(b) != np.isnan(bo)
    # the same comparison after a few sweeps, before any chaotic growth of rounding differences
    e10 = Engine(arr, precision=args.precision)
    e10.init()
    e10.run_fixed(10)
    b10 = e10.beliefs()
    e10.close()
    bp10 = O.OracleBP(og, threads=os.cpu_count() or 1)
    bp10.init()
    bp10.run_fixed(1e-6, 10, 1)
    err10 = float(np.nanmax(np.abs(b10 - bp10.lowpass())))
    labels = g.var_labels()
    stm = np.searchsorted(labels, np.arange(int(fl.info["n_inputs"])))
    stm = stm[(stm < labels.size)]
    stm = stm[labels[stm] < fl.info["n_inputs"]]
    rho = float(spearmanr(b[stm], bo[stm]).statistic)
    rho_lo = float(spearmanr(b[stm], b_lo[stm]).statistic)
    top = {}
    for k in (10, 100):
        a_ = set(stm[np.argsort(-b[stm], kind="stable")[:k]].tolist())
        o_ = set(stm[np.argsort(-bo[stm], kind="stable")[:k]].tolist())
        top["top%d_overlap" % k] = len(a_ & o_) / k
    ms = statistics.median(times)
    return {"metric": "edge msg updates/s (tolerance run)", "value": 2.0 * E * info["sweeps"] / (ms / 1e3),
            "unit": "updates/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "dtype": "f32" if args.precision == 32 else "f64", "data": "synthetic (seeded fault-localisation-shaped generator)",
            "config": {"workload": "fault localisation, %d tuples, OR fan-in log-uniform 1-4096, %d clamps, tol 1e-6, "
                                   "maxiter 500, FP%d" % (fl.info["n_tuples"], len(clamps), args.precision),
                       "vars": int(arr["n_vars"]), "edge_slots": E, "warp_factors": st["warp_factors"],
                       "huge_factors": st["huge_factors"]},
            "ms_per_solve": ms, "sweeps": info["sweeps"], "oracle_sweeps": bp.iters,
            "max_belief_error_vs_fp64_oracle": float(np.nanmax(np.abs(b - bo))),
            "belief_error_quantiles": {str(qq): float(np.nanquantile(np.abs(b - bo), qq)) for qq in (0.5, 0.99, 0.999)},
            "vars_off_by_more_than_1e-5": int(np.sum(np.abs(b - bo) > 1e-5)),
            "max_belief_error_after_10_sweeps": err10,
            "oracle_final_residual_converged": bool(bp.iters < 500),
            "nan_beliefs": {"engine": int(np.isnan(b).sum()), "oracle": int(np.isnan(bo).sum()),
                            "same_positions": bool(np.array_equal(np.isnan(b), np.isnan(bo)))},
            "ranking": dict(statements=int(stm.size), spearman=rho, spearman_vs_logodds_oracle=rho_lo, **top),
            "vs_logodds_oracle": {
                "max_belief_error": float(np.nanmax(np.abs(b - b_lo))),
                "vars_off_by_more_than_1e-5": int(np.sum(np.abs(b - b_lo) > 1e-5)),
                "nan_same_positions": bool(np.array_equal(np.isnan(b), np.isnan(b_lo))),
                "oracle_sweeps": bl.iters,
                "oracle": "the PARALL recurrence in FP64 log-odds (no probability products, no underflow)"},
            "underflow": {
                "events": n_uf, "tainted_vars": int(tainted.sum()),
                "off_by_more_than_1e-5_vs_reference_arith": int(off_ref.sum()),
                "of_those_tainted": int((off_ref & tainted).sum()),
                "of_those_untainted": int((off_ref & ~tainted).sum()),
                "nan_mismatch_untainted": int((off_ref_nan & ~tainted).sum()),
                "tracked_run_sweeps": bt.iters,
                "meaning": "tainted: the reference-arithmetic belief depends on a probability product that "
                           "underflowed to an exact zero"},
            "cpu_oracle_seconds": t_cpu, "cpu_cores": os.cpu_count()}


class Clocks:
    """nvidia-smi samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), "fastlbp_clocks_%d_%d.csv" % (os.getpid(), index))

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic():
    """DRAM bytes per launch from the committed ncu summary (profiles/)."""
    path = os.path.join(ROOT, "profiles", "traffic_cfg1.txt")
    out = {}
    if os.path.exists(path):
        for line in open(path):
            if line.startswith("TRAFFIC "):
                _, name, val = line.split()[:3]
                out[name] = float(val)
    return out


def oracle_leg(fl, args, sweeps):
    """The FP64 oracle (CPU restatement of the reference's PARALL arithmetic),
    OpenMP over all host cores, on the same graph: init + `sweeps` sweeps with
    the run's damping, then beliefs. Its time is the CPU baseline; its
    beliefs are the parity reference of the engine's FP32 ones."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O

    cores = os.cpu_count() or 1
    g = O.OracleGraph.from_factors(fl)
    bp = O.OracleBP(g, damping=args.damping, threads=cores)
    bp.init()
    E = bp.E
    t0 = time.perf_counter()
    bp.run_fixed(1e-9, sweeps, 1)
    dt = time.perf_counter() - t0
    base = {"value": 2.0 * E * sweeps / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": "%d FP64 sweeps of the same graph (damping %g) from init by the oracle's OpenMP loop, %.1f s"
                      % (sweeps, args.damping, dt)}
    return base, bp.lowpass()


def sweep_timing(eng, args, stream, flush, world):
    """Device time of `steps` steps (init + run_fixed(sweeps) + beliefs) with
    CUDA events on the engine stream, L2 flushed before every step; max over
    ranks. Returns (total ms, launches, clock record)."""
    import torch

    for _ in range(args.warmup):
        eng.init()
        eng.run_fixed(args.sweeps)
    torch.cuda.synchronize()
    barrier(world)
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    times, launches = [], 0
    for _ in range(args.steps):
        flush.zero_()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        eng.init()
        info = eng.run_fixed(args.sweeps)
        e.record(stream)
        times.append((s, e))
        launches += info["launches"]
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    total_ms = allreduce_max(sum(s.elapsed_time(e) for s, e in times), world)
    return total_ms, launches, clk


def pass_timing(eng, args, flush):
    """Average device time of each pass (ms) with the sweeps replayed from
    CUDA graphs: the engine's timing mode records CUDA events by event nodes
    of the captured graph around every factor and variable pass."""
    import torch

    eng.set_kernel_timing(True)
    for _ in range(max(1, min(args.steps, 3))):
        flush.zero_()
        eng.init()
        eng.run_fixed(args.sweeps)
    torch.cuda.synchronize()
    f_ms, v_ms, f_n, v_n = eng.kernel_times()
    eng.set_kernel_timing(False)
    return {"factor_pass": f_ms / max(f_n, 1), "var_pass": v_ms / max(v_n, 1)}


def run_ours(args, rank, world, local):
    import torch

    from fastlbp_b200 import Engine

    fl, arr = graph_arrays(args)
    E = int(arr["factor_offsets"][-1])
    F = int(arr["factor_offsets"].size - 1)
    V = int(arr["n_vars"])
    stream = torch.cuda.current_stream()
    eng = Engine(arr, precision=args.precision, damping=args.damping, stream=stream.cuda_stream)
    if args.forms == "auto":
        tuned = eng.autotune(args.sweeps)
    else:
        ff, vf = (int(x) for x in args.forms.split(","))
        eng.set_tuning(ff, vf)
        tuned = None
    forms = eng.tuning()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    total_ms, launches, clk = sweep_timing(eng, args, stream, flush, world)
    updates = 2.0 * E * args.sweeps * args.steps * world
    value = updates / (total_ms / 1e3)
    b_engine = eng.beliefs()  # after init + the last step's sweeps

    per = pass_timing(eng, args, flush)
    # Algorithmic bytes per launch (per-unit figures x units): factor pass
    # 12 B per edge slot + 16 B per factor; variable pass 12 B per slot + 12 B per variable.
    # Damping mixes every slot's new f->v message with its previous one, so a
    # damped sweep must also read the previous message of every slot once:
    # + 4 B per slot, counted in the pass that applies the damping (the
    # variable pass). The undamped figures are kept beside them.
    alg_undamped = {"factor_pass": 12.0 * E + 16.0 * F, "var_pass": 12.0 * E + 12.0 * V}
    damp_bytes = 4.0 * E if args.damping != 0.0 else 0.0
    alg = {"factor_pass": alg_undamped["factor_pass"], "var_pass": alg_undamped["var_pass"] + damp_bytes}
    dom = max(per, key=per.get)
    peak, peak_kind = peaks()
    traffic = ncu_traffic().get(dom)
    sweep_ms = total_ms / (args.steps * args.sweeps)
    # Each pass's time in the plain graph-replayed sweeps of the timed steps:
    # its share of the event-timed sweep (event nodes add a little time to
    # every pass) times the graph-replayed sweep time.
    replay = {k: v / sum(per.values()) * sweep_ms for k, v in per.items()}
    achieved = alg[dom] / (replay[dom] / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": traffic, "alg_bytes_per_launch": alg[dom],
                "launch_ms": {k: round(v, 5) for k, v in replay.items()},
                "launch_ms_event_mode": {k: round(v, 5) for k, v in per.items()},
                "frac_event_mode": round(alg[dom] / (per[dom] / 1e3) / 1e9 / peak, 4),
                "timing": "pass share of the sweep (CUDA events from event nodes of graph-replayed sweeps) x the "
                          "graph-replayed sweep time of the timed steps (CUDA events on the launching stream)",
                "per_kernel": {k: {"achieved": round(alg[k] / (replay[k] / 1e3) / 1e9, 1),
                                   "frac": round(alg[k] / (replay[k] / 1e3) / 1e9 / peak, 4),
                                   "alg_bytes_per_launch": alg[k], "traffic": ncu_traffic().get(k)}
                               for k in replay},
                "sweep_ms_graph_replay": round(sweep_ms, 5),
                "sweep_frac": round((24.0 * E + 16.0 * F + 12.0 * V + damp_bytes) / (sweep_ms / 1e3) / 1e9 / peak, 4),
                "damping_bytes_per_sweep": damp_bytes,
                "undamped_bytes": {"frac": round(alg_undamped[dom] / (replay[dom] / 1e3) / 1e9 / peak, 4),
                                   "alg_bytes_per_launch": alg_undamped[dom],
                                   "sweep_frac": round((24.0 * E + 16.0 * F + 12.0 * V) / (sweep_ms / 1e3) / 1e9 / peak,
                                                       4),
                                   "note": "per-unit figures without the previous-message read that damping needs"}}

    # End to end through the C ABI with host arrays.
    e2e_ms, h2d, phases = [], 0, []
    out = np.zeros(V)
    for i in range(args.e2e_steps + 1 if args.e2e_steps > 0 else 0):
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        t0 = time.perf_counter()
        eng2 = Engine(arr, precision=args.precision, damping=args.damping, stream=stream.cuda_stream)
        eng2.set_tuning(forms["factor_form"], forms["var_form"])
        t1 = time.perf_counter()
        eng2.init()
        eng2.run_fixed(args.sweeps)
        t2 = time.perf_counter()
        eng2.beliefs(out)  # one host buffer over the steps, as a serving loop keeps it
        e.record(stream)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        wall = (t3 - t0) * 1e3
        st2 = eng2.stats()
        h2d = st2["h2d_bytes"]
        phases.append({"create": (t1 - t0) * 1e3, "init_run": (t2 - t1) * 1e3, "beliefs": (t3 - t2) * 1e3,
                       "create_layout": st2["create_us_layout"] / 1e3, "create_alloc": st2["create_us_alloc"] / 1e3,
                       "create_upload": st2["create_us_upload"] / 1e3, "create_rest": st2["create_us_rest"] / 1e3})
        eng2.close()
        if i > 0:  # the first call pays one-time kernel configuration
            e2e_ms.append(max(s.elapsed_time(e), wall))
    # median over steps: a step's host allocations and frees vary with the host's memory state
    e2e_mean = statistics.median(e2e_ms) if e2e_ms else float("nan")  # --e2e-steps 0: profiling runs only
    e2e_val = 2.0 * E * args.sweeps * world / (allreduce_max(e2e_mean, world) / 1e3)

    # Like for like with the reference arm (which has no damping): the same
    # sweeps undamped, in FP32 and in FP64 (the reference's own precision).
    undamped = {}
    if args.damping != 0.0:
        for prec in (32, 64):
            e0 = Engine(arr, precision=prec, damping=0.0, stream=stream.cuda_stream)
            if prec == args.precision:
                e0.set_tuning(forms["factor_form"], forms["var_form"])
            a0 = argparse.Namespace(**vars(args))
            a0.steps = max(3, min(args.steps, 5))
            ms0, _, _ = sweep_timing(e0, a0, stream, flush, world)
            undamped["fp%d" % prec] = {"value": 2.0 * E * args.sweeps * a0.steps * world / (ms0 / 1e3),
                                       "ms_per_step": ms0 / a0.steps}
            e0.close()

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.precision == 32 else "f64",
            "data": "synthetic (seeded Bingo-style generator)",
            "config": {"workload": "1M-tuple Bingo-style graph, 200 PARALL sweeps, damping 0.1, FP32 log-odds",
                       "vars": V, "factors": F, "edge_slots": E, "sweeps": args.sweeps, "damping": args.damping,
                       "seed": args.seed, "scale": args.scale, "replicas": world,
                       "l2": "256 MB buffer written between timed steps; working set > L2",
                       "kernel_forms": eng.tuning(), "autotune": tuned},
            "roofline": roofline, "clocks": clk, "gpu_launches": launches,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": V * 8,
                    "ms_per_step": e2e_mean,
                    "phases_ms": {k: round(statistics.median(p[k] for p in phases[1:]), 2) for k in phases[0]}
                    if len(phases) > 1 else None},
            "undamped": undamped}
    eng.close()
    if rank == 0 and world == 1 and args.cpu_seconds > 0:
        base, b_oracle = oracle_leg(fl, args, args.sweeps)
        line["cpu_baseline"] = base
        nan_same = bool(np.array_equal(np.isnan(b_engine), np.isnan(b_oracle)))
        err = float(np.nanmax(np.abs(b_engine - b_oracle)))
        line["parity"] = {"belief_error_vs_fp64_oracle": err, "tolerance": 1e-5, "within": bool(err <= 1e-5 and nan_same),
                          "vars_compared": V, "nan_positions_equal": nan_same,
                          "oracle": "reference arithmetic, FP64, init + %d sweeps, damping %g" % (args.sweeps, args.damping)}
    extras = [x for x in args.extras.split(",") if x and x != "none"]
    for name in extras:
        try:
            line[name] = {"batched": batched_record, "adjoint": adjoint_record,
                          "sets": sets_record}[name](args, rank, world, local)
        except Exception as ex:  # a sub-record must not cost the main line
            line[name] = {"error": "%s: %s" % (type(ex).__name__, ex)}
    return line


def _make_arrays(job):
    kind, i = job
    (batch_graph_arrays if kind == "batch" else adjoint_graph_arrays)(i)
    return i


def arrays_parallel(kind, indices):
    """Graph arrays of the batched-serving (kind "batch") or gradient
    ("adjoint") sets, generated on all host cores (a spawn-started process
    pool: no worker inherits a CUDA context) and cached in the temp dir."""
    import multiprocessing as mp

    todo = [i for i in indices if not os.path.exists(os.path.join(
        tempfile.gettempdir(), ("fastlbp_b200_cfg3_s3_g%d.npz" if kind == "batch" else "fastlbp_b200_cfg4_s4_g%d.npz") % i))]
    if len(todo) > 1:
        with mp.get_context("spawn").Pool(min(len(todo), os.cpu_count() or 1)) as pool:
            pool.map(_make_arrays, [(kind, i) for i in todo], chunksize=1)
    load = batch_graph_arrays if kind == "batch" else adjoint_graph_arrays
    return [load(i) for i in indices]


def batched_record(args, rank, world, local):
    """Sub-record of the default line: batched serving (512 uneven Bingo-style
    graphs, 1 k-200 k tuples, 1-50 clamps each, per-graph tol 1e-6, maxiter
    500, FP32) in one BatchEngine against the plain form (one engine per
    graph, solved in turn) on the same graphs; graphs dealt to ranks by size.
    Median of 5 steps of each, device work timed by the wall clock around
    whole solves (init + run, results on the device), max over ranks."""
    import torch

    from fastlbp_b200 import BatchEngine, Engine, workloads
    from fastlbp_b200.shard import partition

    tol, maxiter, steps = 1e-6, 500, 5
    sizes = workloads.config3_sizes(args.graphs)
    mine = partition(sizes, world)[rank]
    arrays = arrays_parallel("batch", mine)
    be = BatchEngine(arrays, precision=32)
    plain = [Engine(a, precision=32) for a in arrays]
    tuned = be.autotune_batch(tol, maxiter)
    for e in plain:  # each plain engine takes the tuner's choice for its size class (timed once per class)
        e.autotune(maxiter, tol=tol, reps=2)
    plain_forms = sorted({(e.tuning()["factor_form"], e.tuning()["var_form"]) for e in plain})
    be.init()
    be.run_batch_tol(tol, maxiter)  # captures the sweep graphs
    # A plain solve is a new engine's: the sweep count that maxiter limits
    # and the tolerance rule's previous beliefs start afresh each time
    # (as the batched engine's per-graph state does).
    for e in plain:
        e.reset_counts()
        e.init()
        e.run_tol(tol, maxiter, 1e9)
    torch.cuda.synchronize()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    tb, tp = [], []
    for _ in range(steps):
        barrier(world)
        t0 = time.perf_counter()
        be.init()
        sweeps, reasons = be.run_batch_tol(tol, maxiter)
        tb.append(time.perf_counter() - t0)
        barrier(world)
        t0 = time.perf_counter()
        psweeps = []
        for e in plain:
            e.reset_counts()
            e.init()
            psweeps.append(e.run_tol(tol, maxiter, 1e9)["sweeps"])
        tp.append(time.perf_counter() - t0)
    clk = clocks.stop()
    allb = be.beliefs()
    diff = max((float(np.max(np.abs(be.beliefs_of(k, allb) - e.beliefs()))) if e.n_vars else 0.0
                for k, e in enumerate(plain)), default=0.0)
    t_b = allreduce_max(statistics.median(tb), world)
    t_p = allreduce_max(statistics.median(tp), world)
    E = float(sum(int(a["factor_offsets"][-1]) for a in arrays))
    rec = {"metric": "graphs/s (batched, per-graph tol 1e-6)", "value": args.graphs / t_b, "unit": "graphs/s",
           "plain": args.graphs / t_p, "batched_over_plain": t_p / t_b, "steps": steps, "statistic": "median",
           "graphs": args.graphs, "graphs_this_rank": len(mine), "edge_slots_this_rank": E,
           "sweeps": {"min": int(sweeps.min()), "median": float(np.median(sweeps)), "max": int(sweeps.max()),
                      "same_as_plain": bool(sweeps.tolist() == psweeps)},
           "max_belief_diff_batched_vs_plain": diff, "seconds": {"batched": t_b, "plain": t_p},
           "kernel_forms": be.tuning(), "plain_kernel_forms": [list(x) for x in plain_forms], "clocks": clk,
           "scaling": "strong: the graphs are dealt to the ranks"}
    be.close()
    for e in plain:
        e.close()
    return rec


def sets_record(args, rank, world, local):
    """Sub-record of the default line: the alarm-ranking loop's re-solves as
    evidence sets. One 50 k-tuple graph (config-0 laws) and its first 64
    labelled alarms; set k clamps labels 0..k (the evidence after the k-th
    label), FP32, init + tolerance run (tol 1e-6, maxiter 500) per set. One
    SetsEngine over all sets against one engine per set (flbp_clamp_vars on
    a new engine, solved in turn), both built before timing (construction
    seconds reported apart); sets dealt to ranks. Median of 5 steps of
    each, whole solves timed by the wall clock (results on the device),
    max over ranks."""
    import torch

    from fastlbp_b200 import CausalFactorGraph, Engine, SetsEngine, workloads
    from fastlbp_b200.shard import partition

    tol, maxiter, steps, n_sets = 1e-6, 500, 5, 64
    fl, alarms, y = workloads.config4_graph(0)
    g = CausalFactorGraph.from_factors(fl)
    arrays = g.graph_arrays()
    idx = [g.findVar(int(a)) for a in alarms[:n_sets]]
    vals = [int(v) for v in y[:n_sets]]
    mine = partition(np.ones(n_sets), world)[rank]
    sets = [{idx[j]: vals[j] for j in range(k + 1)} for k in mine]
    t0 = time.perf_counter()
    se = SetsEngine(arrays, sets, precision=32)
    t_create_sets = time.perf_counter() - t0
    t0 = time.perf_counter()
    sep = []
    for cl in sets:
        e = Engine(arrays, precision=32)
        e.set_tuning(1, 1)  # the direct form of the sets engine
        e.clamp(list(cl.keys()), list(cl.values()))
        sep.append(e)
    t_create_sep = time.perf_counter() - t0
    se.init()
    se.run_sets_tol(tol, maxiter)  # captures the sweep graphs
    for e in sep:
        e.reset_counts()
        e.init()
        e.run_tol(tol, maxiter, 1e9)
    torch.cuda.synchronize()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    ts, tp = [], []
    for _ in range(steps):
        barrier(world)
        t0 = time.perf_counter()
        se.init()
        sweeps, _ = se.run_sets_tol(tol, maxiter)
        ts.append(time.perf_counter() - t0)
        barrier(world)
        t0 = time.perf_counter()
        psweeps = []
        for e in sep:
            e.reset_counts()
            e.init()
            psweeps.append(e.run_tol(tol, maxiter, 1e9)["sweeps"])
        tp.append(time.perf_counter() - t0)
    clk = clocks.stop()
    got = se.beliefs()
    diff = max(float(np.nanmax(np.abs(got[k] - e.beliefs()))) for k, e in enumerate(sep))
    t_s = allreduce_max(statistics.median(ts), world)
    t_p = allreduce_max(statistics.median(tp), world)
    rec = {"metric": "evidence sets/s (tol 1e-6)", "value": n_sets / t_s, "unit": "sets/s",
           "separate": n_sets / t_p, "sets_over_separate": t_p / t_s, "steps": steps, "statistic": "median",
           "sets": n_sets, "sets_this_rank": len(mine), "edge_slots": int(arrays["factor_offsets"][-1]),
           "sweeps": {"min": int(sweeps.min()), "median": float(np.median(sweeps)), "max": int(sweeps.max()),
                      "same_as_separate": bool(sweeps.tolist() == psweeps)},
           "max_belief_diff_sets_vs_separate": diff, "seconds": {"sets": t_s, "separate": t_p},
           "construct_seconds": {"sets": t_create_sets, "separate": t_create_sep}, "clocks": clk,
           "scaling": "strong: the sets are dealt to the ranks"}
    se.close()
    for e in sep:
        e.close()
    return rec


def adjoint_record(args, rank, world, local):
    """Sub-record of the default line: gradient through T = 100 undamped
    sweeps from init (checkpoints every 10, FP32) of the BCE loss on 200
    labelled alarms per graph, 64 graphs of 50 k tuples in one BatchEngine
    (graphs dealt to ranks), against a forward solve (init + 100 sweeps +
    beliefs) of the same engine; device buffers. Median of 5 steps, max over
    ranks. The gradient is checked against central differences by
    --workload adjoint and the tests."""
    import torch

    from fastlbp_b200 import BatchEngine
    from fastlbp_b200.shard import partition

    T, K, n_graphs, steps = 100, 10, 64, 5
    mine = partition(np.ones(n_graphs), world)[rank]
    arrays = arrays_parallel("adjoint", mine)
    be = BatchEngine(arrays, precision=32)
    idx = np.concatenate([be.var_off[k] + a["label_vars"] for k, a in enumerate(arrays)])
    y = np.concatenate([a["labels"] for a in arrays])
    dev = torch.device("cuda", local)
    idx_d, y_d = torch.as_tensor(idx, device=dev), torch.as_tensor(y, device=dev)
    b_d = torch.empty(be.n_vars, dtype=torch.float64, device=dev)
    gp_d = torch.empty(be.n_factors, dtype=torch.float64, device=dev)

    def forward():
        be.init()
        be.run_fixed(T)
        be.beliefs_device(b_d)

    def gradient():
        be.adjoint_forward(T, K, fetch=False)
        be.beliefs_device(b_d)
        bb = b_d[idx_d].clamp(1e-300, 1.0 - 1e-16)
        g = torch.zeros_like(b_d)
        g.index_put_((idx_d,), -y_d / bb + (1 - y_d) / (1 - bb), accumulate=True)
        be.adjoint_backward_device(g, gp_d)

    def timed(fn):
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    forward()
    gradient()
    clocks = Clocks(torch.cuda.current_device())
    clocks.start()
    tf, tg = [], []
    for _ in range(steps):
        tf.append(timed(forward))
        tg.append(timed(gradient))
    clk = clocks.stop()
    t_f = allreduce_max(statistics.median(tf), world)
    t_g = allreduce_max(statistics.median(tg), world)
    rec = {"metric": "gradient time / forward-solve time", "value": t_g / t_f, "unit": "ratio",
           "higher_is_better": False, "target": 3.0, "steps": steps, "statistic": "median",
           "seconds": {"forward_solve": t_f, "gradient": t_g}, "graphs": n_graphs, "graphs_this_rank": len(mine),
           "sweeps": T, "checkpoint_every": K, "finite_gradient": bool(torch.isfinite(gp_d).all().item()),
           "clocks": clk}
    be.close()
    return rec


def run_reference(args, rank, world):
    """FastLBP's own code (oracle/_ref/ref_bp, compiled from its sources) on the
    same graph. The reference path exists only as GPU code; it has no damping,
    so it runs the same sweep count undamped."""
    if rank != 0:
        return None
    # The graph file comes from the seeded generator alone (plain Python and
    # numpy): nothing of this repository's library is loaded in this arm.
    from fastlbp_b200 import workloads

    fl = workloads.config1(args.seed, scale=args.scale)
    ref_bp = os.path.join(ROOT, "oracle", "_ref", "ref_bp")
    base = {"metric": METRIC, "unit": UNIT, "impl": "reference", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "data": "synthetic (seeded Bingo-style generator)",
            "config": {"workload": "1M-tuple Bingo-style graph, 200 PARALL sweeps, FP64 (reference has no damping)",
                       "sweeps": args.sweeps, "seed": args.seed, "scale": args.scale}}
    import torch
    if not (os.path.exists(ref_bp) and torch.cuda.is_available()):
        return dict(base, unavailable="oracle/_ref/ref_bp not built on this machine")
    path = os.path.join(tempfile.gettempdir(), "fastlbp_ref_cfg1_s%d_x%g.causal_fg" % (args.seed, args.scale))
    if not os.path.exists(path):
        fl.write(path)
    rep = args.warmup + args.steps
    r = subprocess.run([ref_bp, path, "-", "-", "fixed", str(args.sweeps), "repeat", str(rep)],
                       capture_output=True, text=True, timeout=3000)
    if r.returncode != 0:
        return dict(base, unavailable="reference run failed: " + (r.stderr or r.stdout)[-200:])
    d = json.loads(r.stdout.strip().splitlines()[-1])
    E = int(d["slots"])
    base["config"]["edge_slots"] = E
    runs = d["run_event_all_s"][args.warmup:]
    cons = d["construct_all_s"][args.warmup:]
    value = 2.0 * E * args.sweeps / statistics.mean(runs)
    # end to end as a FastLBP user pays it per solve: construct (host edge
    # records + H2D) + run; the file read is reported apart
    e2e_s = statistics.mean(runs) + statistics.mean(cons)
    line = dict(base, value=value, ms_per_step=statistics.mean(runs) * 1e3, dtype="f64",
                reference_construct_s=statistics.mean(cons), reference_read_s=d["read_s"])
    line["cpu_baseline"] = {"value": value, "unit": UNIT, "kind": "reference", "cores": 1,
                            "sample": "FastLBP CausalBP (updates=PARALL) built from its sources, run(tol, %d, 1) "
                                      "on the B200 from one host thread; its path has no CPU implementation" % args.sweeps}
    line["e2e"] = {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                   "excludes": "CausalBP construction (host edge records + their copy to the device) and the "
                               "file read; see e2e_with_construct"}
    line["e2e_with_construct"] = {"value": 2.0 * E * args.sweeps / e2e_s, "unit": UNIT, "ms_per_step": e2e_s * 1e3,
                                  "includes": "CausalBP construction + run(tol, %d, 1), per solve" % args.sweeps}
    line["gpu_launches"] = None
    return line


def main():
    args = parse()
    maybe_spawn(args)
    rank, world, local = dist_setup(args)
    if args.plan_only:
        line = run_plan(args, rank, world)
    elif args.impl == "reference":
        line = run_reference(args, rank, world)
    elif args.workload == "batch":
        line = run_batch(args, rank, world, local)
    elif args.workload == "fl":
        line = run_fl(args, rank, world, local)
    elif args.workload == "adjoint":
        line = run_adjoint(args, rank, world, local)
    elif args.workload == "bingo":
        line = run_bingo(args, rank, world, local)
    elif args.workload == "seq":
        line = run_seq(args, rank, world, local)
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
