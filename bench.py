#!/usr/bin/env python
"""Benchmark: whole Louvain runs on one B200 per rank, nido's options.

Default workload (one GPU): the many-graph batch the metric is quoted on
("graphs/s, p99 latency batched vs plain"): 4,096 independent graphs, vertex
counts log-uniform in [100, 1e6] scaled to a total of 1.5e9 directed edges,
half SBM and half R-MAT, average degree U[8, 64], integer weights U{1..8} as
FP64, seed 4, nido defaults -b 2 -t 1e-6 -i 500.  A step is one batched run of
every graph to completion (all phases, coarsening included) from the packed
CSR resident in HBM.  The same line carries the plain comparison (the same
engine one graph at a time on a systematic sample of the graphs) and the
serving replay's p50/p99 latency (Poisson arrivals of the serving workload).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload many|serve|rmat22|planted|sbm]

Prints one JSON line.  `value` is graphs/s over all ranks from CUDA events on
the engine's stream; `e2e` is the same metric through the public C ABI with
host buffers (pinned H2D upload of the CSR, run, D2H of the partition inside
the timed region).  `roofline` covers the move phase (all degree-tier kernels
of a sweep): algorithmic bytes 16*E + 32*V per sweep (int32 ids, FP64
weights) over the device time of the move kernels.  For N > 1 the ranks are
independent replicas (no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0}

# DRAM bytes the move kernels move per algorithmic byte (16 B per edge +
# 32 B per vertex per sweep): ncu dram__bytes_read.sum + dram__bytes_write.sum
# of one-kernel, two-launch captures of the warp, CTA-S, CTA-M, CTA-XA and
# CTA-XL tiers on R-MAT scale 20, edge-weighted (cold cache per launch).
MOVE_TRAFFIC_PER_ALGO_BYTE = 1.01


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except OSError:
        return PEAKS_FALLBACK, "fallback"


WORKLOADS = {
    "rmat22": dict(desc="R-MAT scale 22 (4,194,304 vertices), edge factor 16, (0.57,0.19,0.19,0.05), "
                        "symmetrised, self-loops and duplicates removed, weights 1.0, seed 2",
                   nbatches=2, tau=1e-6),
    "rmat20": dict(desc="R-MAT scale 20 (1,048,576 vertices), edge factor 16, (0.57,0.19,0.19,0.05), "
                        "symmetrised, self-loops and duplicates removed, weights 1.0, seed 2 (profiling case)",
                   nbatches=2, tau=1e-6),
    "planted": dict(desc="planted partition 65,536 vertices (256 blocks of 256), average degree 32, 80% intra, "
                         "weights U[0.5,1.5], duplicates summed, seed 1", nbatches=1, tau=1e-6),
    "sbm": dict(desc="SBM 16,777,216 vertices, power-law community sizes (2.5, 16..65,536), average degree 32, "
                     "70% intra, lognormal(0,0.5) weights, seed 3", nbatches=32, tau=1e-6),
    "serve": dict(desc="serving stream: Poisson arrivals, vertex counts log-uniform [1e3, 1e7], 50/50 SBM "
                       "(power-law communities 2.5, 16..65,536, average degree 32, 70% intra) / R-MAT "
                       "(edge factor 16), weights U[0.5,1.5], HBM budget 150 GB, seed 5", nbatches=2, tau=1e-6),
    "many": dict(desc="many-graph batch: 4,096 independent graphs, vertex counts log-uniform [100, 1e6] scaled "
                      "to a total of 1.5e9 directed edges (clamped >= 100), 50/50 SBM (power-law communities "
                      "2.5, 16..65,536, 70% intra) / R-MAT (0.57,0.19,0.19,0.05), average degree U[8,64], "
                      "integer weights U{1..8} as FP64, seed 4", nbatches=2, tau=1e-6),
}


def config_of(args, wl, world):
    """The workload's description: the same keys and values on both arms."""
    c = {"workload": args.workload, "graph": wl["desc"], "nbatches": wl["nbatches"], "tau": wl["tau"],
         "max_iter": 500, "parallelism": f"replicas x{world}",
         "l2": ("CSR of 24 MB fits in L2; runs are not flushed" if args.workload == "planted"
                else "inputs larger than L2 (126 MB): no flush needed")}
    if args.workload == "many":
        c["ngraphs"] = args.many_graphs
        c["edge_cap"] = args.many_edges
        if args.many_graphs != 4096 or args.many_edges != 1.5e9:
            c["graph"] += f" [reduced: {args.many_graphs} graphs, {args.many_edges:.3g} edge cap]"
    if args.workload == "serve":
        c.update(requests=args.serve_requests, rate_per_s=args.serve_rate, vmax=args.serve_vmax,
                 workers=args.serve_workers, hbm_budget_gb=args.serve_budget_gb)
    return c


def make_graph(capi, name):
    from nido_b200 import workloads
    return workloads.single_graph(name)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def reduce_max(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


SMALL_GRAPH_EDGES = 8_000_000  # whole CPU runs are timed directly below this size


def cpu_baseline_sample(G, wl, threads):
    """The CPU oracle (a port of the reference's algorithm, all host threads)
    on the same graph.  Small graphs: one whole run.  Large graphs: the first
    Louvain phase capped at 3 iterations, without coarsening; returns the
    time and the edges it visited (one modularity sweep before the loop, then
    one move and one modularity sweep per iteration)."""
    from oracle import oracle as orc
    small = G.ne <= SMALL_GRAPH_EDGES
    t0 = time.perf_counter()
    _, st = orc.louvain(G.off, G.adj, G.w, nbatches=wl["nbatches"], tau=wl["tau"],
                        max_loops=500 if small else 3, max_phases=200 if small else 1)
    el = time.perf_counter() - t0
    scanned = 0.0
    for p in range(st.phases):
        scanned += st.ne_phase[p] * (1 + 2 * st.loops_phase[p])
    return el, scanned, st, small


def run_ours(args, world, rank, local):
    import torch

    from nido_b200 import capi
    wl = WORKLOADS[args.workload]
    torch.cuda.set_device(local)
    G = make_graph(capi, args.workload)
    ctx = capi.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream())
    g = capi.Graph(ctx, G, wl["nbatches"])
    outbuf = np.empty(G.nv, np.int64)  # page-locked result buffer, reused every step
    capi.host_register(outbuf)
    for _ in range(args.warmup):
        g.run(tau=wl["tau"], out=outbuf)
    barrier(world)
    torch.cuda.synchronize()
    ctx.sync()
    sampler = ClockSampler(local)
    sampler.start()
    l0 = capi.lib().nido_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    stats = [g.run(tau=wl["tau"], out=outbuf)[1] for _ in range(args.steps)]
    e1.record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    launches = int(capi.lib().nido_launch_count() - l0)
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    barrier(world)
    ms_max = reduce_max(ms, world)
    move_ms = sum(s.move_ms for s in stats)
    move_bytes = sum(s.move_bytes for s in stats)
    # device time per run by section (CUDA events; the rest is batching,
    # commits, per-phase preparation and host round trips)
    n = len(stats)
    breakdown = {"move": move_ms / n, "modularity": sum(s.q_ms for s in stats) / n,
                 "aggregation": sum(s.agg_ms for s in stats) / n}
    breakdown["other"] = sum(s.total_ms for s in stats) / n - sum(breakdown.values())
    sweeps = sum(s.total_loops for s in stats)
    edges_per_run = stats[0].edges_scanned
    # edges a whole run visits in the CPU oracle's count (one modularity sweep
    # per phase plus a move and a modularity sweep per loop), from the GPU
    # run's per-phase sizes and loops: the trajectory is the same
    st0 = stats[0]
    visits_per_run = sum(st0.ne_phase[p] * (1 + 2 * st0.loops_phase[p]) for p in range(min(st0.phases, 200)))
    final_q = stats[-1].final_q

    # end to end through the C ABI: pinned host CSR -> upload -> run -> partition
    for a in (G.off, G.adj, G.w):
        capi.host_register(a)
    g.close()
    h2d = G.off.nbytes + G.adj.nbytes + G.w.nbytes
    d2h = 8 * G.nv
    barrier(world)
    torch.cuda.synchronize()
    ctx.sync()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        with capi.Graph(ctx, G, wl["nbatches"]) as g2:
            part, _ = g2.run(tau=wl["tau"], out=outbuf)
    f1.record(stream)
    ctx.sync()
    torch.cuda.synchronize()
    e2e_ms = reduce_max(f0.elapsed_time(f1), world)
    for a in (G.off, G.adj, G.w, outbuf):
        capi.host_unregister(a)

    color = None
    if args.color_batches:
        # conflict-free colour-class batches against the edge-balanced -b cuts
        with capi.Graph(ctx, G, wl["nbatches"]) as g3:
            for _ in range(args.warmup):
                g3.run(tau=wl["tau"], color_batches=True)
            ctx.sync()
            c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            c0.record(stream)
            cst = [g3.run(tau=wl["tau"], color_batches=True)[1] for _ in range(args.steps)]
            c1.record(stream)
            ctx.sync()
            cms = c0.elapsed_time(c1)
        color = {"graphs_per_s": args.steps / (cms * 1e-3), "final_q": cst[-1].final_q,
                 "phases": cst[-1].phases, "loops": cst[-1].total_loops,
                 "edge_balanced": {"graphs_per_s": args.steps / sec_of(ms), "final_q": final_q,
                                   "nbatches": wl["nbatches"]}}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        el, scanned, st, small = cpu_baseline_sample(G, wl, threads)
        if small:
            cpu = {"value": 1.0 / el, "unit": "graphs/s", "cores": threads, "kind": "port",
                   "sample": f"CPU oracle (port of the reference's algorithm), one whole run, {el:.2f} s"}
        else:
            run_s = el * visits_per_run / scanned
            cpu = {"value": 1.0 / run_s, "unit": "graphs/s", "cores": threads, "kind": "port",
                   "sample": f"CPU oracle (port of the reference's algorithm): first phase, {st.total_loops} "
                             f"iterations, no coarsening ({el:.1f} s, {scanned:.3g} edges visited), scaled to a "
                             f"whole run by edges visited ({visits_per_run:.4g} per run: one modularity sweep per "
                             f"phase plus a move and a modularity sweep per loop, from the GPU run's phases)"}
    ctx.close()
    if rank != 0:
        return None
    pk, pk_kind = peaks()
    achieved = move_bytes / (move_ms * 1e-3) / 1e9 if move_ms > 0 else 0.0
    sec = ms_max * 1e-3
    return {
        "metric": "graphs/s", "value": world * args.steps / sec, "unit": "graphs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "ours",
        "config": config_of(args, wl, world),
        "graph_size": {"nv": G.nv, "ne": G.ne}, "device_layout": "int32 ids, int64 offsets, FP64 weights",
        "edges_scanned_per_s": world * edges_per_run * args.steps / sec,
        "move_sweeps_per_run": sweeps / args.steps, "final_q": final_q,
        "loop_graph_build_ms_per_run": sum(s.host_ms[7] for s in stats) / n,
        "breakdown_ms_per_run": breakdown,
        "e2e": {"value": world * args.steps / (e2e_ms * 1e-3), "unit": "graphs/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / pk["hbm_gbs"],
                     "traffic": MOVE_TRAFFIC_PER_ALGO_BYTE * move_bytes / sweeps,
                     "algorithmic_bytes": move_bytes / sweeps,
                     "kernel": "move phase (degree-tier kernels of one sweep; per-sweep bytes)",
                     "traffic_kind": "ncu DRAM bytes per algorithmic byte of the move-tier kernels (one-kernel captures, R-MAT scale 20), scaled",
                     "peak_kind": pk_kind},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
        "color_batches": color,
    }


def sec_of(ms):
    return ms * 1e-3


def run_many(args, world, rank, local):
    """Many graphs per step: one nido_batch_run over the packed set against
    the same engine run one graph at a time (nido_run per graph, graph
    resident), on a systematic sample of the graphs."""
    import torch

    from nido_b200 import capi
    from nido_b200 import workloads as W
    wl = WORKLOADS["many"]
    torch.cuda.set_device(local)
    t0 = time.perf_counter()
    vbase, U, (V, d, kind) = W.many_graphs_packed(args.many_graphs, 4, args.many_edges)
    gen_s = time.perf_counter() - t0
    ng = len(vbase) - 1
    ctx = capi.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream())
    B = capi.Batch(ctx, nbatches=wl["nbatches"], packed=(vbase, U))
    outbuf = np.empty(U.nv, np.int64)  # page-locked result buffer, reused every step
    capi.host_register(outbuf)
    for _ in range(args.warmup):
        res = B.run(tau=wl["tau"], out=outbuf)
    barrier(world)
    ctx.sync()
    sampler = ClockSampler(local)
    sampler.start()
    l0 = capi.lib().nido_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    runs = [B.run(tau=wl["tau"], out=outbuf) for _ in range(args.steps)]
    e1.record(stream)
    ctx.sync()
    launches = int(capi.lib().nido_launch_count() - l0)
    ms = e0.elapsed_time(e1)
    clocks = sampler.stop()
    parts, q, ph, lo, st = runs[-1]
    B.close()
    ms_max = reduce_max(ms, world)
    move_ms = sum(r[4].move_ms for r in runs)
    move_bytes = sum(r[4].move_bytes for r in runs)

    # the same engine one graph at a time on every stride-th graph
    stride = max(1, ng // args.plain_sample)
    sample = list(range(0, ng, stride))
    plain_ms, dq, mismatch = 0.0, 0.0, 0
    for i in sample:
        Gi = W.unpack(vbase, U, i)
        with capi.Graph(ctx, Gi, wl["nbatches"]) as g:
            g.run(tau=wl["tau"])
            ctx.sync()
            p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            p0.record(stream)
            cl, sti = g.run(tau=wl["tau"])
            p1.record(stream)
            ctx.sync()
            plain_ms += p0.elapsed_time(p1)
        dq = max(dq, abs(sti.final_q - q[i]))
        mismatch += int(not np.array_equal(cl, parts[i]))
    plain_gps = len(sample) / (plain_ms * 1e-3)

    # end to end: pinned host CSR -> upload -> batched run -> partitions
    for a in (U.off, U.adj, U.w):
        capi.host_register(a)
    barrier(world)
    ctx.sync()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.steps):
        with capi.Batch(ctx, nbatches=wl["nbatches"], packed=(vbase, U)) as b2:
            b2.run(tau=wl["tau"], out=outbuf)
    f1.record(stream)
    ctx.sync()
    e2e_ms = reduce_max(f0.elapsed_time(f1), world)
    for a in (U.off, U.adj, U.w, outbuf):
        capi.host_unregister(a)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as orc
        threads = os.cpu_count() or 1
        done, t_cpu = 0, 0.0
        for i in sample:  # whole oracle runs on the sampled graphs, about 20 s of CPU work
            Gi = W.unpack(vbase, U, i)
            c0 = time.perf_counter()
            orc.louvain(Gi.off, Gi.adj, Gi.w, nbatches=wl["nbatches"], tau=wl["tau"])
            t_cpu += time.perf_counter() - c0
            done += 1
            if t_cpu > 20.0:
                break
        cpu = {"value": done / t_cpu, "unit": "graphs/s", "cores": threads, "kind": "port",
               "sample": f"CPU oracle (port of the reference's algorithm), whole runs of {done} of the "
                         f"sampled graphs ({t_cpu:.1f} s)"}
    ctx.close()
    serving = None
    if not args.no_serve and world == 1:
        # the metric's latency half: the serving workload's Poisson replay
        serving = serve_replay(args, local)
    if rank != 0:
        return None
    pk, pk_kind = peaks()
    achieved = move_bytes / (move_ms * 1e-3) / 1e9 if move_ms > 0 else 0.0
    sec = ms_max * 1e-3
    return {
        "metric": "graphs/s", "value": world * ng * args.steps / sec, "unit": "graphs/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "impl": "ours",
        "config": config_of(args, wl, world),
        "set": {"ngraphs": ng, "nv": U.nv, "ne": U.ne, "generation_s": round(gen_s, 1)},
        "plain": {"graphs_per_s": world * plain_gps, "sampled_graphs": len(sample),
                  "batched_over_plain": (ng * args.steps / sec) / plain_gps,
                  "max_abs_dq_vs_plain": dq, "partition_mismatches": mismatch},
        "edges_scanned_per_s": world * st.edges_scanned * args.steps / sec,
        "e2e": {"value": world * ng * args.steps / (e2e_ms * 1e-3), "unit": "graphs/s",
                "h2d_bytes_per_step": U.off.nbytes + U.adj.nbytes + U.w.nbytes + vbase.nbytes,
                "d2h_bytes_per_step": 8 * U.nv + 24 * ng},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / pk["hbm_gbs"],
                     "traffic": MOVE_TRAFFIC_PER_ALGO_BYTE * move_bytes / max(1, sum(r[4].total_loops for r in runs)),
                     "algorithmic_bytes": move_bytes / max(1, sum(r[4].total_loops for r in runs)),
                     "kernel": "move phase (degree-tier kernels of one sweep over all graphs; per-sweep bytes)",
                     "traffic_kind": "ncu DRAM bytes per algorithmic byte of the move-tier kernels (one-kernel captures, R-MAT scale 20), scaled",
                     "peak_kind": pk_kind},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "gpu_launches": launches,
        "kernel_launches_per_step": launches / args.steps,
        "breakdown_ms_per_step": {"move": move_ms / len(runs), "modularity": sum(r[4].q_ms for r in runs) / len(runs),
                                  "aggregation": sum(r[4].agg_ms for r in runs) / len(runs),
                                  "other": ms_max / args.steps - (move_ms + sum(r[4].q_ms + r[4].agg_ms
                                                                               for r in runs)) / len(runs)},
        "loop_graph_build_ms_per_step": sum(r[4].host_ms[7] for r in runs) / len(runs),
        "host_sections_ms_per_step": {
            k: sum(r[4].host_ms[i] for r in runs) / len(runs)
            for i, k in enumerate(("reset", "sweeps", "list_rebuilds", "phase_end_aggregation_emit",
                                   "phase_setup", "download"))},
        "latency_ms": serving["latency_ms"] if serving else None,
        "serving": ({k: serving[k] for k in ("graphs_per_s", "requests", "latency_ms", "overlap", "workload")}
                    if serving else None),
    }


def serve_replay(args, local):
    """A stream of requests with Poisson arrivals through the request loop
    (nido_server_*): graphs/s from first arrival to last result, and the
    latency (arrival to result in host memory) of every request."""
    from nido_b200 import capi
    from nido_b200 import workloads as W
    wl = WORKLOADS["serve"]
    t0 = time.perf_counter()
    arr, V, kind = W.serving_requests(args.serve_requests, args.serve_rate, 5, 1e3, args.serve_vmax)
    graphs = [W.make_request(int(v), int(k), 5_000_003 + i) for i, (v, k) in enumerate(zip(V, kind))]
    gen_s = time.perf_counter() - t0
    budget = int(args.serve_budget_gb * 1e9)
    srv = capi.Server(local, budget, workers=args.serve_workers)
    warm = [W.make_request(2000 + 500 * i, i % 2, 77 + i) for i in range(3)]
    for t in [srv.submit(g, wl["nbatches"], wl["tau"]) for g in warm]:
        srv.wait(t)
    l0 = capi.lib().nido_launch_count()
    tickets = [None] * len(graphs)
    start = time.perf_counter()

    def submitter():
        for i, g in enumerate(graphs):
            dt = arr[i] - (time.perf_counter() - start)
            if dt > 0:
                time.sleep(dt)
            tickets[i] = srv.submit(g, wl["nbatches"], wl["tau"])

    th = threading.Thread(target=submitter)
    th.start()
    th.join()
    infos = [srv.wait(t)[1] for t in tickets]
    wall = time.perf_counter() - start
    launches = int(capi.lib().nido_launch_count() - l0)
    srv.close()
    lat = np.array([i.latency_ms for i in infos])
    dev_ms = float(sum(i.device_ms for i in infos))
    return {
        "graphs_per_s": len(graphs) / wall, "wall_s": wall, "requests": len(graphs),
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                       "max": float(lat.max()), "mean_queue": float(np.mean([i.queue_ms for i in infos]))},
        "overlap": {"sum_device_ms": dev_ms, "wall_ms": wall * 1e3, "concurrency": dev_ms / (wall * 1e3)},
        "workload": {"graph": wl["desc"], "rate_per_s": args.serve_rate, "vmax": args.serve_vmax,
                     "workers": args.serve_workers, "hbm_budget_bytes": budget,
                     "total_edges": int(sum(g.ne for g in graphs)), "generation_s": round(gen_s, 1)},
        "h2d_bytes": int(sum(g.off.nbytes + g.adj.nbytes + g.w.nbytes for g in graphs)),
        "d2h_bytes": int(sum(8 * g.nv for g in graphs)),
        "launches": launches,
    }


def run_serve(args, world, rank, local):
    """The serving workload on its own: one step is the whole replay."""
    sampler = ClockSampler(local)
    barrier(world)
    sampler.start()
    r = serve_replay(args, local)
    clocks = sampler.stop()
    wall_max = reduce_max(r["wall_s"], world)
    if rank != 0:
        return None
    return {
        "metric": "graphs/s", "value": world * r["requests"] / wall_max, "unit": "graphs/s", "n_gpus": world,
        "steps": 1, "warmup": 3, "ms_per_step": wall_max * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "ours",
        "config": config_of(args, WORKLOADS["serve"], world),
        "requests": r["requests"], "serving": r["workload"],
        "latency_ms": r["latency_ms"], "overlap": r["overlap"],
        "e2e": {"value": world * r["requests"] / wall_max, "unit": "graphs/s",
                "h2d_bytes_per_step": r["h2d_bytes"], "d2h_bytes_per_step": r["d2h_bytes"]},
        "roofline": None,
        "cpu_baseline": None,
        "clocks": clocks,
        "gpu_launches": r["launches"],
    }


def run_reference_set(args, world, wl):
    """Reference arm of the graph-set workloads: whole CPU-oracle runs, all
    host threads, one graph after another (the reference runs one graph per
    process).  Every step runs whole graphs drawn in order from the set until
    about --ref-step-s seconds have passed; the step's time is what it took."""
    from nido_b200 import workloads as W
    from oracle import oracle as orc
    threads = os.cpu_count() or 1
    if args.workload == "many":
        Vp, dp, kp = W.many_graph_plan(args.many_graphs, 4, args.many_edges)
        stride = max(1, len(Vp) // args.plain_sample)
        items = [(int(Vp[i]), float(dp[i]), int(kp[i]), i) for i in range(0, len(Vp), stride)]
        make = lambda it: W.make_one(it[0], it[1], it[2], 3, 4 * 1_000_003 + it[3])  # W_INT8
    else:
        _, Vs, ks = W.serving_requests(args.serve_requests, args.serve_rate, 5, 1e3, args.serve_vmax)
        items = [(int(v), int(k), i) for i, (v, k) in enumerate(zip(Vs, ks))]
        make = lambda it: W.make_request(it[0], it[1], 5_000_003 + it[2])
    pos, steps = 0, []
    for step in range(args.warmup + args.steps):
        done, el = 0, 0.0
        while el < args.ref_step_s:
            G = make(items[pos % len(items)])
            pos += 1
            c0 = time.perf_counter()
            orc.louvain(G.off, G.adj, G.w, nbatches=wl["nbatches"], tau=wl["tau"])
            el += time.perf_counter() - c0
            done += 1
        if step >= args.warmup:
            steps.append((done, el))
    total_s = sum(t[1] for t in steps)
    value = sum(t[0] for t in steps) / total_s
    sample = (f"CPU oracle (port of the reference's algorithm), {threads} threads: each step whole runs of "
              f"graphs drawn in order from the {args.workload} set's systematic sample, about "
              f"{args.ref_step_s:g} s ({sum(t[0] for t in steps)} graphs in {total_s:.1f} s over {len(steps)} steps)")
    return {
        "metric": "graphs/s", "value": value, "unit": "graphs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / len(steps), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": config_of(args, wl, world),
        "graphs_per_step": [t[0] for t in steps],
        "cpu_baseline": {"value": value, "unit": "graphs/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "graphs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_reference(args, world, rank):
    """The reference's path on the host cores: the CPU oracle (a port of nido's
    algorithm; nido itself has no CPU implementation), all threads.  Every
    step is one whole Louvain run of the workload's graph, timed as it runs."""
    if rank != 0:
        return None
    from nido_b200 import capi
    from oracle import oracle as orc
    wl = WORKLOADS[args.workload]
    if args.workload in ("many", "serve"):
        return run_reference_set(args, world, wl)
    G = make_graph(capi, args.workload)
    threads = os.cpu_count() or 1
    times, final_q = [], None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        _, st = orc.louvain(G.off, G.adj, G.w, nbatches=wl["nbatches"], tau=wl["tau"])
        el = time.perf_counter() - t0
        final_q = st.final_q
        if i >= args.warmup:
            times.append(el)
    total_s = sum(times)
    value = len(times) / total_s
    sample = (f"CPU oracle (port of the reference's algorithm), {threads} threads, one whole run per step "
              f"({total_s:.1f} s for {len(times)} runs)")
    return {
        "metric": "graphs/s", "value": value, "unit": "graphs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * total_s / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": config_of(args, wl, world),
        "graph_size": {"nv": G.nv, "ne": G.ne},
        "cpu_baseline": {"value": value, "unit": "graphs/s", "cores": threads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "graphs/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "final_q": final_q,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="many")
    ap.add_argument("--no-serve", action="store_true", help="many: skip the serving replay's latency figures")
    ap.add_argument("--color-batches", action="store_true",
                    help="one-graph workloads: also time colour-class batches against the -b cuts")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--many-graphs", type=int, default=4096)
    ap.add_argument("--many-edges", type=float, default=1.5e9)
    ap.add_argument("--plain-sample", type=int, default=256, help="graphs run one at a time for the comparison")
    ap.add_argument("--serve-requests", type=int, default=24)
    ap.add_argument("--serve-rate", type=float, default=4.0, help="Poisson arrival rate, requests per second")
    ap.add_argument("--serve-vmax", type=float, default=1e7)
    ap.add_argument("--serve-workers", type=int, default=4)
    ap.add_argument("--serve-budget-gb", type=float, default=150.0)
    ap.add_argument("--ref-step-s", type=float, default=8.0,
                    help="reference arm of the graph sets: seconds of whole CPU runs per step")
    args = ap.parse_args()
    if args.warmup < 3:
        raise SystemExit("--warmup must be at least 3")
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        out = run_reference(args, world, rank)
    elif args.workload == "many":
        out = run_many(args, world, rank, local)
    elif args.workload == "serve":
        out = run_serve(args, world, rank, local)
    else:
        out = run_ours(args, world, rank, local)
    if out is not None:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
