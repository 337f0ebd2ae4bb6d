#!/usr/bin/env python3
"""Benchmark: SSSP GTEPS with delta-stepping on RMAT-24 (uint32 weights).

Workload (one GPU, the metric's configuration): RMAT scale 24, edge factor 16,
a,b,c,d = .57,.19,.19,.05, symmetrised, self-loops and duplicates removed,
uint32 weights U{1..255}; 16 seeded random sources with nonzero degree.  A
step is one single-source solve by the library's persistent delta-stepping
kernel (fixed Near-Far delta, or the learned policy with --policy learned).
Steps cycle through the 16 sources.

value  = sum over timed steps of reached edges / device time (GTEPS), inputs
         resident in HBM (graph 4+ GB > L2, so no L2 flush is needed).
e2e    = the same through the public C ABI with the per-step input (source id)
         copied from pinned host memory and the whole distance array copied
         back to pinned host memory inside the timed region.
roofline: algorithmic bytes of one solve = 8*m_r (dst+weight of each reached
         arc) + 8*n_r (rowptr pairs of reached vertices) + 8*n (label init and
         final write) over the persistent kernel's CUDA-event time, against
         the measured HBM copy bandwidth.
cpu_baseline / --impl reference: the reference's CPU path (min-plus
         Bellman-Ford, numpy, pytorch_testing/.../minplus_bellman_ford.py:51-102)
         restated in oracle/pyoracle.py, timed on a bounded row sample of one
         iteration and scaled to a full solve (iterations x rows).

Multi-GPU (torchrun, --gpus N): replicas; every rank holds its own copy of
the graph and solves its share of the sources (no collective on the data
path); value = all ranks' reached edges / max-over-ranks time.

Other workloads of the same library (one JSON line each, same keys):
  --workload sssp --graph grid : the 4096 x 4096 road-like grid (4-neighbour,
                                 bidirectional, 2 % shortcuts, weights
                                 ceil(lognormal(5, 1))), 16 sources;
  --workload policy            : learned schedule vs the fixed Near-Far delta on
                                 RMAT-24 and the 4096^2 grid, distances compared;
  --workload minplus           : dense min-plus GEMM, N = 8192, int32 (fp32 in
                                 detail), p = 0.3 present, roofline against the
                                 calibrated CUDA-core (min,+) rate;
  --workload spgemm            : CSR x CSR min-plus SpGEMM, ER 2^20, degree 8;
  --workload serve             : 64 resident graphs, 8192 Poisson queries,
                                 batched server vs one-at-a-time solves.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rips2026-amd_b200"))

SCALE = int(os.environ.get("B2_BENCH_SCALE", "24"))
EDGE_FACTOR = 16
SEED = 1
NSRC = 16


def load_peaks() -> tuple[float, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profile_traffic(graph: str = "rmat") -> float | None:
    """dram bytes per launch of the persistent kernel from the committed ncu summary."""
    name = "sssp_delta_rmat24.md" if graph == "rmat" else "sssp_delta_grid4096.md"
    p = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(p):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1].strip())
    except OSError:
        pass
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.rows: list[list[str]] = []
        self.proc = None
        self.th = None
        self.active = False

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.th = threading.Thread(target=self._read, daemon=True)
        self.th.start()

    def _read(self):
        for line in self.proc.stdout:
            if self.active:
                self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def pick_sources(hg, k: int, seed: int) -> list[int]:
    rng = np.random.default_rng(seed)
    deg = np.diff(hg.rowptr)
    out = []
    while len(out) < k:
        s = int(rng.integers(0, hg.n))
        if deg[s] > 0:
            out.append(s)
    return out


def shard_sources(sources: list[int], rank: int, world: int) -> list[int]:
    """Replicas: rank r solves sources r, r + world, ... (every rank at least one)."""
    return sources[rank::world] if world <= len(sources) else [sources[rank % len(sources)]]


def reduce_over_ranks(times, counts, device, distributed: bool):
    """Max over ranks of the timed intervals, sum of the work counts; every
    rank calls it once, in the same order (one MAX then one SUM all-reduce)."""
    import torch
    import torch.distributed as dist
    tt = torch.tensor([float(x) for x in times], dtype=torch.float64, device=device)
    tot = torch.tensor([float(x) for x in counts], dtype=torch.float64, device=device)
    if distributed:
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        dist.all_reduce(tot, op=dist.ReduceOp.SUM)
    return tt.tolist(), tot.tolist()


def cpu_reference_sample(hg, iterations: int, budget_s: float = 12.0) -> dict:
    """Time the reference's min-plus BF iteration (numpy port) on a row sample,
    rows split over all host threads (numpy's gather and reduceat release the
    GIL), and scale it to a full iteration."""
    from concurrent.futures import ThreadPoolExecutor
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    gi = hg  # symmetric weights: incoming CSR == outgoing CSR
    n = gi.n
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    # rows whose arcs fit ~1/4 of the graph per timing run
    target = max(1, gi.m // 4)
    rows = int(np.searchsorted(gi.rowptr, target))
    rows = max(1, min(rows, n))
    arcs = int(gi.rowptr[rows])
    d = np.full(n, np.inf)
    d[0] = 0.0
    d[np.random.default_rng(0).integers(0, n, n // 4)] = 1.0   # a partially reached label vector
    bounds = np.searchsorted(gi.rowptr[: rows + 1], np.linspace(0, arcs, cores + 1)).tolist()
    bounds[0], bounds[-1] = 0, rows
    parts = []
    for a, b in zip(bounds[:-1], bounds[1:]):
        if b <= a:
            continue
        e0, e1 = int(gi.rowptr[a]), int(gi.rowptr[b])
        parts.append((a, b, gi.rowptr[a:b + 1].astype(np.int64) - e0, gi.colind[e0:e1],
                      gi.weights[e0:e1].astype(np.float64)))

    def one(p):
        a, b, rp, ci, dv = p
        return np.minimum(d[a:b], pyoracle.tropical_spmv(rp, ci, dv, d))

    t0 = time.perf_counter()
    reps = 0
    with ThreadPoolExecutor(max_workers=len(parts)) as ex:
        while True:
            list(ex.map(one, parts))
            reps += 1
            if time.perf_counter() - t0 > budget_s / 2 or reps >= 3:
                break
    dt = (time.perf_counter() - t0) / reps
    per_iter = dt * gi.m / max(arcs, 1)
    return {"seconds_per_iteration": per_iter, "iterations": iterations,
            "sample": f"{reps}x tropical_spmv over rows [0,{rows}) = {arcs} arcs of {gi.m} on {len(parts)} "
                      f"threads, scaled to all arcs and {iterations} Bellman-Ford iterations",
            "cores": len(parts)}


def cpu_iterations_and_dijkstra(hg, source: int) -> tuple[int, float]:
    """Jacobi BF round count for `source` from the oracle's (dist, hops)
    Dijkstra, and that Dijkstra's single-core time."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    t0 = time.perf_counter()
    iters, _ = pyoracle.bf_iterations_u32(hg.rowptr, hg.colind, hg.weights, source)
    return iters, time.perf_counter() - t0


def reference_arm(args, hg, sources, config) -> dict:
    """The reference's CPU Bellman-Ford (numpy port) on this workload, host cores only."""
    iters, t_dij = cpu_iterations_and_dijkstra(hg, sources[0])
    smp = cpu_reference_sample(hg, iters)
    t_solve = smp["seconds_per_iteration"] * smp["iterations"]
    deg = np.diff(hg.rowptr)
    reached_edges = float(deg[deg > 0].sum())   # every vertex with an edge is in the giant component
    gteps = reached_edges / t_solve / 1e9
    return {"metric": "sssp_gteps", "value": gteps, "unit": "GTEPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_solve * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config, "impl": "reference",
            "cpu_baseline": {"value": gteps, "unit": "GTEPS", "cores": smp["cores"], "kind": "port",
                             "sample": smp["sample"]},
            "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "detail": {"cpu_dijkstra_1core_seconds": t_dij, "bf_iterations": iters}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--policy", default="fixed", choices=["fixed", "learned"])
    ap.add_argument("--method", default="delta", choices=["delta", "bf", "adds"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--trace-out", default=None, help="write one traced solve's phase list (JSON)")
    ap.add_argument("--workload", default="sssp", choices=["sssp", "policy", "minplus", "spgemm", "serve"])
    ap.add_argument("--graph", default="rmat", choices=["rmat", "grid"])
    ap.add_argument("--n", type=int, default=8192, help="minplus: matrix order")
    ap.add_argument("--rate", type=float, default=10000.0, help="serve: Poisson arrival rate (queries/s)")
    ap.add_argument("--queries", type=int, default=8192, help="serve: queries")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.workload != "sssp":
        if int(os.environ.get("RANK", "0")) != 0:
            return   # the extra workloads are single-GPU measurements (rank 0)
        fn = {"policy": workload_policy, "minplus": workload_minplus, "spgemm": workload_spgemm,
              "serve": workload_serve}[args.workload]
        print(json.dumps(fn(args)), flush=True)
        return

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    import torch
    import torch.distributed as dist
    distributed = world > 1 and args.impl == "ours"
    if args.impl == "reference" and rank != 0:
        return   # the reference arm is rank 0's CPU run; other ranks do no work
    if distributed:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))

    import b200sssp
    t_gen = time.time()
    if args.graph == "grid":
        side = 1 << (SCALE // 2)
        hg = b200sssp.gen_grid(side, side, 0.02, 5.0, 1.0, SEED)
        config = {"workload": f"grid{side}x{side}_4nbr_bidir_2pct_shortcuts_u32lognormal5-1_{args.method}_sssp",
                  "rows": side, "cols": side, "shortcut_frac": 0.02, "weights": "uint32 ceil(lognormal(5, 1))"}
    else:
        hg = b200sssp.gen_rmat(SCALE, EDGE_FACTOR, 0.57, 0.19, 0.19, 1, 255, SEED)
        config = {"workload": f"rmat{SCALE}_ef{EDGE_FACTOR}_sym_u32w1-255_{args.method}_sssp", "scale": SCALE,
                  "edge_factor": EDGE_FACTOR, "weights": "uint32 U{1..255}"}
    t_gen = time.time() - t_gen
    sources = pick_sources(hg, NSRC, SEED)
    config.update({"n": hg.n, "m": hg.m, "sources": NSRC, "method": args.method, "policy": args.policy,
                   "l2": "inputs larger than L2 (graph %.1f GB); no flush" % ((8 * hg.m + 8 * hg.n) / 1e9)})

    if args.impl == "reference":
        if rank == 0:
            line = reference_arm(args, hg, sources, config)
            print(json.dumps(line), flush=True)
        if distributed:
            dist.destroy_process_group()
        return

    g = b200sssp.Graph.from_host(hg, "u32")
    my_sources = shard_sources(sources, rank, world)
    stream = torch.cuda.Stream()
    opts = {}
    if args.policy == "learned":
        opts["policy"] = 1
    # reached edges per source (TEPS numerator), measured once outside timing
    reach = {}
    for s in my_sources:
        _, _, st = g.sssp(s, method=args.method, collect_reach=1, stream=stream, **opts)
        reach[s] = (st["reached"], st["reached_edges"])
    dist_out = torch.empty(g.n, dtype=torch.int32, device="cuda")
    for i in range(args.warmup):
        g.sssp(my_sources[i % len(my_sources)], method=args.method, out=dist_out, stream=stream, **opts)

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    sampler.active = True
    kernel_ms = []
    edges = 0
    bytes_alg = 0
    if distributed:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    st_last = None
    for i in range(args.steps):
        s = my_sources[i % len(my_sources)]
        _, _, st = g.sssp(s, method=args.method, out=dist_out, stream=stream, **opts)
        kernel_ms.append(st["kernel_ms"])
        nr, er = reach[s]
        edges += er
        bytes_alg += 8 * er + 8 * nr + 8 * g.n
        st_last = st
    e1.record(stream)
    torch.cuda.synchronize()
    t_dev = e0.elapsed_time(e1) / 1e3
    if distributed:
        dist.barrier()

    # e2e through the public API: the graph stays resident (uploaded once, as
    # a serving process holds it), the source id goes in by value and every
    # step's full distance array comes back to pinned host memory.
    h_dist = torch.empty(g.n, dtype=torch.int32, pin_memory=True)
    torch.cuda.synchronize()
    e2 = torch.cuda.Event(enable_timing=True)
    e3 = torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    e2e_edges = 0
    for i in range(args.steps):
        s = my_sources[i % len(my_sources)]
        g.sssp(s, method=args.method, out=dist_out, stream=stream, **opts)
        with torch.cuda.stream(stream):
            h_dist.copy_(dist_out, non_blocking=True)
        e2e_edges += reach[s][1]
    e3.record(stream)
    torch.cuda.synchronize()
    t_e2e = e2.elapsed_time(e3) / 1e3
    sampler.active = False
    sampler.stop()

    # max over ranks
    (t_dev, t_e2e), (edges_all, e2e_all) = reduce_over_ranks([t_dev, t_e2e], [edges, e2e_edges], "cuda",
                                                             distributed)

    if args.trace_out and rank == 0:
        _, _, stt = g.sssp(my_sources[0], method=args.method, out=dist_out, stream=stream, trace=1, **opts)
        with open(args.trace_out, "w") as f:
            json.dump({"stats": stt, "phases": g.trace()}, f)

    peak, peak_kind = load_peaks()
    avg_kernel_s = float(np.mean(kernel_ms)) / 1e3
    achieved = (bytes_alg / args.steps) / avg_kernel_s / 1e9
    line = {
        "metric": "sssp_gteps", "value": edges_all / t_dev / 1e9, "unit": "GTEPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_dev / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic", "config": config,
        "e2e": {"value": e2e_all / t_e2e / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 4 * g.n,
                "note": "graph resident; source id passed by value; distances copied to pinned host"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": profile_traffic(args.graph),
                     "peak_kind": peak_kind,
                     "kernel": "k_sssp<WU32,false,kModeDelta>",
                     "bytes_alg_per_launch": bytes_alg / args.steps,
                     "avg_kernel_ms": avg_kernel_s * 1e3},
        "detail": {"phases_per_solve": st_last["phases"], "buckets": st_last["iterations_used"],
                   "delta": st_last["delta_used"], "edges_scanned_last": st_last["edges_scanned"],
                   "improvements_last": st_last["improvements"], "pushes_last": st_last["pushes"],
                   "reached_edges_mean": float(np.mean([v[1] for v in reach.values()])),
                   "grid_blocks": st_last["grid_blocks"], "gen_seconds": t_gen},
    }
    clocks = sampler.summary()
    line["clocks"] = clocks
    if rank == 0 and not args.no_cpu_baseline:
        iters, t_dij = cpu_iterations_and_dijkstra(hg, sources[0])
        smp = cpu_reference_sample(hg, iters)
        t_solve = smp["seconds_per_iteration"] * smp["iterations"]
        cpu = float(np.mean([v[1] for v in reach.values()])) / t_solve / 1e9
        line["cpu_baseline"] = {"value": cpu, "unit": "GTEPS", "cores": smp["cores"], "kind": "port",
                                "sample": smp["sample"], "cpu_dijkstra_1core_seconds": t_dij}
    g.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if distributed:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Extra single-GPU workloads.  Each returns the contract's JSON line.
def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _line(metric, value, unit, args, ms_per_step, dtype, config, **extra):
    out = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": dtype, "data": "synthetic", "config": config}
    out.update(extra)
    return out


def workload_minplus(args):
    """Dense min-plus GEMM C = A (min,+) A, N x N, int32 (fp32 in detail).

    A step is one product.  value = 2 N^3 (min,+) ops per product / device
    time (Gop/s); roofline: (min,+) pairs per second against the calibrated
    rate of the same instruction mix on registers (b2_minplus_calibrate).
    e2e: A copied from pinned host memory and C back, per step.
    cpu_baseline: the reference's chunked torch min-plus (block 16) on all
    host threads over a row sample, scaled to N rows."""
    import ctypes as C
    import torch
    from b200sssp import _lib, minplus
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    N = args.n
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    res = {}
    for name, dt in (("int32", torch.int32), ("fp32", torch.float32)):
        pres = torch.rand(N, N, device="cuda", generator=g) < 0.3
        if dt == torch.int32:
            A = torch.randint(1, 1001, (N, N), device="cuda", generator=g, dtype=torch.int32)
            A[~pres] = minplus.MISSING_I32
        else:
            A = torch.rand(N, N, device="cuda", generator=g)
            A[~pres] = float("inf")
        A.fill_diagonal_(0)
        del pres
        Cm = torch.empty_like(A)
        for _ in range(args.warmup):
            minplus.minplus_gemm(A, A, out=Cm)
        sampler = ClockSampler(0)
        sampler.start()
        time.sleep(0.3)
        sampler.active = True
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(args.steps):
            minplus.minplus_gemm(A, A, out=Cm)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / args.steps
        # e2e through the public call with host buffers
        hA = A.cpu().pin_memory()
        hC = torch.empty_like(hA).pin_memory()
        dA = torch.empty_like(A)
        torch.cuda.synchronize()
        e2, e3 = _events()
        e2.record()
        for _ in range(args.steps):
            dA.copy_(hA, non_blocking=True)
            minplus.minplus_gemm(dA, dA, out=Cm)
            hC.copy_(Cm, non_blocking=True)
        e3.record()
        torch.cuda.synchronize()
        ms_e2e = e2.elapsed_time(e3) / args.steps
        sampler.active = False
        sampler.stop()
        r = C.c_double()
        _lib.check(_lib.lib().b2_minplus_calibrate(1 if dt == torch.float32 else 0, C.byref(r)), "calibrate")
        pairs = float(N) ** 3
        res[name] = {"ms": ms, "gops": 2 * pairs / ms / 1e6, "pairs_per_s": pairs / ms * 1e3,
                     "calibrated_pairs_per_s": r.value, "frac": pairs / ms * 1e3 / r.value,
                     "e2e_ms": ms_e2e, "e2e_gops": 2 * pairs / ms_e2e / 1e6, "clocks": sampler.summary(),
                     "bytes": 4 * N * N}
        del A, Cm, dA, hA, hC
        torch.cuda.empty_cache()
    # CPU baseline: reference chunked torch min-plus on a row sample
    import pyoracle
    rng = np.random.default_rng(SEED)
    rows = 8
    Ah = np.where(rng.uniform(size=(rows, N)) < 0.3, rng.uniform(size=(rows, N)), np.inf).astype(np.float32)
    Bh = np.where(rng.uniform(size=(N, N)) < 0.3, rng.uniform(size=(N, N)), np.inf).astype(np.float32)
    t0 = time.perf_counter()
    pyoracle.min_plus_matmul_chunked(Ah, Bh, block=16)
    t_cpu = (time.perf_counter() - t0) * N / rows
    cpu_gops = 2 * float(N) ** 3 / t_cpu / 1e9
    head = res["int32"]
    return _line("minplus_gops", head["gops"], "Gop/s", args, head["ms"], "int32",
                 {"workload": f"dense_minplus_gemm_N{N}_int32_p0.3_w1-1000", "N": N, "present_p": 0.3,
                  "l2": "operands %.0f MB each > L2; no flush" % (head["bytes"] / 1e6)},
                 e2e={"value": head["e2e_gops"], "unit": "Gop/s", "h2d_bytes_per_step": head["bytes"],
                      "d2h_bytes_per_step": head["bytes"]},
                 gpu_launches=args.steps,
                 roofline={"bound": "alu", "achieved": head["pairs_per_s"] / 1e12,
                           "peak": head["calibrated_pairs_per_s"] / 1e12, "unit": "T (min,+) pairs/s",
                           "frac": head["frac"], "traffic": None, "peak_kind": "calibrated (b2_minplus_calibrate)",
                           "kernel": "k_minplus_tma<int>"},
                 clocks=head["clocks"],
                 cpu_baseline={"value": cpu_gops, "unit": "Gop/s", "cores": __import__("torch").get_num_threads(),
                               "kind": "port",
                               "sample": f"reference chunked torch min-plus (block 16), fp32, {rows} x {N} times "
                                         f"{N} x {N}, scaled to {N} rows"},
                 detail={"fp32": res["fp32"], "int32": res["int32"]})


def workload_spgemm(args):
    """CSR x CSR min-plus SpGEMM C = A (min,+) A on a directed ER graph, n =
    2^20, m = 8 n, int32 weights U{1..1000} (fp32 = w / 1001 in detail).

    A step is one call (outputs allocated by the callee, freed after the
    step).  value = candidate products per second (G/s); roofline: bytes of
    A, the gathered B rows and C over the step time, against the measured HBM
    bandwidth.  cpu_baseline: the oracle's C SpGEMM on a row sample (the
    reference has no CPU SpGEMM)."""
    import torch
    import b200sssp
    from b200sssp import minplus
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    n = 1 << 20
    hg = b200sssp.gen_er(n, 8 * n, 1, 1000, SEED)
    deg = np.diff(hg.rowptr)
    cand = int(deg[hg.colind].sum())
    res = {}
    for name in ("int32", "fp32"):
        vals = hg.weights.view(np.int32) if name == "int32" else (hg.weights.astype(np.float32) / 1001.0)
        Am = (torch.from_numpy(hg.rowptr).cuda(), torch.from_numpy(hg.colind).cuda(), torch.from_numpy(vals).cuda(),
              n)
        for _ in range(args.warmup):
            out = minplus.minplus_spgemm(Am, Am)
        nnz_c = int(out[1].numel())
        del out
        torch.cuda.synchronize()
        ts = []
        e0, e1 = _events()
        for _ in range(args.steps):
            e0.record()
            out = minplus.minplus_spgemm(Am, Am)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
            del out
        ms = float(np.mean(ts))
        bytes_alg = (8 * (n + 1) + 8 * hg.m) + 8 * cand + (8 * (n + 1) + 8 * nnz_c)
        res[name] = {"ms": ms, "ms_min": float(np.min(ts)), "gcand_per_s": cand / ms / 1e6, "nnz_c": nnz_c,
                     "bytes_alg": bytes_alg, "achieved_gbs": bytes_alg / ms / 1e6}
        # e2e: host CSR in, host CSR out
        hrp, hci, hv = (torch.from_numpy(hg.rowptr).pin_memory(), torch.from_numpy(hg.colind).pin_memory(),
                        torch.from_numpy(vals).pin_memory())
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            dA = (hrp.cuda(non_blocking=True), hci.cuda(non_blocking=True), hv.cuda(non_blocking=True), n)
            o = minplus.minplus_spgemm(dA, dA)
            host = [x.cpu() for x in o]
        torch.cuda.synchronize()
        res[name]["e2e_ms"] = (time.perf_counter() - t0) * 1e3 / args.steps
        res[name]["h2d"] = int(hrp.numel() * 8 + hci.numel() * 4 + hv.numel() * 4)
        res[name]["d2h"] = int(sum(x.numel() * x.element_size() for x in host))
        del Am, dA, o, host
        torch.cuda.empty_cache()
    # CPU: the oracle's SpGEMM on the first rows
    rows = 1 << 15
    rp = hg.rowptr[: rows + 1]
    A = (rp, hg.colind[: rp[-1]], hg.weights[: rp[-1]].view(np.int32))
    B = (hg.rowptr, hg.colind, hg.weights.view(np.int32))
    t0 = time.perf_counter()
    pyoracle.minplus_spgemm(A, B, n)
    t_cpu = (time.perf_counter() - t0) * n / rows
    head = res["int32"]
    peak, peak_kind = load_peaks()
    return _line("spgemm_gcand_per_s", head["gcand_per_s"], "G candidates/s", args, head["ms"], "int32",
                 {"workload": "minplus_spgemm_er2^20_deg8_AxA_int32", "n": n, "m": hg.m, "candidates": cand,
                  "l2": "A %.0f MB + expansion > L2; no flush" % ((8 * n + 8 * hg.m) / 1e6)},
                 e2e={"value": cand / head["e2e_ms"] / 1e6, "unit": "G candidates/s", "h2d_bytes_per_step": head["h2d"],
                      "d2h_bytes_per_step": head["d2h"]},
                 gpu_launches=args.steps * 8,
                 roofline={"bound": "hbm", "achieved": head["achieved_gbs"], "peak": peak, "unit": "GB/s",
                           "frac": head["achieved_gbs"] / peak, "traffic": None, "peak_kind": peak_kind,
                           "kernel": "k_rows_warp<int>", "bytes_alg_per_step": head["bytes_alg"]},
                 cpu_baseline={"value": cand / t_cpu / 1e9, "unit": "G candidates/s", "cores": 1, "kind": "port",
                               "sample": f"oracle C SpGEMM over rows [0,{rows}) of A x A, scaled to {n} rows "
                                         "(the reference has no CPU SpGEMM)"},
                 detail=res)


def _policy_eval(g, sources, method="delta"):
    from b200sssp import policy as pol
    return pol.compare(g, sources, method=method, reps=2)


def workload_policy(args):
    """Learned schedule (shipped weights) vs the fixed Near-Far delta on the
    held-out RMAT-24 and 4096^2 grid graphs (uint32 weights), 8 sources each,
    same kernels; distances compared word for word.  value = learned GTEPS
    over both graphs; detail carries each graph's fixed / learned times."""
    import torch
    import b200sssp
    from b200sssp import policy as pol
    p = pol.activate_default()
    out = {}
    tot_e = 0.0
    tot_fixed = tot_learned = 0.0
    for name in ("rmat", "grid"):
        if name == "rmat":
            hg = b200sssp.gen_rmat(SCALE, EDGE_FACTOR, 0.57, 0.19, 0.19, 1, 255, SEED)
        else:
            side = 1 << (SCALE // 2)
            hg = b200sssp.gen_grid(side, side, 0.02, 5.0, 1.0, SEED)
        srcs = pick_sources(hg, 8, SEED)
        g = b200sssp.Graph.from_host(hg, "u32")
        del hg
        reach = 0.0
        for s in srcs:
            _, _, st = g.sssp(s, collect_reach=1)
            reach += st["reached_edges"]
        r = _policy_eval(g, srcs)
        r["decision"] = p.decide(pol.graph_features(g))
        r["fixed_gteps"] = reach / r["fixed_ms"] / 1e6
        r["learned_gteps"] = reach / r["learned_ms"] / 1e6
        out[name] = r
        tot_e += reach
        tot_fixed += r["fixed_ms"]
        tot_learned += r["learned_ms"]
        g.close()
    p.deactivate()
    return _line("sssp_gteps_learned_schedule", tot_e / tot_learned / 1e6, "GTEPS", args,
                 tot_learned / 16, "u32",
                 {"workload": f"learned_vs_fixed_delta_rmat{SCALE}_and_grid{1 << (SCALE // 2)}_u32", "sources": 8},
                 gpu_launches=32,
                 detail={"speedup_over_fixed": tot_fixed / tot_learned, "fixed_gteps": tot_e / tot_fixed / 1e6,
                         "graphs": out})


def workload_serve(args):
    """Batched serving: 64 resident graphs (32 grids 64^2 .. 2048^2, 32 RMAT
    scale 12 .. 20, uint32 weights as in the SSSP workloads), Poisson arrivals
    at --rate, --queries single-source queries with uniform sources; results
    land in pinned host memory.  value = completed queries per second; p50 /
    p99 from arrival to result in host memory.  The one-at-a-time baseline
    (same library, one full-GPU solve per query) runs 1024 queries."""
    import b200sssp
    from b200sssp import serving
    t0 = time.time()
    graphs = []
    for i in range(32):
        side = int(round(64 * (2048 / 64) ** (i / 31)))
        graphs.append(b200sssp.Graph.from_host(b200sssp.gen_grid(side, side, 0.02, 5.0, 1.0, seed=100 + i), "u32"))
    for i in range(32):
        sc = 12 + (i * 9) // 32
        graphs.append(b200sssp.Graph.from_host(b200sssp.gen_rmat(sc, 16, 0.57, 0.19, 0.19, 1, 255, seed=200 + i),
                                               "u32"))
    t_gen = time.time() - t0
    srv = serving.Server(hbm_budget=120 << 30)
    for g in graphs:
        srv.add_graph(g)
        g.sssp(0, collect_reach=1)          # warm the one-at-a-time path: workspace, light counts
    srv.run_load(256, rate_qps=0.0, seed=99, mode="server")                  # warm-up
    rep = srv.run_load(args.queries, rate_qps=args.rate, seed=SEED, mode="server")
    light = srv.run_load(2048, rate_qps=1000.0, seed=SEED + 1, mode="server")      # below capacity
    seq = srv.run_load(1024, rate_qps=0.0, seed=SEED, mode="sequential")
    srv.close()
    # the same server with per-graph autotuning (team kind x bucket constant, timed at registration)
    t0 = time.time()
    srv = serving.Server(hbm_budget=120 << 30, autotune=True)
    for g in graphs:
        srv.add_graph(g)
    t_tune = time.time() - t0
    configs = [srv.graph_config(i) for i in range(len(graphs))]
    srv.run_load(256, rate_qps=0.0, seed=99, mode="server")
    tuned = srv.run_load(args.queries, rate_qps=args.rate, seed=SEED, mode="server")
    tuned_light = srv.run_load(2048, rate_qps=1000.0, seed=SEED + 1, mode="server")
    srv.close()
    tuned["tune_seconds"] = t_tune
    tuned["clusters"] = sum(c["cluster_team"] for c in configs)
    tuned["delta_scales"] = {str(k): sum(1 for c in configs if c["delta_scale"] == k) for k in (2.0, 4.0, 8.0)}
    tuned["light_load_1000qps"] = tuned_light
    if tuned["qps"] > rep["qps"]:
        rep, light = tuned, tuned_light
    return _line("serve_qps", rep["qps"], "queries/s", args, 1e3 / max(rep["qps"], 1e-9), "u32",
                 {"workload": f"serve_64graphs_{args.queries}q_poisson{int(args.rate)}qps", "graphs": 64,
                  "queries": args.queries, "rate_qps": args.rate, "hbm_budget_gb": 120},
                 e2e={"value": rep["qps"], "unit": "queries/s", "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": "distance array of the query's graph"},
                 gpu_launches=None,
                 detail={"p50_us": rep["p50_us"], "p99_us": rep["p99_us"], "server": rep, "sequential": seq,
                         "light_load_1000qps": light, "autotuned": tuned,
                         "speedup_over_sequential_qps": rep["qps"] / max(seq["qps"], 1e-9),
                         "graph_gen_s": t_gen})


if __name__ == "__main__":
    main()
