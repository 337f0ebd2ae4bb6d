#!/usr/bin/env python3
"""Benchmark: SSSP GTEPS with delta-stepping on RMAT-24 (uint32 weights).

Headline workload (one GPU, the metric's configuration): RMAT scale 24, edge
factor 16, a,b,c,d = .57,.19,.19,.05, symmetrised, self-loops and duplicates
removed, uint32 weights U{1..255}; 16 seeded random sources with nonzero
degree.  A step is one single-source solve by the library's persistent
delta-stepping kernel (fixed Near-Far delta, or the learned policy with
--policy learned).  Steps cycle through the 16 sources.

value  = reached edges of the timed steps / device time (GTEPS), inputs
         resident in HBM (graph 4+ GB > L2, so no L2 flush is needed).
e2e    = the same through the public C ABI, every step's whole distance array
         copied back to pinned host memory inside the timed region.  The graph
         stays resident (the reference's DeviceCsrF32 entry points take a
         device CSR the same way) and the source id goes in by value, so no
         host-to-device bytes move per step.
roofline: algorithmic bytes of one solve = 8*m_r (dst+weight of each reached
         arc) + 8*n_r (rowptr pairs of reached vertices) + 8*n (label init and
         final write) over the persistent kernel's CUDA-event time, against
         the measured HBM copy bandwidth.
parity : outside the timed region, the distances of the first two sources
         are compared word for word with the oracle's CPU Dijkstra, and those
         of the first source with the reference's own Bellman-Ford (below).
cpu_baseline: one whole solve of the reference's CPU Bellman-Ford
         (pytorch_testing/.../minplus_bellman_ford.py:51-102, track_pred=False),
         restated in oracle/pyoracle.py, every round's tropical SpMV split into
         row blocks over all host threads.
--impl reference: that CPU Bellman-Ford alone, W warm-up and K timed whole
         solves cycling through the same 16 sources, on a graph built by the
         oracle's generator twin (oracle/oracle_gen.c, pinned byte for byte to
         the library's generator by tests/test_graph_gen_twin.py), so the
         process never loads libb200sssp.so.

detail (N = 1 only; --no-extras skips it): the other configurations measured
in the same run -- the 4096^2 grid (GTEPS, roofline, parity), the FP32-weight
variants of both graphs, the ADDS schedule on both graphs, learned vs fixed
delta, a short serving run, dense min-plus N = 8192 (int32 and fp32, sampled
rows checked), min-plus SpGEMM on ER 2^20, and the small Bellman-Ford config
(ER n = 4096, m = 32768) with the reference's CPU Bellman-Ford beside it.

Multi-GPU (torchrun, --gpus N): replicas; every rank holds its own copy of
the graph and solves its share of the sources (no collective on the data
path); value = all ranks' reached edges / max-over-ranks time.

Single workloads (one JSON line each, same keys):
  --graph grid                 : the grid as the headline;
  --workload policy|minplus|spgemm|serve|c1 : one configuration alone.
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
import traceback

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rips2026-amd_b200"))

SCALE = int(os.environ.get("B2_BENCH_SCALE", "24"))
EDGE_FACTOR = 16
SEED = 1
NSRC = 16
GRID_SIDE = 1 << (SCALE // 2)


def oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle
    return pyoracle


def host_threads() -> int:
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


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
        time.sleep(0.3)
        self.active = True

    def _read(self):
        for line in self.proc.stdout:
            if self.active:
                self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        self.active = False
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


def pick_sources(rowptr: np.ndarray, k: int, seed: int) -> list[int]:
    rng = np.random.default_rng(seed)
    deg = np.diff(rowptr)
    n = deg.shape[0]
    out = []
    while len(out) < k:
        s = int(rng.integers(0, n))
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


def build_workload(kind: str, with_library: bool):
    """(rowptr, colind, weights u32, fweights f32, config) of the RMAT-24 or grid
    workload: by the library's generator, or by the oracle's twin (same bytes)."""
    if kind == "grid":
        args = (GRID_SIDE, GRID_SIDE, 0.02, 5.0, 1.0, SEED)
        config = {"workload": f"grid{GRID_SIDE}x{GRID_SIDE}_4nbr_bidir_2pct_shortcuts_u32lognormal5-1",
                  "rows": GRID_SIDE, "cols": GRID_SIDE, "shortcut_frac": 0.02,
                  "weights": "uint32 ceil(lognormal(5, 1))"}
        if with_library:
            import b200sssp
            hg = b200sssp.gen_grid(*args)
        else:
            hg = oracle().gen_grid(*args)
    else:
        args = (SCALE, EDGE_FACTOR, 0.57, 0.19, 0.19, 1, 255, SEED)
        config = {"workload": f"rmat{SCALE}_ef{EDGE_FACTOR}_sym_u32w1-255", "scale": SCALE,
                  "edge_factor": EDGE_FACTOR, "weights": "uint32 U{1..255}"}
        if with_library:
            import b200sssp
            hg = b200sssp.gen_rmat(*args)
        else:
            hg = oracle().gen_rmat(*args)
    if with_library:
        return hg.rowptr, hg.colind, hg.weights, hg.fweights, config
    return (*hg, config)


def incoming(rowptr, colind, weights, symmetric: bool):
    """INCOMING CSR of an outgoing one (the reference Bellman-Ford's
    orientation).  Symmetric graphs with symmetric weights are their own
    transpose."""
    if symmetric:
        return rowptr, colind, weights
    n = rowptr.shape[0] - 1
    src = np.repeat(np.arange(n, dtype=np.int32), np.diff(rowptr))
    order = np.argsort(colind, kind="stable")
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(np.bincount(colind, minlength=n), out=rp[1:])
    return rp, src[order], weights[order]


def dijkstras(rowptr, colind, weights, sources) -> list[np.ndarray]:
    """The oracle's C Dijkstra for several sources at once (one host thread
    each; ctypes releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor
    orc = oracle()
    with ThreadPoolExecutor(max_workers=max(1, len(sources))) as ex:
        return list(ex.map(lambda s: orc.dijkstra(rowptr, colind, weights, int(s)), sources))


def reference_bf_to_u32(d: np.ndarray) -> np.ndarray:
    """float64 distances of the reference Bellman-Ford as uint32 words
    (+inf -> 0xFFFFFFFF); exact for integer distances below 2^32."""
    out = np.full(d.shape[0], 0xFFFFFFFF, np.uint32)
    fin = np.isfinite(d)
    out[fin] = d[fin].astype(np.uint64).astype(np.uint32)
    return out


def reference_solves(A, sources, steps: int, warmup: int):
    """W untimed and K timed whole solves of the reference's CPU Bellman-Ford
    (row-parallel form), cycling through `sources`."""
    orc = oracle()
    for i in range(warmup):
        orc.sssp_min_plus_bellman_ford_rows(A, sources[i % len(sources)])
    times, results = [], []
    for i in range(steps):
        s = sources[i % len(sources)]
        t0 = time.perf_counter()
        d, used, conv, neg = orc.sssp_min_plus_bellman_ford_rows(A, s)
        times.append(time.perf_counter() - t0)
        results.append((s, d, used, conv))
    return times, results


def reached_edges(rowptr, d: np.ndarray) -> float:
    deg = np.diff(rowptr)
    return float(deg[np.isfinite(d)].sum())


def reference_arm(args) -> dict:
    """The reference's CPU Bellman-Ford on this workload, host cores only, on a
    graph built without the library (the oracle's generator twin)."""
    orc = oracle()
    t_gen = time.time()
    rp, ci, w, fw, config = build_workload(args.graph, with_library=False)
    t_gen = time.time() - t_gen
    sources = pick_sources(rp, NSRC, SEED)
    irp, ici, iw = incoming(rp, ci, w, symmetric=args.graph == "rmat")
    A = orc.RowBlocks(irp, ici, iw.astype(np.float64))
    times, results = reference_solves(A, sources, args.steps, args.warmup)
    A.close()
    total = float(sum(times))
    edges = sum(reached_edges(rp, d) for _, d, _, _ in results)
    gteps = edges / total / 1e9
    config.update({"n": int(rp.shape[0] - 1), "m": int(rp[-1]), "sources": NSRC, "method": "reference_bf"})
    return {"metric": "sssp_gteps", "value": gteps, "unit": "GTEPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config, "impl": "reference",
            "cpu_baseline": {"value": gteps, "unit": "GTEPS", "cores": A.threads, "kind": "port",
                             "sample": f"{args.steps} whole solves of the reference min-plus Bellman-Ford "
                                       f"(numpy port, rounds split into {len(A.blocks)} row blocks over "
                                       f"{A.threads} host threads), {args.warmup} warm-up solves before"},
            "e2e": {"value": gteps, "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "detail": {"rounds_per_solve": [r[2] for r in results], "converged": all(r[3] for r in results),
                       "solve_seconds": times, "graph_gen_seconds": t_gen,
                       "graph_source": "oracle generator twin",
                       "repo_native_libs_mapped": repo_libs_mapped()}}


def repo_libs_mapped() -> list[str]:
    """Shared objects of this repository mapped into this process."""
    try:
        with open("/proc/self/maps") as f:
            libs = {ln.split()[-1] for ln in f if ln.rstrip().endswith(".so") and ROOT in ln}
        return sorted(os.path.relpath(p, ROOT) for p in libs)
    except OSError:
        return []


# ---------------------------------------------------------------------------
# the GPU arm
def sssp_run(g, sources, args, method="delta", opts=None, sampler_gpu=None, dist_out=None):
    """Reach pass, warm-up and K timed solves of one graph; returns the timing
    record and each source's distances from the reach pass."""
    import torch
    opts = dict(opts or {})
    stream = torch.cuda.Stream()
    dt = torch.float32 if g.weight == "f32" else torch.int32
    reach, dists = {}, {}
    for s in sources:
        d, _, st = g.sssp(s, method=method, collect_reach=1, stream=stream, **opts)
        reach[s] = (st["reached"], st["reached_edges"])
        dists[s] = d
    dist_out = dist_out if dist_out is not None else torch.empty(g.n, dtype=dt, device="cuda")
    for i in range(args.warmup):
        g.sssp(sources[i % len(sources)], method=method, out=dist_out, stream=stream, **opts)
    sampler = ClockSampler(sampler_gpu) if sampler_gpu is not None else None
    if sampler:
        sampler.start()
    kernel_ms, edges, bytes_alg, st_last = [], 0, 0, None
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(args.steps):
        s = sources[i % len(sources)]
        _, _, st = g.sssp(s, method=method, out=dist_out, stream=stream, **opts)
        kernel_ms.append(st["kernel_ms"])
        nr, er = reach[s]
        edges += er
        bytes_alg += 8 * er + 8 * nr + 8 * g.n
        st_last = st
    e1.record(stream)
    torch.cuda.synchronize()
    t_dev = e0.elapsed_time(e1) / 1e3
    if sampler:
        sampler.stop()
    return {"t_dev": t_dev, "edges": edges, "bytes_alg": bytes_alg, "kernel_ms": kernel_ms, "st": st_last,
            "reach": reach, "clocks": sampler.summary() if sampler else None, "stream": stream,
            "dist_out": dist_out}, dists


def roofline(bytes_alg_per_launch, avg_kernel_s, kernel, traffic):
    peak, peak_kind = load_peaks()
    achieved = bytes_alg_per_launch / avg_kernel_s / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "peak_kind": peak_kind, "kernel": kernel,
            "bytes_alg_per_launch": bytes_alg_per_launch, "avg_kernel_ms": avg_kernel_s * 1e3}


def parity_check(rp, ci, w, dists_gpu: dict, sources, weight: str) -> dict:
    """Word-for-word comparison of GPU distances with the oracle's Dijkstra."""
    t0 = time.time()
    refs = dijkstras(rp, ci, w, sources)
    mism = 0
    for s, ref in zip(sources, refs):
        got = dists_gpu[s].cpu().numpy()
        got = got.view(np.uint32) if weight == "u32" else got
        mism += int(np.count_nonzero(got.view(np.uint32) != ref.view(np.uint32)))
    return {"sources_checked": len(sources), "mismatches": mism,
            "against": f"oracle C Dijkstra ({'uint32' if weight == 'u32' else 'float32'}), word for word",
            "seconds": time.time() - t0}


def headline(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    import torch
    import torch.distributed as dist
    distributed = world > 1
    if distributed:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    import b200sssp
    t_gen = time.time()
    rp, ci, w, fw, config = build_workload(args.graph, with_library=True)
    t_gen = time.time() - t_gen
    config["workload"] += f"_{args.method}_sssp"
    sources = pick_sources(rp, NSRC, SEED)
    n, m = rp.shape[0] - 1, int(rp[-1])
    config.update({"n": n, "m": m, "sources": NSRC, "method": args.method, "policy": args.policy,
                   "l2": "inputs larger than L2 (graph %.1f GB); no flush" % ((8 * m + 8 * n) / 1e9)})
    g = b200sssp.Graph.from_arrays(rp, ci, w, weight="u32")
    my_sources = shard_sources(sources, rank, world)
    opts = {"policy": 1} if args.policy == "learned" else {}
    run, dists = sssp_run(g, my_sources, args, method=args.method, opts=opts, sampler_gpu=local)
    if distributed:
        dist.barrier()
    # e2e through the public API: the graph stays resident, the source id goes
    # in by value and every step's full distance array comes back to pinned host
    stream, dist_out = run["stream"], run["dist_out"]
    h_dist = torch.empty(g.n, dtype=torch.int32, pin_memory=True)
    torch.cuda.synchronize()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    e2e_edges = 0
    for i in range(args.steps):
        s = my_sources[i % len(my_sources)]
        g.sssp(s, method=args.method, out=dist_out, stream=stream, **opts)
        with torch.cuda.stream(stream):
            h_dist.copy_(dist_out, non_blocking=True)
        e2e_edges += run["reach"][s][1]
    e3.record(stream)
    torch.cuda.synchronize()
    t_e2e = e2.elapsed_time(e3) / 1e3
    (t_dev, t_e2e), (edges_all, e2e_all) = reduce_over_ranks([run["t_dev"], t_e2e], [run["edges"], e2e_edges],
                                                             "cuda", distributed)
    if args.trace_out and rank == 0:
        _, _, stt = g.sssp(my_sources[0], method=args.method, out=dist_out, stream=stream, trace=1, **opts)
        with open(args.trace_out, "w") as f:
            json.dump({"stats": stt, "phases": g.trace()}, f)
    st = run["st"]
    kernel = f"k_sssp<WU32,false,kModeDelta>"
    line = {
        "metric": "sssp_gteps", "value": edges_all / t_dev / 1e9, "unit": "GTEPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_dev / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic", "config": config,
        "e2e": {"value": e2e_all / t_e2e / 1e9, "unit": "GTEPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 4 * g.n,
                "note": "graph resident in HBM (uploaded once, like the reference's device-CSR entry points); "
                        "source id passed by value; the whole distance array copied to pinned host per step"},
        "gpu_launches": args.steps,
        "roofline": roofline(run["bytes_alg"] / args.steps, float(np.mean(run["kernel_ms"])) / 1e3, kernel,
                             profile_traffic(args.graph)),
        "clocks": run["clocks"],
        "detail": {"phases_per_solve": st["phases"], "buckets": st["iterations_used"],
                   "delta": st["delta_used"], "edges_scanned_last": st["edges_scanned"],
                   "improvements_last": st["improvements"], "pushes_last": st["pushes"],
                   "heavy_pulls_last": st["heavy_pulls"],
                   "reached_edges_mean": float(np.mean([v[1] for v in run["reach"].values()])),
                   "grid_blocks": st["grid_blocks"], "gen_seconds": t_gen},
    }
    ctx = None
    if rank == 0 and world == 1:
        chk = my_sources[:2]
        line["parity"] = parity_check(rp, ci, w, dists, chk, "u32")
        if not args.no_cpu_baseline:
            line["cpu_baseline"], bf_match = cpu_baseline(rp, ci, w, args.graph == "rmat", my_sources[0],
                                                          dists[my_sources[0]])
            line["parity"]["reference_bf_mismatches"] = bf_match
        ctx = {"g": g, "sources": my_sources, "rp": rp, "ci": ci, "w": w, "fw": fw, "run": run}
    else:
        g.close()
    if distributed:
        dist.destroy_process_group()
    return line, ctx, rank


def cpu_baseline(rp, ci, w, symmetric: bool, source: int, gpu_dist) -> tuple[dict, int]:
    """One whole solve of the reference's CPU Bellman-Ford (row-parallel numpy
    port, all host threads) from `source`; its distances are compared with
    the GPU's word for word."""
    orc = oracle()
    irp, ici, iw = incoming(rp, ci, w, symmetric)
    A = orc.RowBlocks(irp, ici, iw.astype(np.float64))
    t0 = time.perf_counter()
    d, used, conv, neg = orc.sssp_min_plus_bellman_ford_rows(A, source)
    dt = time.perf_counter() - t0
    A.close()
    got = gpu_dist.cpu().numpy().view(np.uint32)
    mism = int(np.count_nonzero(reference_bf_to_u32(d) != got))
    return ({"value": reached_edges(rp, d) / dt / 1e9, "unit": "GTEPS", "cores": A.threads, "kind": "port",
             "sample": f"one whole solve (source {source}, {used} rounds + the negative-cycle round) of the "
                       f"reference min-plus Bellman-Ford, numpy port, {len(A.blocks)} row blocks over "
                       f"{A.threads} host threads",
             "seconds": dt}, mism)


# ---------------------------------------------------------------------------
# detail: the other configurations, measured in the same run (N = 1)
def _graph_line(g, sources, args, rp, ci, w, weight, kind, method="delta", opts=None, check=1):
    run, dists = sssp_run(g, sources, args, method=method, opts=opts, sampler_gpu=0)
    st = run["st"]
    wt = "WF32" if weight == "f32" else "WU32"
    out = {"gteps": run["edges"] / run["t_dev"] / 1e9, "ms_per_solve": run["t_dev"] / args.steps * 1e3,
           "roofline": roofline(run["bytes_alg"] / args.steps, float(np.mean(run["kernel_ms"])) / 1e3,
                                f"k_adds<{wt},false>" if method == "adds" else f"k_sssp<{wt},false,kModeDelta>",
                                profile_traffic(kind) if weight == "u32" and method == "delta" else None),
           "phases": st["phases"], "buckets": st["iterations_used"], "delta": st["delta_used"],
           "delta_final": st["delta_final"], "edges_scanned_last": st["edges_scanned"], "clocks": run["clocks"]}
    if method == "adds":
        out["work_items_last"] = st["work_items"]
        out["active_buckets_max_last"] = st["active_buckets_max"]
    if check:
        out["parity"] = parity_check(rp, ci, w if weight == "u32" else np.ascontiguousarray(w, np.float32),
                                     dists, sources[:check], weight)
    return out


def detail_graphs(args, ctx, out: dict):
    import b200sssp
    # the headline graph's ADDS schedule and FP32-weight variant
    g, srcs = ctx["g"], ctx["sources"]
    head = "rmat" if args.graph == "rmat" else "grid"
    out[f"{head}_adds"] = _guard(lambda: _graph_line(g, srcs, args, ctx["rp"], ctx["ci"], ctx["w"], "u32", head,
                                                     method="adds"))
    gf = b200sssp.Graph.from_arrays(ctx["rp"], ctx["ci"], ctx["fw"], weight="f32")
    out[f"{head}_f32"] = _guard(lambda: _graph_line(gf, srcs, args, ctx["rp"], ctx["ci"], ctx["fw"], "f32", head))
    gf.close()
    # the other graph
    other = "grid" if head == "rmat" else "rmat"
    rp, ci, w, fw, config = build_workload(other, with_library=True)
    osrcs = pick_sources(rp, NSRC, SEED)
    go = b200sssp.Graph.from_arrays(rp, ci, w, weight="u32")
    rec = _guard(lambda: _graph_line(go, osrcs, args, rp, ci, w, "u32", other))
    if isinstance(rec, dict):
        rec["config"] = config
        rec["n"], rec["m"] = int(rp.shape[0] - 1), int(rp[-1])
    out[other] = rec
    out[f"{other}_adds"] = _guard(lambda: _graph_line(go, osrcs, args, rp, ci, w, "u32", other, method="adds"))
    gf = b200sssp.Graph.from_arrays(rp, ci, fw, weight="f32")
    out[f"{other}_f32"] = _guard(lambda: _graph_line(gf, osrcs, args, rp, ci, fw, "f32", other))
    gf.close()
    # learned schedule vs fixed Near-Far delta on both graphs
    graphs = {head: (g, srcs), other: (go, osrcs)}
    out["policy"] = _guard(lambda: policy_compare(graphs))
    go.close()


def _guard(fn):
    try:
        return fn()
    except Exception as e:   # one configuration's failure must not hide the others
        return {"error": f"{type(e).__name__}: {e}", "trace": traceback.format_exc(limit=3)}


def policy_compare(graphs: dict) -> dict:
    from b200sssp import policy as pol
    p = pol.activate_default()
    res = {}
    try:
        for name, (g, srcs) in graphs.items():
            r = pol.compare(g, srcs[:8], reps=2)
            r["network_output"] = p.decide(pol.graph_features(g))
            if not r["policy_used"]:
                r["note"] = ("features outside the training graphs' range: the fixed Near-Far schedule runs "
                             "(the network's output above is not applied)")
            res[name] = r
    finally:
        p.deactivate()
    w = pol.load_weights()
    res["training"] = {k: (float(w[k]) if k in w else None) for k in
                       ("n_graphs", "cv_geo_speedup", "cv_slower_frac", "cv_worst", "cv_oracle_geo_speedup",
                        "dead_zone")}
    res["training"]["cv_folds"] = int(w["cv_folds"]) if "cv_folds" in w else None
    return res


def detail_c1(args) -> dict:
    """The small Bellman-Ford configuration: directed ER n = 4096, m = 32768,
    uint32 weights U{1..100}, source 0.  GPU Bellman-Ford per solve beside the
    reference's own CPU Bellman-Ford (serial numpy port, like the reference)
    and the oracle's Dijkstra, all three compared word for word."""
    import torch
    import b200sssp
    orc = oracle()
    hg = b200sssp.gen_er(4096, 32768, 1, 100, SEED)
    g = b200sssp.Graph.from_host(hg, "u32")
    d = torch.empty(g.n, dtype=torch.int32, device="cuda")
    for _ in range(max(3, args.warmup)):
        g.sssp(0, method="bf", out=d)
    ks = []
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = max(20, args.steps)
    e0.record()
    for _ in range(reps):
        _, _, st = g.sssp(0, method="bf", out=d)
        ks.append(st["kernel_ms"])
    e1.record()
    torch.cuda.synchronize()
    wall_us = e0.elapsed_time(e1) / reps * 1e3
    gpu = d.cpu().numpy().view(np.uint32)
    rounds = st["iterations_used"]
    d_delta, _, _ = g.sssp(0, method="delta")
    g.close()
    inc = hg.transpose()
    t0 = time.perf_counter()
    ref_runs = 0
    while True:
        ref, used, conv, neg = orc.sssp_min_plus_bellman_ford(inc.rowptr, inc.colind, inc.weights.astype(np.float64),
                                                             0)
        ref_runs += 1
        if time.perf_counter() - t0 > 2.0 or ref_runs >= 10:
            break
    t_ref = (time.perf_counter() - t0) / ref_runs
    t0 = time.perf_counter()
    dj = orc.dijkstra(hg.rowptr, hg.colind, hg.weights, 0)
    t_dj = time.perf_counter() - t0
    deg = np.diff(hg.rowptr)
    m_r = float(deg[gpu != 0xFFFFFFFF].sum())
    return {"workload": "er4096_m32768_u32w1-100_bf_source0", "gpu_bf_us_per_solve": wall_us,
            "gpu_bf_kernel_us": float(np.mean(ks)) * 1e3, "gpu_bf_gteps": m_r / (wall_us * 1e-6) / 1e9,
            "bf_rounds": rounds, "reference_bf_rounds": used, "reference_bf_seconds": t_ref,
            "reference_bf_gteps": m_r / t_ref / 1e9, "reference_runs": ref_runs,
            "cpu_dijkstra_seconds": t_dj,
            "parity": {"gpu_bf_vs_dijkstra_mismatches": int(np.count_nonzero(gpu != dj)),
                       "reference_bf_vs_dijkstra_mismatches": int(np.count_nonzero(reference_bf_to_u32(ref) != dj)),
                       "gpu_delta_vs_dijkstra_mismatches": int(np.count_nonzero(
                           d_delta.cpu().numpy().view(np.uint32) != dj))},
            "cpu_baseline": {"kind": "port", "cores": 1, "sample": "whole solves of the reference min-plus "
                             "Bellman-Ford (serial numpy port)"}}


def minplus_measure(args, N: int, steps: int, check_rows: int) -> dict:
    """Dense min-plus C = A (min,+) A, N x N, int32 and fp32 (p = 0.3 present)."""
    import ctypes as C
    import torch
    from b200sssp import _lib, minplus
    orc = oracle()
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
        for _ in range(max(3, args.warmup)):
            minplus.minplus_gemm(A, A, out=Cm, check_status=False)
        minplus.status()
        sampler = ClockSampler(0)
        sampler.start()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            minplus.minplus_gemm(A, A, out=Cm, check_status=False)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        minplus.status()
        # e2e through the public call with host buffers
        hA = A.cpu().pin_memory()
        hC = torch.empty_like(hA).pin_memory()
        dA = torch.empty_like(A)
        torch.cuda.synchronize()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record()
        for _ in range(steps):
            dA.copy_(hA, non_blocking=True)
            minplus.minplus_gemm(dA, dA, out=Cm, check_status=False)
            hC.copy_(Cm, non_blocking=True)
        e3.record()
        torch.cuda.synchronize()
        ms_e2e = e2.elapsed_time(e3) / steps
        minplus.status()
        sampler.stop()
        # parity on sampled rows: C[rows] == oracle (A[rows] (min,+) A), word for word
        rows = np.random.default_rng(SEED).choice(N, size=min(check_rows, N), replace=False)
        Ah = hA.numpy()
        ref = orc.minplus_gemm(np.ascontiguousarray(Ah[rows]), Ah)
        mism = int(np.count_nonzero(hC.numpy()[rows].view(np.uint32) != ref.view(np.uint32)))
        r = C.c_double()
        _lib.check(_lib.lib().b2_minplus_calibrate(1 if dt == torch.float32 else 0, C.byref(r)), "calibrate")
        pairs = float(N) ** 3
        res[name] = {"ms": ms, "gops": 2 * pairs / ms / 1e6, "pairs_per_s": pairs / ms * 1e3,
                     "calibrated_pairs_per_s": r.value, "frac_of_calibrated_alu": pairs / ms * 1e3 / r.value,
                     "e2e_ms": ms_e2e, "e2e_gops": 2 * pairs / ms_e2e / 1e6, "clocks": sampler.summary(),
                     "bytes": 4 * N * N, "parity": {"rows_checked": int(rows.shape[0]), "mismatches": mism,
                                                    "against": "oracle C min-plus GEMM, word for word"}}
        del A, Cm, dA, hA, hC
        torch.cuda.empty_cache()
    # CPU baseline: the reference's chunked torch min-plus on a row sample
    rng = np.random.default_rng(SEED)
    rows = 8
    Ah = np.where(rng.uniform(size=(rows, N)) < 0.3, rng.uniform(size=(rows, N)), np.inf).astype(np.float32)
    Bh = np.where(rng.uniform(size=(N, N)) < 0.3, rng.uniform(size=(N, N)), np.inf).astype(np.float32)
    t0 = time.perf_counter()
    orc.min_plus_matmul_chunked(Ah, Bh, block=16)
    t_cpu = (time.perf_counter() - t0) * N / rows
    res["cpu_baseline"] = {"value": 2 * float(N) ** 3 / t_cpu / 1e9, "unit": "Gop/s",
                           "cores": __import__("torch").get_num_threads(), "kind": "port",
                           "sample": f"reference chunked torch min-plus (block 16), fp32, {rows} x {N} times "
                                     f"{N} x {N}, scaled to {N} rows"}
    return res


def spgemm_measure(args, steps: int, check_rows: int) -> dict:
    """CSR x CSR min-plus SpGEMM C = A (min,+) A on a directed ER graph, n = 2^20,
    m = 8 n, int32 weights U{1..1000} (fp32 = w / 1001)."""
    import torch
    import b200sssp
    from b200sssp import minplus
    orc = oracle()
    n = 1 << 20
    hg = b200sssp.gen_er(n, 8 * n, 1, 1000, SEED)
    deg = np.diff(hg.rowptr)
    cand = int(deg[hg.colind].sum())
    peak, peak_kind = load_peaks()
    res = {"n": n, "m": hg.m, "candidates": cand}
    for name in ("int32", "fp32"):
        vals = hg.weights.view(np.int32) if name == "int32" else (hg.weights.astype(np.float32) / np.float32(1001.0))
        Am = (torch.from_numpy(hg.rowptr).cuda(), torch.from_numpy(hg.colind).cuda(), torch.from_numpy(vals).cuda(),
              n)
        for _ in range(max(3, args.warmup)):
            out = minplus.minplus_spgemm(Am, Am)
        nnz_c = int(out[1].numel())
        # parity on sampled rows against the oracle's C SpGEMM (columns sorted on both sides)
        rows = np.sort(np.random.default_rng(SEED).choice(n, size=check_rows, replace=False))
        crp = out[0].cpu().numpy()
        cci = out[1].cpu().numpy()
        cv = out[2].cpu().numpy()
        mism = 0
        for r in rows:
            a0, a1 = hg.rowptr[r], hg.rowptr[r + 1]
            Ar = (np.array([0, a1 - a0], np.int64), hg.colind[a0:a1], vals[a0:a1])
            rrp, rci, rv = orc.minplus_spgemm(Ar, (hg.rowptr, hg.colind, vals), n)
            o = np.argsort(rci, kind="stable")
            got_c = cci[crp[r]:crp[r + 1]]
            got_v = cv[crp[r]:crp[r + 1]]
            if not (np.array_equal(got_c, rci[o]) and np.array_equal(got_v.view(np.uint32), rv[o].view(np.uint32))):
                mism += 1
        del out
        torch.cuda.synchronize()
        ts = []
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(steps):
            e0.record()
            out = minplus.minplus_spgemm(Am, Am)
            e1.record()
            torch.cuda.synchronize()
            ts.append(e0.elapsed_time(e1))
            del out
        ms = float(np.mean(ts))
        bytes_alg = (8 * (n + 1) + 8 * hg.m) + 8 * cand + (8 * (n + 1) + 8 * nnz_c)
        res[name] = {"ms": ms, "ms_min": float(np.min(ts)), "gcand_per_s": cand / ms / 1e6, "nnz_c": nnz_c,
                     "bytes_alg": bytes_alg, "achieved_gbs": bytes_alg / ms / 1e6,
                     "frac_of_hbm": bytes_alg / ms / 1e6 / peak, "peak_kind": peak_kind,
                     "parity": {"rows_checked": int(rows.shape[0]), "rows_mismatched": mism,
                                "against": "oracle C SpGEMM, sorted columns, word for word"}}
        del Am
        torch.cuda.empty_cache()
    # CPU: the oracle's SpGEMM on the first rows (the reference has no CPU SpGEMM)
    rows = 1 << 15
    rp = hg.rowptr[: rows + 1]
    A = (rp, hg.colind[: rp[-1]], hg.weights[: rp[-1]].view(np.int32))
    B = (hg.rowptr, hg.colind, hg.weights.view(np.int32))
    t0 = time.perf_counter()
    orc.minplus_spgemm(A, B, n)
    t_cpu = (time.perf_counter() - t0) * n / rows
    res["cpu_baseline"] = {"value": cand / t_cpu / 1e9, "unit": "G candidates/s", "cores": 1, "kind": "port",
                           "sample": f"oracle C SpGEMM over rows [0,{rows}) of A x A, scaled to {n} rows "
                                     "(the reference has no CPU SpGEMM)"}
    res["hg"] = hg
    return res


def serve_measure(queries: int, rate: float, light_queries: int, seq_queries: int, autotune: bool) -> dict:
    """64 resident graphs (32 grids 64^2 .. 2048^2, 32 RMAT scale 12 .. 20), Poisson
    single-source queries; continuous-batching server vs one-at-a-time solves."""
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
    rep = srv.run_load(queries, rate_qps=rate, seed=SEED, mode="server")
    light = srv.run_load(light_queries, rate_qps=1000.0, seed=SEED + 1, mode="server")      # below capacity
    heavy = srv.run_load(queries, rate_qps=50000.0, seed=SEED + 2, mode="server")           # the top of 1k-50k q/s
    seq = srv.run_load(seq_queries, rate_qps=0.0, seed=SEED, mode="sequential")
    srv.close()
    out = {"server": rep, "light_load_1000qps": light, "heavy_load_50000qps": heavy, "sequential": seq,
           "speedup_over_sequential_qps": rep["qps"] / max(seq["qps"], 1e-9), "graph_gen_s": t_gen,
           "p50_us": rep["p50_us"], "p99_us": rep["p99_us"]}
    if autotune:
        t0 = time.time()
        srv = serving.Server(hbm_budget=120 << 30, autotune=True)
        for g in graphs:
            srv.add_graph(g)
        t_tune = time.time() - t0
        configs = [srv.graph_config(i) for i in range(len(graphs))]
        srv.run_load(256, rate_qps=0.0, seed=99, mode="server")
        tuned = srv.run_load(queries, rate_qps=rate, seed=SEED, mode="server")
        tuned["light_load_1000qps"] = srv.run_load(light_queries, rate_qps=1000.0, seed=SEED + 1, mode="server")
        srv.close()
        tuned["tune_seconds"] = t_tune
        tuned["clusters"] = sum(c["cluster_team"] for c in configs)
        out["autotuned"] = tuned
    for g in graphs:
        g.close()
    return out


def run_extras(args, ctx, line):
    import torch
    detail = line.setdefault("detail", {})
    detail_graphs(args, ctx, detail)
    ctx["g"].close()
    torch.cuda.empty_cache()
    detail["serve"] = _guard(lambda: serve_measure(4096, 10000.0, 1024, 512, autotune=False))
    torch.cuda.empty_cache()
    detail["minplus_N8192"] = _guard(lambda: minplus_measure(args, 8192, 3, 64))
    sp = _guard(lambda: spgemm_measure(args, 3, 512))
    if isinstance(sp, dict):
        sp.pop("hg", None)
    detail["spgemm_er2^20"] = sp
    detail["c1_bf_small"] = _guard(lambda: detail_c1(args))


# ---------------------------------------------------------------------------
# single workloads (one JSON line each)
def _line(metric, value, unit, args, ms_per_step, dtype, config, **extra):
    out = {"metric": metric, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
           "dtype": dtype, "data": "synthetic", "config": config}
    out.update(extra)
    return out


def workload_minplus(args):
    """Dense min-plus GEMM, N x N: value = 2 N^3 (min,+) ops per product / device
    time (Gop/s); roofline against the calibrated rate of the same
    instruction mix on registers (b2_minplus_calibrate)."""
    N = args.n
    res = minplus_measure(args, N, args.steps, 64)
    head = res["int32"]
    return _line("minplus_gops", head["gops"], "Gop/s", args, head["ms"], "int32",
                 {"workload": f"dense_minplus_gemm_N{N}_int32_p0.3_w1-1000", "N": N, "present_p": 0.3,
                  "l2": "operands %.0f MB each > L2; no flush" % (head["bytes"] / 1e6)},
                 e2e={"value": head["e2e_gops"], "unit": "Gop/s", "h2d_bytes_per_step": head["bytes"],
                      "d2h_bytes_per_step": head["bytes"]},
                 gpu_launches=args.steps,
                 roofline={"bound": "alu", "achieved": head["pairs_per_s"] / 1e12,
                           "peak": head["calibrated_pairs_per_s"] / 1e12, "unit": "T (min,+) pairs/s",
                           "frac": head["frac_of_calibrated_alu"], "traffic": None,
                           "peak_kind": "calibrated (b2_minplus_calibrate)", "kernel": "k_minplus_tma<int>"},
                 clocks=head["clocks"], cpu_baseline=res["cpu_baseline"], parity=head["parity"],
                 detail={"fp32": res["fp32"], "int32": res["int32"]})


def workload_spgemm(args):
    """CSR x CSR min-plus SpGEMM on ER 2^20, degree 8: value = candidate
    products per second; roofline: bytes of A, the gathered B rows and C."""
    res = spgemm_measure(args, args.steps, 512)
    hg = res.pop("hg")
    n = hg.n
    head = res["int32"]
    peak, peak_kind = load_peaks()
    # e2e: host CSR in, host CSR out
    import torch
    from b200sssp import minplus
    vals = hg.weights.view(np.int32)
    hrp, hci, hv = (torch.from_numpy(hg.rowptr).pin_memory(), torch.from_numpy(hg.colind).pin_memory(),
                    torch.from_numpy(vals).pin_memory())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        dA = (hrp.cuda(non_blocking=True), hci.cuda(non_blocking=True), hv.cuda(non_blocking=True), n)
        o = minplus.minplus_spgemm(dA, dA)
        host = [x.cpu() for x in o]
    torch.cuda.synchronize()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    h2d = int(hrp.numel() * 8 + hci.numel() * 4 + hv.numel() * 4)
    d2h = int(sum(x.numel() * x.element_size() for x in host))
    return _line("spgemm_gcand_per_s", head["gcand_per_s"], "G candidates/s", args, head["ms"], "int32",
                 {"workload": "minplus_spgemm_er2^20_deg8_AxA_int32", "n": n, "m": hg.m,
                  "candidates": res["candidates"],
                  "l2": "A %.0f MB + expansion > L2; no flush" % ((8 * n + 8 * hg.m) / 1e6)},
                 e2e={"value": res["candidates"] / e2e_ms / 1e6, "unit": "G candidates/s", "h2d_bytes_per_step": h2d,
                      "d2h_bytes_per_step": d2h},
                 gpu_launches=args.steps * 8,
                 roofline={"bound": "hbm", "achieved": head["achieved_gbs"], "peak": peak, "unit": "GB/s",
                           "frac": head["achieved_gbs"] / peak, "traffic": None, "peak_kind": peak_kind,
                           "kernel": "k_rows_warp<int>", "bytes_alg_per_step": head["bytes_alg"]},
                 cpu_baseline=res["cpu_baseline"], parity=head["parity"], detail=res)


def workload_policy(args):
    """Learned schedule (shipped weights) vs the fixed Near-Far delta on the
    held-out RMAT-24 and 4096^2 grid graphs, 8 sources each, distances compared
    word for word.  value = learned GTEPS over both graphs."""
    import b200sssp
    graphs, reach = {}, {}
    for name in ("rmat", "grid"):
        rp, ci, w, fw, _ = build_workload(name, with_library=True)
        srcs = pick_sources(rp, 8, SEED)
        g = b200sssp.Graph.from_arrays(rp, ci, w, weight="u32")
        reach[name] = sum(g.sssp(s, collect_reach=1)[2]["reached_edges"] for s in srcs)
        graphs[name] = (g, srcs)
    res = policy_compare(graphs)
    for name, (g, _) in graphs.items():
        res[name]["fixed_gteps"] = reach[name] / res[name]["fixed_ms"] / 1e6
        res[name]["learned_gteps"] = reach[name] / res[name]["learned_ms"] / 1e6
        g.close()
    tot_e = sum(reach.values())
    tot_f = sum(res[k]["fixed_ms"] for k in graphs)
    tot_l = sum(res[k]["learned_ms"] for k in graphs)
    return _line("sssp_gteps_learned_schedule", tot_e / tot_l / 1e6, "GTEPS", args, tot_l / 16, "u32",
                 {"workload": f"learned_vs_fixed_delta_rmat{SCALE}_and_grid{GRID_SIDE}_u32", "sources": 8},
                 gpu_launches=32,
                 detail={"speedup_over_fixed": tot_f / tot_l, "fixed_gteps": tot_e / tot_f / 1e6, "graphs": res})


def workload_serve(args):
    """Batched serving: value = completed queries per second at --rate; p50 /
    p99 from arrival to result in host memory."""
    rep = serve_measure(args.queries, args.rate, 2048, 1024, autotune=True)
    best = rep["autotuned"] if rep["autotuned"]["qps"] > rep["server"]["qps"] else rep["server"]
    return _line("serve_qps", best["qps"], "queries/s", args, 1e3 / max(best["qps"], 1e-9), "u32",
                 {"workload": f"serve_64graphs_{args.queries}q_poisson{int(args.rate)}qps", "graphs": 64,
                  "queries": args.queries, "rate_qps": args.rate, "hbm_budget_gb": 120},
                 e2e={"value": best["qps"], "unit": "queries/s", "h2d_bytes_per_step": 0,
                      "d2h_bytes_per_step": "distance array of the query's graph"},
                 gpu_launches=None, detail=rep)


def workload_c1(args):
    r = detail_c1(args)
    return _line("bf_small_us_per_solve", r["gpu_bf_us_per_solve"], "us", args, r["gpu_bf_us_per_solve"] / 1e3,
                 "u32", {"workload": r["workload"]}, higher_is_better=False, gpu_launches=args.steps,
                 cpu_baseline={"value": r["reference_bf_seconds"] * 1e6, "unit": "us", "cores": 1, "kind": "port",
                               "sample": r["cpu_baseline"]["sample"]},
                 parity=r["parity"], detail=r)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--policy", default="fixed", choices=["fixed", "learned"])
    ap.add_argument("--method", default="delta", choices=["delta", "bf", "adds"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="headline only (skip the detail configurations)")
    ap.add_argument("--trace-out", default=None, help="write one traced solve's phase list (JSON)")
    ap.add_argument("--workload", default="sssp", choices=["sssp", "policy", "minplus", "spgemm", "serve", "c1"])
    ap.add_argument("--graph", default="rmat", choices=["rmat", "grid"])
    ap.add_argument("--n", type=int, default=8192, help="minplus: matrix order")
    ap.add_argument("--rate", type=float, default=10000.0, help="serve: Poisson arrival rate (queries/s)")
    ap.add_argument("--queries", type=int, default=8192, help="serve: queries")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:   # the reference arm is rank 0's CPU run; other ranks do no work
            print(json.dumps(reference_arm(args)), flush=True)
        return
    if args.workload != "sssp":
        if rank != 0:
            return   # the single workloads are single-GPU measurements (rank 0)
        fn = {"policy": workload_policy, "minplus": workload_minplus, "spgemm": workload_spgemm,
              "serve": workload_serve, "c1": workload_c1}[args.workload]
        print(json.dumps(fn(args)), flush=True)
        return
    line, ctx, rank = headline(args)
    if ctx is not None and not args.no_extras:
        t0 = time.time()
        run_extras(args, ctx, line)
        line["detail"]["extras_seconds"] = time.time() - t0
    elif ctx is not None:
        ctx["g"].close()
    if rank == 0:
        print(json.dumps(line, default=float), flush=True)


if __name__ == "__main__":
    main()
