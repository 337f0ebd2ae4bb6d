"""Generate the golden fixtures under tests/golden/ from the REFERENCE's own code.

Run in a container that has the reference checkout (read-only):

    python tests/golden/make_golden.py /path/to/rips2026-amd

It imports the reference's Python path (pytorch_testing/...) and records its
outputs on seeded inputs.  The fixtures are what pins the oracle
(tests/test_oracle_golden.py) and the CUDA path (tests/test_gpu_*.py); the
reference itself is not needed afterwards.

Fixtures written:
  bf_py.npz         reference sssp_min_plus_bellman_ford (minplus_bellman_ford.py:51-102)
                    on: the RRG worked example (test_minplus_bellman_ford.py:174-219),
                    seeded random graphs with float weights, DAGs with negative
                    weights, a negative cycle, and the n=4096 / m=32768 ER graph
                    with uint32 weights U{1..100}, source 0.
  dense_kats.npz    the 14 known-answer cases of
                    HIP_kernel/bellman_ford/tests/test_correctness.cpp:246-528 with
                    their expected distances, plus the reference python BF result.
  minplus.npz       reference min_plus_matmul (matrix_mult_chunked.py:1-23), fp32
                    and int32-as-float64, on seeded matrices with +inf / missing entries.
  bucketed.npz      reference bucketted_bellman_ford (bucketed_bellman_ford:1-71,
                    device="cpu") on seeded graphs, several deltas.
  tiny_gr.json      the five-vertex graph of Charlotte_ADS_Float_Attempt/tools/make_tiny_gr.py
                    and its expected distances (check_tiny_output.py:10).
  tiny.gr           that graph as the reference's own tool writes it (Lonestar binary .gr),
                    with tiny_gr.json's expected distances read from check_tiny_output.py.
                    `python tests/golden/make_golden.py REF --only tiny` regenerates these two.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def load_reference(ref: str):
    pt = os.path.join(ref, "pytorch_testing")
    sys.path[:0] = [pt, os.path.join(pt, "bellman_ford_attempts", "Attempt1_June23")]
    import minplus_algebra as ma  # noqa: E402
    import minplus_bellman_ford as mbf  # noqa: E402
    import torch  # noqa: E402
    import time  # noqa: E402
    ns_mm = {"torch": torch, "time": time}
    exec(open(os.path.join(pt, "matrix_mult_attempts", "matrix_mult_chunked.py")).read(), ns_mm)
    ns_bk = {"torch": torch, "time": time}
    exec(open(os.path.join(pt, "bellman_ford_attempts", "bucketed_bellman_ford")).read(), ns_bk)
    return ma, mbf, ns_mm["min_plus_matmul"], ns_bk["bucketted_bellman_ford"]


def edges_to_incoming(n, edges):
    """(u, v, w) list -> incoming CSR with parallel edges min-reduced, columns sorted."""
    best = {}
    for u, v, w in edges:
        k = (v, u)
        if k not in best or w < best[k]:
            best[k] = w
    rows = [[] for _ in range(n)]
    for (v, u), w in best.items():
        rows[v].append((u, w))
    rp = [0]
    ci, dv = [], []
    for v in range(n):
        for u, w in sorted(rows[v]):
            ci.append(u)
            dv.append(w)
        rp.append(len(ci))
    return np.array(rp, np.int64), np.array(ci, np.int32), np.array(dv, np.float64)


def random_edges(n, n_edges, seed, lo, hi, dag=False):
    rng = np.random.default_rng(seed)
    seen, out = set(), []
    while len(out) < n_edges:
        u, v = (int(x) for x in rng.integers(0, n, 2))
        if u == v or (u, v) in seen or (dag and v <= u):
            if dag and len(seen) >= n * (n - 1) // 2:
                break
            continue
        seen.add((u, v))
        out.append((u, v, float(rng.uniform(lo, hi))))
    return out


def main(ref: str) -> None:
    ma, mbf, min_plus_matmul, bucketted_bellman_ford = load_reference(ref)
    import torch
    import scipy.sparse as sp

    # ---------------------------------------------------------------- bf_py
    cases = []
    rrg = [(0, 1, 1.5), (0, 4, 0.7), (1, 7, 0.3), (1, 5, 0.4), (4, 5, 0.3), (4, 6, 1.1), (5, 6, 1.0),
           (5, 8, 1.2), (6, 9, 2.1), (7, 6, 2.1), (8, 9, 2.5)]
    cases.append(("rrg_example", 10, rrg, 0, None))
    for t in range(12):
        rng = np.random.default_rng(100 + t)
        n = int(rng.integers(10, 120))
        cases.append((f"random_{t}", n, random_edges(n, int(n * rng.uniform(2, 6)), 200 + t, 0.5, 20.0), 0, None))
    for t in range(4):
        n = 30 + 10 * t
        cases.append((f"dag_negative_{t}", n, random_edges(n, 3 * n, 300 + t, -5.0, 20.0, dag=True), 0, None))
    cases.append(("negative_cycle", 3, [(0, 1, 1.0), (1, 2, -5.0), (2, 1, 1.0)], 0, 3))
    cases.append(("hop_limited", 40, random_edges(40, 160, 7, 0.5, 20.0), 0, 3))
    cases.append(("single_node", 1, [], 0, None))
    cases.append(("disconnected", 3, [(0, 1, 1.0)], 0, None))
    out = {}
    for name, n, edges, src, mi in cases:
        A = ma.tropical_matrix_from_edges(n, edges)
        r = mbf.sssp_min_plus_bellman_ford(A, src, max_iters=mi)
        rp, ci, dv = edges_to_incoming(n, edges)
        out[f"{name}/rowptr"] = rp
        out[f"{name}/colind"] = ci
        out[f"{name}/data"] = dv
        out[f"{name}/meta"] = np.array([n, src, -1 if mi is None else mi, r.iterations_used, int(r.converged),
                                        int(r.has_negative_cycle)], np.int64)
        out[f"{name}/dist"] = r.dist
        out[f"{name}/pred"] = r.pred
    # C1: ER n=4096, m=32768, uint32 U{1..100}, source 0 (library generator, seed 0)
    sys.path.insert(0, os.path.join(REPO, "rips2026-amd_b200"))
    import b200sssp
    g = b200sssp.gen_er(4096, 32768, 1, 100, 0)
    gi = g.transpose()
    A = sp.csr_matrix((gi.weights.astype(np.float64), gi.colind, gi.rowptr), shape=(g.n, g.n))
    r = mbf.sssp_min_plus_bellman_ford(A, 0, track_pred=False)
    out["c1_er4096/out_rowptr"] = g.rowptr
    out["c1_er4096/out_colind"] = g.colind
    out["c1_er4096/weights"] = g.weights
    out["c1_er4096/meta"] = np.array([g.n, 0, -1, r.iterations_used, int(r.converged), int(r.has_negative_cycle)],
                                     np.int64)
    out["c1_er4096/dist"] = r.dist
    out["names"] = np.array([c[0] for c in cases] + ["c1_er4096"])
    np.savez_compressed(os.path.join(HERE, "bf_py.npz"), **out)

    # ---------------------------------------------------------------- dense KATs
    I = float("inf")
    kats = []

    def add(name, n, src, edges, expected):
        A = ma.tropical_matrix_from_edges(n, edges)
        r = mbf.sssp_min_plus_bellman_ford(A, src)
        ea = np.array(edges, np.float64).reshape(-1, 3)
        kats.append((name, np.array([n, src, r.iterations_used], np.int64), ea,
                     np.array(expected, np.float64), np.asarray(r.dist, np.float64)))

    def exp(n, pairs):
        e = [I] * n
        for k, v in pairs:
            e[k] = v
        return e

    def flat(n, mat):   # dense incoming: mat[v*n+u] = w(u->v)
        return [(u, v, mat[v * n + u]) for v in range(n) for u in range(n) if mat[v * n + u] != I]

    add("single_vertex", 1, 0, [], exp(1, [(0, 0.0)]))
    add("two_vertices_unreachable", 2, 0, [], exp(2, [(0, 0.0)]))
    add("flattened_diamond_positive", 4, 0,
        flat(4, [I, I, I, I, 2.0, I, I, I, 5.0, 1.0, I, I, I, 4.0, 1.0, I]),
        exp(4, [(0, 0.0), (1, 2.0), (2, 3.0), (3, 4.0)]))
    add("flattened_negative_edges_no_cycle", 5, 0,
        flat(5, [I, I, I, I, 2.0, 6.0, I, I, -2.0, I, 7.0, 8.0, I, I, I, I, 5.0, -3.0, I, 7.0, I, -4.0, 9.0, I, I]),
        exp(5, [(0, 0.0), (1, 2.0), (2, 7.0), (3, 4.0), (4, -2.0)]))
    add("sparse_disconnected_components", 6, 0, [(0, 1, 3.0), (1, 2, 4.0), (3, 4, 1.0), (4, 5, 1.0)],
        exp(6, [(0, 0.0), (1, 3.0), (2, 7.0)]))
    add("sparse_zero_weight_edges", 6, 0,
        [(0, 1, 0.0), (0, 2, 5.0), (1, 2, 0.0), (2, 3, 0.0), (1, 4, 2.0), (4, 5, 0.0), (3, 5, 4.0)],
        exp(6, [(0, 0.0), (1, 0.0), (2, 0.0), (3, 0.0), (4, 2.0), (5, 2.0)]))
    add("sparse_duplicate_edges_keep_min", 5, 0,
        [(0, 1, 10.0), (0, 1, 3.0), (1, 2, 4.0), (0, 2, 20.0), (2, 3, 1.0), (1, 3, 100.0), (3, 4, -2.0)],
        exp(5, [(0, 0.0), (1, 3.0), (2, 7.0), (3, 8.0), (4, 6.0)]))
    add("sparse_source_not_zero", 7, 3,
        [(3, 0, 2.0), (3, 4, 1.0), (4, 5, 1.0), (5, 6, 1.0), (0, 1, 3.0), (1, 2, 3.0), (3, 2, 10.0), (6, 2, -4.0)],
        exp(7, [(0, 2.0), (1, 5.0), (2, -1.0), (3, 0.0), (4, 1.0), (5, 2.0), (6, 3.0)]))
    add("sparse_negative_edges_branching", 8, 0,
        [(0, 1, 4.0), (0, 2, 1.0), (2, 1, -2.0), (1, 3, 2.0), (2, 3, 5.0), (3, 4, 1.0), (1, 5, 10.0),
         (4, 5, -1.0), (5, 6, 2.0), (2, 7, 8.0), (6, 7, -3.0)],
        exp(8, [(0, 0.0), (1, -1.0), (2, 1.0), (3, 1.0), (4, 2.0), (5, 1.0), (6, 3.0), (7, 0.0)]))
    add("sparse_unreachable_negative_edges", 5, 0, [(0, 1, 2.0), (1, 2, 2.0), (3, 4, -5.0)],
        exp(5, [(0, 0.0), (1, 2.0), (2, 4.0)]))
    e, x = [], [I] * 100   # 10x10 right/down grid
    for r_ in range(10):
        for c_ in range(10):
            node = r_ * 10 + c_
            x[node] = float(2 * r_ + c_)
            if c_ + 1 < 10:
                e.append((node, node + 1, 1.0))
            if r_ + 1 < 10:
                e.append((node, node + 10, 2.0))
    add("sparse_grid_10x10_directed_right_down", 100, 0, e, x)
    e = [(f, t, float(t - f) if f < t else float(100 + f - t)) for f in range(10) for t in range(10) if f != t]
    add("dense_complete_10_positive_cycles", 10, 0, e, [float(i) for i in range(10)])
    e = [(0, v, float(v)) for v in range(1, 1024)]
    for f in range(1024):
        for off in range(-16, 49):
            if off == 0:
                continue
            t = (f + off + 1024) % 1024
            e.append((f, t, float(t - f) + float((abs(off) % 5) + 1)))
    add("medium_connected_1024_local_density", 1024, 0, e, [float(i) for i in range(1024)])
    e = [(0, v, float((v % 97) + 1)) for v in range(1, 10000)] + [(0, 5000, 1.0), (5000, 9999, -5.0)]
    x = [0.0] + [float((v % 97) + 1) for v in range(1, 10000)]
    x[5000] = 1.0
    x[9999] = -4.0
    add("large_sparse_star_10000_with_two_hop_improvement", 10000, 0, e, x)
    kz = {"names": np.array([k[0] for k in kats])}
    for name, meta, ea, expd, pyd in kats:
        kz[f"{name}/meta"], kz[f"{name}/edges"] = meta, ea
        kz[f"{name}/expected"], kz[f"{name}/python_dist"] = expd, pyd
    np.savez_compressed(os.path.join(HERE, "dense_kats.npz"), **kz)

    # ---------------------------------------------------------------- minplus
    rng = np.random.default_rng(11)
    mm = {}
    for t, (M, K, N) in enumerate([(33, 47, 29), (64, 64, 64), (17, 100, 5)]):
        A = rng.uniform(0, 1, (M, K)).astype(np.float32)
        B = rng.uniform(0, 1, (K, N)).astype(np.float32)
        A[rng.uniform(size=A.shape) < 0.6] = np.inf
        B[rng.uniform(size=B.shape) < 0.6] = np.inf
        Cr = min_plus_matmul(torch.from_numpy(A), torch.from_numpy(B), block=16).numpy()
        mm[f"f32_{t}/A"], mm[f"f32_{t}/B"], mm[f"f32_{t}/C"] = A, B, Cr
        Ai = rng.integers(1, 1001, (M, K)).astype(np.int64)
        Bi = rng.integers(1, 1001, (K, N)).astype(np.int64)
        Ai[rng.uniform(size=Ai.shape) < 0.7] = 1073741823
        Bi[rng.uniform(size=Bi.shape) < 0.7] = 1073741823
        Ci = min_plus_matmul(torch.from_numpy(Ai.astype(np.float64)), torch.from_numpy(Bi.astype(np.float64)),
                             block=16).numpy()
        mm[f"i32_{t}/A"], mm[f"i32_{t}/B"], mm[f"i32_{t}/C"] = Ai.astype(np.int32), Bi.astype(np.int32), Ci
    np.savez_compressed(os.path.join(HERE, "minplus.npz"), **mm)

    # ---------------------------------------------------------------- bucketed
    bk = {}
    for t, (n, deg, delta) in enumerate([(300, 4, 5.0), (500, 8, 20.0), (200, 3, 1.0)]):
        rng = np.random.default_rng(40 + t)
        src = rng.integers(0, n, n * deg)
        dst = rng.integers(0, n, n * deg)
        keep = src != dst
        src, dst = src[keep], dst[keep]
        w = rng.integers(1, 50, src.shape[0]).astype(np.float32)
        order = np.lexsort((dst, src))
        src, dst, w = src[order], dst[order], w[order]
        rowptr = np.zeros(n + 1, np.int64)
        np.add.at(rowptr, src + 1, 1)
        rowptr = np.cumsum(rowptr)
        d = bucketted_bellman_ford(torch.from_numpy(rowptr), torch.from_numpy(dst.astype(np.int64)),
                                   torch.from_numpy(w), 0, n, delta=delta, device="cpu").numpy()
        bk[f"b{t}/rowptr"], bk[f"b{t}/col"], bk[f"b{t}/w"] = rowptr, dst.astype(np.int32), w
        bk[f"b{t}/dist"], bk[f"b{t}/delta"] = d, np.array([delta], np.float32)
    np.savez_compressed(os.path.join(HERE, "bucketed.npz"), **bk)

    tiny_fixtures(ref)
    print("fixtures written to", HERE)


def tiny_fixtures(ref: str) -> None:
    """The reference's tiny Lonestar graph, written by its own make_tiny_gr.py, and the
    expected distances of its check_tiny_output.py."""
    import runpy
    import subprocess
    tools = os.path.join(ref, "HIP_kernel", "faster_GPU_algo", "Charlotte_ADS_Float_Attempt", "tools")
    gr = os.path.join(HERE, "tiny.gr")
    subprocess.run([sys.executable, os.path.join(tools, "make_tiny_gr.py"), gr], check=True)
    expected = runpy.run_path(os.path.join(tools, "check_tiny_output.py"), run_name="golden")["EXPECTED"]
    raw = open(gr, "rb").read()
    _, _, n, m = np.frombuffer(raw[:32], np.uint64).tolist()
    ends = np.frombuffer(raw[32:32 + 8 * n], np.uint64)
    dst = np.frombuffer(raw[32 + 8 * n:32 + 8 * n + 4 * m], np.uint32)
    off = 32 + 8 * n + 4 * m + (4 if m % 2 else 0)
    w = np.frombuffer(raw[off:off + 4 * m], np.float32)
    tiny = {"n": int(n), "out_rowptr": [0] + ends.astype(int).tolist(), "out_colind": dst.astype(int).tolist(),
            "weights": w.astype(float).tolist(), "source": 0,
            "expected": [None if np.isinf(expected[v]) else float(expected[v]) for v in range(int(n))]}
    with open(os.path.join(HERE, "tiny_gr.json"), "w") as f:
        json.dump(tiny, f)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if a != "--only" and a != "tiny"]
    ref_dir = args[0] if args else os.environ.get("B2_REFERENCE_DIR", "")
    if not ref_dir or not os.path.isdir(ref_dir):
        sys.exit("usage: make_golden.py <reference checkout> [--only tiny]  (or set B2_REFERENCE_DIR)")
    if "--only" in sys.argv:
        tiny_fixtures(ref_dir)
    else:
        main(ref_dir)
