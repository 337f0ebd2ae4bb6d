"""Oracle: CPU restatement of the reference algorithms -- test infrastructure.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker (or as the timed CPU baseline).  The product
path (libb200sssp.so and the b200sssp package) never imports it.

Two parts:
  * liboracle.so (oracle.c, built by build_oracle()): Dijkstra u32/f32/f64,
    Jacobi Bellman-Ford, dense min-plus, SpGEMM, shortest-path-tree check.
  * numpy ports of the reference's Python path, operation for operation:
      tropical_spmv            <- pytorch_testing/bellman_ford_attempts/Attempt1_June23/minplus_algebra.py:58-102
      sssp_min_plus_bellman_ford <- .../Attempt1_June23/minplus_bellman_ford.py:51-102 (track_pred=False)
      min_plus_matmul_chunked  <- pytorch_testing/matrix_mult_attempts/matrix_mult_chunked.py:1-23
      delta_bucket_count       <- bucket_index rule, HIP_kernel/delta_stepping/src/delta_stepping_hip_CSR.cpp:233-239
    These are what bench.py times as the reference CPU implementation.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRCS = [os.path.join(HERE, "oracle.c"), os.path.join(HERE, "oracle_gen.c")]

_lib = None


def build_oracle(force: bool = False) -> str:
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(f) for f in SRCS):
        tmp = LIB + ".tmp"
        subprocess.run(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off", "-pthread", "-o", tmp,
                        *SRCS, "-lm"], check=True)
        os.replace(tmp, LIB)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build_oracle()
        L = C.CDLL(LIB)
        P = C.c_void_p
        i64 = C.c_int64
        L.orc_dijkstra_u32.argtypes = [i64, P, P, P, i64, P]
        L.orc_dijkstra_f32.argtypes = [i64, P, P, P, i64, P]
        L.orc_dijkstra_u32_hops.argtypes = [i64, P, P, P, i64, P, P]
        L.orc_dijkstra_u32_hops.restype = i64
        L.orc_dijkstra_f64.argtypes = [i64, P, P, P, i64, P]
        L.orc_dijkstra_u32_from.argtypes = [i64, P, P, P, i64, P, C.c_int]
        L.orc_dijkstra_f32_from.argtypes = [i64, P, P, P, i64, P, C.c_int]
        L.orc_bf_jacobi_f32.argtypes = [i64, P, P, P, i64, i64, C.c_int, P, P]
        L.orc_bf_jacobi_f64.argtypes = [i64, P, P, P, i64, i64, C.c_int, P, P]
        L.orc_minplus_gemm_f32.argtypes = [P, P, P, i64, i64, i64, i64, i64, i64]
        L.orc_minplus_gemm_i32.argtypes = [P, P, P, i64, i64, i64, i64, i64, i64]
        for nm in ("orc_minplus_spgemm_f32", "orc_minplus_spgemm_i32"):
            getattr(L, nm).argtypes = [i64, i64, i64, P, P, P, P, P, P, P, P, P, i64]
            getattr(L, nm).restype = i64
        L.orc_validate_spt.argtypes = [i64, P, P, P, C.c_int, i64, P, P]
        L.orc_validate_spt.restype = C.c_int
        pp = C.POINTER(C.c_void_p)
        L.orc_gen_rmat.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint32, C.c_uint32,
                                   C.c_uint64, C.c_int, C.POINTER(i64), C.POINTER(i64), pp, pp, pp]
        L.orc_gen_grid.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_uint64, C.c_int,
                                   C.POINTER(i64), C.POINTER(i64), pp, pp, pp, C.POINTER(C.c_uint32)]
        L.orc_free.argtypes = [P]
        _lib = L
    return _lib


def _host_threads() -> int:
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


def _take(ptr: C.c_void_p, count: int, dtype) -> np.ndarray:
    """Copy a malloc'd C array into numpy and free it."""
    L = lib()
    try:
        if count == 0:
            return np.zeros(0, dtype)
        buf = (C.c_char * (count * np.dtype(dtype).itemsize)).from_address(ptr.value)
        return np.frombuffer(buf, dtype=dtype, count=count).copy()
    finally:
        L.orc_free(ptr)


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             wmin: int = 1, wmax: int = 255, seed: int = 0, threads: int | None = None):
    """Twin of the library's RMAT generator (oracle_gen.c): OUTGOING CSR
    (rowptr int64, colind int32, weights uint32, fweights float32), the same
    bytes as b2_gen_rmat for the same arguments."""
    L = lib()
    n, m = C.c_int64(), C.c_int64()
    rp, ci, w = C.c_void_p(), C.c_void_p(), C.c_void_p()
    r = L.orc_gen_rmat(scale, edge_factor, a, b, c, wmin, wmax, seed, threads or _host_threads(), C.byref(n),
                       C.byref(m), C.byref(rp), C.byref(ci), C.byref(w))
    if r != 0:
        raise ValueError(f"orc_gen_rmat failed ({r})")
    rowptr = _take(rp, n.value + 1, np.int64)
    colind = _take(ci, m.value, np.int32)
    weights = _take(w, m.value, np.uint32)
    fweights = weights.astype(np.float32) / np.float32(float(wmax) + 1.0)
    return rowptr, colind, weights, fweights


def gen_grid(rows: int, cols: int, shortcut_frac: float = 0.02, mu: float = 5.0, sigma: float = 1.0,
             seed: int = 0, threads: int | None = None):
    """Twin of the library's road-like grid generator (oracle_gen.c): the same
    bytes as b2_gen_grid (float weights w / (max w + 1))."""
    L = lib()
    n, m = C.c_int64(), C.c_int64()
    rp, ci, w = C.c_void_p(), C.c_void_p(), C.c_void_p()
    mx = C.c_uint32()
    r = L.orc_gen_grid(rows, cols, shortcut_frac, mu, sigma, seed, threads or _host_threads(), C.byref(n),
                       C.byref(m), C.byref(rp), C.byref(ci), C.byref(w), C.byref(mx))
    if r != 0:
        raise ValueError(f"orc_gen_grid failed ({r})")
    rowptr = _take(rp, n.value + 1, np.int64)
    colind = _take(ci, m.value, np.int32)
    weights = _take(w, m.value, np.uint32)
    fweights = weights.astype(np.float32) / np.float32(float(mx.value) + 1.0)
    return rowptr, colind, weights, fweights


def _p(a: np.ndarray) -> int:
    return a.ctypes.data


def _csr(rowptr, colind):
    return np.ascontiguousarray(rowptr, np.int64), np.ascontiguousarray(colind, np.int32)


def dijkstra(rowptr, colind, weights, source: int) -> np.ndarray:
    """OUTGOING CSR.  uint32 weights -> uint32 dist (0xFFFFFFFF unreachable);
    float32 -> float32 (+inf); float64 -> float64."""
    rp, ci = _csr(rowptr, colind)
    n = rp.shape[0] - 1
    w = np.ascontiguousarray(weights)
    if w.dtype == np.uint32:
        d = np.empty(n, np.uint32)
        lib().orc_dijkstra_u32(n, _p(rp), _p(ci), _p(w), source, _p(d))
    elif w.dtype == np.float32:
        d = np.empty(n, np.float32)
        lib().orc_dijkstra_f32(n, _p(rp), _p(ci), _p(w), source, _p(d))
    else:
        w = w.astype(np.float64)
        d = np.empty(n, np.float64)
        lib().orc_dijkstra_f64(n, _p(rp), _p(ci), _p(w), source, _p(d))
    return d


def dijkstra_warm(rowptr, colind, weights, source: int, initial: np.ndarray) -> np.ndarray:
    """Dijkstra that keeps `initial` as upper bounds and starts from the source
    alone (hip_adds::sssp with initialize_distances = false): uint32 or float32."""
    rp, ci = _csr(rowptr, colind)
    n = rp.shape[0] - 1
    w = np.ascontiguousarray(weights)
    if w.dtype == np.uint32:
        out = np.array(initial, dtype=np.uint32, copy=True)
        lib().orc_dijkstra_u32_from(n, _p(rp), _p(ci), _p(w), source, _p(out), 1)
    else:
        w = np.ascontiguousarray(w, np.float32)
        out = np.array(initial, dtype=np.float32, copy=True)
        lib().orc_dijkstra_f32_from(n, _p(rp), _p(ci), _p(w), source, _p(out), 1)
    return out


def bf_iterations_u32(rowptr, colind, weights, source: int) -> tuple[int, np.ndarray]:
    """Jacobi Bellman-Ford iteration count (max min-hop shortest path + 1) and
    the distances, from a (dist, hops) Dijkstra on OUTGOING CSR."""
    rp, ci = _csr(rowptr, colind)
    n = rp.shape[0] - 1
    w = np.ascontiguousarray(weights, np.uint32)
    d = np.empty(n, np.uint32)
    h = np.empty(n, np.uint32)
    mx = lib().orc_dijkstra_u32_hops(n, _p(rp), _p(ci), _p(w), source, _p(d), _p(h))
    return int(mx) + 1, d


def bf_jacobi(in_rowptr, in_colind, weights, source: int, max_iters: int = -1, detect_negative: bool = False):
    """INCOMING CSR Jacobi BF.  Returns (dist, iterations_used, converged, negative_cycle, first_unchanged)."""
    rp, ci = _csr(in_rowptr, in_colind)
    n = rp.shape[0] - 1
    w = np.ascontiguousarray(weights)
    out = np.zeros(4, np.int64)
    if w.dtype == np.float32:
        d = np.empty(n, np.float32)
        lib().orc_bf_jacobi_f32(n, _p(rp), _p(ci), _p(w), source, max_iters, int(detect_negative), _p(d), _p(out))
    else:
        w = w.astype(np.float64)
        d = np.empty(n, np.float64)
        lib().orc_bf_jacobi_f64(n, _p(rp), _p(ci), _p(w), source, max_iters, int(detect_negative), _p(d), _p(out))
    return d, int(out[0]), bool(out[1]), bool(out[2]), int(out[3])


def minplus_gemm(A: np.ndarray, B: np.ndarray) -> np.ndarray:
    M, K = A.shape
    N = B.shape[1]
    A = np.ascontiguousarray(A)
    B = np.ascontiguousarray(B)
    Cm = np.empty((M, N), A.dtype)
    fn = lib().orc_minplus_gemm_f32 if A.dtype == np.float32 else lib().orc_minplus_gemm_i32
    fn(_p(A), _p(B), _p(Cm), M, N, K, K, N, N)
    return Cm


def minplus_spgemm(A, B, ncols_b: int):
    """A, B = (rowptr int64, colind int32, values f32|i32).  Returns (rowptr, colind, values), sorted rows."""
    arp, aci = _csr(A[0], A[1])
    brp, bci = _csr(B[0], B[1])
    av = np.ascontiguousarray(A[2])
    bv = np.ascontiguousarray(B[2])
    M = arp.shape[0] - 1
    K = brp.shape[0] - 1
    fn = lib().orc_minplus_spgemm_f32 if av.dtype == np.float32 else lib().orc_minplus_spgemm_i32
    nnz = fn(M, K, ncols_b, _p(arp), _p(aci), _p(av), _p(brp), _p(bci), _p(bv), None, None, None, 0)
    crp = np.empty(M + 1, np.int64)
    cci = np.empty(max(nnz, 1), np.int32)
    cv = np.empty(max(nnz, 1), av.dtype)
    fn(M, K, ncols_b, _p(arp), _p(aci), _p(av), _p(brp), _p(bci), _p(bv), _p(crp), _p(cci), _p(cv), nnz)
    return crp, cci[:nnz], cv[:nnz]


def validate_spt(rowptr, colind, weights, source: int, dist: np.ndarray, pred: np.ndarray) -> int:
    rp, ci = _csr(rowptr, colind)
    w = np.ascontiguousarray(weights)
    kind = 0 if w.dtype == np.uint32 else 1
    d = np.ascontiguousarray(dist, np.uint32 if kind == 0 else np.float32)
    pr = np.ascontiguousarray(pred, np.int32)
    return lib().orc_validate_spt(rp.shape[0] - 1, _p(rp), _p(ci), _p(w), kind, source, _p(d), _p(pr))


# ---------------------------------------------------------------------------
# numpy ports of the reference's Python path
INF = np.float64(np.inf)


def tropical_spmv(indptr: np.ndarray, indices: np.ndarray, data: np.ndarray, d: np.ndarray) -> np.ndarray:
    """d_new[v] = min over row v of d[indices] + data (INCOMING CSR; empty rows +inf)."""
    n = indptr.shape[0] - 1
    if indices.shape[0] == 0:
        return np.full(n, INF)
    candidates = d[indices] + data
    has = indptr[1:] > indptr[:-1]
    out = np.full(n, INF)
    if not np.any(has):
        return out
    out[has] = np.minimum.reduceat(candidates, indptr[:-1][has])
    return out


def sssp_min_plus_bellman_ford(indptr, indices, data, source: int, max_iters: int | None = None,
                               iteration_hook=None):
    """Returns (dist float64, iterations_used, converged, has_negative_cycle)."""
    indptr = np.asarray(indptr, np.int64)
    indices = np.asarray(indices)
    data = np.asarray(data, np.float64)
    n = indptr.shape[0] - 1
    if max_iters is None:
        max_iters = n - 1
    d = np.full(n, INF)
    d[source] = 0.0
    converged = False
    used = 0
    for it in range(max_iters):
        used = it + 1
        d_new = np.minimum(d, tropical_spmv(indptr, indices, data, d))
        if iteration_hook is not None:
            iteration_hook(used)
        if np.array_equal(d_new, d) or np.all(np.isclose(d_new, d) | (np.isinf(d_new) & np.isinf(d))):
            d = d_new
            converged = True
            break
        d = d_new
    d_check = np.minimum(d, tropical_spmv(indptr, indices, data, d))
    neg = not np.all(np.isclose(d_check, d) | (np.isinf(d_check) & np.isinf(d)))
    return d, used, converged, neg


class RowBlocks:
    """An INCOMING CSR cut into row blocks of about equal arc counts, one per
    host thread, for the row-parallel form of sssp_min_plus_bellman_ford."""

    def __init__(self, indptr, indices, data, threads: int | None = None):
        indptr = np.asarray(indptr, np.int64)
        self.n = indptr.shape[0] - 1
        self.m = int(indptr[-1])
        self.threads = max(1, threads or _host_threads())
        cuts = np.searchsorted(indptr, np.linspace(0, self.m, self.threads + 1)).tolist()
        cuts[0], cuts[-1] = 0, self.n
        self.blocks = []
        for a, b in zip(cuts[:-1], cuts[1:]):
            if b <= a:
                continue
            e0, e1 = int(indptr[a]), int(indptr[b])
            self.blocks.append((a, b, indptr[a:b + 1] - e0, np.asarray(indices[e0:e1]),
                                np.asarray(data[e0:e1], np.float64)))
        from concurrent.futures import ThreadPoolExecutor
        self.pool = ThreadPoolExecutor(max_workers=len(self.blocks) or 1)

    def relax(self, d: np.ndarray) -> np.ndarray:
        """np.minimum(d, tropical_spmv(A, d)), block by block (numpy's gather
        and reduceat release the GIL, so the blocks run in parallel)."""
        out = np.empty_like(d)

        def one(blk):
            a, b, rp, ci, dv = blk
            out[a:b] = np.minimum(d[a:b], tropical_spmv(rp, ci, dv, d))

        list(self.pool.map(one, self.blocks))
        return out

    def close(self):
        self.pool.shutdown()


def sssp_min_plus_bellman_ford_rows(A: RowBlocks, source: int, max_iters: int | None = None):
    """sssp_min_plus_bellman_ford (minplus_bellman_ford.py:51-102, track_pred=False)
    with every round's tropical SpMV split into row blocks over host threads:
    the same rounds, the same stopping test and the same negative-cycle round,
    so the same (dist, iterations_used, converged, has_negative_cycle)."""
    n = A.n
    if max_iters is None:
        max_iters = n - 1
    d = np.full(n, INF)
    d[source] = 0.0
    converged = False
    used = 0
    for it in range(max_iters):
        used = it + 1
        d_new = A.relax(d)
        if np.array_equal(d_new, d) or np.all(np.isclose(d_new, d) | (np.isinf(d_new) & np.isinf(d))):
            d = d_new
            converged = True
            break
        d = d_new
    d_check = A.relax(d)
    neg = not np.all(np.isclose(d_check, d) | (np.isinf(d_check) & np.isinf(d)))
    return d, used, converged, neg


def min_plus_matmul_chunked(A: np.ndarray, B: np.ndarray, block: int = 16) -> np.ndarray:
    """C = A (min,+) B by k-blocks of broadcast add + min (the reference's chunked torch loop)."""
    import torch
    At = torch.from_numpy(np.ascontiguousarray(A))
    Bt = torch.from_numpy(np.ascontiguousarray(B))
    m, n = At.shape
    p = Bt.shape[1]
    Cm = torch.full((m, p), float("inf"), dtype=At.dtype)
    for k0 in range(0, n, block):
        k1 = min(k0 + block, n)
        partial = At[:, k0:k1].unsqueeze(-1) + Bt[k0:k1, :].unsqueeze(0)
        Cm = torch.minimum(Cm, partial.amin(dim=1))
    return Cm.numpy()


def delta_bucket_count(dist: np.ndarray, delta, weight: str) -> int:
    """Number of distinct buckets among reached distances = the reference's
    delta-stepping iterations_used when it converges."""
    if weight == "u32":
        d = np.asarray(dist, np.uint32)
        d = d[d != 0xFFFFFFFF].astype(np.uint64)
        return int(np.unique(d // np.uint64(int(delta))).shape[0])
    d = np.asarray(dist, np.float32)
    d = d[np.isfinite(d)]
    inv = np.float32(1.0) / np.float32(delta)
    b = np.floor(d * inv).astype(np.float64)
    b = np.clip(b, 0, float(0x3fffffff - 1))
    return int(np.unique(b).shape[0])


# ---- schedule-policy MLP in FP64 (no reference counterpart) ------------------
# Layout of the 5955 parameters: W1[64x24] b1[64] W2[64x64] b2[64] W3[3x64] b3[3].
def bf16_round(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float32."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _mlp_unpack(params):
    p = np.asarray(params, np.float64)
    o = 0
    out = []
    for shape in ((64, 24), (64,), (64, 64), (64,), (3, 64), (3,)):
        k = int(np.prod(shape))
        out.append(p[o:o + k].reshape(shape))
        o += k
    assert o == 5955 == p.size
    return out


def mlp_forward(params, Xn):
    """Outputs (B x 3) for standardized features Xn, FP64 throughout."""
    W1, b1, W2, b2, W3, b3 = _mlp_unpack(params)
    h1 = np.maximum(Xn @ W1.T + b1, 0.0)
    h2 = np.maximum(h1 @ W2.T + b2, 0.0)
    return h2 @ W3.T + b3


def mlp_loss_grad(params, Xn, T):
    """Mean loss sum_k (y_k - t_k)^2 over the three outputs and its gradient
    with respect to the 5955 parameters, FP64."""
    W1, b1, W2, b2, W3, b3 = _mlp_unpack(params)
    Xn = np.asarray(Xn, np.float64)
    T = np.asarray(T, np.float64)
    B = Xn.shape[0]
    a1 = Xn @ W1.T + b1
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ W2.T + b2
    h2 = np.maximum(a2, 0.0)
    y = h2 @ W3.T + b3
    e = y - T
    loss = (e ** 2).sum(1)
    dy = 2.0 * e / B
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    dh2 = (dy @ W3) * (a2 > 0)
    gW2 = dh2.T @ h1
    gb2 = dh2.sum(0)
    dh1 = (dh2 @ W2) * (a1 > 0)
    gW1 = dh1.T @ Xn
    gb1 = dh1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return float(loss.mean()), g
