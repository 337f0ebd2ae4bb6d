"""b200sssp: B200-native SSSP and min-plus products (Python side).

Thin host layer over the C ABI in include/b200sssp.h (libb200sssp.so built
in-tree).  Device buffers are torch CUDA tensors; every solve runs the
library's CUDA kernels and nothing else: there is no CPU path here.

    g = b200sssp.Graph.from_host(hg)           # resident outgoing CSR
    dist, pred, st = g.sssp(0, method="delta")  # one persistent launch
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import B2Error, LibraryMissing, check, default_opts, lib  # noqa: F401

__all__ = ["HostGraph", "Graph", "gen_er", "gen_rmat", "gen_grid", "B2Error", "LibraryMissing",
           "minplus_gemm", "apsp", "minplus_spgemm", "csrbin_read", "csrbin_write", "dimacs_read",
           "dimacs_to_csrbin", "lonestar_read", "lonestar_write"]


# ---------------------------------------------------------------------------
@dataclass
class HostGraph:
    """CSR in host memory (numpy).  orientation: 'outgoing' or 'incoming'."""
    n: int
    rowptr: np.ndarray      # int64[n+1]
    colind: np.ndarray      # int32[m]
    weights: np.ndarray     # uint32[m]
    fweights: np.ndarray    # float32[m]
    orientation: str = "outgoing"

    @property
    def m(self) -> int:
        return int(self.colind.shape[0])

    def transpose(self) -> "HostGraph":
        src = _to_hostcsr(self)
        out = _lib.HostCSR()
        check(lib().b2_host_csr_transpose(C.byref(src), C.byref(out)), "transpose")
        hg = _from_hostcsr(out, "incoming" if self.orientation == "outgoing" else "outgoing")
        return hg

    def out_degree(self) -> np.ndarray:
        if self.orientation != "outgoing":
            raise ValueError("out_degree needs an outgoing CSR")
        return np.diff(self.rowptr)


def _from_hostcsr(h: _lib.HostCSR, orientation: str) -> HostGraph:
    n, m = int(h.n), int(h.m)
    try:
        rowptr = np.ctypeslib.as_array(h.rowptr, shape=(n + 1,)).copy()
        colind = np.ctypeslib.as_array(h.colind, shape=(max(m, 1),))[:m].copy()
        w = np.ctypeslib.as_array(h.weights, shape=(max(m, 1),))[:m].copy()
        fw = (np.ctypeslib.as_array(h.fweights, shape=(max(m, 1),))[:m].copy()
              if bool(h.fweights) else w.astype(np.float32))
    finally:
        lib().b2_host_csr_free(C.byref(h))
    return HostGraph(n, rowptr, colind, w, fw, orientation)


def _to_hostcsr(g: HostGraph) -> _lib.HostCSR:
    h = _lib.HostCSR()
    h.n, h.m = g.n, g.m
    g.rowptr = np.ascontiguousarray(g.rowptr, np.int64)
    g.colind = np.ascontiguousarray(g.colind, np.int32)
    g.weights = np.ascontiguousarray(g.weights, np.uint32)
    g.fweights = np.ascontiguousarray(g.fweights, np.float32)
    h.rowptr = g.rowptr.ctypes.data_as(C.POINTER(C.c_int64))
    h.colind = g.colind.ctypes.data_as(C.POINTER(C.c_int32))
    h.weights = g.weights.ctypes.data_as(C.POINTER(C.c_uint32))
    h.fweights = g.fweights.ctypes.data_as(C.POINTER(C.c_float))
    return h


def gen_er(n: int, m: int, wmin: int = 1, wmax: int = 100, seed: int = 0) -> HostGraph:
    """Directed Erdos-Renyi: m distinct arcs, no self-loops, U{wmin..wmax} weights."""
    h = _lib.HostCSR()
    check(lib().b2_gen_er(n, m, wmin, wmax, seed, C.byref(h)), "gen_er")
    return _from_hostcsr(h, "outgoing")


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             wmin: int = 1, wmax: int = 255, seed: int = 0) -> HostGraph:
    """Symmetrised RMAT (self-loops and duplicates removed), U{wmin..wmax} weights."""
    h = _lib.HostCSR()
    check(lib().b2_gen_rmat(scale, edge_factor, a, b, c, wmin, wmax, seed, C.byref(h)), "gen_rmat")
    return _from_hostcsr(h, "outgoing")


def gen_grid(rows: int, cols: int, shortcut_frac: float = 0.02, mu: float = 5.0, sigma: float = 1.0,
             seed: int = 0) -> HostGraph:
    """4-neighbour bidirectional grid + random long-range shortcut pairs, ceil(lognormal) weights."""
    h = _lib.HostCSR()
    check(lib().b2_gen_grid(rows, cols, shortcut_frac, mu, sigma, seed, C.byref(h)), "gen_grid")
    return _from_hostcsr(h, "outgoing")


def csrbin_write(path: str, g: HostGraph) -> None:
    """Write an INCOMING float CSR as a RIPSCSR1 .csrbin file."""
    if g.orientation != "incoming":
        raise ValueError("RIPSCSR1 stores incoming CSR")
    rp = np.ascontiguousarray(g.rowptr, np.int64)
    ci = np.ascontiguousarray(g.colind, np.int32)
    fv = np.ascontiguousarray(g.fweights, np.float32)
    check(lib().b2_csrbin_write(path.encode(), g.n, g.m, rp.ctypes.data, ci.ctypes.data, fv.ctypes.data),
          "csrbin_write")


def csrbin_read(path: str) -> HostGraph:
    h = _lib.HostCSR()
    check(lib().b2_csrbin_read(path.encode(), C.byref(h)), "csrbin_read")
    return _from_hostcsr(h, "incoming")


def dimacs_read(path: str) -> tuple[HostGraph, int, int]:
    """DIMACS shortest-path .gr text as an INCOMING float CSR, read like the
    reference's gr_to_csr converter; returns (graph, declared arcs, arc lines read)."""
    h = _lib.HostCSR()
    declared, loaded = C.c_int64(), C.c_int64()
    check(lib().b2_dimacs_read(path.encode(), C.byref(h), C.byref(declared), C.byref(loaded)), "dimacs_read")
    return _from_hostcsr(h, "incoming"), declared.value, loaded.value


def dimacs_to_csrbin(gr_path: str, csrbin_path: str) -> int:
    """The reference converter: DIMACS .gr -> RIPSCSR1 .csrbin; returns the arcs kept."""
    nnz = C.c_int64()
    check(lib().b2_dimacs_to_csrbin(gr_path.encode(), csrbin_path.encode(), C.byref(nnz)), "dimacs_to_csrbin")
    return nnz.value


def lonestar_read(path: str, float_weights: bool = True) -> HostGraph:
    """Galois / Lonestar binary .gr (version 1) as an OUTGOING CSR; 4-byte edge data
    read as float (the ADDS port's reading) or as uint32."""
    h = _lib.HostCSR()
    check(lib().b2_lonestar_read(path.encode(), 1 if float_weights else 0, C.byref(h)), "lonestar_read")
    return _from_hostcsr(h, "outgoing")


def lonestar_write(path: str, g: HostGraph, float_weights: bool = True) -> None:
    """Write an OUTGOING CSR as Lonestar .gr version 1 (fweights or uint32 weights)."""
    if g.orientation != "outgoing":
        raise ValueError("Lonestar .gr stores outgoing CSR")
    h = _to_hostcsr(g)
    check(lib().b2_lonestar_write(path.encode(), C.byref(h), 1 if float_weights else 0), "lonestar_write")


# ---------------------------------------------------------------------------
def _torch():
    import torch
    return torch


def _stream_ptr(stream) -> int:
    torch = _torch()
    if stream is None:
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


_METHODS = {"bf": "b2_sssp_bf", "delta": "b2_sssp_delta", "adds": "b2_sssp_adds"}


class Graph:
    """A resident graph on the current CUDA device (outgoing packed CSR + workspace)."""

    def __init__(self, handle: int, weight: str):
        self._h = C.c_void_p(handle)
        self.weight = weight
        info = _lib.GraphInfo()
        check(lib().b2_graph_info_get(self._h, C.byref(info)), "graph_info")
        self.n, self.m = int(info.n), int(info.m)

    @classmethod
    def from_arrays(cls, rowptr, colind, values, *, orientation: str = "outgoing",
                    weight: str | None = None, stream=None) -> "Graph":
        """Arrays may be numpy (host) or torch CUDA tensors (device)."""
        torch = _torch()
        on_dev = isinstance(rowptr, torch.Tensor) and rowptr.is_cuda
        keep = []
        if on_dev:
            rp = rowptr.contiguous(); ci = colind.contiguous().to(torch.int32); vv = values.contiguous()
            if weight is None:
                weight = "f32" if vv.dtype == torch.float32 else "u32"
            if weight == "u32" and vv.dtype != torch.int32:
                vv = vv.to(torch.int64).to(torch.int32)  # same bits for values < 2^31
            bits = 64 if rp.dtype == torch.int64 else 32
            keep = [rp, ci, vv]
            ptrs = (rp.data_ptr(), ci.data_ptr(), vv.data_ptr())
            n = rp.numel() - 1
            nnz = ci.numel()
        else:
            rp = np.ascontiguousarray(rowptr)
            bits = 64 if rp.dtype.itemsize == 8 else 32
            rp = rp.astype(np.int64 if bits == 64 else np.uint32, copy=False)
            ci = np.ascontiguousarray(colind, np.int32)
            vv = np.ascontiguousarray(values)
            if weight is None:
                weight = "f32" if vv.dtype.kind == "f" else "u32"
            vv = vv.astype(np.float32 if weight == "f32" else np.uint32, copy=False)
            keep = [rp, ci, vv]
            ptrs = (rp.ctypes.data, ci.ctypes.data, vv.ctypes.data)
            n = rp.shape[0] - 1
            nnz = ci.shape[0]
        csr = _lib.CSR()
        csr.rows = csr.cols = n
        csr.nnz = nnz
        csr.rowptr, csr.colind, csr.values = ptrs
        csr.rowptr_bits = bits
        csr.weight_type = _lib.W_F32 if weight == "f32" else _lib.W_U32
        csr.orientation = _lib.OUTGOING if orientation == "outgoing" else _lib.INCOMING
        csr.on_device = 1 if on_dev else 0
        h = C.c_void_p()
        st = _stream_ptr(stream)
        check(lib().b2_graph_create(C.byref(csr), C.c_void_p(st), C.byref(h)), "graph_create")
        del keep
        return cls(h.value, weight)

    @classmethod
    def from_host(cls, g: HostGraph, weight: str = "u32", stream=None) -> "Graph":
        vals = g.weights if weight == "u32" else g.fweights
        return cls.from_arrays(g.rowptr, g.colind, vals, orientation=g.orientation, weight=weight,
                               stream=stream)

    def info(self) -> dict:
        info = _lib.GraphInfo()
        check(lib().b2_graph_info_get(self._h, C.byref(info)), "graph_info")
        return {k: getattr(info, k) for k, _ in info._fields_}

    def set_degree_order(self, stream=None) -> None:
        """Renumber vertices internally by out-degree (inputs / outputs keep input ids)."""
        check(lib().b2_graph_set_degree_order(self._h, C.c_void_p(_stream_ptr(stream))), "set_degree_order")

    @property
    def degree_ordered(self) -> bool:
        return bool(lib().b2_graph_degree_ordered(self._h))

    def delta_heuristic(self, scale: float = 16.0) -> float:
        d = C.c_double()
        check(lib().b2_delta_heuristic(self._h, scale, C.byref(d)), "delta_heuristic")
        return d.value

    def sssp(self, source: int, method: str = "delta", pred: bool = False, out=None, out_pred=None,
             stream=None, **opts):
        """Run one solve; returns (dist tensor, pred tensor | None, stats dict).
        opts are b2_sssp_opts fields; progress=callable(dict) is called once per
        finished round (BF) or bucket (delta, ADDS) while the solve runs."""
        torch = _torch()
        dt = torch.float32 if self.weight == "f32" else torch.int32
        dist = out if out is not None else torch.empty(self.n, dtype=dt, device="cuda")
        pr = None
        if pred:
            pr = out_pred if out_pred is not None else torch.empty(self.n, dtype=torch.int32, device="cuda")
        progress = opts.pop("progress", None)
        o = default_opts(**opts)
        keep = None
        if progress is not None:
            # called from this thread while the kernel runs, once per round / bucket
            def _cb(p, _user):
                q = p.contents
                progress({"iteration": q.iteration, "max_iters": q.max_iters, "changed": bool(q.changed),
                          "elapsed_ms": q.elapsed_ms})
            keep = _lib.PROGRESS_FN(_cb)
            o.progress = C.cast(keep, C.c_void_p)
        st = _lib.Stats()
        fn = getattr(lib(), _METHODS[method])
        rc = fn(self._h, source, C.c_void_p(dist.data_ptr()),
                C.c_void_p(pr.data_ptr() if pr is not None else 0), C.byref(o),
                C.c_void_p(_stream_ptr(stream)), C.byref(st))
        site = f" at device site {st.device_error_site}" if rc != _lib.SUCCESS and st.device_error_site else ""
        check(rc, f"sssp[{method}]{site}")
        del keep
        return dist, pr, st.as_dict()

    def trace(self) -> list[dict]:
        """Per-phase trace of the last solve run with trace=1."""
        cap = 4096
        buf = (_lib.TraceEntry * cap)()
        n = C.c_int32()
        check(lib().b2_graph_trace(self._h, C.cast(buf, C.c_void_p), cap, C.byref(n)), "graph_trace")
        kinds = {1: "relax", 2: "commit", 3: "split", 4: "probe", 5: "output", 7: "fused", 8: "pull"}
        out = []
        for e in buf[: n.value]:
            out.append({"kind": kinds.get(e.kind & 0xff, str(e.kind)) + ("-heavy" if e.kind & 0x100 else "")
                        + ("-dense" if e.kind & 0x200 else ""),
                        "frontier": e.frontier, "hub_chunks": e.hub_chunks, "bucket": e.bucket,
                        "t_us": e.t_ns / 1e3})
        return out

    def close(self) -> None:
        if self._h:
            lib().b2_graph_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def bf_dense(adj, source: int, out=None, stream=None, **opts):
    """Bellman-Ford over a dense incoming adjacency (adj[v, u] = w(u->v), +inf = no edge)
    on the GPU; returns (dist tensor, stats dict)."""
    torch = _torch()
    if adj.dim() != 2 or adj.shape[0] != adj.shape[1] or adj.dtype != torch.float32 or not adj.is_contiguous():
        raise ValueError("square contiguous float32 CUDA matrix required")
    n = adj.shape[0]
    dist = out if out is not None else torch.empty(n, dtype=torch.float32, device=adj.device)
    o = default_opts(**opts)
    st = _lib.Stats()
    check(lib().b2_sssp_bf_dense(C.c_void_p(adj.data_ptr()), n, source, C.c_void_p(dist.data_ptr()), C.byref(o),
                                 C.c_void_p(_stream_ptr(stream)), C.byref(st)), "bf_dense")
    return dist, st.as_dict()


def dist_to_numpy(dist, weight: str) -> np.ndarray:
    """Device distances -> float64 numpy with +inf for unreachable."""
    a = dist.cpu().numpy()
    if weight == "u32":
        u = a.view(np.uint32)
        out = u.astype(np.float64)
        out[u == 0xFFFFFFFF] = np.inf
        return out
    return a.astype(np.float64)


# min-plus entry points are defined in .minplus (imported lazily by users)
from .minplus import minplus_gemm, apsp, minplus_spgemm  # noqa: E402
