"""Batched continuous serving of single-source queries (b2_server_* in the C ABI).

No counterpart in the reference.  A ``Server`` keeps resident graphs and a
device arena of a fixed HBM budget; ``submit`` queues a query, the engine
admits queries whose arena slot fits, runs them in batch launches where one
thread block solves one query, and each query completes on its own as soon
as its result is in the caller's buffer (page-locked host memory or device
memory).

    srv = Server(hbm_budget=8 << 30)
    gid = srv.add_graph(graph)                  # a b200sssp.Graph (must outlive srv)
    out = srv.result_buffer(graph)              # page-locked host tensor
    t = srv.submit(gid, source, out)
    srv.progress(wait_all=True)
    done = srv.poll()                           # [{"ticket", "status", "latency_us", ...}]
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_size_t), ("max_batch", C.c_int32), ("lanes", C.c_int32),
                ("max_inflight", C.c_int32), ("blocks_per_sm", C.c_int32), ("timeout_ms", C.c_double),
                ("delta_scale", C.c_double), ("big_vertices", C.c_int32), ("autotune", C.c_int32),
                ("reserved", C.c_int32 * 2)]


class Completion(C.Structure):
    _fields_ = [("ticket", C.c_uint64), ("status", C.c_int32), ("graph_id", C.c_int32),
                ("source", C.c_uint32), ("phases", C.c_uint32), ("edges_scanned", C.c_uint64),
                ("reached", C.c_uint64), ("reached_edges", C.c_uint64), ("latency_us", C.c_double)]


class ServerInfo(C.Structure):
    _fields_ = [("graphs", C.c_int32), ("blocks", C.c_uint32), ("pending", C.c_int64),
                ("running", C.c_int64), ("completed_unpolled", C.c_int64), ("arena_bytes", C.c_size_t),
                ("arena_used", C.c_size_t)]


class LoadOpts(C.Structure):
    _fields_ = [("queries", C.c_int64), ("rate_qps", C.c_double), ("seed", C.c_uint64), ("mode", C.c_int32),
                ("with_pred", C.c_int32), ("host_result_bytes", C.c_size_t), ("graph_ids", C.c_void_p),
                ("n_graph_ids", C.c_int32), ("reserved0", C.c_int32), ("checksums", C.c_void_p),
                ("query_graph", C.c_void_p), ("query_source", C.c_void_p), ("reserved", C.c_int32 * 4)]


class LoadReport(C.Structure):
    _fields_ = [("completed", C.c_int64), ("failed", C.c_int64), ("elapsed_s", C.c_double), ("qps", C.c_double),
                ("p50_us", C.c_double), ("p99_us", C.c_double), ("mean_us", C.c_double), ("max_us", C.c_double),
                ("gteps", C.c_double), ("reached_edges", C.c_uint64), ("reserved", C.c_double * 4)]


def _as_dict(st) -> dict:
    return {k: getattr(st, k) for k, _ in st._fields_ if not k.startswith("reserved")}


def slot_bytes(n: int, with_pred: bool = False) -> int:
    return int(lib().b2_server_slot_bytes(n, 1 if with_pred else 0))


class Server:
    def __init__(self, hbm_budget: int = 1 << 30, max_batch: int = 512, lanes: int = 16,
                 max_inflight: int = 8192, timeout_ms: float = 20000.0, delta_scale: float = 4.0,
                 blocks_per_sm: int = 0, big_vertices: int = 0, autotune: bool = False):
        o = ServerOpts()
        lib().b2_server_opts_default(C.byref(o))
        o.hbm_budget_bytes = hbm_budget
        o.max_batch = max_batch
        o.lanes = lanes
        o.max_inflight = max_inflight
        o.timeout_ms = timeout_ms
        o.delta_scale = delta_scale
        o.blocks_per_sm = blocks_per_sm
        o.big_vertices = big_vertices
        o.autotune = 1 if autotune else 0
        h = C.c_void_p()
        check(lib().b2_server_create(C.byref(o), C.byref(h)), "server_create")
        self._h = h
        self._graphs = []      # keep the Graph objects alive

    def add_graph(self, g) -> int:
        gid = C.c_int32()
        check(lib().b2_server_add_graph(self._h, g._h, C.byref(gid)), "server_add_graph")
        self._graphs.append(g)
        return gid.value

    def graph_config(self, graph_id: int) -> dict:
        """Team, bucket-width constant and autotuned flag of a graph's queries."""
        team, tuned = C.c_int32(), C.c_int32()
        scale = C.c_double()
        check(lib().b2_server_graph_config(self._h, graph_id, C.byref(team), C.byref(scale), C.byref(tuned)),
              "server_graph_config")
        return {"cluster_team": bool(team.value), "delta_scale": scale.value, "tuned": bool(tuned.value)}

    @staticmethod
    def result_buffer(g, pinned: bool = True):
        """A result tensor for g: page-locked host memory (or CUDA memory)."""
        import torch
        dt = torch.float32 if g.weight == "f32" else torch.int32
        if pinned:
            return torch.empty(g.n, dtype=dt).pin_memory()
        return torch.empty(g.n, dtype=dt, device="cuda")

    def submit(self, graph_id: int, source: int, out, out_pred=None) -> int:
        t = C.c_uint64()
        check(lib().b2_server_submit(self._h, graph_id, source, C.c_void_p(out.data_ptr()),
                                     C.c_void_p(out_pred.data_ptr() if out_pred is not None else 0),
                                     C.byref(t)), "server_submit")
        return t.value

    def cancel(self, ticket: int) -> bool:
        return lib().b2_server_cancel(self._h, C.c_uint64(ticket)) == _lib.SUCCESS

    def progress(self, wait_all: bool = False) -> None:
        check(lib().b2_server_progress(self._h, 1 if wait_all else 0), "server_progress")

    def poll(self, capacity: int = 4096) -> list[dict]:
        buf = (Completion * capacity)()
        n = C.c_int32()
        check(lib().b2_server_poll(self._h, C.cast(buf, C.c_void_p), capacity, C.byref(n)), "server_poll")
        return [_as_dict(buf[i]) for i in range(n.value)]

    def info(self) -> dict:
        st = ServerInfo()
        check(lib().b2_server_info(self._h, C.byref(st)), "server_info")
        return _as_dict(st)

    def run_load(self, queries: int, rate_qps: float = 0.0, seed: int = 1, mode: str = "server",
                 with_pred: bool = False, host_result_bytes: int = 1 << 30, graph_ids=None,
                 record: bool = False) -> dict:
        """Poisson load (rate_qps <= 0: all at t = 0).  mode 'server' or
        'sequential' (one full-GPU solve at a time).  record=True also returns
        per-query graph, source and result checksum arrays."""
        o = LoadOpts()
        lib().b2_load_opts_default(C.byref(o))
        o.queries = queries
        o.rate_qps = rate_qps
        o.seed = seed
        o.mode = 1 if mode == "sequential" else 0
        o.with_pred = 1 if with_pred else 0
        o.host_result_bytes = host_result_bytes
        keep = []
        if graph_ids is not None:
            ids = np.ascontiguousarray(graph_ids, np.int32)
            keep.append(ids)
            o.graph_ids = ids.ctypes.data
            o.n_graph_ids = ids.size
        if record:
            cs = np.zeros(queries, np.uint64)
            qg = np.zeros(queries, np.int32)
            qs = np.zeros(queries, np.uint32)
            o.checksums, o.query_graph, o.query_source = cs.ctypes.data, qg.ctypes.data, qs.ctypes.data
        rep = LoadReport()
        check(lib().b2_server_run_load(self._h, C.byref(o), C.byref(rep)), "server_run_load")
        out = _as_dict(rep)
        if record:
            out.update(checksums=cs, query_graph=qg, query_source=qs)
        return out

    def close(self) -> None:
        if self._h:
            lib().b2_server_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def checksum_words(a: np.ndarray) -> int:
    """The load generator's 64-bit hash of a result's distance words."""
    w = np.ascontiguousarray(a).view(np.uint32)
    h = 0x9E3779B97F4A7C15
    M = (1 << 64) - 1
    for i, x in enumerate(w.tolist()):
        h = (((h ^ x) * 0x100000001B3) + i) & M
    return h
