"""ctypes binding of libb200sssp.so (the C ABI declared in include/b200sssp.h).

The shared library is built in-tree by rips2026-amd_b200/build.py.  Loading it
never falls back to anything else: if the file is missing, LibraryMissing is
raised and nothing runs.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "libb200sssp.so")


class LibraryMissing(RuntimeError):
    pass


class B2Error(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        super().__init__(f"{what}: {status_string(status)} ({status})" if what else status_string(status))


# ---- enums -----------------------------------------------------------------
SUCCESS, INVALID_ARGUMENT, CUDA_ERROR, OUT_OF_MEMORY, POOL_EXHAUSTED, BUCKET_OVERFLOW, \
    DEVICE_ERROR, TIMEOUT, NOT_SUPPORTED, INVALID_INDEX, INVALID_ROWPTR, INVALID_WEIGHT, CANCELLED = range(13)
W_U32, W_F32 = 0, 1
INCOMING, OUTGOING = 0, 1
BF_CHECKED, BF_NO_CHECKS, BF_VAR_CHECKS = 0, 1, 2


class CSR(C.Structure):
    _fields_ = [("rows", C.c_int64), ("cols", C.c_int64), ("nnz", C.c_int64),
                ("rowptr", C.c_void_p), ("colind", C.c_void_p), ("values", C.c_void_p),
                ("rowptr_bits", C.c_int32), ("weight_type", C.c_int32),
                ("orientation", C.c_int32), ("on_device", C.c_int32)]


class GraphInfo(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("weight_type", C.c_int32),
                ("max_out_degree", C.c_int32), ("mean_weight", C.c_double),
                ("mean_degree", C.c_double), ("device_bytes", C.c_size_t)]


class Opts(C.Structure):
    _fields_ = [("max_iters", C.c_int32), ("bf_check", C.c_int32), ("check_interval", C.c_int32),
                ("policy", C.c_int32), ("delta", C.c_double), ("delta_scale", C.c_double),
                ("hub_degree", C.c_uint32), ("fusion_threshold", C.c_uint32),
                ("pull_fraction", C.c_float), ("grid_blocks", C.c_uint32),
                ("timeout_ms", C.c_double), ("collect_reach", C.c_int32),
                ("detect_negative_cycle", C.c_int32), ("light_heavy", C.c_int32), ("trace", C.c_int32),
                ("dense_fraction", C.c_float), ("worklist_capacity", C.c_uint32), ("keep_distances", C.c_int32),
                ("active_buckets", C.c_uint32), ("adds_fixed_delta", C.c_int32), ("progress", C.c_void_p),
                ("progress_user", C.c_void_p), ("max_active_buckets", C.c_uint32),
                ("reserved", C.c_int32 * 2)]


class Progress(C.Structure):
    _fields_ = [("iteration", C.c_int32), ("max_iters", C.c_int32), ("changed", C.c_int32),
                ("reserved", C.c_int32), ("elapsed_ms", C.c_double)]


PROGRESS_FN = C.CFUNCTYPE(None, C.POINTER(Progress), C.c_void_p)


class TraceEntry(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("frontier", C.c_uint32), ("hub_chunks", C.c_uint32),
                ("bucket", C.c_uint32), ("t_ns", C.c_uint64)]


class Stats(C.Structure):
    _fields_ = [("iterations_used", C.c_int32), ("converged", C.c_int32),
                ("has_negative_cycle", C.c_int32), ("phases", C.c_int32),
                ("edges_scanned", C.c_uint64), ("improvements", C.c_uint64),
                ("pushes", C.c_uint64), ("reached", C.c_uint64), ("reached_edges", C.c_uint64),
                ("delta_used", C.c_double), ("kernel_ms", C.c_float), ("device_error", C.c_uint32),
                ("grid_blocks", C.c_uint32), ("first_unchanged", C.c_uint32),
                ("local_subphases", C.c_uint32), ("delta_updates", C.c_uint32),
                ("delta_final", C.c_double), ("policy_used", C.c_uint32), ("heavy_pulls", C.c_uint32),
                ("work_items", C.c_uint64), ("active_buckets_max", C.c_uint32), ("device_error_site", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class HostCSR(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("rowptr", C.POINTER(C.c_int64)),
                ("colind", C.POINTER(C.c_int32)), ("weights", C.POINTER(C.c_uint32)),
                ("fweights", C.POINTER(C.c_float))]


# Every symbol include/b200sssp.h declares, with its signature.
_P = C.c_void_p
_SIGS = {
    "b2_status_string": (C.c_char_p, [C.c_int]),
    "b2_abi_version": (C.c_int, []),
    "b2_sssp_opts_default": (None, [C.POINTER(Opts)]),
    "b2_device_free": (C.c_int, [_P]),
    "b2_device_copy": (C.c_int, [_P, _P, C.c_size_t, _P]),
    "b2_graph_create": (C.c_int, [C.POINTER(CSR), _P, C.POINTER(_P)]),
    "b2_graph_destroy": (C.c_int, [_P]),
    "b2_graph_info_get": (C.c_int, [_P, C.POINTER(GraphInfo)]),
    "b2_graph_set_degree_order": (C.c_int, [_P, _P]),
    "b2_graph_degree_ordered": (C.c_int32, [_P]),
    "b2_delta_heuristic": (C.c_int, [_P, C.c_double, C.POINTER(C.c_double)]),
    "b2_graph_trace": (C.c_int, [_P, _P, C.c_int32, C.POINTER(C.c_int32)]),
    "b2_sssp_bf": (C.c_int, [_P, C.c_uint32, _P, _P, C.POINTER(Opts), _P, C.POINTER(Stats)]),
    "b2_sssp_delta": (C.c_int, [_P, C.c_uint32, _P, _P, C.POINTER(Opts), _P, C.POINTER(Stats)]),
    "b2_sssp_adds": (C.c_int, [_P, C.c_uint32, _P, _P, C.POINTER(Opts), _P, C.POINTER(Stats)]),
    "b2_sssp_bf_dense": (C.c_int, [_P, C.c_int32, C.c_uint32, _P, C.POINTER(Opts), _P, C.POINTER(Stats)]),
    "b2_minplus_gemm_f32": (C.c_int, [_P, _P, _P] + [C.c_int32] * 6 + [_P]),
    "b2_minplus_gemm_i32": (C.c_int, [_P, _P, _P] + [C.c_int32] * 6 + [_P]),
    "b2_apsp_f32": (C.c_int, [_P, C.c_int32, _P, C.POINTER(C.c_int32)]),
    "b2_apsp_i32": (C.c_int, [_P, C.c_int32, _P, C.POINTER(C.c_int32)]),
    "b2_apsp_f32_noalloc": (C.c_int, [_P, C.c_int32, _P, C.POINTER(C.c_int32)]),
    "b2_minplus_status": (C.c_int, [_P]),
    "b2_minplus_calibrate": (C.c_int, [C.c_int32, C.POINTER(C.c_double)]),
    "b2_minplus_spgemm_f32": (C.c_int, [C.POINTER(CSR), C.POINTER(CSR), C.POINTER(_P), C.POINTER(_P),
                                        C.POINTER(_P), C.POINTER(C.c_int64), _P]),
    "b2_minplus_spgemm_i32": (C.c_int, [C.POINTER(CSR), C.POINTER(CSR), C.POINTER(_P), C.POINTER(_P),
                                        C.POINTER(_P), C.POINTER(C.c_int64), _P]),
    "b2_minplus_spgemm_plan": (C.c_int, [C.POINTER(CSR), C.POINTER(CSR), _P, C.POINTER(_P), C.POINTER(C.c_int64)]),
    "b2_minplus_spgemm_fill": (C.c_int, [_P, _P, _P, _P, _P]),
    "b2_minplus_spgemm_plan_free": (C.c_int, [_P]),
    "b2_policy_param_count": (C.c_int32, []),
    "b2_policy_create": (C.c_int, [C.c_uint64, C.POINTER(_P)]),
    "b2_policy_destroy": (C.c_int, [_P]),
    "b2_policy_set_params": (C.c_int, [_P, _P, _P, _P]),
    "b2_policy_get_params": (C.c_int, [_P, _P, _P, _P]),
    "b2_policy_set_dead_zone": (C.c_int, [_P, C.c_float]),
    "b2_policy_set_feature_range": (C.c_int, [_P, _P, _P]),
    "b2_policy_forward": (C.c_int, [_P, _P, C.c_int32, _P]),
    "b2_policy_gradient": (C.c_int, [_P, _P, _P, C.c_int32, _P, C.POINTER(C.c_float)]),
    "b2_policy_train": (C.c_int, [_P, _P, _P, C.c_int32, C.c_int32, C.c_float, C.c_float,
                                  C.POINTER(C.c_float)]),
    "b2_policy_activate": (C.c_int, [_P]),
    "b2_graph_features": (C.c_int, [_P, _P]),
    "b2_server_opts_default": (None, [_P]),
    "b2_server_create": (C.c_int, [_P, C.POINTER(_P)]),
    "b2_server_destroy": (C.c_int, [_P]),
    "b2_server_add_graph": (C.c_int, [_P, _P, C.POINTER(C.c_int32)]),
    "b2_server_graph_config": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                         C.POINTER(C.c_int32)]),
    "b2_server_slot_bytes": (C.c_size_t, [C.c_int64, C.c_int32]),
    "b2_server_submit": (C.c_int, [_P, C.c_int32, C.c_uint32, _P, _P, C.POINTER(C.c_uint64)]),
    "b2_server_cancel": (C.c_int, [_P, C.c_uint64]),
    "b2_server_progress": (C.c_int, [_P, C.c_int32]),
    "b2_server_poll": (C.c_int, [_P, _P, C.c_int32, C.POINTER(C.c_int32)]),
    "b2_server_info": (C.c_int, [_P, _P]),
    "b2_load_opts_default": (None, [_P]),
    "b2_server_run_load": (C.c_int, [_P, _P, _P]),
    "b2_gen_er": (C.c_int, [C.c_int64, C.c_int64, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(HostCSR)]),
    "b2_gen_rmat": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint32,
                              C.c_uint32, C.c_uint64, C.POINTER(HostCSR)]),
    "b2_gen_grid": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_uint64,
                              C.POINTER(HostCSR)]),
    "b2_host_csr_free": (None, [C.POINTER(HostCSR)]),
    "b2_host_csr_transpose": (C.c_int, [C.POINTER(HostCSR), C.POINTER(HostCSR)]),
    "b2_csrbin_write": (C.c_int, [C.c_char_p, C.c_int64, C.c_int64, _P, _P, _P]),
    "b2_csrbin_read": (C.c_int, [C.c_char_p, C.POINTER(HostCSR)]),
    "b2_dimacs_read": (C.c_int, [C.c_char_p, C.POINTER(HostCSR), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]),
    "b2_dimacs_to_csrbin": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(C.c_int64)]),
    "b2_lonestar_read": (C.c_int, [C.c_char_p, C.c_int32, C.POINTER(HostCSR)]),
    "b2_lonestar_write": (C.c_int, [C.c_char_p, C.POINTER(HostCSR), C.c_int32]),
}

_lib = None


def lib() -> C.CDLL:
    """Load the in-tree library once; raise LibraryMissing if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise LibraryMissing(f"{LIB_PATH} not built (run rips2026-amd_b200/build.py)")
    L = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def declared_symbols() -> list[str]:
    return sorted(_SIGS)


def status_string(s: int) -> str:
    try:
        return lib().b2_status_string(int(s)).decode()
    except LibraryMissing:
        return f"status {s}"


def check(status: int, what: str = "") -> None:
    if status != SUCCESS:
        raise B2Error(status, what)


def default_opts(**kw) -> Opts:
    o = Opts()
    lib().b2_sssp_opts_default(C.byref(o))
    if os.environ.get("B2_TIMEOUT_MS"):
        o.timeout_ms = float(os.environ["B2_TIMEOUT_MS"])
    for k, v in kw.items():
        if not hasattr(o, k):
            raise TypeError(f"unknown option {k}")
        setattr(o, k, v)
    return o
