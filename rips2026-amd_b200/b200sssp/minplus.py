"""Min-plus (tropical) products on the GPU through the C ABI.

minplus_gemm(A, B)  -> C[i,j] = min_k A[i,k] + B[k,j]   (torch CUDA tensors)
apsp(D)             -> repeated squaring in place, returns the number of products
minplus_spgemm(A, B)-> CSR x CSR (device tensors in, device tensors out)

Interface of the reference: minplus_gemm_f32 (HIP_kernel/minplus_mm/src/minplus_hip.hpp:24-33),
minplus_sparse::minplus_spgemm_csr_f32 (minplus_sparse_hip.hpp:64-150), and the
pytorch prototype min_plus_matmul (pytorch_testing/matrix_mult_attempts/matrix_mult_chunked.py:1-23).
"""
from __future__ import annotations

import ctypes as C

from . import _lib
from ._lib import check, lib

MISSING_I32 = 1073741823  # INT32_MAX // 2


def _torch():
    import torch
    return torch


def _sp(stream):
    torch = _torch()
    return torch.cuda.current_stream().cuda_stream if stream is None else (
        stream if isinstance(stream, int) else stream.cuda_stream)


def minplus_gemm(A, B, out=None, stream=None, check_status: bool = True):
    """C = A (min,+) B on the GPU.  The product is asynchronous on `stream`;
    with check_status (default) the call waits for it and raises B2Error
    (B2_TIMEOUT) if one of its bounded shared-memory waits gave up.  Callers
    issuing many products can pass False and call status(stream) once."""
    torch = _torch()
    if A.dtype != B.dtype or A.dim() != 2 or B.dim() != 2 or A.shape[1] != B.shape[0]:
        raise ValueError("A (MxK) and B (KxN) must be 2-D with matching inner size and dtype")
    if A.stride(1) != 1 or B.stride(1) != 1:
        raise ValueError("row-major (unit column stride) operands required")
    M, K = A.shape
    N = B.shape[1]
    if out is None:
        out = torch.empty((M, N), dtype=A.dtype, device=A.device)
    fn = {torch.float32: lib().b2_minplus_gemm_f32, torch.int32: lib().b2_minplus_gemm_i32}.get(A.dtype)
    if fn is None:
        raise TypeError("float32 or int32 operands required")
    check(fn(C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()), C.c_void_p(out.data_ptr()), M, N, K,
             A.stride(0), B.stride(0), out.stride(0), C.c_void_p(_sp(stream))), "minplus_gemm")
    if check_status:
        status(stream)
    return out


def status(stream=None) -> None:
    """Wait for `stream`; raise B2Error if a min-plus product issued since the
    last GEMM / APSP call began gave up a bounded wait (b2_minplus_status)."""
    check(lib().b2_minplus_status(C.c_void_p(_sp(stream))), "minplus_status")


def apsp(D, stream=None) -> int:
    torch = _torch()
    if D.dim() != 2 or D.shape[0] != D.shape[1] or not D.is_contiguous():
        raise ValueError("square contiguous matrix required")
    n = C.c_int32()
    fn = {torch.float32: lib().b2_apsp_f32, torch.int32: lib().b2_apsp_i32}[D.dtype]
    check(fn(C.c_void_p(D.data_ptr()), D.shape[0], C.c_void_p(_sp(stream)), C.byref(n)), "apsp")
    return n.value


def _csr_view(rowptr, colind, values, ncols):
    torch = _torch()
    c = _lib.CSR()
    c.rows = rowptr.numel() - 1
    c.cols = ncols
    c.nnz = colind.numel()
    c.rowptr = rowptr.data_ptr()
    c.colind = colind.data_ptr() if colind.numel() else None
    c.values = values.data_ptr() if values.numel() else None
    c.rowptr_bits = 64
    c.weight_type = _lib.W_F32 if values.dtype == torch.float32 else _lib.W_U32
    c.orientation = _lib.OUTGOING
    c.on_device = 1
    return c


def minplus_spgemm(A, B, stream=None):
    """A, B: (rowptr int64, colind int32, values f32|i32, ncols).  Returns (rowptr, colind, values)
    as torch CUDA tensors.  The product is computed into library scratch
    (b2_minplus_spgemm_plan), the outputs are allocated by torch at their exact
    size and filled on `stream` (b2_minplus_spgemm_fill)."""
    torch = _torch()
    a = _csr_view(*A)
    b = _csr_view(*B)
    if a.weight_type != b.weight_type:
        raise TypeError("A and B must have the same value dtype")
    is_f = A[2].dtype == torch.float32
    plan = C.c_void_p()
    nnz = C.c_int64()
    sp = C.c_void_p(_sp(stream))
    check(lib().b2_minplus_spgemm_plan(C.byref(a), C.byref(b), sp, C.byref(plan), C.byref(nnz)), "minplus_spgemm")
    try:
        dev = A[0].device
        rp = torch.empty(a.rows + 1, dtype=torch.int64, device=dev)
        ci = torch.empty(nnz.value, dtype=torch.int32, device=dev)
        vv = torch.empty(nnz.value, dtype=torch.float32 if is_f else torch.int32, device=dev)
    except BaseException:
        lib().b2_minplus_spgemm_plan_free(plan)
        raise
    check(lib().b2_minplus_spgemm_fill(plan, C.c_void_p(rp.data_ptr()), C.c_void_p(ci.data_ptr() if nnz.value else 0),
                                       C.c_void_p(vv.data_ptr() if nnz.value else 0), sp), "minplus_spgemm_fill")
    return rp, ci, vv


def minplus_spgemm_callee_alloc(A, B, stream=None):
    """The reference's one-call form (b2_minplus_spgemm_f32 / _i32: outputs
    allocated by the library, freed here after their copy into torch tensors)."""
    torch = _torch()
    a = _csr_view(*A)
    b = _csr_view(*B)
    is_f = A[2].dtype == torch.float32
    prp, pci, pv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    nnz = C.c_int64()
    fn = lib().b2_minplus_spgemm_f32 if is_f else lib().b2_minplus_spgemm_i32
    check(fn(C.byref(a), C.byref(b), C.byref(prp), C.byref(pci), C.byref(pv), C.byref(nnz),
             C.c_void_p(_sp(stream))), "minplus_spgemm")
    return _adopt(prp.value, pci.value, pv.value, a.rows, nnz.value, torch.float32 if is_f else torch.int32)


def _adopt(prp, pci, pv, rows, nnz, vdtype):
    """Copy callee-allocated device arrays into torch tensors and cudaFree them."""
    torch = _torch()
    rp = torch.empty(rows + 1, dtype=torch.int64, device="cuda")
    ci = torch.empty(nnz, dtype=torch.int32, device="cuda")
    vv = torch.empty(nnz, dtype=vdtype, device="cuda")
    try:
        for t, p in ((rp, prp), (ci, pci), (vv, pv)):
            if p and t.numel():
                check(lib().b2_device_copy(C.c_void_p(t.data_ptr()), C.c_void_p(p),
                                           t.numel() * t.element_size(), None), "device_copy")
    finally:
        for p in (prp, pci, pv):
            if p:
                lib().b2_device_free(C.c_void_p(p))
    return rp, ci, vv
