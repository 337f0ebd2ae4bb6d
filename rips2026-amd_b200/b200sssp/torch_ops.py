"""torch.ops.b200sssp: the reference's pytorch_testing entry points as torch
custom operators on CUDA tensors (importing this module registers them).

  torch.ops.b200sssp.sssp_min_plus_bellman_ford(rowptr, colind, values, source, max_iters=-1)
      <- sssp_min_plus_bellman_ford
         (pytorch_testing/bellman_ford_attempts/Attempt1_June23/minplus_bellman_ford.py:51-102).
      INCOMING CSR (row v, column u = w(u -> v)), float32 or int32 weights; max_iters < 0
      means n - 1.  Returns (dist, pred int64 (-1 = none), iterations_used, converged,
      has_negative_cycle), with the reference's extra relaxation round for the cycle check.
      float32 weights may be negative (the reference's float64 rules, negative cycles
      included) and give float32 distances.  int32 weights are solved as exact unsigned
      integers and give int32 distances (0xFFFFFFFF bits = unreachable); they must be
      nonnegative (a negative one raises ValueError: pass float32 values for those).
  torch.ops.b200sssp.bucketted_bellman_ford(rowptr, col, weight, source, num_nodes, delta=1.0)
      <- bucketted_bellman_ford (pytorch_testing/bellman_ford_attempts/bucketed_bellman_ford:1-71).
      OUTGOING CSR, float32 weights; delta-stepping with bucket width `delta`; returns dist.
  torch.ops.b200sssp.min_plus_matmul(A, B)
      <- min_plus_matmul (pytorch_testing/matrix_mult_attempts/matrix_mult_chunked.py:1-23).
      Row-major float32 or int32 operands; returns C = A (min,+) B.

Each call runs the library's CUDA kernels on the current torch stream.  There
is no CPU path: tensors on any other device are refused with a ValueError.
"""
from __future__ import annotations

import torch

from . import Graph
from .minplus import minplus_gemm


def _need_cuda(*ts: torch.Tensor) -> None:
    for t in ts:
        if not (isinstance(t, torch.Tensor) and t.is_cuda):
            raise ValueError("b200sssp ops take CUDA tensors (there is no CPU path)")


def _stream():
    return torch.cuda.current_stream()


@torch.library.custom_op("b200sssp::sssp_min_plus_bellman_ford", mutates_args=())
def sssp_min_plus_bellman_ford(rowptr: torch.Tensor, colind: torch.Tensor, values: torch.Tensor, source: int,
                               max_iters: int = -1) -> tuple[torch.Tensor, torch.Tensor, int, bool, bool]:
    _need_cuda(rowptr, colind, values)
    if values.dtype == torch.float32:
        weight = "f32"
    elif values.dtype == torch.int32:
        if values.numel() and bool((values < 0).any()):
            raise ValueError("negative int32 weights: pass float32 values for negative weights")
        weight = "u32"
    else:
        raise TypeError("values must be float32 or int32")
    g = Graph.from_arrays(rowptr, colind, values, orientation="incoming", weight=weight, stream=_stream())
    try:
        dist, pred, st = g.sssp(int(source), method="bf", pred=True, max_iters=int(max_iters),
                                detect_negative_cycle=1, stream=_stream())
    finally:
        g.close()
    return dist, pred.to(torch.int64), int(st["iterations_used"]), bool(st["converged"]), \
        bool(st["has_negative_cycle"])


@sssp_min_plus_bellman_ford.register_fake
def _(rowptr, colind, values, source, max_iters=-1):
    n = rowptr.shape[0] - 1
    dt = torch.float32 if values.dtype == torch.float32 else torch.int32
    return (values.new_empty(n, dtype=dt), rowptr.new_empty(n, dtype=torch.int64), 0, False, False)


@torch.library.custom_op("b200sssp::bucketted_bellman_ford", mutates_args=())
def bucketted_bellman_ford(rowptr: torch.Tensor, col: torch.Tensor, weight: torch.Tensor, source: int,
                           num_nodes: int, delta: float = 1.0) -> torch.Tensor:
    _need_cuda(rowptr, col, weight)
    if rowptr.shape[0] != num_nodes + 1:
        raise ValueError("rowptr must hold num_nodes + 1 offsets")
    g = Graph.from_arrays(rowptr.to(torch.int64), col.to(torch.int32), weight.to(torch.float32),
                          orientation="outgoing", weight="f32", stream=_stream())
    try:
        dist, _, _ = g.sssp(int(source), method="delta", delta=float(delta), stream=_stream())
    finally:
        g.close()
    return dist


@bucketted_bellman_ford.register_fake
def _(rowptr, col, weight, source, num_nodes, delta=1.0):
    return weight.new_empty(num_nodes, dtype=torch.float32)


@torch.library.custom_op("b200sssp::min_plus_matmul", mutates_args=())
def min_plus_matmul(A: torch.Tensor, B: torch.Tensor) -> torch.Tensor:
    _need_cuda(A, B)
    return minplus_gemm(A.contiguous(), B.contiguous(), stream=_stream())


@min_plus_matmul.register_fake
def _(A, B):
    return A.new_empty((A.shape[0], B.shape[1]))
