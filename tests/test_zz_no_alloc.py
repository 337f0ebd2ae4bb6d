"""Allocation-free APSP entry point (b2_apsp_f32_noalloc) through the C ABI.

Callers that cannot allocate device memory while they run (a plugin whose
host owns the device memory pool, a serving loop with a fixed memory budget)
use b2_apsp_f32_noalloc, whose scratch is a fixed module array.  This checks
it against the allocating b2_apsp_f32 on two calls in a row: the shared
scratch keeps the previous call's contents, so the second call must not be
affected by the first.  The kernel is the same, so results must be
bit-identical.  The file is named to run after every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _apsp(L, fn, D):
    sq = C.c_int32()
    st = fn(C.c_void_p(D.data_ptr()), D.shape[0], None, C.byref(sq))
    return st, sq.value


def test_noalloc_apsp_matches_allocating_entry_point(b2, cuda):
    torch = cuda
    from b200sssp import _lib
    L = _lib.lib()
    rng = np.random.default_rng(2026)
    # two calls in a row, the second smaller than the first, then the exact fit
    # (a 2048 x 2048 matrix fills the scratch up to the change flag) and the
    # one-vertex case (nothing to square)
    for n in (700, 301, 2048, 1):
        D = rng.uniform(0, 1, (n, n)).astype(np.float32)
        D[rng.uniform(size=D.shape) < (0.97 if n < 1000 else 0.995)] = np.inf
        np.fill_diagonal(D, 0)
        a = torch.from_numpy(D).cuda()
        b = a.clone()
        st_a, sq_a = _apsp(L, L.b2_apsp_f32, a)
        st_b, sq_b = _apsp(L, L.b2_apsp_f32_noalloc, b)
        torch.cuda.synchronize()
        assert st_a == 0 and st_b == 0
        assert sq_a == sq_b
        assert np.array_equal(a.cpu().numpy(), b.cpu().numpy())


def test_noalloc_apsp_rejects_sizes_past_its_scratch(b2, cuda):
    torch = cuda
    from b200sssp import _lib
    L = _lib.lib()
    D = torch.zeros((2049, 2049), dtype=torch.float32, device="cuda")
    st, _ = _apsp(L, L.b2_apsp_f32_noalloc, D)
    assert st == _lib.NOT_SUPPORTED
