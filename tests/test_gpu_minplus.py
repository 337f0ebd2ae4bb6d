"""GPU parity: dense min-plus GEMM (int32, fp32) and APSP repeated squaring.

Bit-exact against the oracle (min over k of one rounded addition is exact in
any order), against the reference's chunked torch min_plus_matmul fixtures,
and APSP against all-pairs Dijkstra.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
MISS = 1073741823


def _rand(rng, shape, dtype, p_missing):
    if dtype == np.float32:
        a = rng.uniform(0, 1, shape).astype(np.float32)
        a[rng.uniform(size=shape) < p_missing] = np.inf
    else:
        a = rng.integers(1, 1001, shape).astype(np.int32)
        a[rng.uniform(size=shape) < p_missing] = MISS
    return a


@pytest.mark.parametrize("dtype", [np.float32, np.int32])
@pytest.mark.parametrize("shape", [(128, 128, 128), (256, 384, 96), (33, 47, 29), (130, 257, 75), (1, 1, 1),
                                   (300, 5, 1000), (512, 64, 513)])
def test_gemm_matches_oracle(b2, orc, cuda, dtype, shape):
    torch = cuda
    M, K, N = shape
    rng = np.random.default_rng(M * 7 + K * 3 + N)
    A = _rand(rng, (M, K), dtype, 0.5)
    B = _rand(rng, (K, N), dtype, 0.5)
    C = b2.minplus_gemm(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()).cpu().numpy()
    assert np.array_equal(C, orc.minplus_gemm(A, B))


@pytest.mark.parametrize("dtype", [np.float32, np.int32])
def test_gemm_strided_and_unaligned_operands(b2, orc, cuda, dtype):
    """Leading dimensions larger than the width, and ones TMA cannot describe
    (not a multiple of 16 bytes) -> the plain-load kernel; same results."""
    torch = cuda
    rng = np.random.default_rng(3)
    for lda_pad, ldb_pad in ((0, 0), (4, 8), (1, 3)):
        M, K, N = 150, 70, 140
        A = _rand(rng, (M, K + lda_pad), dtype, 0.4)
        B = _rand(rng, (K, N + ldb_pad), dtype, 0.4)
        At = torch.from_numpy(A).cuda()[:, :K]
        Bt = torch.from_numpy(B).cuda()[:, :N]
        C = b2.minplus_gemm(At, Bt).cpu().numpy()
        assert np.array_equal(C, orc.minplus_gemm(A[:, :K].copy(), B[:, :N].copy())), (lda_pad, ldb_pad)


def test_gemm_nan_and_inf_semantics(b2, orc, cuda):
    torch = cuda
    rng = np.random.default_rng(9)
    A = rng.uniform(-1, 1, (64, 80)).astype(np.float32)
    B = rng.uniform(-1, 1, (80, 96)).astype(np.float32)
    A[rng.uniform(size=A.shape) < 0.1] = np.nan
    B[rng.uniform(size=B.shape) < 0.1] = np.inf
    A[rng.uniform(size=A.shape) < 0.05] = -np.inf
    C = b2.minplus_gemm(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()).cpu().numpy()
    R = orc.minplus_gemm(A, B)
    assert np.array_equal(np.isnan(C), np.isnan(R))
    ok = ~np.isnan(R)
    assert np.array_equal(C[ok], R[ok])


def test_reference_chunked_fixtures(b2, golden, cuda):
    torch = cuda
    z = golden("minplus.npz")
    for t in range(3):
        A, B, Cr = z[f"f32_{t}/A"], z[f"f32_{t}/B"], z[f"f32_{t}/C"]
        C = b2.minplus_gemm(torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()).cpu().numpy()
        assert np.array_equal(C, Cr)
        Ai, Bi, Ci = z[f"i32_{t}/A"], z[f"i32_{t}/B"], z[f"i32_{t}/C"]
        C = b2.minplus_gemm(torch.from_numpy(Ai).cuda(), torch.from_numpy(Bi).cuda()).cpu().numpy()
        assert np.array_equal(C, np.minimum(Ci, MISS).astype(np.int32))


def test_invalid_arguments(b2, cuda):
    torch = cuda
    A = torch.zeros((4, 4), dtype=torch.float32, device="cuda")
    from b200sssp import _lib
    import ctypes as C
    L = _lib.lib()
    p = C.c_void_p(A.data_ptr())
    assert L.b2_minplus_gemm_f32(p, p, p, 4, 4, 4, 3, 4, 4, None) == _lib.INVALID_ARGUMENT  # lda < K
    assert L.b2_minplus_gemm_f32(p, p, p, 0, 4, 4, 4, 4, 4, None) == _lib.INVALID_ARGUMENT
    assert L.b2_minplus_gemm_f32(None, p, p, 4, 4, 4, 4, 4, 4, None) == _lib.INVALID_ARGUMENT


@pytest.mark.parametrize("dtype", [np.float32, np.int32])
@pytest.mark.parametrize("n", [2, 57, 200])
def test_apsp_matches_all_pairs_dijkstra(b2, orc, cuda, dtype, n):
    torch = cuda
    rng = np.random.default_rng(n)
    D = _rand(rng, (n, n), dtype, 0.9)
    np.fill_diagonal(D, 0)
    Dt = torch.from_numpy(D).cuda()
    sq = b2.apsp(Dt)
    got = Dt.cpu().numpy()
    # oracle: Dijkstra from every source on the outgoing CSR of D
    missing = np.isinf(D) if dtype == np.float32 else (D >= MISS)
    rows, cols = np.nonzero(~missing)
    rp = np.zeros(n + 1, np.int64)
    np.add.at(rp, rows + 1, 1)
    rp = np.cumsum(rp)
    w = D[rows, cols]
    if dtype == np.int32:
        w = w.astype(np.uint32)
    for s in range(n):
        ref = orc.dijkstra(rp, cols.astype(np.int32), w, s)
        if dtype == np.int32:
            ref = np.where(ref == 0xFFFFFFFF, MISS, np.minimum(ref, MISS)).astype(np.int32)
            assert np.array_equal(got[s], ref), s
        else:
            # squaring sums paths in tree order, Dijkstra left to right: float
            # addition is not associative, so agreement is within 1e-6 relative
            assert np.array_equal(np.isinf(got[s]), np.isinf(ref)), s
            fin = np.isfinite(ref)
            assert np.allclose(got[s][fin], ref[fin], rtol=1e-6, atol=0), s
    # bit-exact against the same squarings done by the oracle
    Dc = D.copy()
    for _ in range(sq):
        Dc = orc.minplus_gemm(Dc, Dc)
    assert np.array_equal(got, Dc)
    assert 0 <= sq <= int(np.ceil(np.log2(max(n - 1, 1))))


def test_calibration_reports_a_rate(b2, cuda):
    from b200sssp import _lib
    import ctypes as C
    r = C.c_double()
    assert _lib.lib().b2_minplus_calibrate(0, C.byref(r)) == 0
    assert r.value > 1e12      # >1 T (min,+) pairs/s on a B200
    assert _lib.lib().b2_minplus_calibrate(1, C.byref(r)) == 0
    assert r.value > 1e12
