"""GPU parity: CSR x CSR min-plus SpGEMM vs the oracle (bit-exact; sorted rows)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
MISS = 1073741823


def _rand_csr(rng, R, C, dens, dtype, dup=False):
    rows, cols, vals = [], [], []
    for r in range(R):
        k = rng.binomial(C, dens) if C else 0
        cs = rng.choice(C, size=k, replace=False) if k else np.zeros(0, int)
        if dup and k:
            cs = np.concatenate([cs, rng.choice(cs, size=max(1, k // 3))])
        rng.shuffle(cs)
        rows += [r] * len(cs)
        cols += cs.tolist()
        if dtype == np.float32:
            v = rng.uniform(0, 1, len(cs)).astype(np.float32)
            v[rng.uniform(size=len(cs)) < 0.05] = np.inf
            v[rng.uniform(size=len(cs)) < 0.03] = np.nan
        else:
            v = rng.integers(1, 1001, len(cs)).astype(np.int32)
            v[rng.uniform(size=len(cs)) < 0.1] = MISS
        vals += v.tolist()
    rp = np.zeros(R + 1, np.int64)
    np.add.at(rp, np.array(rows, np.int64) + 1, 1)
    return np.cumsum(rp), np.array(cols, np.int32), np.array(vals, dtype)


def _gpu(b2, torch, A, B, ncols_b):
    ta = (torch.from_numpy(A[0]).cuda(), torch.from_numpy(A[1]).cuda(), torch.from_numpy(A[2]).cuda(),
          int(B[0].shape[0] - 1))
    tb = (torch.from_numpy(B[0]).cuda(), torch.from_numpy(B[1]).cuda(), torch.from_numpy(B[2]).cuda(), ncols_b)
    rp, ci, v = b2.minplus_spgemm(ta, tb)
    return rp.cpu().numpy(), ci.cpu().numpy(), v.cpu().numpy()


@pytest.mark.parametrize("dtype", [np.float32, np.int32])
@pytest.mark.parametrize("shape", [(40, 30, 50, 0.2), (200, 150, 120, 0.05), (1, 1, 1, 1.0), (64, 64, 64, 0.0),
                                   (300, 40, 500, 0.3)])
def test_spgemm_matches_oracle(b2, orc, cuda, dtype, shape):
    M, K, N, d = shape
    rng = np.random.default_rng(M + K + N)
    A = _rand_csr(rng, M, K, d, dtype, dup=True)
    B = _rand_csr(rng, K, N, d, dtype, dup=True)
    got = _gpu(b2, cuda, A, B, N)
    ref = orc.minplus_spgemm(A, B, N)
    assert np.array_equal(got[0], ref[0])
    assert np.array_equal(got[1], ref[1])
    assert np.array_equal(got[2], ref[2])


def test_spgemm_graph_square(b2, orc, cuda):
    """A (x) A on an ER graph: two-hop shortest path lengths (config C2s shape, scaled down)."""
    g = b2.gen_er(1 << 14, 8 << 14, 1, 1000, 5)
    A = (g.rowptr, g.colind, g.weights.astype(np.int32))
    got = _gpu(b2, cuda, A, A, g.n)
    ref = orc.minplus_spgemm(A, A, g.n)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)
    Af = (g.rowptr, g.colind, g.fweights)
    got = _gpu(b2, cuda, Af, Af, g.n)
    ref = orc.minplus_spgemm(Af, Af, g.n)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


def test_spgemm_invalid_inputs(b2, cuda):
    torch = cuda
    rp = torch.tensor([0, 1, 2], dtype=torch.int64, device="cuda")
    ci = torch.tensor([0, 5], dtype=torch.int32, device="cuda")         # 5 >= K
    v = torch.tensor([1.0, 2.0], dtype=torch.float32, device="cuda")
    good_ci = torch.tensor([0, 1], dtype=torch.int32, device="cuda")
    with pytest.raises(b2.B2Error) as e:
        b2.minplus_spgemm((rp, ci, v, 2), (rp, good_ci, v, 2))
    assert e.value.status == 9
    bad_rp = torch.tensor([0, 2, 1], dtype=torch.int64, device="cuda")
    with pytest.raises(b2.B2Error) as e:
        b2.minplus_spgemm((bad_rp, good_ci, v, 2), (rp, good_ci, v, 2))
    assert e.value.status == 10
    with pytest.raises(b2.B2Error) as e:      # A.cols != B.rows
        b2.minplus_spgemm((rp, good_ci, v, 3), (rp, good_ci, v, 2))
    assert e.value.status == 1


@pytest.mark.parametrize("dtype", [np.float32, np.int32])
def test_spgemm_row_sizes_across_sort_widths(b2, orc, cuda, dtype):
    """Rows whose candidate counts sit on every register-sort width boundary
    (32 x 1 .. 32 x 16) and just past the one-warp limit (512), where rows
    switch to expand-sort-compress; columns collide heavily so runs are long."""
    rng = np.random.default_rng(17)
    K, N = 700, 97
    blen = np.where(np.arange(K) < 600, 1, rng.integers(2, 9, K))      # rows 0..599 hold one entry
    brp = np.concatenate([[0], np.cumsum(blen)]).astype(np.int64)
    bci = rng.integers(0, N, int(brp[-1])).astype(np.int32)
    targets = [1, 2, 31, 32, 33, 63, 64, 65, 127, 128, 129, 255, 256, 257, 511, 512, 513, 640, 2000]
    rows, vals = [], []
    for t in targets:
        if t <= 600:
            cols = rng.permutation(600)[:t]
        else:
            cols = np.concatenate([rng.permutation(600), rng.integers(600, K, (t - 600) // 4 + 1)])
        rows.append(cols.astype(np.int32))
    arp = np.concatenate([[0], np.cumsum([len(r) for r in rows])]).astype(np.int64)
    aci = np.concatenate(rows)
    if dtype == np.float32:
        av = rng.uniform(0, 1, aci.size).astype(np.float32)
        bv = rng.uniform(0, 1, bci.size).astype(np.float32)
        av[rng.uniform(size=av.size) < 0.02] = np.inf
    else:
        av = rng.integers(1, 1000, aci.size).astype(np.int32)
        bv = rng.integers(1, 1000, bci.size).astype(np.int32)
        bv[rng.uniform(size=bv.size) < 0.02] = MISS
    A, B = (arp, aci, av), (brp, bci, bv)
    got = _gpu(b2, cuda, A, B, N)
    ref = orc.minplus_spgemm(A, B, N)
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("dtype", ["f32", "i32"])
def test_plan_fill_equals_callee_allocated_form(b2, orc, cuda, dtype):
    """The two-step form (b2_minplus_spgemm_plan / _fill into caller buffers)
    and the reference's one-call form (library-allocated outputs) give the
    same words; an unfilled plan is released by b2_minplus_spgemm_plan_free."""
    torch = cuda
    import ctypes as C
    from b200sssp import _lib, minplus
    hg = b2.gen_er(30000, 240000, 1, 1000, 91)
    vals = hg.weights.view(np.int32) if dtype == "i32" else hg.weights.astype(np.float32) / np.float32(1001)
    A = (torch.from_numpy(hg.rowptr).cuda(), torch.from_numpy(hg.colind).cuda(), torch.from_numpy(vals).cuda(), hg.n)
    p1 = minplus.minplus_spgemm(A, A)
    p2 = minplus.minplus_spgemm_callee_alloc(A, A)
    for x, y in zip(p1, p2):
        assert x.dtype == y.dtype and torch.equal(x, y)
    ref = orc.minplus_spgemm((hg.rowptr, hg.colind, vals), (hg.rowptr, hg.colind, vals), hg.n)
    assert np.array_equal(p1[0].cpu().numpy(), ref[0])
    assert np.array_equal(p1[1].cpu().numpy(), ref[1])
    assert np.array_equal(p1[2].cpu().numpy().view(np.uint32), ref[2].view(np.uint32))
    a = minplus._csr_view(*A)
    plan, nnz = C.c_void_p(), C.c_int64()
    assert _lib.lib().b2_minplus_spgemm_plan(C.byref(a), C.byref(a), None, C.byref(plan), C.byref(nnz)) == 0
    assert nnz.value == p1[1].numel()
    assert _lib.lib().b2_minplus_spgemm_plan_free(plan) == 0
