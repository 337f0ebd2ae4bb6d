"""GPU: the asynchronous ADDS worklist kernel (b2_sssp_adds).

Distances are bit-exact against the oracle's Dijkstra (uint32 and float32),
predecessors form shortest-path trees, repeated solves on one handle agree,
small worklists, a tiny bucket width (many window epochs and far-pile
splits), a fixed width and every starting active-bucket count give the same
words.  The warm start (hip_adds::Options::initialize_distances = false,
hip_adds_sssp.hpp:64-66) keeps the caller's distances as upper bounds and
matches the oracle's warm Dijkstra, in input ids on degree-ordered graphs too.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

INF = 0xFFFFFFFF


def _graphs(b2):
    return {"rmat15": b2.gen_rmat(15, 16, seed=61), "grid300": b2.gen_grid(300, 280, 0.02, seed=62),
            "er": b2.gen_er(20000, 160000, 1, 100, 63)}


@pytest.mark.parametrize("weight", ["u32", "f32"])
def test_adds_exact_with_pred(b2, orc, cuda, weight):
    for name, hg in _graphs(b2).items():
        g = b2.Graph.from_host(hg, weight)
        w = hg.weights if weight == "u32" else hg.fweights
        deg = np.diff(hg.rowptr)
        for s in (int(np.argmax(deg)), int(np.flatnonzero(deg)[7])):
            ref = orc.dijkstra(hg.rowptr, hg.colind, w, s)
            d, p, st = g.sssp(s, method="adds", pred=True)
            got = d.cpu().numpy()
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), (name, s)
            assert orc.validate_spt(hg.rowptr, hg.colind, w, s, got, p.cpu().numpy()) == 0, (name, s)
            assert st["converged"] == 1 and st["work_items"] > 0
            d2, _, _ = g.sssp(s, method="adds")
            assert np.array_equal(d2.cpu().numpy().view(np.uint32), ref.view(np.uint32)), (name, s)
        g.close()


@pytest.mark.parametrize("opts", [{"delta": 1.0}, {"delta": 3.0, "adds_fixed_delta": 1}, {"active_buckets": 1},
                                  {"active_buckets": 32}, {"hub_degree": 64}, {"grid_blocks": 7},
                                  {"active_buckets": 1, "max_active_buckets": 1}, {"max_active_buckets": 4}])
def test_adds_schedule_options_keep_words(b2, orc, cuda, opts):
    hg = b2.gen_rmat(14, 16, seed=64)
    g = b2.Graph.from_host(hg, "u32")
    ref = orc.dijkstra(hg.rowptr, hg.colind, hg.weights, 3)
    d, _, st = g.sssp(3, method="adds", **opts)
    assert np.array_equal(d.cpu().numpy().view(np.uint32), ref)
    if opts.get("delta") == 1.0:
        assert st["phases"] > 1 and st["delta_updates"] > 0 and st["delta_final"] > 1.0
    if opts.get("adds_fixed_delta"):
        assert st["delta_updates"] == 0 and st["delta_final"] == 3.0
    if opts.get("max_active_buckets"):
        assert st["active_buckets_max"] <= opts["max_active_buckets"]
    g.close()


@pytest.mark.parametrize("weight", ["u32", "f32"])
@pytest.mark.parametrize("ordered", [False, True])
def test_adds_warm_start(b2, orc, cuda, weight, ordered):
    torch = cuda
    hg = b2.gen_rmat(14, 16, seed=65)
    g = b2.Graph.from_host(hg, weight)
    if ordered:
        g.set_degree_order()
    w = hg.weights if weight == "u32" else hg.fweights
    rng = np.random.default_rng(66)
    cold = orc.dijkstra(hg.rowptr, hg.colind, w, 9)
    # upper bounds: infinity, the cold answer with noise above it, and a few
    # values below it (kept: a warm start trusts its bounds)
    if weight == "u32":
        init = np.full(hg.n, INF, np.uint32)
        pick = rng.choice(hg.n, hg.n // 3, replace=False)
        fin = cold[pick] != INF
        init[pick[fin]] = cold[pick[fin]] + rng.integers(0, 40, int(fin.sum())).astype(np.uint32)
        low = rng.choice(hg.n, 50, replace=False)
        init[low] = np.minimum(cold[low], 3).astype(np.uint32)
        dt = torch.int32
        t = torch.from_numpy(init.view(np.int32).copy()).cuda()
    else:
        init = np.full(hg.n, np.inf, np.float32)
        pick = rng.choice(hg.n, hg.n // 3, replace=False)
        init[pick] = cold[pick] + rng.uniform(0, 0.2, pick.shape[0]).astype(np.float32)
        low = rng.choice(hg.n, 50, replace=False)
        init[low] = np.minimum(cold[low], np.float32(0.01))
        dt = torch.float32
        t = torch.from_numpy(init.copy()).cuda()
    want = orc.dijkstra_warm(hg.rowptr, hg.colind, w, 9, init)
    d, _, st = g.sssp(9, method="adds", out=t, keep_distances=1)
    assert d.dtype == dt
    assert np.array_equal(d.cpu().numpy().view(np.uint32), want.view(np.uint32))
    # with predecessors the distances are the same words
    t2 = torch.from_numpy(init.view(np.int32).copy() if weight == "u32" else init.copy()).cuda()
    d2, p2, _ = g.sssp(9, method="adds", out=t2, keep_distances=1, pred=True)
    assert np.array_equal(d2.cpu().numpy().view(np.uint32), want.view(np.uint32))
    pr = p2.cpu().numpy()
    assert pr[9] == -1
    # a cold solve afterwards is exact again
    d3, _, _ = g.sssp(9, method="adds")
    assert np.array_equal(d3.cpu().numpy().view(np.uint32), cold.view(np.uint32))
    g.close()


def test_warm_start_is_adds_only(b2, cuda):
    from b200sssp import _lib
    hg = b2.gen_er(1000, 8000, 1, 100, 67)
    g = b2.Graph.from_host(hg, "u32")
    for m in ("delta", "bf"):
        with pytest.raises(_lib.B2Error) as ei:
            g.sssp(0, method=m, keep_distances=1)
        assert ei.value.status == _lib.NOT_SUPPORTED
    g.close()


def test_adds_small_worklist_is_pool_exhausted(b2, orc, cuda):
    from b200sssp import _lib
    hg = b2.gen_rmat(15, 16, seed=68)
    g = b2.Graph.from_host(hg, "u32")
    with pytest.raises(_lib.B2Error) as ei:
        g.sssp(2, method="adds", worklist_capacity=16)
    assert ei.value.status == _lib.POOL_EXHAUSTED
    d, _, _ = g.sssp(2, method="adds")
    assert np.array_equal(d.cpu().numpy().view(np.uint32), orc.dijkstra(hg.rowptr, hg.colind, hg.weights, 2))
    g.close()
