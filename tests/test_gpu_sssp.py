"""GPU parity: Bellman-Ford and delta-stepping kernels vs the oracle.

Distances must be bit-exact (uint32 and float32: the float fixpoint of
relaxation is unique, so a float32 Dijkstra reproduces it); against the
reference's float64 python path float32 results agree within 1e-6 relative.
Iteration counts follow the reference's rules exactly.  Predecessor arrays are
checked as shortest-path trees.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

INF_U = 0xFFFFFFFF


def _graph(b2, hg, weight):
    return b2.Graph.from_host(hg, weight=weight)


def _np(t):
    return t.cpu().numpy()


def _dist_u32(t):
    return _np(t).view(np.uint32)


def _raw(t, weight):
    return _dist_u32(t) if weight == "u32" else _np(t)


def _gpu_vs_dijkstra(b2, orc, hg, weight, sources, method="delta", pred=False, **opts):
    g = _graph(b2, hg, weight)
    w = hg.weights if weight == "u32" else hg.fweights
    for s in sources:
        dist, pr, st = g.sssp(int(s), method=method, pred=pred, **opts)
        ref = orc.dijkstra(hg.rowptr, hg.colind, w, int(s))
        got = _dist_u32(dist) if weight == "u32" else _np(dist)
        assert np.array_equal(got, ref), (method, weight, s, int(np.sum(got != ref)))
        if pred:
            code = orc.validate_spt(hg.rowptr, hg.colind, w, int(s), got, _np(pr))
            assert code == 0, (method, weight, s, code)
        yield got, st
    g.close()


@pytest.mark.parametrize("weight", ["u32", "f32"])
@pytest.mark.parametrize("method", ["bf", "delta"])
def test_er_c1_exact(b2, orc, cuda, weight, method):
    hg = b2.gen_er(4096, 32768, 1, 100, 0)
    for _ in _gpu_vs_dijkstra(b2, orc, hg, weight, [0, 1, 4095], method=method):
        pass


def test_c1_matches_reference_python_bf(b2, golden, cuda):
    z = golden("bf_py.npz")
    hg = b2.gen_er(4096, 32768, 1, 100, 0)
    g = _graph(b2, hg, "u32")
    for method in ("bf", "delta"):
        dist, _, st = g.sssp(0, method=method)
        d = _dist_u32(dist).astype(np.float64)
        d[_dist_u32(dist) == INF_U] = np.inf
        assert np.array_equal(d, z["c1_er4096/dist"]), method
    dist, _, st = g.sssp(0, method="bf")
    assert st["iterations_used"] == int(z["c1_er4096/meta"][3]) and st["converged"] == 1


@pytest.mark.parametrize("weight", ["u32", "f32"])
@pytest.mark.parametrize("method", ["bf", "delta"])
def test_rmat_and_grid_exact_with_pred(b2, orc, cuda, weight, method):
    for hg in (b2.gen_rmat(13, 16, seed=2), b2.gen_grid(96, 80, 0.02, seed=3)):
        deg = np.diff(hg.rowptr)
        srcs = [int(np.argmax(deg)), int(np.nonzero(deg)[0][7]), 0 if deg[0] else int(np.nonzero(deg)[0][0])]
        for _ in _gpu_vs_dijkstra(b2, orc, hg, weight, srcs, method=method, pred=True):
            pass


@pytest.mark.parametrize("delta", [1, 3, 40, 255, 100000])
def test_delta_bucket_counts_and_windows(b2, orc, cuda, delta):
    hg = b2.gen_rmat(12, 8, seed=5)
    for got, st in _gpu_vs_dijkstra(b2, orc, hg, "u32", [int(np.argmax(np.diff(hg.rowptr)))], delta=float(delta)):
        assert st["iterations_used"] == orc.delta_bucket_count(got, delta, "u32")
        assert st["converged"] == 1


@pytest.mark.parametrize("delta", [0.003, 0.05, 0.7, 9.0])
def test_delta_float_bucket_rule(b2, orc, cuda, delta):
    hg = b2.gen_grid(48, 40, 0.02, seed=8)
    for got, st in _gpu_vs_dijkstra(b2, orc, hg, "f32", [5], delta=delta):
        assert st["iterations_used"] == orc.delta_bucket_count(got, np.float32(delta), "f32")


def test_delta_max_iters_partial_state(b2, orc, cuda):
    """After k buckets: vertices of the first k buckets are final, every other
    vertex holds min over settled u of d[u] + w (reference loop semantics,
    delta_stepping_hip_CSR.cpp:701-780)."""
    hg = b2.gen_er(2000, 12000, 1, 60, 4)
    g = _graph(b2, hg, "u32")
    final = orc.dijkstra(hg.rowptr, hg.colind, hg.weights, 0)
    delta = 16
    fin = final[final != INF_U].astype(np.int64)
    buckets = np.unique(fin // delta)
    for k in (1, 2, 5, len(buckets) - 1, len(buckets), len(buckets) + 3):
        dist, _, st = g.sssp(0, method="delta", delta=float(delta), max_iters=k)
        got = _dist_u32(dist)
        settled_b = set(buckets[:k].tolist())
        settled = np.array([d != INF_U and (int(d) // delta) in settled_b for d in final])
        exp = np.full(hg.n, INF_U, np.uint64)
        exp[settled] = final[settled]
        src = np.repeat(np.arange(hg.n), np.diff(hg.rowptr))
        msk = settled[src]
        cand = final[src[msk]].astype(np.uint64) + hg.weights[msk]
        dst = hg.colind[msk]
        np.minimum.at(exp, dst, np.minimum(cand, INF_U))
        exp[settled] = final[settled]
        assert np.array_equal(got, exp.astype(np.uint32)), k
        assert st["iterations_used"] == min(k, len(buckets))
        assert st["converged"] == (1 if k >= len(buckets) else 0)


def test_bf_iterations_hop_limits_and_negative_weights(b2, orc, golden, cuda):
    z = golden("bf_py.npz")
    for name in [str(x) for x in z["names"]]:
        if name == "c1_er4096":
            continue
        n, src, mi, iters, conv, neg = (int(x) for x in z[f"{name}/meta"])
        rp, ci, dv = z[f"{name}/rowptr"], z[f"{name}/colind"], z[f"{name}/data"]
        dv32 = dv.astype(np.float32)
        g = b2.Graph.from_arrays(rp, ci, dv32, orientation="incoming", weight="f32")
        dist, _, st = g.sssp(src, method="bf", max_iters=mi, detect_negative_cycle=1)
        got = _np(dist)
        od, oused, oconv, oneg, _ = orc.bf_jacobi(rp, ci, dv32, src, mi, detect_negative=True)
        assert np.array_equal(got, od), name
        assert st["iterations_used"] == oused == iters, name
        assert bool(st["converged"]) == oconv == bool(conv), name
        assert bool(st["has_negative_cycle"]) == oneg == bool(neg), name
        ref = z[f"{name}/dist"]
        fin = np.isfinite(ref)
        assert np.array_equal(np.isfinite(got), fin), name
        if not neg:
            assert np.allclose(got[fin], ref[fin], rtol=1e-6, atol=1e-5), name
        g.close()


def test_dense_known_answers_on_gpu_bf(b2, golden, cuda):
    z = golden("dense_kats.npz")
    for name in [str(x) for x in z["names"]]:
        n, src, py_iters = (int(x) for x in z[f"{name}/meta"])
        e = z[f"{name}/edges"]
        if e.shape[0]:
            order = np.lexsort((e[:, 0], e[:, 1]))
            e = e[order]
        rp = np.zeros(n + 1, np.int64)
        np.add.at(rp, e[:, 1].astype(np.int64) + 1, 1)
        rp = np.cumsum(rp)
        g = b2.Graph.from_arrays(rp, e[:, 0].astype(np.int32), e[:, 2].astype(np.float32),
                                 orientation="incoming", weight="f32")
        dist, _, st = g.sssp(src, method="bf")
        got = _np(dist).astype(np.float64)
        exp = z[f"{name}/expected"]
        both = np.isinf(got) & np.isinf(exp)
        with np.errstate(invalid="ignore"):
            ok = both | (np.abs(got - exp) <= 1e-4 * (1 + np.abs(got) + np.abs(exp)))
        assert ok.all(), name
        if n > 1:
            assert st["iterations_used"] == py_iters, name
        g.close()


def test_variants_no_checks_and_single_vertex(b2, cuda):
    g = b2.Graph.from_arrays(np.array([0, 0], np.int64), np.zeros(0, np.int32), np.zeros(0, np.uint32))
    dist, _, st = g.sssp(0, method="bf")
    assert _dist_u32(dist).tolist() == [0] and st["iterations_used"] == 0 and st["converged"] == 0
    dist, _, st = g.sssp(0, method="delta")
    assert _dist_u32(dist).tolist() == [0]


def test_unreachable_zero_weights_duplicates(b2, orc, cuda):
    # duplicate arcs 0->1 (9, 3), zero-weight arcs 0->2 and 1->3, isolated vertex 5
    rp = np.array([0, 3, 4, 5, 5, 5, 5], np.int64)
    ci = np.array([1, 1, 2, 3, 4], np.int32)
    w = np.array([9, 3, 0, 0, 7], np.uint32)
    for method in ("bf", "delta"):
        g = b2.Graph.from_arrays(rp, ci, w)
        dist, pr, _ = g.sssp(0, method=method, pred=True)
        assert _dist_u32(dist).tolist() == [0, 3, 0, 3, 7, INF_U], method
        assert _np(pr).tolist() == [-1, 0, 0, 1, 2, -1], method


def test_incoming_orientation_same_answer(b2, orc, cuda):
    hg = b2.gen_rmat(11, 8, seed=9)
    hg.weights = (hg.weights * 3 + np.arange(hg.m, dtype=np.uint32) % 7).astype(np.uint32)  # asymmetric
    gi = hg.transpose()
    a = b2.Graph.from_host(hg, "u32")
    b = b2.Graph.from_arrays(gi.rowptr, gi.colind, gi.weights, orientation="incoming", weight="u32")
    for method in ("bf", "delta"):
        da, _, _ = a.sssp(3, method=method)
        db, _, _ = b.sssp(3, method=method)
        assert np.array_equal(_dist_u32(da), _dist_u32(db))
        assert np.array_equal(_dist_u32(da), orc.dijkstra(hg.rowptr, hg.colind, hg.weights, 3))


def test_invalid_inputs_rejected(b2, cuda):
    with pytest.raises(b2.B2Error) as e:
        b2.Graph.from_arrays(np.array([0, 2, 1], np.int64), np.array([1, 0], np.int32), np.array([1, 1], np.uint32))
    assert e.value.status == 10  # INVALID_ROWPTR
    with pytest.raises(b2.B2Error) as e:
        b2.Graph.from_arrays(np.array([0, 1, 2], np.int64), np.array([1, 5], np.int32), np.array([1, 1], np.uint32))
    assert e.value.status == 9   # INVALID_INDEX
    with pytest.raises(b2.B2Error) as e:
        b2.Graph.from_arrays(np.array([0, 1, 1], np.int64), np.array([1], np.int32), np.array([np.nan], np.float32))
    assert e.value.status == 11  # INVALID_WEIGHT
    g = b2.Graph.from_arrays(np.array([0, 1, 1], np.int64), np.array([1], np.int32), np.array([-1.0], np.float32))
    with pytest.raises(b2.B2Error) as e:
        g.sssp(0, method="delta")
    assert e.value.status == 11  # delta needs nonnegative weights
    d, _, _ = g.sssp(0, method="bf")
    assert _np(d).tolist() == [0.0, -1.0]
    with pytest.raises(b2.B2Error):
        g.sssp(7, method="bf")


def test_repeatable_and_large_properties(b2, orc, cuda):
    hg = b2.gen_rmat(17, 16, seed=11)
    g = _graph(b2, hg, "u32")
    s = int(np.argmax(np.diff(hg.rowptr)))
    d1, p1, st1 = g.sssp(s, method="delta", pred=True, collect_reach=1)
    d2, p2, _ = g.sssp(s, method="delta", pred=True)
    d3, _, _ = g.sssp(s, method="bf")
    assert np.array_equal(_np(d1), _np(d2)) and np.array_equal(_np(p1), _np(p2))
    assert np.array_equal(_np(d1), _np(d3))
    ref = orc.dijkstra(hg.rowptr, hg.colind, hg.weights, s)
    assert np.array_equal(_dist_u32(d1), ref)
    reached = ref != INF_U
    assert st1["reached"] == int(reached.sum())
    assert st1["reached_edges"] == int(np.diff(hg.rowptr)[reached].sum())


def test_light_heavy_split_is_schedule_only(b2, orc, cuda):
    """Relaxing light edges per sub-phase and heavy edges once per settled
    vertex changes work, never distances or the bucket count."""
    for hg in (b2.gen_rmat(12, 16, seed=21), b2.gen_grid(64, 64, 0.02, seed=22)):
        for weight in ("u32", "f32"):
            g = _graph(b2, hg, weight)
            delta = 40.0 if weight == "u32" else 0.03
            d1, _, s1 = g.sssp(3, method="delta", delta=delta, light_heavy=1)
            d0, _, s0 = g.sssp(3, method="delta", delta=delta, light_heavy=0)
            assert np.array_equal(_np(d1), _np(d0))
            assert s1["iterations_used"] == s0["iterations_used"]
            w = hg.weights if weight == "u32" else hg.fweights
            ref = orc.dijkstra(hg.rowptr, hg.colind, w, 3)
            got = _dist_u32(d1) if weight == "u32" else _np(d1)
            assert np.array_equal(got, ref)
            g.close()


def test_phase_trace(b2, cuda):
    hg = b2.gen_rmat(12, 8, seed=23)
    g = _graph(b2, hg, "u32")
    _, _, st = g.sssp(0, method="delta", trace=1)
    tr = g.trace()
    assert len(tr) == st["phases"]
    assert tr[-1]["kind"] == "output"
    ts = [e["t_us"] for e in tr]
    assert ts == sorted(ts)
    assert any(e["kind"] == "relax-heavy" for e in tr)
    _, _, st = g.sssp(0, method="bf", trace=1)
    assert len(g.trace()) == st["phases"]


def test_dense_bf_known_answers(b2, golden, cuda):
    """bellman_ford_minplus_hip's dense path on the reference's 14 KATs
    (HIP_kernel/bellman_ford/tests/test_correctness.cpp), n <= 1024 dense."""
    torch = cuda
    z = golden("dense_kats.npz")
    for name in [str(x) for x in z["names"]]:
        n, src, py_iters = (int(x) for x in z[f"{name}/meta"])
        if n > 1024:
            continue
        adj = np.full((n, n), np.inf, np.float32)
        for u, v, w in z[f"{name}/edges"]:
            u, v = int(u), int(v)
            adj[v, u] = min(adj[v, u], np.float32(w))
        dist, st = b2.bf_dense(torch.from_numpy(adj).cuda(), src)
        got = _np(dist).astype(np.float64)
        exp = z[f"{name}/expected"]
        both = np.isinf(got) & np.isinf(exp)
        with np.errstate(invalid="ignore"):
            ok = both | (np.abs(got - exp) <= 1e-4 * (1 + np.abs(got) + np.abs(exp)))
        assert ok.all(), name
        if n > 1:
            assert st["iterations_used"] == py_iters, name


@pytest.mark.parametrize("fusion", [64, 4096, 1 << 30])
def test_bucket_fusion_is_schedule_only(b2, orc, cuda, fusion):
    """Small light frontiers run by one block (bucket fusion) give the same
    distances, predecessor trees and bucket counts as the grid-wide schedule."""
    for hg, weight, delta in ((b2.gen_grid(80, 70, 0.02, seed=31), "u32", 500.0),
                              (b2.gen_rmat(12, 16, seed=32), "f32", 0.1),
                              (b2.gen_er(3000, 15000, 1, 50, 33), "u32", 7.0)):
        g = _graph(b2, hg, weight)
        w = hg.weights if weight == "u32" else hg.fweights
        d0, _, s0 = g.sssp(1, method="delta", delta=delta, fusion_threshold=0)
        d1, p1, s1 = g.sssp(1, method="delta", delta=delta, fusion_threshold=fusion, pred=True)
        assert np.array_equal(_np(d0), _np(d1))
        assert s0["iterations_used"] == s1["iterations_used"]
        assert s1["local_subphases"] > 0
        got = _dist_u32(d1) if weight == "u32" else _np(d1)
        assert np.array_equal(got, orc.dijkstra(hg.rowptr, hg.colind, w, 1))
        assert orc.validate_spt(hg.rowptr, hg.colind, w, 1, got, _np(p1)) == 0
        dk, _, sk = g.sssp(1, method="delta", delta=delta, fusion_threshold=fusion, max_iters=3)
        dr, _, sr = g.sssp(1, method="delta", delta=delta, fusion_threshold=0, max_iters=3)
        assert np.array_equal(_np(dk), _np(dr)) and sk["converged"] == sr["converged"]
        g.close()


@pytest.mark.parametrize("weight", ["u32", "f32"])
def test_adds_adaptive_width_exact(b2, orc, cuda, weight):
    """ADDS schedule: bucket width adapted at window boundaries (re-based
    windows); distances must stay exact and predecessors a shortest-path tree."""
    for hg in (b2.gen_rmat(13, 16, seed=41), b2.gen_grid(100, 90, 0.02, seed=42), b2.gen_er(5000, 40000, 1, 200, 43)):
        g = _graph(b2, hg, weight)
        w = hg.weights if weight == "u32" else hg.fweights
        deg = np.diff(hg.rowptr)
        src = int(np.argmax(deg))
        ref = orc.dijkstra(hg.rowptr, hg.colind, w, src)
        for delta in (0.0, 1.0 if weight == "u32" else 1e-4):
            d, p, st = g.sssp(src, method="adds", delta=delta, pred=True)
            got = _dist_u32(d) if weight == "u32" else _np(d)
            assert np.array_equal(got, ref), (delta, int(np.sum(got != ref)))
            assert orc.validate_spt(hg.rowptr, hg.colind, w, src, got, _np(p)) == 0
            assert st["converged"] == 1
            if delta:
                assert st["delta_updates"] > 0 and st["delta_final"] > delta
        g.close()


@pytest.mark.parametrize("weight", ["u32", "f32"])
def test_degree_order_keeps_input_ids(b2, orc, cuda, weight):
    """A graph renumbered internally by degree answers in input ids: distances
    bit-exact, predecessors a shortest-path tree, for every method, from the
    server too, and the same words as the graph in input order."""
    from b200sssp import serving
    hg = b2.gen_rmat(13, 16, seed=21)
    w = hg.weights if weight == "u32" else hg.fweights
    plain = b2.Graph.from_host(hg, weight)
    g = b2.Graph.from_host(hg, weight)
    assert not g.degree_ordered
    g.set_degree_order()
    g.set_degree_order()                      # idempotent
    assert g.degree_ordered
    for s in (0, 77, hg.n - 1):
        ref = orc.dijkstra(hg.rowptr, hg.colind, w, s)
        for method in ("delta", "bf", "adds"):
            d, p, st = g.sssp(s, method=method, pred=True)
            got = _raw(d, weight)
            assert np.array_equal(got, ref), method
            assert orc.validate_spt(hg.rowptr, hg.colind, w, s, got, p.cpu().numpy()) == 0
            d0, _, st0 = plain.sssp(s, method=method)
            assert np.array_equal(got, _raw(d0, weight))
            if method != "adds":   # ADDS adapts its bucket width as it goes: the count is its schedule's
                assert st["iterations_used"] == st0["iterations_used"]
        d, _, st = g.sssp(s, collect_reach=1)
        _, _, st0 = plain.sssp(s, collect_reach=1)
        assert (st["reached"], st["reached_edges"]) == (st0["reached"], st0["reached_edges"])
    srv = serving.Server(hbm_budget=64 << 20)
    gid = srv.add_graph(g)
    outs = []
    for s in (5, 901):
        out = srv.result_buffer(g)
        pr = cuda.empty(g.n, dtype=cuda.int32).pin_memory()
        srv.submit(gid, s, out, pr)
        outs.append((s, out, pr))
    srv.progress(wait_all=True)
    assert all(c["status"] == 0 for c in srv.poll())
    for s, out, pr in outs:
        ref = orc.dijkstra(hg.rowptr, hg.colind, w, s)
        got = out.numpy().view(np.uint32) if weight == "u32" else out.numpy()
        assert np.array_equal(got, ref)
        assert orc.validate_spt(hg.rowptr, hg.colind, w, s, got, pr.numpy()) == 0
    srv.close()
    f = __import__("b200sssp.policy", fromlist=["graph_features"]).graph_features(g)
    assert np.isfinite(f).all()
    g.close()
    plain.close()


@pytest.mark.parametrize("weight", ["u32", "f32"])
def test_pull_heavy_pass_matches_push(b2, orc, cuda, weight):
    """The pull direction of the heavy pass (forced with a tiny switch point)
    gives the push pass's words exactly: distances, predecessors (smallest id
    among equal distances) and bucket counts, also on a degree-ordered graph.
    The asynchronous ADDS kernel has no heavy pass: the switch point leaves
    its distances exact."""
    graphs = [b2.gen_rmat(13, 16, seed=31), b2.gen_er(3000, 24000, 1, 1000, seed=32),
              b2.gen_grid(40, 50, 0.05, seed=33)]
    for k, hg in enumerate(graphs):
        w = hg.weights if weight == "u32" else hg.fweights
        g = b2.Graph.from_host(hg, weight)
        if k == 0:
            g.set_degree_order()
        for s in (0, hg.n // 3):
            ref = orc.dijkstra(hg.rowptr, hg.colind, w, s)
            da, _, sa = g.sssp(s, method="adds", pull_fraction=1e-9)
            assert np.array_equal(_raw(da, weight), ref) and sa["heavy_pulls"] == 0
        for method in ("delta",):
            for s in (0, hg.n // 3):
                ref = orc.dijkstra(hg.rowptr, hg.colind, w, s)
                dp, pp, sp = g.sssp(s, method=method, pred=True, pull_fraction=0.0)
                dq, pq, sq = g.sssp(s, method=method, pred=True, pull_fraction=1e-9)
                assert sp["heavy_pulls"] == 0 and sq["heavy_pulls"] > 0
                assert np.array_equal(_raw(dq, weight), ref)
                assert np.array_equal(_raw(dq, weight), _raw(dp, weight))
                assert np.array_equal(pq.cpu().numpy(), pp.cpu().numpy())
                assert sq["iterations_used"] == sp["iterations_used"]
                d2, _, _ = g.sssp(s, method=method, pull_fraction=1e-9)      # no predecessors
                assert np.array_equal(_raw(d2, weight), ref)
        g.close()


def test_pull_switch_point(b2, orc, cuda):
    """A dense skewed graph solved from its biggest hub pulls the heavy pass of
    its first bucket once the members' heavy edges pass the switch point, and
    still matches the oracle; a sparse grid never builds the incoming CSR."""
    hg = b2.gen_rmat(15, 32, seed=41)
    g = b2.Graph.from_host(hg, "u32")
    hub = int(np.argmax(np.diff(hg.rowptr)))
    d, _, st = g.sssp(hub, pull_fraction=2.0)
    assert st["heavy_pulls"] >= 1
    assert np.array_equal(_raw(d, "u32"), orc.dijkstra(hg.rowptr, hg.colind, hg.weights, hub))
    _, _, st = g.sssp(hub, pull_fraction=1e6)       # switch point never reached: push only
    assert st["heavy_pulls"] == 0
    grid = b2.gen_grid(64, 64, 0.0, seed=42)
    gg = b2.Graph.from_host(grid, "u32")
    gg.sssp(0, pull_fraction=0.0)                                # workspace allocated, push only
    before = gg.info()["device_bytes"]
    _, _, st = gg.sssp(0)
    assert st["heavy_pulls"] == 0
    assert gg.info()["device_bytes"] == before                   # no incoming CSR for a sparse grid
    g.close()
    gg.close()


@pytest.mark.parametrize("weight", ["u32", "f32"])
def test_stamp_sweep_matches_queue(b2, orc, cuda, weight):
    """Frontiers found by sweeping the push / bucket stamps (forced on every
    phase with a tiny threshold) give the queue path's words exactly:
    distances, predecessors and bucket counts, on a grid, an ER graph and a
    degree-ordered RMAT graph.  (Block-local sub-phases always read their
    queues; a threshold of one keeps them out of the way.)  The asynchronous
    ADDS kernel has no phases to sweep: the option leaves its distances
    exact."""
    graphs = [b2.gen_grid(60, 70, 0.02, seed=51), b2.gen_er(3000, 24000, 1, 1000, seed=52),
              b2.gen_rmat(13, 16, seed=53)]
    for k, hg in enumerate(graphs):
        w = hg.weights if weight == "u32" else hg.fweights
        g = b2.Graph.from_host(hg, weight)
        if k == 2:
            g.set_degree_order()
        for s in (0, hg.n // 2):
            ref = orc.dijkstra(hg.rowptr, hg.colind, w, s)
            da, _, _ = g.sssp(s, method="adds", dense_fraction=1e-9)
            assert np.array_equal(_raw(da, weight), ref)
        for method in ("delta",):
            for s in (0, hg.n // 2):
                ref = orc.dijkstra(hg.rowptr, hg.colind, w, s)
                dq, pq, sq = g.sssp(s, method=method, pred=True, dense_fraction=-1.0, fusion_threshold=1)
                dd, pd, sd = g.sssp(s, method=method, pred=True, dense_fraction=1e-9, fusion_threshold=1,
                                    trace=1)
                assert any(e["kind"].endswith("-dense") for e in g.trace())
                assert np.array_equal(_raw(dd, weight), ref)
                assert np.array_equal(_raw(dq, weight), ref)
                assert np.array_equal(pd.cpu().numpy(), pq.cpu().numpy())
                assert sd["iterations_used"] == sq["iterations_used"]
                d2, _, _ = g.sssp(s, method=method, dense_fraction=1e-9)      # no predecessors
                assert np.array_equal(_raw(d2, weight), ref)
        g.close()


def test_stamp_sweep_default_follows_degree(b2, cuda):
    """By default a low-degree grid sweeps its large frontiers and a skewed
    RMAT graph keeps reading its queues."""
    grid = b2.Graph.from_host(b2.gen_grid(128, 128, 0.02, seed=54), "u32")
    grid.sssp(0, trace=1)
    assert any(e["kind"].endswith("-dense") for e in grid.trace())
    rm = b2.Graph.from_host(b2.gen_rmat(14, 16, seed=55), "u32")
    rm.sssp(0, trace=1)
    assert not any(e["kind"].endswith("-dense") for e in rm.trace())
    grid.close()
    rm.close()


def test_reference_tiny_lonestar_known_answer(b2, cuda):
    """The reference's tiny Lonestar graph (tests/golden/tiny.gr, written by its
    make_tiny_gr.py) solved from the file: every method gives the distances of
    its check_tiny_output.py."""
    import json
    import os
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    t = json.load(open(os.path.join(golden, "tiny_gr.json")))
    exp = np.array([np.inf if x is None else x for x in t["expected"]], np.float32)
    g = b2.Graph.from_host(b2.lonestar_read(os.path.join(golden, "tiny.gr")), "f32")
    for method in ("bf", "delta", "adds"):
        d, _, st = g.sssp(t["source"], method=method)
        assert np.array_equal(_np(d), exp), method
    g.close()


@pytest.mark.parametrize("method", ["bf", "delta", "adds"])
def test_live_progress_callback(b2, orc, cuda, method):
    """The progress callback runs while the kernel runs: one call per round
    (BF) or bucket (delta, ADDS), in order, the first well before the solve
    returns; BF's last round reports no change (bf_hip_CSR.cpp:79-95), and
    delta-stepping's last bucket reports no successor."""
    import time
    hg = b2.gen_grid(512, 512, 0.0, seed=77)
    g = _graph(b2, hg, "u32")
    g.sssp(0, method=method)   # warm: workspace, light counts
    calls = []
    t0 = time.perf_counter()
    d, _, st = g.sssp(0, method=method, progress=lambda p: calls.append((time.perf_counter(), p)))
    t1 = time.perf_counter()
    assert np.array_equal(_dist_u32(d), orc.dijkstra(hg.rowptr, hg.colind, hg.weights, 0))
    its = [p["iteration"] for _, p in calls]
    assert its == list(range(1, st["iterations_used"] + 1))
    assert all(p["changed"] for _, p in calls[:-1]) and not calls[-1][1]["changed"]
    ms = [p["elapsed_ms"] for _, p in calls[:-1]]
    assert all(a <= b for a, b in zip(ms, ms[1:]))
    if method == "bf":
        assert len(calls) > 100
        # published while running: the first report precedes the return by
        # a good part of the solve
        assert calls[0][0] - t0 < 0.5 * (t1 - t0)
    g.close()
