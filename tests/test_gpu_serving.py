"""GPU: batched serving -- per-query parity with the oracle, isolation (same
words alone and in a mix), HBM-budget admission, cancellation, refusals, the
per-query time budget, and the load generator's accounting."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def srvmod(b2, cuda):
    from b200sssp import serving
    return serving


@pytest.fixture(scope="module")
def graphs(b2, cuda):
    specs = [("er", b2.gen_er(3000, 24000, 1, 1000, seed=1), "u32"),
             ("rmat", b2.gen_rmat(13, 16, seed=2), "u32"),
             ("grid", b2.gen_grid(70, 50, 0.02, seed=3), "u32"),
             ("rmatf", b2.gen_rmat(12, 8, seed=4), "f32"),
             ("gridf", b2.gen_grid(40, 40, 0.0, seed=5), "f32")]
    return [(name, hg, b2.Graph.from_host(hg, w), w) for name, hg, w in specs]


def _raw(t, weight):
    a = t.cpu().numpy()
    return a.view(np.uint32) if weight == "u32" else a


def _w(hg, weight):
    return hg.weights if weight == "u32" else hg.fweights


def test_server_matches_oracle(srvmod, graphs, orc):
    srv = srvmod.Server(hbm_budget=256 << 20)
    jobs = []
    for name, hg, g, w in graphs:
        gid = srv.add_graph(g)
        rng = np.random.default_rng(len(name))
        for s in rng.integers(0, g.n, 6):
            out = srv.result_buffer(g)
            jobs.append((srv.submit(gid, int(s), out), hg, w, int(s), out))
    srv.progress(wait_all=True)
    done = {c["ticket"]: c for c in srv.poll()}
    assert len(done) == len(jobs)
    for t, hg, w, s, out in jobs:
        assert done[t]["status"] == 0
        ref = orc.dijkstra(hg.rowptr, hg.colind, _w(hg, w), s)
        assert np.array_equal(_raw(out, w), ref)
        reached = int(np.count_nonzero(ref != (0xFFFFFFFF if w == "u32" else np.inf)))
        assert done[t]["reached"] == reached
    srv.close()


def test_server_predecessors_match_full_solver(srvmod, graphs, orc, cuda):
    torch = cuda
    srv = srvmod.Server(hbm_budget=256 << 20)
    for name, hg, g, w in graphs:
        gid = srv.add_graph(g)
        for s in (0, g.n // 2):
            out = srv.result_buffer(g)
            pr = torch.empty(g.n, dtype=torch.int32).pin_memory()
            t = srv.submit(gid, s, out, pr)
            srv.progress(wait_all=True)
            (c,) = srv.poll()
            assert c["ticket"] == t and c["status"] == 0
            d_full, p_full, _ = g.sssp(s, method="delta", pred=True)
            assert np.array_equal(_raw(out, w), _raw(d_full, w))
            assert np.array_equal(pr.numpy(), p_full.cpu().numpy())
            got = _raw(out, w)
            assert orc.validate_spt(hg.rowptr, hg.colind, _w(hg, w), s, got, pr.numpy()) == 0
    srv.close()


def test_isolation_alone_and_in_the_mix(srvmod, graphs, cuda):
    """A query's words do not depend on the other queries of its batches."""
    name, hg, g, w = graphs[1]
    srv = srvmod.Server(hbm_budget=512 << 20)
    gids = [srv.add_graph(x[2]) for x in graphs]
    alone = srv.result_buffer(g)
    srv.submit(gids[1], 7, alone)
    srv.progress(wait_all=True)
    srv.poll()
    rng = np.random.default_rng(0)
    mix, bufs = [], []
    for i in range(600):
        k = int(rng.integers(0, len(graphs)))
        gg = graphs[k][2]
        out = srv.result_buffer(gg)
        bufs.append(out)
        mix.append(srv.submit(gids[k], int(rng.integers(0, gg.n)), out))
        if i == 300:
            mine = srv.result_buffer(g)
            mt = srv.submit(gids[1], 7, mine)
    srv.progress(wait_all=True)
    res = {c["ticket"]: c for c in srv.poll()}
    assert all(res[t]["status"] == 0 for t in mix) and res[mt]["status"] == 0
    assert np.array_equal(_raw(mine, w), _raw(alone, w))
    srv.close()


def test_hbm_budget_admission(srvmod, graphs, orc):
    name, hg, g, w = graphs[0]
    slot = srvmod.slot_bytes(g.n)
    srv = srvmod.Server(hbm_budget=2 * slot + 4096)       # two queries at a time
    gid = srv.add_graph(g)
    big = graphs[1][2]                                    # larger graph: never fits
    gbig = srv.add_graph(big)
    with pytest.raises(Exception) as e:
        srv.submit(gbig, 0, srv.result_buffer(big))
    assert getattr(e.value, "status", None) == 3         # B2_OUT_OF_MEMORY
    outs = [(s, srv.result_buffer(g)) for s in range(0, 40, 2)]
    ts = [srv.submit(gid, s, o) for s, o in outs]
    srv.progress()
    assert srv.info()["arena_used"] <= 2 * slot + 4096
    srv.progress(wait_all=True)
    done = {c["ticket"]: c for c in srv.poll()}
    for t, (s, o) in zip(ts, outs):
        assert done[t]["status"] == 0
        assert np.array_equal(_raw(o, w), orc.dijkstra(hg.rowptr, hg.colind, _w(hg, w), s))
    assert srv.info()["arena_used"] == 0
    srv.close()


def test_cancel_and_refusals(srvmod, graphs, b2, cuda):
    torch = cuda
    name, hg, g, w = graphs[2]
    srv = srvmod.Server(hbm_budget=64 << 20)
    gid = srv.add_graph(g)
    outs = [srv.result_buffer(g) for _ in range(5)]
    ts = [srv.submit(gid, i, o) for i, o in enumerate(outs)]
    assert srv.cancel(ts[2])
    assert not srv.cancel(123456789)
    srv.progress(wait_all=True)
    done = {c["ticket"]: c for c in srv.poll()}
    assert done[ts[2]]["status"] == 12                    # B2_CANCELLED
    assert all(done[t]["status"] == 0 for i, t in enumerate(ts) if i != 2)
    ref, _, _ = g.sssp(4, method="delta")
    assert np.array_equal(_raw(outs[4], w), _raw(ref, w))
    with pytest.raises(b2.B2Error) as e:                 # source out of range
        srv.submit(gid, g.n, outs[0])
    assert e.value.status == 1
    pageable = torch.empty(g.n, dtype=torch.int32)        # not page-locked: refused
    with pytest.raises(b2.B2Error) as e:
        srv.submit(gid, 0, pageable)
    assert e.value.status == 1
    rp = np.array([0, 1, 1], np.int64)
    neg = b2.Graph.from_arrays(rp, np.array([1], np.int32), np.array([-1.0], np.float32))
    with pytest.raises(b2.B2Error) as e:
        srv.add_graph(neg)
    assert e.value.status == 11
    srv.close()


def test_device_result_buffers(srvmod, graphs, cuda):
    name, hg, g, w = graphs[3]
    srv = srvmod.Server(hbm_budget=64 << 20)
    gid = srv.add_graph(g)
    out = srv.result_buffer(g, pinned=False)
    srv.submit(gid, 3, out)
    srv.progress(wait_all=True)
    (c,) = srv.poll()
    assert c["status"] == 0
    ref, _, _ = g.sssp(3, method="delta")
    assert np.array_equal(_raw(out, w), _raw(ref, w))
    srv.close()


def test_time_budget_reports_timeout(srvmod, graphs):
    """A per-query budget that runs out ends that query with B2_TIMEOUT; the
    server keeps serving (no device fault, the kernel returns)."""
    name, hg, g, w = graphs[2]
    srv = srvmod.Server(hbm_budget=64 << 20, timeout_ms=1e-6)
    gid = srv.add_graph(g)
    out = srv.result_buffer(g)
    srv.submit(gid, 0, out)
    srv.progress(wait_all=True)
    (c,) = srv.poll()
    assert c["status"] == 7                               # B2_TIMEOUT
    srv.close()
    ok = srvmod.Server(hbm_budget=64 << 20)
    gid = ok.add_graph(g)
    ok.submit(gid, 0, out)
    ok.progress(wait_all=True)
    (c,) = ok.poll()
    assert c["status"] == 0
    ok.close()


@pytest.mark.parametrize("mode", ["server", "sequential"])
def test_load_generator_results(srvmod, graphs, cuda, mode):
    srv = srvmod.Server(hbm_budget=256 << 20)
    for x in graphs:
        srv.add_graph(x[2])
    rep = srv.run_load(120, rate_qps=20000.0 if mode == "server" else 0.0, seed=5, mode=mode, record=True)
    assert rep["completed"] == 120 and rep["failed"] == 0
    assert rep["p50_us"] > 0 and rep["p99_us"] >= rep["p50_us"]
    for i in range(0, 120, 11):
        _, hg, g, w = graphs[int(rep["query_graph"][i])]
        d, _, _ = g.sssp(int(rep["query_source"][i]), method="delta")
        assert srvmod.checksum_words(d.cpu().numpy()) == int(rep["checksums"][i])
    srv.close()


@pytest.mark.parametrize("big_vertices", [1, 4000])
def test_cluster_teams_match_oracle_and_solver(srvmod, graphs, orc, cuda, big_vertices):
    """Queries on big graphs are solved by a cluster of blocks sharing the lead
    block's state through distributed shared memory: distances equal the
    oracle's, predecessors equal the full-GPU solver's, and a query's words do
    not change when it runs among others (every graph a cluster, or a mix)."""
    torch = cuda
    srv = srvmod.Server(hbm_budget=512 << 20, big_vertices=big_vertices)
    gids = [srv.add_graph(x[2]) for x in graphs]
    jobs = []
    for (name, hg, g, w), gid in zip(graphs, gids):
        for s in (0, g.n // 2, g.n - 1):
            out = srv.result_buffer(g)
            pr = torch.empty(g.n, dtype=torch.int32).pin_memory()
            jobs.append((srv.submit(gid, s, out, pr), hg, g, w, s, out, pr))
    # a mix of plain queries around them
    rng = np.random.default_rng(3)
    for _ in range(200):
        k = int(rng.integers(0, len(graphs)))
        srv.submit(gids[k], int(rng.integers(0, graphs[k][2].n)), srv.result_buffer(graphs[k][2]))
    srv.progress(wait_all=True)
    done = {c["ticket"]: c for c in srv.poll()}
    assert all(c["status"] == 0 for c in done.values())
    for t, hg, g, w, s, out, pr in jobs:
        ref = orc.dijkstra(hg.rowptr, hg.colind, _w(hg, w), s)
        assert np.array_equal(_raw(out, w), ref)
        _, p_full, _ = g.sssp(s, method="delta", pred=True)
        assert np.array_equal(pr.numpy(), p_full.cpu().numpy())
        reached = int(np.count_nonzero(ref != (0xFFFFFFFF if w == "u32" else np.inf)))
        assert done[t]["reached"] == reached
    rep = srv.run_load(200, rate_qps=0.0, seed=9, record=True)
    assert rep["completed"] == 200 and rep["failed"] == 0
    for i in range(0, 200, 17):
        _, hg, g, w = graphs[int(rep["query_graph"][i])]
        ref = orc.dijkstra(hg.rowptr, hg.colind, _w(hg, w), int(rep["query_source"][i]))
        assert int(rep["checksums"][i]) == srvmod.checksum_words(ref)
    srv.close()


def test_autotuned_server_matches_oracle(srvmod, graphs, orc):
    """With autotune the server times each graph under every team kind and
    bucket-width constant before admitting queries; answers stay exact."""
    srv = srvmod.Server(hbm_budget=512 << 20, autotune=True)
    gids = [srv.add_graph(x[2]) for x in graphs[:3]]
    for gid in gids:
        cfg = srv.graph_config(gid)
        assert cfg["tuned"] and cfg["delta_scale"] in (2.0, 4.0, 8.0)
    jobs = []
    for (name, hg, g, w), gid in zip(graphs[:3], gids):
        for s in (0, g.n // 3):
            out = srv.result_buffer(g)
            jobs.append((srv.submit(gid, s, out), hg, w, s, out))
    srv.progress(wait_all=True)
    done = {c["ticket"]: c for c in srv.poll()}
    for t, hg, w, s, out in jobs:
        assert done[t]["status"] == 0
        assert np.array_equal(_raw(out, w), orc.dijkstra(hg.rowptr, hg.colind, _w(hg, w), s))
    srv.close()
