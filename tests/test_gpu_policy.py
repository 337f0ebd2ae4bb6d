"""GPU: the schedule-policy MLP kernels against the FP64 oracle, training,
and the learned schedule in the solve path (distances unchanged)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pol(b2, cuda):
    from b200sssp import policy
    yield policy
    policy.Policy.deactivate()


def _bf16_params(P, orc):
    return orc.bf16_round(P).astype(np.float64)


def test_forward_matches_fp64_oracle(pol, orc):
    p = pol.Policy(seed=11)
    P, mu, sg = p.params()
    rng = np.random.default_rng(0)
    X = rng.normal(size=(37, 24)).astype(np.float32)
    Y = p.forward(X)
    Xn = (X.astype(np.float64) - mu) / sg
    ref = orc.mlp_forward(_bf16_params(P, orc), Xn)
    assert np.allclose(Y, ref, rtol=1e-4, atol=1e-4)     # FP32 accumulation vs FP64


def test_features_past_the_training_range_are_clamped(pol, orc):
    """Raw features outside the range set by training (or from the weight file)
    score like the nearest in-range features; clearing the range restores plain
    normalization."""
    p = pol.Policy(seed=5)
    rng = np.random.default_rng(1)
    X = rng.normal(size=(64, 24)).astype(np.float32)
    T = rng.normal(size=(64, 3)).astype(np.float32)
    p.train(X, T, epochs=5)                          # first training call sets the range from X
    lo, hi = X.min(axis=0), X.max(axis=0)
    Xo = (X[:8] * 4.0).astype(np.float32)            # mostly past the range
    assert np.array_equal(p.forward(Xo), p.forward(np.clip(Xo, lo, hi)))
    p.set_feature_range(None, None)
    P, mu, sg = p.params()
    ref = orc.mlp_forward(_bf16_params(P, orc), (Xo.astype(np.float64) - mu) / sg)
    assert np.allclose(p.forward(Xo), ref, rtol=1e-4, atol=1e-4)
    p.set_feature_range(lo, hi)
    assert np.array_equal(p.forward(Xo), p.forward(np.clip(Xo, lo, hi)))
    p.close()


def test_gradient_matches_fp64_oracle(pol, orc):
    p = pol.Policy(seed=5)
    rng = np.random.default_rng(1)
    X = rng.normal(size=(50, 24)).astype(np.float32)
    T = np.c_[rng.normal(size=50), rng.uniform(6, 12, 50), rng.uniform(1, 8, 50)].astype(np.float32)
    # non-trivial normalization
    P, _, _ = p.params()
    mu = rng.normal(size=24).astype(np.float32)
    sg = rng.uniform(0.5, 2.0, 24).astype(np.float32)
    p.set_params(P, mu, sg)
    G, loss = p.gradient(X, T)
    Xn = (X.astype(np.float64) - mu.astype(np.float64)) / sg.astype(np.float64)
    ref_loss, ref = orc.mlp_loss_grad(_bf16_params(P, orc), Xn, T)
    assert abs(loss - ref_loss) <= 1e-4 * max(1.0, abs(ref_loss))
    scale = np.abs(ref).max()
    assert np.abs(G - ref).max() <= 1e-4 * scale
    assert np.linalg.norm(G - ref) <= 1e-4 * np.linalg.norm(ref)


def test_training_is_deterministic_and_fits(pol):
    rng = np.random.default_rng(2)
    X = rng.normal(size=(64, 24)).astype(np.float32)
    w = rng.normal(size=24)
    T = np.c_[np.tanh(X @ w / 5) * 3, np.where(X[:, 0] > 0, 10.0, 6.0), np.where(X[:, 1] < 0, 8.0, 3.0)]
    T = T.astype(np.float32)
    a, b = pol.Policy(seed=3), pol.Policy(seed=3)
    la = a.train(X, T, epochs=600, lr=3e-3)
    lb = b.train(X, T, epochs=600, lr=3e-3)
    assert la == lb
    assert np.array_equal(a.params()[0], b.params()[0])
    _, l0 = pol.Policy(seed=3).gradient(X, T)
    assert la < 0.25 * l0
    Y = a.forward(X)
    assert ((Y[:, 1] > 8.0) == (T[:, 1] > 8.0)).mean() > 0.9


def _raw(d, weight):
    a = d.cpu().numpy()
    return a.view(np.uint32) if weight == "u32" else a


def _set_constant(p, y):
    """All weights zero, output biases = y: the policy outputs y for every graph."""
    P = np.zeros(5955, np.float32)
    P[-3:] = y
    p.set_params(P, np.zeros(24, np.float32), np.ones(24, np.float32))


@pytest.mark.parametrize("weight", ["u32", "f32"])
def test_policy_sets_schedule_and_keeps_distances(pol, b2, orc, cuda, weight):
    hg = b2.gen_rmat(14, 8, seed=4)
    g = b2.Graph.from_host(hg, weight)
    nf = g.delta_heuristic()
    w = hg.weights if weight == "u32" else hg.fweights
    ref = orc.dijkstra(hg.rowptr, hg.colind, w, 3)
    p = pol.Policy()
    _set_constant(p, [2.0, 6.0, 3.0])             # delta x4, fusion off, pull past 8 n heavy edges
    p.activate()
    d, _, st = g.sssp(3, policy=1)
    assert st["policy_used"] == 1
    want = max(1.0, np.floor(nf * 4.0)) if weight == "u32" else nf * 4.0
    assert st["delta_used"] == pytest.approx(want, rel=1e-12)
    assert np.array_equal(_raw(d, weight), ref)
    _set_constant(p, [-9.0, 10.0, 7.5])            # clamped to /16, fusion threshold 1024, push only
    d2, _, st2 = g.sssp(3, policy=1, trace=1)
    assert st2["policy_used"] == 1
    want = max(1.0, np.floor(nf / 16.0)) if weight == "u32" else nf / 16.0
    assert st2["delta_used"] == pytest.approx(want, rel=1e-12)
    assert st2["heavy_pulls"] == 0
    assert not any(t["kind"].startswith("pull") for t in g.trace())
    assert np.array_equal(_raw(d2, weight), ref)
    pol.Policy.deactivate()                        # no active policy: Near-Far fallback
    d3, _, st3 = g.sssp(3, policy=1)
    assert st3["policy_used"] == 0 and st3["delta_used"] == pytest.approx(
        max(1.0, np.floor(nf)) if weight == "u32" else nf, rel=1e-12)
    assert np.array_equal(_raw(d3, weight), ref)


def test_features_are_cached_and_sane(pol, b2, cuda):
    hg = b2.gen_grid(64, 64, 0.0, 5.0, 1.0, seed=2)
    g = b2.Graph.from_host(hg)
    f = pol.graph_features(g)
    assert f.shape == (24,) and np.isfinite(f).all()
    assert f[0] == pytest.approx(12.0)               # log2 n
    assert f[17] > np.log2(1 + 60)                   # hop depth of a 64 x 64 grid
    assert np.array_equal(f, pol.graph_features(g))


def test_shipped_policy_keeps_distances(pol, b2, orc, cuda):
    """The shipped weights pick the schedule of graphs inside their training
    range (2^14 - 2^22 vertices) and leave graphs outside it on the fixed
    Near-Far schedule; distances and predecessor trees are exact either way."""
    p = pol.activate_default()
    for hg, weight, s, inside in [(b2.gen_rmat(15, 16, seed=9), "u32", 1, True),
                                  (b2.gen_grid(150, 140, 0.02, seed=3), "f32", 5, True),
                                  (b2.gen_er(20000, 160000, 1, 1000, seed=1), "u32", 0, True),
                                  (b2.gen_er(2000, 16000, 1, 1000, seed=2), "u32", 0, False)]:
        g = b2.Graph.from_host(hg, weight)
        w = hg.weights if weight == "u32" else hg.fweights
        ref = orc.dijkstra(hg.rowptr, hg.colind, w, s)
        for method in ("delta", "adds"):
            d, pr, st = g.sssp(s, method=method, policy=1, pred=True)
            assert st["policy_used"] == (1 if inside else 0), (hg.n, method)
            got = _raw(d, weight)
            assert np.array_equal(got, ref)
            assert orc.validate_spt(hg.rowptr, hg.colind, w, s, got, pr.cpu().numpy()) == 0
        g.close()
    p.deactivate()


def test_dead_zone_keeps_near_far_delta(pol, b2, cuda):
    """A predicted change of delta inside the dead zone is ignored: the solve
    uses the Near-Far delta; outside it the multiplier applies."""
    hg = b2.gen_rmat(13, 8, seed=6)
    g = b2.Graph.from_host(hg, "f32")
    nf = g.delta_heuristic()
    p = pol.Policy()
    _set_constant(p, [0.375, 6.0, 3.0])             # (exact in bfloat16)
    p.set_dead_zone(0.5)
    p.activate()
    _, _, st = g.sssp(0, policy=1)
    assert st["policy_used"] == 1 and st["delta_used"] == pytest.approx(nf, rel=1e-12)
    p.set_dead_zone(0.25)
    _, _, st = g.sssp(0, policy=1)
    assert st["delta_used"] == pytest.approx(nf * 2.0 ** 0.375, rel=1e-6)
    assert p.decide(pol.graph_features(g))["delta_mult"] == pytest.approx(2.0 ** 0.375, rel=1e-6)
    pol.Policy.deactivate()
    g.close()


def test_trained_policy_gains_on_held_out_graphs(pol, b2, orc, cuda):
    """What the trained network gains over the method without it.  A policy is
    trained with the library's own kernels on 80 % of the shipped sweep
    dataset and decides for the held-out 20 %: the time of each decision, read
    off that graph's measured sweep table, beats the fixed Near-Far schedule
    in geometric mean.  Live solves with the decisions on regenerated
    held-out graphs give the fixed schedule's distances word for word."""
    import os
    X, _, TT, info = pol.load_dataset(os.path.join(os.path.dirname(pol.DEFAULT_WEIGHTS), "policy_dataset.npz"))
    idx = np.random.default_rng(11).permutation(len(X))
    test, train = idx[: len(X) // 5], idx[len(X) // 5:]
    T = np.array([pol.robust_label(a, 0.03) for a in TT], np.float32)
    p = pol.Policy(seed=11)
    p.train(X[train], T[train], epochs=800, lr=3e-3, weight_decay=1e-2)
    Y = p.forward(X[test])
    sp = np.array([pol.decision_speedup(TT[i], y) for i, y in zip(test, Y)])
    gain = float(np.exp(np.log(sp).mean()))
    best = float(np.exp(np.log([TT[i][pol.FIXED_INDEX] / TT[i].min() for i in test]).mean()))
    assert gain > 1.0, (gain, best)
    # live: the decisions change the schedule, never the distances
    p.activate()
    small = [i for i in test if info[i]["n"] <= (1 << 16)][:4]
    for i in small:
        hg, w, wtype, _ = pol.training_graph(int(info[i]["index"]))
        g = b2.Graph.from_arrays(hg.rowptr, hg.colind, w, weight=wtype)
        s = int(np.flatnonzero(np.diff(hg.rowptr))[0])
        d0, _, _ = g.sssp(s)
        d1, _, st = g.sssp(s, policy=1)
        assert st["policy_used"] == 1
        assert np.array_equal(d0.cpu().numpy().view(np.uint32), d1.cpu().numpy().view(np.uint32))
        g.close()
    pol.Policy.deactivate()
    p.close()
