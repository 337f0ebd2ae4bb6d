"""Schedule policy, CPU side: the FP64 MLP oracle against finite differences,
bfloat16 rounding, and the weight-file format (no GPU)."""
import os

import numpy as np
import pytest


def test_oracle_gradient_matches_finite_differences(orc):
    rng = np.random.default_rng(3)
    P = rng.normal(0, 0.2, 5955)
    X = rng.normal(size=(9, 24))
    T = np.c_[rng.normal(size=9), rng.uniform(6, 12, 9), rng.uniform(1, 8, 9)]
    _, g = orc.mlp_loss_grad(P, X, T)
    eps = 1e-6
    for i in rng.choice(5955, 60, replace=False):
        Pp, Pm = P.copy(), P.copy()
        Pp[i] += eps
        Pm[i] -= eps
        fd = (orc.mlp_loss_grad(Pp, X, T)[0] - orc.mlp_loss_grad(Pm, X, T)[0]) / (2 * eps)
        assert abs(fd - g[i]) < 1e-6 * (1 + abs(g[i]))
    # the forward used by the loss is the same function
    y = orc.mlp_forward(P, X)
    assert y.shape == (9, 3)


def test_bf16_round_ties_to_even(orc):
    x = np.array([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, -2.0 - 2 ** -7, 0.0, 1e-40], np.float32)
    got = orc.bf16_round(x)
    assert got[:5].tolist() == [1.0, 1.0, 1.015625, -2.0, 0.0]


def test_weight_file_round_trip(tmp_path, b2):
    from b200sssp import policy as pol
    rng = np.random.default_rng(1)
    P = rng.normal(size=5955).astype(np.float32)
    mu = rng.normal(size=24).astype(np.float32)
    sg = rng.uniform(0.5, 2, 24).astype(np.float32)
    path = os.path.join(tmp_path, "w.npz")
    pol.save_weights(path, P, mu, sg, note=np.int32(5))
    w = pol.load_weights(path)
    assert np.array_equal(w["params"], P) and np.array_equal(w["mu"], mu) and np.array_equal(w["sigma"], sg)
    assert int(w["format_version"]) == pol.FORMAT_VERSION and int(w["note"]) == 5
    bad = dict(w)
    bad["format_version"] = np.int32(99)
    np.savez(path, **bad)
    with pytest.raises(ValueError):
        pol.load_weights(path)
    with pytest.raises(ValueError):
        pol.save_weights(path, P[:-1], mu, sg)


def test_shipped_weights_load(b2):
    from b200sssp import policy as pol
    w = pol.load_weights()
    assert w["params"].dtype == np.float32 and np.isfinite(w["params"]).all()
    assert (w["sigma"] > 0).all()
    assert int(w["n_graphs"]) > 0


def test_label_rule():
    from b200sssp import policy as pol
    times = {(lm, fl, pl): 10.0 for lm in pol.SWEEP_LOG2 for fl in pol.FUSION_LOG2 for pl in pol.PULL_LOG2}
    for lm in (1.5, 2.0, 2.5):
        times[(lm, 10.0, 8.0)] = 5.0          # a flat optimum: x 2^2, fusion 1024, push only
    times[(-1.0, 6.0, 3.0)] = 5.05            # a sharp dip: its neighbours are slow
    y, best = pol.label_from_sweep(times)
    assert y.tolist() == [2.0, 10.0, 8.0] and best == 5.0
    for lm in (-1.5, -1.0, -0.5):
        times[(lm, 6.0, 3.0)] = 5.1           # now flat too and within 3 %: nearer the Near-Far delta
    y, _ = pol.label_from_sweep(times)
    assert y.tolist() == [-1.0, 6.0, 3.0]
    y, _ = pol.label_from_sweep(times, tol=0.0)
    assert y.tolist() == [2.0, 10.0, 8.0]


def test_decoding_matches_the_library_rule():
    """Outputs are log2 values: the multiplier is clamped and has a dead zone,
    fusion is off below 2^7, the heavy pass pushes only above 2^7."""
    from b200sssp import policy as pol
    d = pol.decode([0.3, 9.0, 2.0])
    assert d == {"delta_mult": pytest.approx(2 ** 0.3), "fusion_threshold": 512, "pull_fraction": 4.0}
    assert pol.decode([0.3, 9.0, 2.0], dead_zone=0.5)["delta_mult"] == 1.0
    d = pol.decode([99.0, 6.9, 7.1])
    assert d["delta_mult"] == 2.0 ** 6 and d["fusion_threshold"] == 0 and d["pull_fraction"] == 0.0
    d = pol.decode([-99.0, 30.0, -5.0])
    assert d["delta_mult"] == 2.0 ** -4 and d["fusion_threshold"] == 2 ** 14 and d["pull_fraction"] == 1.0
    L = len(pol.SWEEP_LOG2)
    assert pol.decision_index([99.0, 11.2, 2.1]) == (L - 1, 3, 1)
    assert pol.decision_index([0.1, 6.5, 7.5]) == (pol.SWEEP_LOG2.index(0.0), 0, 3)


def test_robust_label_prefers_flat_side():
    """A sharp minimum next to a cliff loses to a slightly slower flat region;
    the decision cost reads the chosen configuration off the sweep table."""
    from b200sssp import policy as pol
    L = len(pol.SWEEP_LOG2)
    A = np.full((L, 4, 4), 10.0)
    i0 = pol.SWEEP_LOG2.index(0.0)
    f0, p0 = pol.FIXED_INDEX[1], pol.FIXED_INDEX[2]
    A[i0 - 2, f0, p0] = 7.0          # sharp minimum at x 2^-1 ...
    A[i0 - 3, f0, p0] = 30.0         # ... next to a cliff
    A[i0 + 2: i0 + 5, f0, p0] = 8.0  # flat region at x 2^1 .. 2^2
    y = pol.robust_label(A)
    assert y.tolist() == [1.5, 6.0, 3.0]          # middle of the flat region
    assert pol.decision_speedup(A, y) == pytest.approx(10.0 / 8.0)
    assert pol.decision_speedup(A, [-1.0, 0.0, 3.2]) == pytest.approx(10.0 / 7.0)


def test_shipped_dataset_matches_weights():
    from b200sssp import policy as pol
    X, T, TT, info = pol.load_dataset(os.path.join(os.path.dirname(pol.DEFAULT_WEIGHTS), "policy_dataset.npz"))
    assert X.shape[0] == TT.shape[0] == len(info) > 0
    assert TT.shape[1:] == (len(pol.SWEEP_LOG2), len(pol.FUSION_LOG2), len(pol.PULL_LOG2))
    assert np.isfinite(TT).all() and (TT > 0).all()
    w = pol.load_weights()
    assert int(w["n_graphs"]) == X.shape[0]
