"""GPU: torch.ops.b200sssp (the pytorch_testing harness binding) gives the
library's own results: Bellman-Ford words and stats, delta-stepping distances
equal to the oracle, min-plus products equal to the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ops(b2, cuda):
    import b200sssp.torch_ops  # noqa: F401
    return cuda.ops.b200sssp


def test_bellman_ford_op_matches_library(ops, b2, orc, cuda):
    hg = b2.gen_er(2000, 16000, 1, 100, seed=71)
    inc = hg.transpose()
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a)).cuda()
    dist, pred, iters, conv, negc = ops.sssp_min_plus_bellman_ford(
        t(inc.rowptr), t(inc.colind), t(inc.fweights.astype(np.float32)), 5)
    g = b2.Graph.from_host(hg, "f32")
    d2, p2, st = g.sssp(5, method="bf", pred=True, detect_negative_cycle=1)
    assert np.array_equal(dist.cpu().numpy(), d2.cpu().numpy())
    assert np.array_equal(pred.cpu().numpy(), p2.cpu().numpy().astype(np.int64))
    assert (iters, conv, negc) == (st["iterations_used"], bool(st["converged"]), bool(st["has_negative_cycle"]))
    assert np.array_equal(dist.cpu().numpy(), orc.dijkstra(hg.rowptr, hg.colind, hg.fweights.astype(np.float32), 5))
    g.close()


def test_bucketed_op_matches_oracle(ops, b2, orc, cuda):
    hg = b2.gen_er(3000, 24000, 1, 50, seed=72)
    w = hg.fweights.astype(np.float32)
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a)).cuda()
    d = ops.bucketted_bellman_ford(t(hg.rowptr), t(hg.colind.astype(np.int64)), t(w), 0, hg.n, 0.05)
    assert np.array_equal(d.cpu().numpy(), orc.dijkstra(hg.rowptr, hg.colind, w, 0))


def test_min_plus_matmul_op_matches_oracle(ops, orc, cuda):
    rng = np.random.default_rng(73)
    A = rng.uniform(0, 1, (300, 200)).astype(np.float32)
    B = rng.uniform(0, 1, (200, 250)).astype(np.float32)
    A[rng.random(A.shape) < 0.5] = np.inf
    C = ops.min_plus_matmul(cuda.from_numpy(A).cuda(), cuda.from_numpy(B).cuda())
    assert np.array_equal(C.cpu().numpy(), orc.minplus_gemm(A, B))


def test_bellman_ford_op_int32_weights(ops, b2, orc, cuda):
    """int32 weights are solved exactly (int32 distances); a negative int32
    weight is refused, and the same negative weights as float32 go through the
    reference's negative-weight rules, negative-cycle flag included."""
    hg = b2.gen_er(1500, 12000, 1, 100, seed=74)
    inc = hg.transpose()
    t = lambda a: cuda.from_numpy(np.ascontiguousarray(a)).cuda()
    wi = inc.weights.view(np.int32)
    dist, pred, iters, conv, negc = ops.sssp_min_plus_bellman_ford(t(inc.rowptr), t(inc.colind), t(wi), 3)
    assert dist.dtype == cuda.int32
    assert np.array_equal(dist.cpu().numpy().view(np.uint32), orc.dijkstra(hg.rowptr, hg.colind, hg.weights, 3))
    assert conv and not negc
    bad = wi.copy()
    bad[5] = -3
    with pytest.raises(ValueError, match="negative int32"):
        ops.sssp_min_plus_bellman_ford(t(inc.rowptr), t(inc.colind), t(bad), 3)
    # incoming CSR of 0->1 (1), 2->1 (1), 1->2 (-2): the cycle 1->2->1 weighs -1
    rp = np.array([0, 0, 2, 3], np.int64)
    ci = np.array([0, 2, 1], np.int32)
    wf = np.array([1.0, 1.0, -2.0], np.float32)
    dist, pred, iters, conv, negc = ops.sssp_min_plus_bellman_ford(t(rp), t(ci), t(wf), 0)
    assert dist.dtype == cuda.float32 and negc and not conv
