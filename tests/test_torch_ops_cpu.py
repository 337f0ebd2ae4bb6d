"""CPU: the torch.ops binding for the reference's pytorch_testing harness is
registered with the reference's argument lists and refuses non-CUDA tensors
(there is no CPU path)."""
import pytest
import torch


@pytest.fixture(scope="module")
def ops(b2):
    import b200sssp.torch_ops  # noqa: F401  (registers torch.ops.b200sssp.*)
    return torch.ops.b200sssp


def test_schemas(ops):
    bf = str(ops.sssp_min_plus_bellman_ford.default._schema)
    assert "Tensor rowptr, Tensor colind, Tensor values, SymInt source, SymInt max_iters=-1" in bf
    assert "(Tensor, Tensor, SymInt, bool, bool)" in bf
    bk = str(ops.bucketted_bellman_ford.default._schema)
    assert "Tensor rowptr, Tensor col, Tensor weight, SymInt source, SymInt num_nodes, float delta=1." in bk
    assert str(ops.min_plus_matmul.default._schema).endswith("(Tensor A, Tensor B) -> Tensor")


def test_cpu_tensors_are_refused(ops):
    rp = torch.tensor([0, 1, 1], dtype=torch.int64)
    ci = torch.tensor([1], dtype=torch.int32)
    w = torch.tensor([2.0])
    with pytest.raises(ValueError, match="CUDA"):
        ops.sssp_min_plus_bellman_ford(rp, ci, w, 0)
    with pytest.raises(ValueError, match="CUDA"):
        ops.bucketted_bellman_ford(rp, ci, w, 0, 2)
    with pytest.raises(ValueError, match="CUDA"):
        ops.min_plus_matmul(torch.zeros(2, 2), torch.zeros(2, 2))


def test_fake_kernels_follow_the_value_dtype(ops):
    """Under FakeTensorMode (torch.compile tracing) the distance dtype is the
    real op's: float32 for float32 weights, int32 for int32 weights."""
    from torch._subclasses.fake_tensor import FakeTensorMode
    with FakeTensorMode():
        rp = torch.empty(5, dtype=torch.int64)
        ci = torch.empty(4, dtype=torch.int32)
        for vdt, ddt in ((torch.float32, torch.float32), (torch.int32, torch.int32)):
            d, p, *_ = ops.sssp_min_plus_bellman_ford(rp, ci, torch.empty(4, dtype=vdt), 0)
            assert d.dtype == ddt and d.shape == (4,)
            assert p.dtype == torch.int64
