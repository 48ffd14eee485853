"""The PyTorch operator library loads without a GPU, registers every operator with its schema, and has no CPU
kernel: a call with host tensors fails in the dispatcher instead of falling back to the host."""
import pytest
import torch

from mbirjax_b200 import torch_ops


def test_operators_are_registered_with_schemas():
    ops = torch_ops.load()
    for name in torch_ops.OPS:
        op = getattr(ops, name)
        schema = str(op.default._schema)
        assert schema.startswith('mbirjax_b200::' + name + '(')
    assert 'Tensor(a!) flat_recon' in str(ops.vcd_subset_step.default._schema)


def test_no_cpu_kernel():
    ops = torch_ops.load()
    gi = [0, 4, 2, 8, 8, 8, 2, 1, 1, 128]
    gf = [1.0, 1.0, 0.0, 0.0, 1.0, 0.0, float('inf'), 1.0, 1.0, 0.0]
    with pytest.raises((RuntimeError, NotImplementedError)):
        ops.sparse_forward_project(gi, gf, torch.zeros(4), torch.zeros((3, 2)), torch.zeros(3, dtype=torch.int32))
