"""The PyTorch dispatcher operators against the ctypes path over the same C entry points (the same kernels on the
same stream, so the results are bitwise equal), and their argument checks."""
import numpy as np
import pytest
import torch

from mbirjax_b200 import _capi, torch_ops
from cases import make_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_operators_match_the_ctypes_path(cuda, kind):
    ops = torch_ops.load()
    model, geom = make_case(kind, views=16, rows=8, channels=32)
    nr, nc, ns = geom.recon_shape
    gi, gf, views = torch_ops.geometry_args(model)
    g = model._geometry()
    rng = np.random.default_rng(0)
    idx = torch.as_tensor(np.sort(rng.choice(nr * nc, nr * nc // 2, replace=False)).astype(np.int32), device='cuda')
    vox = torch.as_tensor(rng.random((int(idx.shape[0]), ns), dtype=np.float32), device='cuda')
    sino = torch.as_tensor(rng.random(geom.sinogram_shape, dtype=np.float32), device='cuda')
    w = torch.as_tensor(rng.random(geom.sinogram_shape, dtype=np.float32), device='cuda')
    sel = torch.as_tensor([3, 0, 7], dtype=torch.int32, device='cuda')

    assert torch.equal(ops.sparse_forward_project(gi, gf, views, vox, idx), _capi.forward_project(g, vox, idx))
    assert torch.equal(ops.sparse_forward_project(gi, gf, views, vox, idx, sel),
                       _capi.forward_project(g, vox, idx, view_indices=sel))
    assert torch.equal(ops.sparse_back_project(gi, gf, views, sino, idx, None, 2, w, 0.5),
                       _capi.back_project(g, sino, idx, coeff_power=2, weights=w, scale=0.5))
    assert torch.equal(ops.sparse_back_project(gi, gf, views, None, idx, coeff_power=2),
                       _capi.back_project(g, None, idx, coeff_power=2))
    if kind != 'translation':
        assert torch.equal(ops.direct_filter(gi, gf, views, sino), _capi.direct_filter(g, sino))

    params = (np.array([1, 1, 1, 1, 1, 1], dtype=np.float32) / 6, 0.2, 2.0, 1.2, 1.0)
    qa = torch_ops.qparams_args(*params)
    flat = torch.as_tensor(rng.random((nr * nc, ns), dtype=np.float32), device='cuda')
    gh = ops.qggmrf_grad_hess(flat, [nr, nc, ns], idx, qa)
    ref = _capi.qggmrf_grad_hess(flat, (nr, nc, ns), idx, _capi.qggmrf_params(*params))
    assert torch.equal(gh[0], ref[0]) and torch.equal(gh[1], ref[1])
    loss, grad = ops.qggmrf_loss_grad(flat.reshape(nr, nc, ns), qa)
    loss_ref, grad_ref = _capi.qggmrf_loss_grad(flat.reshape(nr, nc, ns), _capi.qggmrf_params(*params))
    assert float(loss) == float(loss_ref) and torch.equal(grad, grad_ref)

    hess = torch.as_tensor(rng.random((nr * nc, ns), dtype=np.float32) + 1.0, device='cuda')
    f1, e1 = flat.clone(), sino.clone()
    f2, e2 = flat.clone(), sino.clone()
    s1 = torch.zeros(4, dtype=torch.float64, device='cuda')
    s2 = torch.zeros(4, dtype=torch.float64, device='cuda')
    ops.vcd_subset_step(gi, gf, views, f1, e1, w, hess, idx, 50.0, qa, s1)
    _capi.vcd_subset_step(g, f2, e2, w, hess, idx, 50.0, _capi.qggmrf_params(*params), s2)
    assert torch.equal(f1, f2) and torch.equal(e1, e2) and torch.equal(s1, s2)


def test_operators_check_their_arguments(cuda):
    ops = torch_ops.load()
    model, geom = make_case('parallel', views=8, rows=4, channels=16)
    gi, gf, views = torch_ops.geometry_args(model)
    nr, nc, ns = geom.recon_shape
    idx = torch.arange(10, dtype=torch.int32, device='cuda')
    with pytest.raises(RuntimeError, match='voxel_values must be Float'):
        ops.sparse_forward_project(gi, gf, views, torch.zeros((10, ns), dtype=torch.float64, device='cuda'), idx)
    with pytest.raises(RuntimeError, match='must be contiguous'):
        ops.sparse_forward_project(gi, gf, views, torch.zeros((ns, 10), device='cuda').t(), idx)
    with pytest.raises(RuntimeError, match='shape'):
        ops.sparse_forward_project(gi, gf, views, torch.zeros((11, ns), device='cuda'), idx)
    with pytest.raises(RuntimeError, match='pixel_indices must be Int'):
        ops.sparse_back_project(gi, gf, views, None, idx.long())
