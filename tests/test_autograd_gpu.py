"""Autograd: the gradient of 0.5 ||W^(1/2)(A x - y)||^2 + qGGMRF(x) through the projector autograd pair and the
qGGMRF loss kernel, checked against central finite differences of the float64 oracle at 64 random voxels
(eps = 1e-3), plus projected gradient descent."""
import numpy as np
import pytest
import torch

import mbirjax_b200 as mb
from mbirjax_b200 import autograd as AG
import oracle as O
from cases import make_case

pytestmark = pytest.mark.gpu


def _oracle_loss(geom, x, y, w, params):
    np.random.seed(0)
    ax = O.forward_project(geom, x, dtype=np.float64)
    r = ax - y
    return 0.5 * float(np.sum(w * r * r)) + O.qggmrf_loss(x, params)


def test_gradient_matches_central_differences(cuda):
    model, geom = make_case('cone', views=16, rows=8, channels=32)
    nr, nc, ns = geom.recon_shape
    rng = np.random.default_rng(0)
    mask = O.get_2d_ror_mask(geom.recon_shape)[:, :, None]
    x = (rng.random(geom.recon_shape) * mask).astype(np.float64)
    np.random.seed(0)
    y = O.forward_project(geom, (x * 0.8 + 0.1 * mask).astype(np.float32), dtype=np.float64)
    w = np.exp(-y / y.max())
    params = (O.get_b_from_nbr_wts([1, 1, 1]), 0.3, 2.0, 1.2, 1.0)

    xt = torch.tensor(x, dtype=torch.float32, device='cuda', requires_grad=True)
    loss = AG.weighted_ls_qggmrf_loss(xt, model, torch.tensor(y, dtype=torch.float32, device='cuda'),
                                      torch.tensor(w, dtype=torch.float32, device='cuda'), params)
    (grad,) = torch.autograd.grad(loss, xt)
    grad = grad.cpu().numpy()
    assert float(loss) == pytest.approx(_oracle_loss(geom, x.astype(np.float32).astype(np.float64), y, w, params),
                                        rel=1e-4)

    ror = np.argwhere(np.broadcast_to(mask, geom.recon_shape))
    picks = ror[rng.choice(len(ror), 64, replace=False)]
    eps = 1e-3
    fd = []
    for i, j, k in picks:
        xp, xm = x.copy(), x.copy()
        xp[i, j, k] += eps
        xm[i, j, k] -= eps
        fd.append((_oracle_loss(geom, xp, y, w, params) - _oracle_loss(geom, xm, y, w, params)) / (2 * eps))
    fd = np.array(fd)
    ag = np.array([grad[i, j, k] for i, j, k in picks])
    assert np.linalg.norm(ag - fd) <= 1e-3 * np.linalg.norm(fd)


def test_projector_pair_is_adjoint_under_autograd(cuda):
    model, geom = make_case('parallel', views=12, rows=6, channels=24)
    x = torch.rand(geom.recon_shape, device='cuda', requires_grad=True)
    y = torch.rand(geom.sinogram_shape, device='cuda')
    ax = AG.forward_project(x, model)
    (gx,) = torch.autograd.grad(torch.sum(ax * y), x)
    # d<Ax, y>/dx = A^T y on the region of reconstruction
    aty = AG.back_project(y, model)
    torch.testing.assert_close(gx, aty, rtol=1e-5, atol=1e-5)
    # view-chunked backward gives the same gradient
    ax2 = AG.forward_project(x, model, 5)
    (gx2,) = torch.autograd.grad(torch.sum(ax2 * y), x)
    torch.testing.assert_close(gx2, gx, rtol=1e-5, atol=1e-5)


def test_projected_gradient_descent_decreases_loss(cuda):
    model, geom = make_case('cone', views=24, rows=8, channels=32)
    from mbirjax_b200.utilities import gen_ellipsoid_phantom
    ph = gen_ellipsoid_phantom(geom.recon_shape, 4, 1, device='cuda')
    y = AG.forward_project(ph, model).detach()
    w = torch.exp(-y / y.max())
    params = (mb.get_b_from_nbr_wts([1, 1, 1]), 0.5, 2.0, 1.2, 1.0)
    v = torch.rand_like(ph)
    for _ in range(15):  # power iteration for the Lipschitz constant of A^T W A
        v = AG.back_project(w * AG.forward_project(v, model), model)
        lip = float(torch.linalg.norm(v))
        v = v / lip
    x, losses = AG.projected_gradient_descent(model, y, w, params, torch.zeros_like(ph), steps=30,
                                              step_size=1.0 / (1.1 * lip))
    assert float(x.min()) >= 0.0
    assert float(losses[-1]) < 0.5 * float(losses[0])
