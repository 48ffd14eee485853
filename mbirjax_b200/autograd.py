"""torch.autograd wrappers of the projector pair and the qGGMRF prior.

``ForwardProject`` maps a full recon (Nr, Nc, S) to a sinogram (V, R, C) with the sparse forward projector over the
region of reconstruction; its backward is the matched adjoint kernel (the back projector), and vice versa for
``BackProject``.  The kernels compute every footprint coefficient on the fly per (view, pixel), so no footprint
table is ever stored, at any size; ``view_chunk`` additionally splits the backward pass into launches of that many
views (the reference has no autograd path: its JAX transpose helper ``get_transpose``,
``tomography_model.py:1834-1855``, is unused on the hot path).  ``QGGMRFLoss`` evaluates ``qggmrf_loss``
(``qggmrf.py:31-65``) and its hand-written gradient kernel in one launch.
"""
import numpy as np
import torch

from . import _capi
from .vcd_utils import get_2d_ror_mask


def _ror_indices(model, device):
    """Sorted flat indices of the region of reconstruction (no RNG draw), cached per model and device."""
    key = (tuple(model.get_params('recon_shape')), str(device))
    cache = getattr(model, '_ror_index_cache', None)
    if cache is None or cache[0] != key:
        recon_shape = model.get_params('recon_shape')
        idx = np.flatnonzero(get_2d_ror_mask(recon_shape).flatten()).astype(np.int32)
        model._ror_index_cache = (key, torch.as_tensor(idx, device=device))
    return model._ror_index_cache[1]


def _back_project_chunked(g, sino, idx, view_chunk):
    if not view_chunk or view_chunk >= g.num_views:
        return _capi.back_project(g, sino, idx)
    out = None
    for v0 in range(0, g.num_views, view_chunk):
        views = torch.arange(v0, min(v0 + view_chunk, g.num_views), dtype=torch.int32, device=sino.device)
        part = _capi.back_project(g, sino, idx, view_indices=views)
        out = part if out is None else out.add_(part)
    return out


class ForwardProject(torch.autograd.Function):
    """recon (Nr, Nc, S) -> A recon (V, R, C); backward = A^T."""

    @staticmethod
    def forward(ctx, recon, model, view_chunk=None):
        g = model._geometry()
        idx = _ror_indices(model, recon.device)
        nr, nc, ns = recon.shape
        vox = recon.detach().reshape(nr * nc, ns)[idx.long()].contiguous()
        ctx.model, ctx.view_chunk, ctx.shape = model, view_chunk, recon.shape
        return _capi.forward_project(g, vox, idx)

    @staticmethod
    def backward(ctx, grad_sino):
        model = ctx.model
        g = model._geometry()
        idx = _ror_indices(model, grad_sino.device)
        cyl = _back_project_chunked(g, grad_sino.contiguous(), idx, ctx.view_chunk)
        nr, nc, ns = ctx.shape
        out = torch.zeros((nr * nc, ns), dtype=torch.float32, device=grad_sino.device)
        out[idx.long()] = cyl
        return out.reshape(ctx.shape), None, None


class BackProject(torch.autograd.Function):
    """sinogram (V, R, C) -> A^T sinogram (Nr, Nc, S) (zero outside the ROR); backward = A."""

    @staticmethod
    def forward(ctx, sino, model):
        g = model._geometry()
        idx = _ror_indices(model, sino.device)
        nr, nc, ns = model.get_params('recon_shape')
        out = torch.zeros((nr * nc, ns), dtype=torch.float32, device=sino.device)
        out[idx.long()] = _capi.back_project(g, sino.detach().contiguous(), idx)
        ctx.model = model
        return out.reshape(nr, nc, ns)

    @staticmethod
    def backward(ctx, grad_recon):
        model = ctx.model
        g = model._geometry()
        idx = _ror_indices(model, grad_recon.device)
        nr, nc, ns = grad_recon.shape
        vox = grad_recon.reshape(nr * nc, ns)[idx.long()].contiguous()
        return _capi.forward_project(g, vox, idx), None


class QGGMRFLoss(torch.autograd.Function):
    """qGGMRF loss of a full recon; the gradient comes from the same kernel launch."""

    @staticmethod
    def forward(ctx, recon, qggmrf_params):
        b, sigma_x, p, q, T = qggmrf_params
        qp = _capi.qggmrf_params(b, sigma_x, p, q, T)
        loss, grad = _capi.qggmrf_loss_grad(recon.detach().contiguous(), qp, need_grad=recon.requires_grad)
        ctx.save_for_backward(grad if grad is not None else torch.empty(0))
        return loss.to(torch.float32)

    @staticmethod
    def backward(ctx, grad_out):
        (grad,) = ctx.saved_tensors
        return grad * grad_out, None


def forward_project(recon, model, view_chunk=None):
    return ForwardProject.apply(recon, model, view_chunk)


def back_project(sino, model):
    return BackProject.apply(sino, model)


def qggmrf_loss(recon, qggmrf_params):
    return QGGMRFLoss.apply(recon, qggmrf_params)


def weighted_ls_qggmrf_loss(recon, model, sinogram, weights, qggmrf_params, view_chunk=None):
    """0.5 * || W^(1/2) (A x - y) ||^2 + qGGMRF(x), summed in float64 (a float64 scalar)."""
    r = forward_project(recon, model, view_chunk) - sinogram
    data = 0.5 * torch.sum(weights * r * r if weights is not None else r * r, dtype=torch.float64)
    return data + qggmrf_loss(recon, qggmrf_params)


def projected_gradient_descent(model, sinogram, weights, qggmrf_params, init, steps, step_size, view_chunk=None):
    """Gradient descent on weighted_ls_qggmrf_loss with projection onto x >= 0 after every step."""
    x = init.detach().clone().requires_grad_(True)
    losses = []
    for _ in range(steps):
        loss = weighted_ls_qggmrf_loss(x, model, sinogram, weights, qggmrf_params, view_chunk)
        (g,) = torch.autograd.grad(loss, x)
        with torch.no_grad():
            x -= step_size * g
            x.clamp_(min=0.0)
        losses.append(loss.detach())
    return x.detach(), torch.stack(losses)
