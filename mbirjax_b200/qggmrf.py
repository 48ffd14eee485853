"""qGGMRF prior: the reference's functions on the mbirjax_b200 kernels.

* ``get_b_from_nbr_wts`` (host): ``qggmrf.py:388-395``
* ``qggmrf_gradient_and_hessian_at_indices``: ``qggmrf.py:118-148`` -> ``mbx_qggmrf_grad_hess``
* ``qggmrf_loss`` / ``qggmrf_loss_and_grad``: ``qggmrf.py:31-65`` -> ``mbx_qggmrf_loss_grad``
"""
import numpy as np
import torch

from . import _capi


def get_b_from_nbr_wts(qggmrf_nbr_wts):
    """[row, col, slice] weights -> 6 normalised directional weights [row+1, row-1, col+1, col-1, slice+1, slice-1]."""
    b = np.array([qggmrf_nbr_wts, qggmrf_nbr_wts]).T.flatten()
    b = b / np.sum(b)
    return tuple(float(v) for v in b)


def _as_cuda(x, dtype):
    if isinstance(x, torch.Tensor):
        return x.to(device='cuda', dtype=dtype).contiguous()
    return torch.as_tensor(np.ascontiguousarray(x), device='cuda').to(dtype).contiguous()


def qggmrf_gradient_and_hessian_at_indices(flat_recon, recon_shape, pixel_indices, qggmrf_params):
    """Surrogate gradient and Hessian diagonal, each (len(pixel_indices), num_slices)."""
    b, sigma_x, p, q, T = qggmrf_params
    qp = _capi.qggmrf_params(b, sigma_x, p, q, T)
    return _capi.qggmrf_grad_hess(_as_cuda(flat_recon, torch.float32), recon_shape,
                                  _as_cuda(pixel_indices, torch.int32), qp)


def qggmrf_loss_and_grad(full_recon, qggmrf_params, need_grad=True):
    """(loss as a float64 device scalar, gradient (Nr, Nc, S) or None)."""
    b, sigma_x, p, q, T = qggmrf_params
    qp = _capi.qggmrf_params(b, sigma_x, p, q, T)
    return _capi.qggmrf_loss_grad(_as_cuda(full_recon, torch.float32), qp, need_grad=need_grad)


def qggmrf_loss(full_recon, qggmrf_params):
    loss, _ = qggmrf_loss_and_grad(full_recon, qggmrf_params, need_grad=False)
    return float(loss)
