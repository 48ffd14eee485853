"""A stand-in for the CUDA library, for CPU tests of the host logic only.

The models' host code (parameters, partitions and their np.random draws, the VCD iteration loop, its statistics
and stopping rule, auto-regularisation, the per-view plugin functions) runs unchanged, on host tensors, while
each library call it makes (``_capi.forward_project``, ``back_project``, ``direct_filter``, ``vcd_subset_step``,
``qggmrf_denoise_step``, ``qggmrf_loss_grad``) is answered by the oracle.  The geometry record is read the way
the library reads it, angle or translation pointer included, so a wrong record shows up as a wrong result.

This is test infrastructure: the product keeps failing loudly without a GPU (``test_compute_without_gpu_fails_
loudly``), and the fixture below patches the package only for the test that requests it.
"""
import ctypes
import math

import numpy as np
import pytest
import torch

import oracle as O
from oracle import denoise as OD

_KINDS = {0: 'parallel', 1: 'cone', 2: 'translation'}


def oracle_geometry_of(g):
    """The OracleGeometry a mbx_geom record describes, its per-view parameters read from the record's pointer."""
    kind = _KINDS[g.kind]
    v = g.num_views
    if kind == 'translation':
        views = np.ctypeslib.as_array((ctypes.c_float * (3 * v)).from_address(g.translations)).reshape(v, 3).copy()
    else:
        views = np.ctypeslib.as_array((ctypes.c_float * v).from_address(g.angles)).copy()
    sdd, mag = g.source_detector_dist, g.magnification
    og = O.OracleGeometry(kind, (v, g.num_det_rows, g.num_det_channels),
                          (g.num_recon_rows, g.num_recon_cols, g.num_recon_slices), views, g.delta_det_channel,
                          g.delta_det_row, g.det_channel_offset, g.det_row_offset, g.delta_voxel,
                          g.recon_slice_offset, sdd, sdd / mag if math.isfinite(sdd) else math.inf, mag,
                          g.psf_radius, g.bp_psf_radius, g.entries_per_cylinder_batch)
    og.delta_recon_row = g.delta_recon_row
    return og


def _np(t):
    return None if t is None else t.detach().numpy()


def _qggmrf(qp):
    return np.array(list(qp.b), dtype=np.float32), qp.sigma_x, qp.p, qp.q, qp.T


def forward_project(geom, voxel_values, pixel_indices, view_indices=None, out=None):
    og = oracle_geometry_of(geom)
    return torch.as_tensor(O.sparse_forward_project(og, _np(voxel_values), _np(pixel_indices), _np(view_indices)))


def back_project(geom, sinogram, pixel_indices, view_indices=None, coeff_power=1, weights=None, scale=1.0, out=None):
    og = oracle_geometry_of(geom)
    if sinogram is None:  # the library's convention: the weights, or ones when there are none either
        sinogram = torch.ones(og.sinogram_shape, dtype=torch.float32) if weights is None else weights
        weights = None
    sino = _np(sinogram) if weights is None else _np(weights * sinogram)
    res = O.sparse_back_project(og, sino, _np(pixel_indices), _np(view_indices), coeff_power=coeff_power)
    return torch.as_tensor(np.float32(scale) * res if scale != 1.0 else res)


def direct_filter(geom, sinogram, out=None):
    og = oracle_geometry_of(geom)
    s = _np(sinogram)
    if og.kind == 'parallel':
        return torch.as_tensor(O.fbp_filter(s, og.delta_voxel))
    return torch.as_tensor(O.fdk_filter(s, og.source_detector_dist, og.magnification, og.delta_voxel,
                                        og.delta_det_row, og.delta_det_channel, og.det_row_offset,
                                        og.det_channel_offset))


def vcd_subset_step(geom, flat_recon, error_sinogram, weights, fm_hessian, pixel_indices, fm_constant, qp, stats,
                    workspace=None, prox_input=None, sigma_prox=0.0, positivity=False):
    og = oracle_geometry_of(geom)
    r, e, ell1, alpha = O.vcd_subset_update(og, _np(flat_recon), _np(error_sinogram), _np(weights), _np(fm_hessian),
                                            _np(pixel_indices), fm_constant, _qggmrf(qp), prox_input=_np(prox_input),
                                            sigma_prox=sigma_prox, positivity=positivity)
    flat_recon.copy_(torch.as_tensor(r))
    error_sinogram.copy_(torch.as_tensor(e))
    stats[0], stats[1] = alpha, ell1


def qggmrf_denoise_step(flat_image, flat_error_image, image_shape, pixel_indices, fm_constant, qp, stats,
                        workspace=None):
    im, er, ell1, alpha = OD.vcd_subset_denoiser(_np(flat_image), _np(flat_error_image), _np(pixel_indices),
                                                 fm_constant, _qggmrf(qp), tuple(image_shape))
    flat_image.copy_(torch.as_tensor(im))
    flat_error_image.copy_(torch.as_tensor(er))
    stats[0], stats[1] = alpha, ell1


def qggmrf_loss_grad(recon, qp, need_grad=True):
    x = _np(recon)
    loss = torch.tensor(O.qggmrf_loss(x, _qggmrf(qp)), dtype=torch.float64)
    return loss, (torch.as_tensor(O.qggmrf_loss_grad(x, _qggmrf(qp))) if need_grad else None)


@pytest.fixture
def oracle_library(monkeypatch):
    """Run the models on the host with the oracle answering their library calls (see the module docstring)."""
    import mbirjax_b200.tomography_model as tm
    from mbirjax_b200 import _capi
    monkeypatch.setattr(tm, '_cuda_device', lambda: torch.device('cpu'))
    for name, fn in (('forward_project', forward_project), ('back_project', back_project),
                     ('direct_filter', direct_filter), ('vcd_subset_step', vcd_subset_step),
                     ('qggmrf_denoise_step', qggmrf_denoise_step), ('qggmrf_loss_grad', qggmrf_loss_grad)):
        monkeypatch.setattr(_capi, name, fn)
    monkeypatch.setattr(_capi, 'vcd_subset_step_workspace', lambda geom, n, device: (None, 0))
    monkeypatch.setattr(_capi, '_workspace', lambda nbytes, device: (None, int(nbytes)))
    return _capi
