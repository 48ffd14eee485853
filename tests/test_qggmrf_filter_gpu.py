"""GPU parity of the qGGMRF kernels (golden vectors of the reference's tests/test_qggmrf.py:81-134, finite
differences) and of the FBP/FDK filter against the oracle."""
import json
import os

import numpy as np
import pytest
import torch

import mbirjax_b200 as mb
from mbirjax_b200 import _capi
import oracle as O
from cases import make_case, rel_l2

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'qggmrf_golden.json')


def test_qggmrf_golden_vectors_on_gpu(cuda):
    g = json.load(open(GOLDEN))
    params = (mb.get_b_from_nbr_wts([1, 1, 1]), g['sigma_x'], g['p'], g['q'], g['T'])
    flat = np.array(g['flat_recon'], dtype=np.float32)
    grad, hess = mb.qggmrf_gradient_and_hessian_at_indices(flat, tuple(g['recon_shape']), np.arange(9), params)
    assert np.allclose(grad.cpu().numpy(), g['grad_ref'])      # np.allclose defaults, as the reference test
    assert np.allclose(hess.cpu().numpy(), g['hess_ref'])


@pytest.mark.parametrize('p,q', [(2.0, 1.2), (1.6, 1.1)])
def test_qggmrf_grad_hess_matches_oracle(cuda, p, q):
    shape = (23, 17, 9)
    rng = np.random.default_rng(4)
    x = rng.random(shape).astype(np.float32)
    flat = x.reshape(-1, shape[2])
    idx = rng.permutation(shape[0] * shape[1])[:150].astype(np.int32)
    params = (mb.get_b_from_nbr_wts([1.0, 0.7, 1.3]), 0.3, p, q, 1.0)
    g_gpu, h_gpu = mb.qggmrf_gradient_and_hessian_at_indices(flat, shape, idx, params)
    g_ref, h_ref = O.qggmrf_gradient_and_hessian_at_indices(flat, shape, idx, params)
    assert rel_l2(g_gpu.cpu().numpy(), g_ref) <= 1e-5
    assert rel_l2(h_gpu.cpu().numpy(), h_ref) <= 1e-5


def test_qggmrf_loss_and_gradient(cuda):
    shape = (11, 13, 7)
    rng = np.random.default_rng(5)
    x = rng.random(shape).astype(np.float32)
    params = (mb.get_b_from_nbr_wts([1, 1, 1]), 0.25, 2.0, 1.2, 1.0)
    loss, grad = mb.qggmrf_loss_and_grad(x, params)
    assert float(loss) == pytest.approx(O.qggmrf_loss(x, params), rel=1e-5)
    assert rel_l2(grad.cpu().numpy(), O.qggmrf_loss_grad(x, params)) <= 1e-5


@pytest.mark.parametrize('kind,kw', [('parallel', {}), ('cone', {}), ('cone', {'sid_factor': 2.0})])
def test_direct_filter_matches_oracle(cuda, kind, kw):
    model, geom = make_case(kind, views=10, rows=6, channels=37, **kw)
    sino = np.random.default_rng(6).random(geom.sinogram_shape).astype(np.float32)
    out = model.direct_filter(sino).cpu().numpy()
    if kind == 'parallel':
        ref = O.fbp_filter(sino, geom.delta_voxel)
    else:
        ref = O.fdk_filter(sino, geom.source_detector_dist, geom.magnification, geom.delta_voxel, geom.delta_det_row,
                           geom.delta_det_channel, geom.det_row_offset, geom.det_channel_offset)
    assert rel_l2(out, ref) <= 1e-5


@pytest.mark.parametrize('kind', ['parallel', 'cone'])
def test_direct_recon_of_phantom(cuda, kind):
    # tests/test_fbp_fdk.py in miniature: FBP/FDK of a forward projection recovers a block phantom
    model, geom = make_case(kind, views=96, rows=8, channels=64)
    nr, nc, ns = geom.recon_shape
    ph = np.zeros(geom.recon_shape, dtype=np.float32)
    ph[nr // 3:2 * nr // 3, nc // 3:2 * nc // 3, :] = 1.0
    sino = model.forward_project(ph)
    rec = model.direct_recon(sino).cpu().numpy()
    inner = (slice(nr // 3 + 3, 2 * nr // 3 - 3), slice(nc // 3 + 3, 2 * nc // 3 - 3), slice(2, ns - 2))
    assert abs(float(np.mean(rec[inner])) - 1.0) < 0.1
    np.random.seed(0)
    ref = O.back_project(geom, O.fbp_filter(O.forward_project(geom, ph), geom.delta_voxel) if kind == 'parallel' else
                         O.fdk_filter(O.forward_project(geom, ph), geom.source_detector_dist, geom.magnification,
                                      geom.delta_voxel, geom.delta_det_row, geom.delta_det_channel))
    assert rel_l2(rec, ref) <= 1e-5


@pytest.mark.parametrize('kind', ['parallel', 'cone'])
def test_fbp_fdk_meets_the_reference_tolerances(cuda, kind):
    """tests/test_fbp_fdk.py through the model API at its own size: the Shepp-Logan phantom of the model, its
    forward projection and the direct recon of that stay under the reference's error bounds; the parallel recon
    also matches the oracle's."""
    from cases import fbp_fdk_model, oracle_geometry, recon_error_stats, FBP_TOLERANCES, FDK_TOLERANCES
    model = fbp_fdk_model(kind)
    phantom = model.gen_modified_3d_sl_phantom()
    assert tuple(phantom.shape) == (128, 128, 128)
    recon = model.direct_recon(model.forward_project(phantom)).cpu().numpy()
    phantom = phantom.cpu().numpy()
    stats = recon_error_stats(recon, phantom)
    for name, bound in (FBP_TOLERANCES if kind == 'parallel' else FDK_TOLERANCES).items():
        assert stats[name] < bound, (name, stats)
    if kind == 'parallel':
        geom = oracle_geometry(model)
        ref = O.back_project(geom, O.fbp_filter(O.forward_project(geom, phantom), geom.delta_voxel))
        assert rel_l2(recon, ref) <= 1e-5
