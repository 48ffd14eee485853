"""CPU tests of the models' host logic end to end, with the oracle answering the library calls
(``fake_library.oracle_library``): the VCD iteration loop of ``recon`` / ``prox_map`` (partitions and the
np.random order of their subsets, the initial alpha, the statistics and the stopping rule), the denoiser's loop,
FBP/FDK, the geometry records of the per-view plugin functions and the autograd wrappers.  The GPU tests check
the same host code with the CUDA library underneath."""
import numpy as np
import pytest

import mbirjax_b200 as mb
import oracle as O
from oracle import denoise as OD
from cases import make_case, rel_l2
from fake_library import oracle_library  # noqa: F401  (fixture)


def _phantom_and_sino(geom, seed, weighted):
    from mbirjax_b200.utilities import gen_ellipsoid_phantom
    ph = gen_ellipsoid_phantom(geom.recon_shape, 4, seed).numpy()
    sino = O.forward_project(geom, ph)
    sino = (sino + np.random.default_rng(seed).normal(0, 0.01 * np.abs(sino).max(), sino.shape)).astype(np.float32)
    w = np.exp(-sino / sino.max()).astype(np.float32) if weighted else None
    return ph, sino, w


@pytest.mark.parametrize('kind,weighted', [('parallel', False), ('cone', True), ('translation', False)])
def test_recon_host_loop_matches_oracle(oracle_library, kind, weighted):
    model, geom = make_case(kind, views=16, rows=4, channels=24)
    _, sino, w = _phantom_and_sino(geom, 1, weighted)
    model.set_params(sharpness=0.0, granularity=[1, 3], partition_sequence=[0, 1], verbose=0)
    np.random.seed(3)
    with pytest.warns(UserWarning) if kind == 'translation' else _no_warning():
        rec, rdict = model.recon(sino, weights=w, max_iterations=3, stop_threshold_change_pct=0, logfile_path=None,
                                 print_logs=False, compute_prior_loss=True)
    np.random.seed(3)
    ref, stats = O.vcd.recon(geom, sino, granularity=[1, 3], partition_sequence=[0, 1], max_iterations=3, weights=w,
                             sharpness=0.0, stop_threshold_change_pct=0,
                             qggmrf_nbr_wts=tuple(model.get_params('qggmrf_nbr_wts')))
    assert rel_l2(rec.numpy(), ref) <= 1e-5
    rp = rdict['recon_params']
    assert rp['num_iterations'] == 3 and list(rp['partition_sequence']) == [0, 1, 1]
    np.testing.assert_allclose(rp['fm_rmse'], stats['fm_rmse'], rtol=1e-5)
    assert rp['regularization_params']['sigma_x'] == pytest.approx(stats['sigma_x'], rel=1e-6)
    assert all(v > 0 for v in rp['prior_loss'])


class _no_warning:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def test_recon_stops_at_the_change_threshold(oracle_library):
    """The loop ends after the first iteration whose relative change is under the threshold, as the oracle's
    (tomography_model.py:1220-1250)."""
    model, geom = make_case('parallel', views=16, rows=4, channels=24)
    _, sino, _ = _phantom_and_sino(geom, 2, False)
    model.set_params(sharpness=0.0, granularity=[2], partition_sequence=[0], verbose=0)
    np.random.seed(5)
    rec, rdict = model.recon(sino, max_iterations=30, stop_threshold_change_pct=2.0, logfile_path=None,
                             print_logs=False)
    np.random.seed(5)
    ref, stats = O.vcd.recon(geom, sino, granularity=[2], partition_sequence=[0], max_iterations=30, sharpness=0.0,
                             stop_threshold_change_pct=2.0)
    n = rdict['recon_params']['num_iterations']
    assert 1 < n < 30 and n == len(stats['fm_rmse'])
    assert rdict['recon_params']['stop_threshold_change_pct'][-1] < 2.0 <= rdict['recon_params']['stop_threshold_change_pct'][-2]
    assert rel_l2(rec.numpy(), ref) <= 1e-5


def test_prox_map_host_loop_matches_oracle(oracle_library):
    model, geom = make_case('parallel', views=16, rows=4, channels=24)
    ph, sino, _ = _phantom_and_sino(geom, 4, False)
    sigma_y, sigma_x, sigma_prox = O.auto_regularization(geom, sino, None, 30.0, 0.0)
    with pytest.warns(UserWarning, match='regularization'):
        model.set_params(sigma_y=float(sigma_y), sigma_x=float(sigma_x), sigma_prox=float(sigma_prox),
                         granularity=[2], partition_sequence=[0], verbose=0, positivity_flag=True)
    prox = (ph + np.random.default_rng(9).normal(0, 0.05, ph.shape)).astype(np.float32)
    np.random.seed(4)
    rec, loss = model.prox_map(prox, sino, max_iterations=2, stop_threshold_change_pct=0, logfile_path=None,
                               print_logs=False)
    np.random.seed(4)
    ref, stats = O.prox_map(geom, prox, sino, sigma_y=sigma_y, sigma_x=sigma_x, sigma_prox=sigma_prox,
                            granularity=[2], partition_sequence=[0], max_iterations=2, stop_threshold_change_pct=0,
                            positivity=True)
    assert rel_l2(rec.numpy(), ref) <= 1e-5
    assert float(rec.min()) >= 0.0
    np.testing.assert_allclose(np.asarray(loss[0]), stats['fm_rmse'], rtol=1e-5)


def test_denoiser_host_loop_matches_oracle(oracle_library):
    from mbirjax_b200.utilities import gen_ellipsoid_phantom
    shape = (20, 18, 6)
    clean = gen_ellipsoid_phantom(shape, 3, 1).numpy()
    noisy = (clean + 0.1 * np.random.default_rng(1).standard_normal(shape)).astype(np.float32)
    den = mb.QGGMRFDenoiser(shape)
    den.set_params(verbose=0)
    np.random.seed(7)
    out, d = den.denoise(noisy, 0.1, max_iterations=3, stop_threshold_change_pct=0, logfile_path=None,
                         print_logs=False)
    small = noisy[::shape[0] // min(20, shape[0])]
    sigma_x = float(np.float32(0.2 * OD._neighbour_std(small, OD._support(small, 0.1))))
    np.random.seed(7)
    partition = O.gen_set_of_pixel_partitions(shape, [16], use_ror_mask=False)[0]
    ref, nmae, alphas = OD.denoise(noisy, partition, 0.1, (O.get_b_from_nbr_wts([1, 1, 1]), sigma_x, 2.0, 1.2, 1.0),
                                   3, 0)
    assert rel_l2(out.numpy(), ref) <= 1e-6
    np.testing.assert_allclose(d['recon_params']['alpha_values'], alphas, rtol=1e-6)


@pytest.mark.parametrize('kind', ['parallel', 'cone'])
def test_direct_recon_host_path_matches_oracle(oracle_library, kind):
    model, geom = make_case(kind, views=20, rows=4, channels=24)
    sino = np.random.default_rng(2).random(geom.sinogram_shape).astype(np.float32)
    rec = model.direct_recon(sino).numpy()
    filt = (O.fbp_filter(sino, geom.delta_voxel) if kind == 'parallel' else
            O.fdk_filter(sino, geom.source_detector_dist, geom.magnification, geom.delta_voxel, geom.delta_det_row,
                         geom.delta_det_channel, geom.det_row_offset, geom.det_channel_offset))
    np.random.seed(0)
    assert rel_l2(rec, O.back_project(geom, filt)) <= 1e-6


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_one_view_records_give_the_oracle_view(oracle_library, kind):
    """The per-view plugin functions' one-view geometry record, read as the library reads it, projects view j
    as the model's geometry does."""
    model, geom = make_case(kind, views=7, rows=4, channels=20)
    nr, nc, ns = geom.recon_shape
    rng = np.random.default_rng(5)
    idx = rng.permutation(nr * nc)[: nr * nc // 2].astype(np.int32)
    x = rng.standard_normal((len(idx), ns)).astype(np.float32)
    view = rng.standard_normal(geom.sinogram_shape[1:]).astype(np.float32)
    pp = model.get_projector_params()
    views = np.asarray(model.get_params(model.get_params('view_params_name')), dtype=np.float32)
    cls = type(model)
    for j in (0, 5):
        fp = cls.forward_project_pixel_batch_to_one_view(x, idx, views[j], pp).numpy()
        np.testing.assert_allclose(fp, O.forward_project_one_view(geom, x, idx, geom.angles[j]), rtol=1e-6,
                                   atol=1e-6)
        bp = cls.back_project_one_view_to_pixel_batch(view, idx, views[j], pp, coeff_power=2).numpy()
        np.testing.assert_allclose(bp, O.back_project_one_view(geom, view, idx, geom.angles[j], coeff_power=2),
                                   rtol=1e-6, atol=1e-6)


def test_autograd_pair_host_logic(oracle_library):
    """mbirjax_b200.autograd on the host: the gradient of <A x, y> is A^T y on the region of reconstruction (zero
    outside), the view-chunked backward adds the same chunks, and the gradient of the weighted least-squares +
    qGGMRF loss matches central differences of the float64 oracle loss."""
    import torch
    from mbirjax_b200 import autograd as AG
    model, geom = make_case('cone', views=10, rows=4, channels=16)
    rng = np.random.default_rng(0)
    x = torch.tensor(rng.random(geom.recon_shape), dtype=torch.float32, requires_grad=True)
    y = torch.tensor(rng.random(geom.sinogram_shape), dtype=torch.float32)
    (gx,) = torch.autograd.grad(torch.sum(AG.forward_project(x, model) * y), x)
    aty = AG.back_project(y, model)
    torch.testing.assert_close(gx, aty, rtol=1e-6, atol=1e-6)
    mask = O.get_2d_ror_mask(geom.recon_shape)[:, :, None].astype(bool)
    assert not np.any(gx.numpy()[~np.broadcast_to(mask, geom.recon_shape)])
    (gx3,) = torch.autograd.grad(torch.sum(AG.forward_project(x, model, 3) * y), x)
    torch.testing.assert_close(gx3, gx, rtol=1e-5, atol=1e-5)

    params = (O.get_b_from_nbr_wts([1, 1, 1]), 0.3, 2.0, 1.2, 1.0)
    x64 = (rng.random(geom.recon_shape) * mask).astype(np.float64)
    y64 = O.forward_project(geom, (0.8 * x64).astype(np.float32), dtype=np.float64)
    w64 = np.exp(-y64 / y64.max())

    def loss64(v):
        r = O.forward_project(geom, v, dtype=np.float64) - y64
        return 0.5 * float(np.sum(w64 * r * r)) + O.qggmrf_loss(v, params)

    xt = torch.tensor(x64, dtype=torch.float32, requires_grad=True)
    loss = AG.weighted_ls_qggmrf_loss(xt, model, torch.tensor(y64, dtype=torch.float32),
                                      torch.tensor(w64, dtype=torch.float32), params)
    (grad,) = torch.autograd.grad(loss, xt)
    assert float(loss.detach()) == pytest.approx(loss64(x64.astype(np.float32).astype(np.float64)), rel=1e-4)
    ror = np.argwhere(np.broadcast_to(mask, geom.recon_shape))
    picks = ror[rng.choice(len(ror), 12, replace=False)]
    eps = 1e-3
    fd, ag = [], []
    for i, j, k in picks:
        xp, xm = x64.copy(), x64.copy()
        xp[i, j, k] += eps
        xm[i, j, k] -= eps
        fd.append((loss64(xp) - loss64(xm)) / (2 * eps))
        ag.append(float(grad[i, j, k]))
    assert np.linalg.norm(np.array(ag) - np.array(fd)) <= 1e-3 * np.linalg.norm(fd)
