"""GPU parity of the VCD subset update and of full reconstructions against the oracle (same partitions,
subset orders and qGGMRF parameters; bar: 1e-4 NRMSE against the oracle's recon after a fixed iteration count)."""
import numpy as np
import pytest
import torch

import mbirjax_b200 as mb
from mbirjax_b200 import _capi
import oracle as O
from cases import make_case, rel_l2

pytestmark = pytest.mark.gpu


def _phantom_and_sino(model, geom, seed, weights=False):
    from mbirjax_b200.utilities import gen_ellipsoid_phantom
    ph = gen_ellipsoid_phantom(geom.recon_shape, 6, seed).numpy()
    np.random.seed(seed)
    sino = O.forward_project(geom, ph)
    sino = sino + np.random.default_rng(seed).normal(0, 0.01 * np.abs(sino).max(), sino.shape).astype(np.float32)
    w = np.exp(-sino / sino.max()).astype(np.float32) if weights else None
    return ph, sino.astype(np.float32), w


@pytest.mark.parametrize('kind,weighted', [('parallel', False), ('parallel', True), ('cone', False), ('cone', True),
                                           ('translation', True)])
def test_subset_step_matches_oracle(cuda, kind, weighted):
    model, geom = make_case(kind, views=24, rows=6, channels=40)
    ph, sino, w = _phantom_and_sino(model, geom, 3, weighted)
    nr, nc, ns = geom.recon_shape
    rng = np.random.default_rng(0)
    flat = (0.9 * ph + 0.05 * rng.random(ph.shape)).astype(np.float32).reshape(-1, ns)
    np.random.seed(1)
    err = (sino - O.forward_project(geom, flat.reshape(geom.recon_shape))).astype(np.float32)
    hess = O.compute_hessian_diagonal(geom, w).reshape(-1, ns)
    np.random.seed(2)
    subset = O.gen_pixel_partition(geom.recon_shape, 3)[1]
    params = (O.get_b_from_nbr_wts([1, 1, 1]), 0.2, 2.0, 1.2, 1.0)
    fm = 1.0 / 0.05 ** 2
    r_ref, e_ref, l1_ref, a_ref = O.vcd_subset_update(geom, flat, err, w, hess, subset, fm, params)

    dev = torch.device('cuda')
    flat_d = torch.as_tensor(flat, device=dev).contiguous()
    err_d = torch.as_tensor(err, device=dev).contiguous()
    w_d = None if w is None else torch.as_tensor(w, device=dev)
    stats = torch.zeros(4, dtype=torch.float64, device=dev)
    _capi.vcd_subset_step(model._geometry(), flat_d, err_d, w_d, torch.as_tensor(hess, device=dev),
                          torch.as_tensor(subset, device=dev), fm, _capi.qggmrf_params(*params), stats)
    st = stats.cpu().numpy()
    assert st[0] == pytest.approx(a_ref, rel=1e-5)
    assert st[1] == pytest.approx(l1_ref, rel=1e-5)
    assert rel_l2(flat_d.cpu().numpy(), r_ref) <= 1e-6
    assert rel_l2(err_d.cpu().numpy(), e_ref) <= 1e-5


def _recon_pair(kind, shape_kw, granularity, iterations, weighted, seed):
    model, geom = make_case(kind, **shape_kw)
    ph, sino, w = _phantom_and_sino(model, geom, seed, weighted)
    model.set_params(sharpness=0.0, snr_db=30.0, granularity=granularity, partition_sequence=[0], verbose=0)
    np.random.seed(seed)
    rec, rdict = model.recon(sino, weights=w, max_iterations=iterations, stop_threshold_change_pct=0,
                             logfile_path=None, print_logs=False)
    np.random.seed(seed)
    ref, stats = O.vcd.recon(geom, sino, granularity=granularity, partition_sequence=[0], max_iterations=iterations,
                             weights=w, sharpness=0.0, snr_db=30.0, stop_threshold_change_pct=0,
                             qggmrf_nbr_wts=tuple(model.get_params('qggmrf_nbr_wts')))
    return rec.cpu().numpy(), ref, rdict, stats, ph


@pytest.mark.parametrize('kind,weighted', [('parallel', False), ('cone', False), ('cone', True),
                                           ('translation', False)])
def test_recon_matches_oracle(cuda, kind, weighted):
    rec, ref, rdict, stats, ph = _recon_pair(kind, dict(views=32, rows=6, channels=48), [4], 5, weighted, 0)
    assert rel_l2(rec, ref) <= 1e-4
    assert rdict['recon_params']['num_iterations'] == 5
    np.testing.assert_allclose(rdict['recon_params']['fm_rmse'], stats['fm_rmse'], rtol=1e-3)
    assert rdict['recon_params']['regularization_params']['sigma_x'] == pytest.approx(stats['sigma_x'], rel=1e-6)


def test_recon_small_parallel_config(cuda):
    """Parallel-beam VCD: 128x128x16 volume, 64 views x 16 rows x 128 channels, 10 ellipsoids (seed 0),
    1% noise, p=2, q=1.2, T=1, sharpness 0, 10 iterations with 4 subsets."""
    from mbirjax_b200.utilities import gen_ellipsoid_phantom
    model, geom = make_case('parallel', views=64, rows=16, channels=128)
    ang = np.linspace(0, np.pi, 64, endpoint=False).astype(np.float32)
    model = mb.ParallelBeamModel((64, 16, 128), ang)
    geom = O.parallel_geometry((64, 16, 128), ang)
    ph = gen_ellipsoid_phantom(geom.recon_shape, 10, 0).numpy()
    np.random.seed(0)
    sino = O.forward_project(geom, ph)
    sino = (sino + np.random.default_rng(0).normal(0, 0.01 * np.abs(sino).max(), sino.shape)).astype(np.float32)
    model.set_params(sharpness=0.0, granularity=[4], partition_sequence=[0], verbose=0)
    np.random.seed(0)
    rec, _ = model.recon(sino, max_iterations=10, stop_threshold_change_pct=0, logfile_path=None, print_logs=False)
    np.random.seed(0)
    ref, _ = O.vcd.recon(geom, sino, granularity=[4], partition_sequence=[0], max_iterations=10, sharpness=0.0,
                         stop_threshold_change_pct=0)
    assert rel_l2(rec.cpu().numpy(), ref) <= 1e-4
    # sanity floor: the iterative recon is closer to the phantom than its FBP initialisation
    fbp = model.direct_recon(sino).cpu().numpy()
    assert rel_l2(rec.cpu().numpy(), ph) < rel_l2(fbp, ph)


def _small_parallel_case(seed=3):
    from mbirjax_b200.utilities import gen_ellipsoid_phantom
    ang = np.linspace(0, np.pi, 32, endpoint=False).astype(np.float32)
    model = mb.ParallelBeamModel((32, 8, 48), ang)
    geom = O.parallel_geometry((32, 8, 48), ang)
    ph = gen_ellipsoid_phantom(geom.recon_shape, 4, seed).numpy()
    sino = O.forward_project(geom, ph)
    sino = (sino + np.random.default_rng(seed).normal(0, 0.02 * np.abs(sino).max(), sino.shape)).astype(np.float32)
    model.set_params(sharpness=0.0, granularity=[4], partition_sequence=[0], verbose=0)
    return model, geom, ph, sino


def test_recon_with_positivity_matches_oracle(cuda):
    """positivity_flag=True: the update of each subset is clipped so no voxel goes below zero, then re-projected
    (tomography_model.py:1497-1507); same recon as the oracle's restatement."""
    model, geom, ph, sino = _small_parallel_case()
    model.set_params(positivity_flag=True)
    np.random.seed(3)
    rec, d = model.recon(sino, max_iterations=4, stop_threshold_change_pct=0, logfile_path=None, print_logs=False)
    rec = rec.cpu().numpy()
    np.random.seed(3)
    ref, stats = O.vcd.recon(geom, sino, granularity=[4], partition_sequence=[0], max_iterations=4, sharpness=0.0,
                             stop_threshold_change_pct=0, positivity=True)
    assert rel_l2(rec, ref) <= 1e-4
    np.testing.assert_allclose(d['recon_params']['alpha_values'], stats['alpha_values'], rtol=1e-4)
    mask = O.get_2d_ror_mask(geom.recon_shape)[:, :, None] > 0
    assert rec[np.broadcast_to(mask, rec.shape)].min() >= -1e-6 * np.abs(rec).max()


def test_prox_map_matches_oracle(cuda):
    """prox_map: VCD with the proximal prior centred on prox_input (tomography_model.py:1660-1697, prior
    gradient (x - v) / sigma_prox^2 and Hessian sigma_prox^2) at the model's sigma_y and sigma_prox."""
    model, geom, ph, sino = _small_parallel_case(seed=4)
    sigma_y, sigma_x, sigma_prox = O.auto_regularization(geom, sino, None, 30.0, 0.0)
    model.set_params(sigma_y=float(sigma_y), sigma_x=float(sigma_x), sigma_prox=float(sigma_prox))
    prox = (ph + np.random.default_rng(9).normal(0, 0.05, ph.shape)).astype(np.float32)
    np.random.seed(4)
    rec, loss = model.prox_map(prox, sino, max_iterations=3, stop_threshold_change_pct=0, logfile_path=None,
                               print_logs=False)
    np.random.seed(4)
    ref, stats = O.prox_map(geom, prox, sino, sigma_y=sigma_y, sigma_x=sigma_x, sigma_prox=sigma_prox,
                            granularity=[4], partition_sequence=[0], max_iterations=3, stop_threshold_change_pct=0)
    assert rel_l2(rec.cpu().numpy(), ref) <= 1e-4
    np.testing.assert_allclose(np.asarray(loss[0]), stats['fm_rmse'], rtol=1e-4)


def test_prox_map_fixed_point(cuda):
    """The reference's proximal-map corner case (tests/test_prox.py): input, initial recon and the noiseless data
    all agree with the phantom, so five iterations leave it in place to 1e-5."""
    from mbirjax_b200.utilities import gen_ellipsoid_phantom
    ang = np.linspace(0, np.pi, 32, endpoint=False).astype(np.float32)
    model = mb.ParallelBeamModel((32, 40, 128), ang)
    phantom = gen_ellipsoid_phantom(model.get_params('recon_shape'), 6, 0)
    sino = model.forward_project(phantom)
    model.set_params(verbose=0)
    np.random.seed(0)
    rec, _ = model.prox_map(phantom, sino, max_iterations=5, init_recon=phantom, logfile_path=None,
                            print_logs=False)
    assert float(torch.max(torch.abs(rec - phantom.to(rec.device)))) < 1e-5


@pytest.mark.parametrize('kind', ['parallel', 'cone'])
def test_vcd_meets_the_reference_tolerances(cuda, kind):
    """tests/test_vcd.py through the model API at its own size: the model's Shepp-Logan phantom, its forward
    projection, and the default recon of that (sharpness 1, multi-granular partitions, at most 15 iterations,
    stop at 0.2%) stay under the reference's error bounds."""
    from cases import vcd_acceptance_model, recon_error_stats, VCD_TOLERANCES
    model = vcd_acceptance_model(kind)
    phantom = model.gen_modified_3d_sl_phantom()
    sino = model.forward_project(phantom)
    model.set_params(verbose=0)
    np.random.seed(0)
    rec, rdict = model.recon(sino, logfile_path=None, print_logs=False)
    assert rdict['recon_params']['num_iterations'] <= 15
    err = recon_error_stats(rec.cpu().numpy(), phantom.cpu().numpy())
    for name, bound in VCD_TOLERANCES[kind].items():
        assert err[name] < bound, (name, err)
