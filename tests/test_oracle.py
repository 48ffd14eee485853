"""CPU tests of the oracle: pinned against the reference's golden vectors, its structural tests and its
end-to-end acceptance bounds at their own sizes (reference tests/test_qggmrf.py:23-172,
tests/test_projectors.py:152-303, tests/test_fbp_fdk.py, tests/test_vcd.py, tests/test_denoiser.py; the bounds are
read from tests/golden/acceptance_bounds.json)."""
import json
import os

import numpy as np
import pytest

import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'qggmrf_golden.json')


def _golden():
    with open(GOLDEN) as f:
        return json.load(f)


def test_qggmrf_golden_vectors():
    g = _golden()
    params = (O.get_b_from_nbr_wts([1, 1, 1]), g['sigma_x'], g['p'], g['q'], g['T'])
    flat = np.array(g['flat_recon'])
    grad, hess = O.qggmrf_gradient_and_hessian_at_indices(flat, tuple(g['recon_shape']), np.arange(flat.shape[0]),
                                                          params)
    # np.allclose defaults, as the reference test (tests/test_qggmrf.py:133-134)
    assert np.allclose(grad, g['grad_ref'])
    assert np.allclose(hess, g['hess_ref'])


def test_b_tilde_definition():
    rng = np.random.default_rng(3)
    p = rng.random() + 1
    q = p - 0.9 * rng.random()
    T = 0.5 + rng.random()
    sigma_x = 0.1 + rng.random()
    delta = 0.1 + rng.random(10)
    b2 = O.get_2_b_tilde(delta, 1.0, ((1,) * 6, sigma_x, p, q, T), dt=np.float64)
    assert np.allclose(b2 / 2, O.b_tilde_by_definition(delta, sigma_x, p, q, T))


def test_qggmrf_loss_gradient_finite_difference():
    # tests/test_qggmrf.py:136-172 shape of test, in float64
    p, q, T, sigma_x = 2.0413, 1.124, 1.46, 0.789
    params = (O.get_b_from_nbr_wts([1, 1, 1]), sigma_x, p, q, T)
    rng = np.random.default_rng(0)
    x = rng.random((3, 3, 3))
    d = rng.random((3, 3, 3))
    eps = 1e-7
    fd = (O.qggmrf_loss(x + eps * d, params) - O.qggmrf_loss(x, params)) / eps
    g_surr, h_surr = O.qggmrf_gradient_and_hessian_at_indices(x.reshape(9, 3), (3, 3, 3), np.arange(9), params,
                                                              dt=np.float64)
    assert np.allclose(fd, np.sum(g_surr.reshape(x.shape) * d), rtol=1e-3)
    g_loss = O.qggmrf_loss_grad(x, params)
    assert np.allclose(fd, np.sum(g_loss * d), rtol=1e-5)
    g_ref, h_ref = O.compute_qggmrf_grad_and_hessian(x, params)
    assert np.allclose(h_ref, h_surr.reshape(x.shape))
    assert np.allclose(g_ref, g_surr.reshape(x.shape))


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_oracle_adjoint_exact_in_float64(kind):
    from cases import make_case
    _, geom = make_case(kind, views=12, rows=6, channels=24)
    nr, nc, ns = geom.recon_shape
    rng = np.random.default_rng(1)
    idx = np.arange(nr * nc)
    x = rng.random((nr * nc, ns))
    y = rng.random(geom.sinogram_shape)
    ax = O.sparse_forward_project(geom, x, idx, dtype=np.float64)
    aty = O.sparse_back_project(geom, y, idx, dtype=np.float64)
    assert abs(np.sum(ax * y) - np.sum(aty * x)) <= 1e-12 * abs(np.sum(ax * y))


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_oracle_hessian_finite_difference(kind):
    # tests/test_projectors.py:264-303
    from cases import make_case
    _, geom = make_case(kind, views=10, rows=6, channels=20)
    nr, nc, ns = geom.recon_shape
    hess = O.compute_hessian_diagonal(geom, dtype=np.float64)
    i, j, k = nr // 3, nc // 2, ns // 2
    x = np.zeros((nr * nc, ns))
    x[i * nc + j, k] = 0.01
    idx = np.arange(nr * nc)
    atax = O.sparse_back_project(geom, O.sparse_forward_project(geom, x, idx, dtype=np.float64), idx,
                                 dtype=np.float64).reshape(nr, nc, ns)
    assert np.isclose(hess[i, j, k], atax[i, j, k] / 0.01)


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_oracle_view_batching(kind):
    # tests/test_projectors.py:152-198; exact here since the oracle rounds consistently
    from cases import make_case
    _, geom = make_case(kind, views=12, rows=6, channels=24)
    nr, nc, ns = geom.recon_shape
    np.random.seed(2)
    idx = O.gen_full_indices(geom.recon_shape)
    x = np.random.rand(len(idx), ns).astype(np.float32)
    full = O.sparse_forward_project(geom, x, idx)
    for j in range(3):
        views = np.arange(j, 12, 3)
        np.testing.assert_array_equal(O.sparse_forward_project(geom, x, idx, views), full[views])
    bp = O.sparse_back_project(geom, full, idx)
    parts = sum(O.sparse_back_project(geom, full, idx, np.arange(j, 12, 3)) for j in range(3))
    assert np.abs(parts - bp).max() <= 1e-5 * np.abs(bp).max()


def test_oracle_partitions_match_reference_contract():
    np.random.seed(0)
    shape = (20, 20, 3)
    p = O.gen_pixel_partition(shape, 7)
    mask = O.get_2d_ror_mask(shape).flatten()
    n = int(mask.sum())
    assert p.shape == (7, int(np.ceil(n / 7)))
    assert np.all(np.diff(p, axis=1) > 0)                       # sorted, no duplicates inside a subset
    assert set(np.unique(p)) == set(np.flatnonzero(mask))       # covers the ROR exactly
    assert list(O.gen_partition_sequence([0, 2, 4], 6)) == [0, 2, 4, 4, 4, 4]


def test_oracle_fbp_recovers_phantom():
    # sanity floor in the spirit of tests/test_fbp_fdk.py: FBP of a forward projection resembles the phantom
    from cases import make_case
    _, geom = make_case('parallel', views=64, rows=2, channels=48)
    nr, nc, ns = geom.recon_shape
    ph = np.zeros(geom.recon_shape, dtype=np.float32)
    ph[16:32, 14:30, :] = 1.0
    sino = O.forward_project(geom, ph)
    rec = O.back_project(geom, O.fbp_filter(sino, geom.delta_voxel))
    inner = (slice(18, 30), slice(16, 28))
    assert abs(float(np.mean(rec[inner])) - 1.0) < 0.1


@pytest.mark.parametrize('kind', ['parallel', 'cone'])
def test_oracle_fbp_fdk_meets_the_reference_tolerances(kind):
    """tests/test_fbp_fdk.py at its own size: the oracle's FBP / FDK of its forward projection of the Shepp-Logan
    phantom stays under the error bounds the reference sets just above its own results (parallel lands at nrmse
    0.2099 against 0.21), which pins the projector and filter scaling, not only their structure."""
    from cases import fbp_fdk_model, oracle_geometry, recon_error_stats, FBP_TOLERANCES, FDK_TOLERANCES
    from mbirjax_b200.utilities import generate_3d_shepp_logan_low_dynamic_range
    geom = oracle_geometry(fbp_fdk_model(kind))
    assert geom.recon_shape == (128, 128, 128)
    phantom = generate_3d_shepp_logan_low_dynamic_range(geom.recon_shape).numpy()
    sino = O.forward_project(geom, phantom)
    if kind == 'parallel':
        filtered, tol = O.fbp_filter(sino, geom.delta_voxel), FBP_TOLERANCES
    else:
        filtered, tol = O.fdk_filter(sino, geom.source_detector_dist, geom.magnification, geom.delta_voxel,
                                     geom.delta_det_row, geom.delta_det_channel, geom.det_row_offset,
                                     geom.det_channel_offset), FDK_TOLERANCES
    stats = recon_error_stats(O.back_project(geom, filtered), phantom)
    for name, bound in tol.items():
        assert stats[name] < bound, (name, stats)


def test_oracle_vcd_meets_the_reference_tolerances():
    """tests/test_vcd.py at its own size, parallel beam (the cone case takes minutes on the CPU and runs on the GPU
    through the model API): the oracle's default multi-granular VCD recon of the Shepp-Logan phantom's forward
    projection stays under the reference's error bounds (it lands at nrmse 0.089 against 0.15)."""
    from cases import vcd_acceptance_model, oracle_geometry, recon_error_stats, VCD_TOLERANCES
    from mbirjax_b200.utilities import generate_3d_shepp_logan_low_dynamic_range
    model = vcd_acceptance_model('parallel')
    geom = oracle_geometry(model)
    phantom = generate_3d_shepp_logan_low_dynamic_range(geom.recon_shape).numpy()
    sino = O.forward_project(geom, phantom)
    np.random.seed(0)
    granularity, sequence = model.get_params(['granularity', 'partition_sequence'])
    rec, stats = O.vcd.recon(geom, sino, granularity=granularity, partition_sequence=sequence, max_iterations=15,
                             sharpness=model.get_params('sharpness'), snr_db=model.get_params('snr_db'),
                             stop_threshold_change_pct=0.2)
    err = recon_error_stats(rec, phantom)
    for name, bound in VCD_TOLERANCES['parallel'].items():
        assert err[name] < bound, (name, err)


def test_oracle_denoiser_meets_the_reference_tolerance():
    """tests/test_denoiser.py::test_qggmrf_denoiser at its own size: the oracle's qGGMRF denoiser (sharpness 0,
    16 subsets, at most 20 iterations, stop at 0.1%) brings a 100^3 Shepp-Logan phantom with noise of std 0.1
    within 20% relative error."""
    from oracle import denoise as OD
    from mbirjax_b200.utilities import generate_3d_shepp_logan_low_dynamic_range
    np.random.seed(0)
    shape = (100, 100, 100)
    phantom = generate_3d_shepp_logan_low_dynamic_range(shape).numpy()
    noisy = (phantom + 0.1 * np.random.randn(*shape)).astype(np.float32)
    small = noisy[::shape[0] // min(20, shape[0])]     # auto_set_regularization_params' view subsample
    sigma_x = float(np.float32(0.2 * OD._neighbour_std(small, OD._support(small, 0.1))))
    partition = O.gen_set_of_pixel_partitions(shape, [16], use_ror_mask=False)[0]
    qp = (O.get_b_from_nbr_wts([1, 1, 1]), sigma_x, 2.0, 1.2, 1.0)
    out, nmae, _ = OD.denoise(noisy, partition, 0.1, qp, 20, 0.1)
    from cases import ACCEPTANCE_BOUNDS
    assert np.linalg.norm(out - phantom) / np.linalg.norm(phantom) < ACCEPTANCE_BOUNDS['denoiser_nrmse']
    assert len(nmae) < 20                               # the 0.1% stop ends it early


def test_shepp_logan_and_cube_phantoms():
    """The reference's test phantoms (utilities.py:658-696, 1034-1056) by known answers: the centre voxel of the
    Shepp-Logan phantom is 1 - 0.8, the volume is symmetric in the slice axis, and its values are sums of the
    listed intensities; the cube is a quarter block of value 1 / max(rows, cols), shifted a column per slice."""
    from mbirjax_b200.utilities import generate_3d_shepp_logan_low_dynamic_range, gen_cube_phantom
    p = generate_3d_shepp_logan_low_dynamic_range((65, 49, 33)).numpy()
    assert p.dtype == np.float32 and p.shape == (65, 49, 33)
    assert p[32, 24, 16] == np.float32(1.0) + np.float32(-0.8)
    np.testing.assert_array_equal(p, p[:, :, ::-1])
    levels = np.array([0.0, 0.1, 0.2, 0.3, 0.4, 1.0])
    assert np.all(np.min(np.abs(np.unique(p)[:, None] - levels[None, :]), axis=1) < 1e-6)
    assert p[0, 0, 0] == 0 and p[32, 24, 0] == 0          # corner and the slice ends lie outside the skull
    c = gen_cube_phantom((16, 20, 5)).numpy()
    assert c.shape == (16, 20, 5)
    for k in range(5):
        rows, cols = np.nonzero(c[:, :, k])
        assert (rows.min(), rows.max()) == (6, 9) and (cols.min(), cols.max()) == (7 + k, 11 + k)
    np.testing.assert_allclose(c[c > 0], 0.2)


def test_oracle_prox_map_fixed_point():
    """The oracle's proximal map leaves a consistent input in place (the reference's tests/test_prox.py corner
    case, on a small volume)."""
    ang = np.linspace(0, np.pi, 8, endpoint=False).astype(np.float32)
    geom = O.parallel_geometry((8, 3, 16), ang)
    x = np.random.default_rng(0).random(geom.recon_shape).astype(np.float32) * O.get_2d_ror_mask(geom.recon_shape)[:, :, None]
    y = O.forward_project(geom, x)
    np.random.seed(0)
    rec, _ = O.prox_map(geom, x, y, sigma_y=1.0, sigma_x=1.0, sigma_prox=1.0, granularity=[2],
                        partition_sequence=[0], max_iterations=2, init_recon=x, stop_threshold_change_pct=0)
    assert np.max(np.abs(rec - x)) < 1e-5


def test_median_filter_golden():
    """The oracle's 27-point median with edge replication reproduces the reference's known answer."""
    from oracle.denoise import median_filter3d
    g = json.load(open(os.path.join(os.path.dirname(GOLDEN), 'median_golden.json')))
    np.testing.assert_array_equal(median_filter3d(np.arange(27).reshape(3, 3, 3)), np.array(g['expected']))


def test_denoiser_noise_estimate_matches_oracle():
    """QGGMRFDenoiser's host-side noise estimate (denoising.py:80-136) agrees with the oracle's restatement."""
    import mbirjax_b200 as mb
    from oracle.denoise import estimate_image_noise_std
    rng = np.random.default_rng(0)
    img = np.zeros((24, 20, 6), np.float32)
    img[4:18, 5:15, 1:5] = 1.0
    img += 0.1 * rng.standard_normal(img.shape).astype(np.float32)
    d = mb.QGGMRFDenoiser(img.shape)
    assert d.estimate_image_noise_std(img) == pytest.approx(estimate_image_noise_std(img), rel=1e-6)
