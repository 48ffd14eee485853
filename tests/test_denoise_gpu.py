"""The qGGMRF denoiser and the median filter (denoising.py of the reference) against the oracle."""
import numpy as np
import pytest
import torch

import mbirjax_b200 as mb
import oracle as O
from oracle import denoise as OD
from cases import rel_l2

pytestmark = pytest.mark.gpu


def test_median_filter_matches_oracle(cuda):
    x = np.random.default_rng(0).standard_normal((17, 13, 9)).astype(np.float32)
    np.testing.assert_array_equal(mb.median_filter3d(x).cpu().numpy(), OD.median_filter3d(x))
    a = np.arange(27, dtype=np.float32).reshape(3, 3, 3)
    np.testing.assert_array_equal(mb.median_filter3d(a).cpu().numpy(), OD.median_filter3d(a))


def _noisy(shape, seed, sigma):
    from mbirjax_b200.utilities import gen_ellipsoid_phantom
    clean = gen_ellipsoid_phantom(shape, 6, seed).numpy()
    return clean, (clean + sigma * np.random.default_rng(seed).standard_normal(shape)).astype(np.float32)


def test_denoise_matches_oracle(cuda):
    """Same partition (np.random), same regularisation, subsets in order: the device denoiser follows the oracle's
    restatement of vcd_subset_denoiser iteration for iteration."""
    shape, sigma_noise = (32, 32, 8), 0.1
    clean, noisy = _noisy(shape, 1, sigma_noise)
    den = mb.QGGMRFDenoiser(shape)
    den.set_params(verbose=0)
    np.random.seed(7)
    out, d = den.denoise(noisy, sigma_noise, max_iterations=4, stop_threshold_change_pct=0, logfile_path=None,
                         print_logs=False)
    # the oracle's side: sigma_x from the subsampled image as auto_set_regularization_params computes it
    step = shape[0] // min(20, shape[0])
    small = noisy[::step]
    recon_std = OD._neighbour_std(small, OD._support(small, sigma_noise))
    sigma_x = float(np.float32(0.2 * recon_std))
    np.random.seed(7)
    partition = O.gen_set_of_pixel_partitions(shape, [16], use_ror_mask=False)[0]
    qp = (O.get_b_from_nbr_wts([1, 1, 1]), sigma_x, 2.0, 1.2, 1.0)
    ref, nmae, alphas = OD.denoise(noisy, partition, sigma_noise, qp, 4, 0)
    assert d['recon_params']['regularization_params']['sigma_x'] == pytest.approx(sigma_x, rel=1e-6)
    assert rel_l2(out.cpu().numpy(), ref) <= 1e-4
    np.testing.assert_allclose(d['recon_params']['alpha_values'], alphas, rtol=1e-4)
    np.testing.assert_allclose(np.array(d['recon_params']['stop_threshold_change_pct']) / 100, nmae, rtol=1e-3)


def test_denoiser_reduces_noise(cuda):
    """The reference's check (tests/test_denoiser.py): denoising a noisy phantom with the known noise level lands
    within 20% relative error of the clean phantom."""
    shape = (64, 64, 32)
    clean, noisy = _noisy(shape, 2, 0.1)
    den = mb.QGGMRFDenoiser(shape)
    den.set_params(sharpness=0.0, verbose=0)
    np.random.seed(0)
    out, _ = den.denoise(noisy, 0.1, max_iterations=20, stop_threshold_change_pct=0.1, logfile_path=None,
                         print_logs=False)
    out = out.cpu().numpy()
    assert np.linalg.norm(out - clean) / np.linalg.norm(clean) < 0.2
    assert np.linalg.norm(out - clean) < np.linalg.norm(noisy - clean)


def test_qggmrf_denoiser_reference_case(cuda):
    """tests/test_denoiser.py::test_qggmrf_denoiser at its own size: a 100^3 Shepp-Logan phantom with noise of std
    0.1, sharpness 0, at most 20 iterations, stop at 0.1%, denoised within 20% relative error."""
    from mbirjax_b200.utilities import generate_3d_shepp_logan_low_dynamic_range
    np.random.seed(0)
    shape = (100, 100, 100)
    phantom = generate_3d_shepp_logan_low_dynamic_range(shape).numpy()
    noisy = phantom + 0.1 * np.random.randn(*shape)
    den = mb.QGGMRFDenoiser(shape)
    den.set_params(sharpness=0.0, verbose=0)
    out, _ = den.denoise(noisy, 0.1, max_iterations=20, stop_threshold_change_pct=0.1, logfile_path=None,
                         print_logs=False)
    from cases import ACCEPTANCE_BOUNDS
    assert np.linalg.norm(out.cpu().numpy() - phantom) / np.linalg.norm(phantom) < ACCEPTANCE_BOUNDS['denoiser_nrmse']
