"""GPU parity of the sparse projectors (through the C ABI) against the oracle.

Bars: forward/back projection within 1e-5 relative L2 of the float32 oracle; adjointness <y, Ax> = <A^T y, x>
within 1e-5 relative to the float64 oracle's value; view subsets and coefficient power 2 likewise.
Test shapes follow the reference's tests/test_projectors.py (adjoint :200-262, Hessian :264-303, view
batching :152-198)."""
import numpy as np
import pytest
import torch

import mbirjax_b200 as mb
from mbirjax_b200 import _capi
import oracle as O
from cases import make_case, oracle_geometry, rel_l2

pytestmark = pytest.mark.gpu

TOL = 1e-5

CASES = [
    ('parallel', dict(views=16, rows=8, channels=32)),
    ('parallel', dict(views=9, rows=5, channels=33)),                       # odd channels, ragged tiles
    ('parallel', dict(views=12, rows=6, channels=40, delta_voxel=3.0, delta_det_row=3.0)),  # psf radius 2
    ('parallel', dict(views=20, rows=3, channels=24, det_channel_offset=1.3)),
    ('cone', dict(views=16, rows=8, channels=32)),
    ('cone', dict(views=16, rows=12, channels=32, sid_factor=2.0)),         # magnification 2
    ('cone', dict(views=10, rows=7, channels=27, det_row_offset=0.7, det_channel_offset=-1.1,
                  recon_slice_offset=0.4)),
    ('cone', dict(views=12, rows=10, channels=30, delta_voxel=2.2)),        # psf radius 2
    # more than 128 detector rows: several 128-row batches, each with its own row anchor, in the forward
    # projection (cone_beam.py:336-358) and several 128-slice batches in the back projection (cone_beam.py:500-541)
    ('cone', dict(views=8, rows=300, channels=24, sdd_factor=40.0)),
    ('cone', dict(views=6, rows=260, channels=20, sdd_factor=30.0, sid_factor=15.0, det_row_offset=0.3)),  # mag. 2
    ('translation', dict(views=16, rows=8, channels=32)),
    ('translation', dict(views=12, rows=10, channels=30, sid_factor=2.0)),  # magnification 2
    ('translation', dict(views=10, rows=7, channels=27, det_row_offset=0.7, det_channel_offset=-1.1,
                         y_spread=3.0)),
    ('translation', dict(views=12, rows=10, channels=30, delta_voxel=2.2)),  # psf radius 2
]


def _ids():
    return ['%s-%d' % (k, i) for i, (k, _) in enumerate(CASES)]


def _case(kind, kw):
    kw = dict(kw)
    params = {k: kw.pop(k) for k in list(kw) if k in ('delta_voxel', 'delta_det_row', 'det_channel_offset',
                                                     'det_row_offset', 'recon_slice_offset')}
    model, _ = make_case(kind, **kw)
    if params:
        model.set_params(no_warning=True, **params)
        if 'delta_voxel' in params:  # re-derive the recon size for the new voxel size, as a user would
            model.auto_set_recon_size(model.get_params('sinogram_shape'), no_warning=True)
    return model, oracle_geometry(model)


@pytest.mark.parametrize('kind,kw', CASES, ids=_ids())
def test_forward_back_parity(cuda, kind, kw):
    model, geom = _case(kind, kw)
    nr, nc, ns = geom.recon_shape
    np.random.seed(7)
    idx = O.gen_full_indices(geom.recon_shape)
    rng = np.random.default_rng(1)
    x = rng.random((len(idx), ns)).astype(np.float32)
    y = rng.random(geom.sinogram_shape).astype(np.float32)

    ax_gpu = model.sparse_forward_project(x, idx).cpu().numpy()
    ax_ref = O.sparse_forward_project(geom, x, idx)
    assert rel_l2(ax_gpu, ax_ref) <= TOL

    aty_gpu = model.sparse_back_project(y, idx).cpu().numpy()
    aty_ref = O.sparse_back_project(geom, y, idx)
    assert rel_l2(aty_gpu, aty_ref) <= TOL

    h_gpu = model.sparse_back_project(y, idx, coeff_power=2).cpu().numpy()
    h_ref = O.sparse_back_project(geom, y, idx, coeff_power=2)
    assert rel_l2(h_gpu, h_ref) <= TOL

    # the unit-weight Hessian diagonal, back-projected from no sinogram at all (the library's unit mode)
    assert rel_l2(model.compute_hessian_diagonal().cpu().numpy(), O.compute_hessian_diagonal(geom)) <= TOL

    # adjointness against the float64 oracle
    ref64 = np.sum(O.sparse_forward_project(geom, x, idx, dtype=np.float64) * y)
    lhs = np.sum(ax_gpu.astype(np.float64) * y)
    rhs = np.sum(aty_gpu.astype(np.float64) * x)
    assert abs(lhs - ref64) <= TOL * abs(ref64)
    assert abs(rhs - ref64) <= TOL * abs(ref64)


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_view_subsets_and_weights(cuda, kind):
    model, geom = make_case(kind, views=15, rows=6, channels=28)
    nr, nc, ns = geom.recon_shape
    rng = np.random.default_rng(3)
    idx = rng.permutation(nr * nc)[: nr * nc // 3].astype(np.int32)       # unsorted sparse subset
    x = rng.standard_normal((len(idx), ns)).astype(np.float32)
    y = rng.standard_normal(geom.sinogram_shape).astype(np.float32)
    w = rng.random(geom.sinogram_shape).astype(np.float32)
    views = np.array([14, 0, 7, 3, 3], dtype=np.int32)
    fp = model.sparse_forward_project(x, idx, view_indices=views).cpu().numpy()
    assert rel_l2(fp, O.sparse_forward_project(geom, x, idx, views)) <= TOL
    bp = model.sparse_back_project(y, idx, view_indices=views).cpu().numpy()
    assert rel_l2(bp, O.sparse_back_project(geom, y, idx, views)) <= TOL
    # fused weights: A^T (w * y)
    g = model._geometry()
    bw = _capi.back_project(g, torch.as_tensor(y, device='cuda'), torch.as_tensor(idx, device='cuda'),
                            weights=torch.as_tensor(w, device='cuda')).cpu().numpy()
    assert rel_l2(bw, O.sparse_back_project(geom, w * y, idx)) <= TOL


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_view_batching_consistency(cuda, kind):
    # tests/test_projectors.py:152-198: interleaved view subsets reassemble the full projection
    model, geom = make_case(kind, views=24, rows=8, channels=32)
    ns = geom.recon_shape[2]
    np.random.seed(1)
    idx = mb.gen_full_indices(geom.recon_shape)
    x = np.random.rand(len(idx), ns).astype(np.float32)
    full = model.sparse_forward_project(x, idx).cpu().numpy()
    y = full
    bp = model.sparse_back_project(y, idx).cpu().numpy()
    parts = np.zeros_like(bp)
    for j in range(5):
        v = np.arange(j, 24, 5)
        np.testing.assert_allclose(model.sparse_forward_project(x, idx, view_indices=v).cpu().numpy(), full[v],
                                   rtol=1e-6, atol=1e-6 * np.abs(full).max())
        parts += model.sparse_back_project(y, idx, view_indices=v).cpu().numpy()
    assert np.abs(parts - bp).max() <= 1e-5 * np.abs(bp).max()


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_hessian_diagonal(cuda, kind):
    model, geom = make_case(kind, views=12, rows=6, channels=24)
    h = model.compute_hessian_diagonal().cpu().numpy()
    assert rel_l2(h, O.compute_hessian_diagonal(geom)) <= TOL
    w = np.random.default_rng(0).random(geom.sinogram_shape).astype(np.float32)
    hw = model.compute_hessian_diagonal(weights=w).cpu().numpy()
    assert rel_l2(hw, O.compute_hessian_diagonal(geom, w)) <= TOL
    # finite-difference check of the Hessian (tests/test_projectors.py:264-303)
    nr, nc, ns = geom.recon_shape
    i, j, k = nr // 3, nc // 2, ns // 2
    xx = np.zeros((nr * nc, ns), dtype=np.float32)
    xx[i * nc + j, k] = 0.01
    idx = np.arange(nr * nc, dtype=np.int32)
    atax = model.sparse_back_project(model.sparse_forward_project(xx, idx), idx).cpu().numpy().reshape(nr, nc, ns)
    assert np.isclose(h[i, j, k], atax[i, j, k] / 0.01, rtol=1e-5)
    # unit weights: the library back-projects no buffer of ones; it must give what a sinogram of ones gives (for
    # parallel beam it projects one slice and writes it to every slice, which are then exactly equal)
    ones = np.ones(geom.sinogram_shape, dtype=np.float32)
    h1 = model.sparse_back_project(ones, idx, coeff_power=2).cpu().numpy().reshape(nr, nc, ns)
    assert rel_l2(h, h1) <= 1e-6
    if kind == 'parallel':
        assert np.array_equal(h, np.broadcast_to(h[:, :, :1], h.shape))


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_full_projection_reference_test_geometry(cuda, kind):
    # the reference's projector-test geometry: 64 views, 40 rows, 128 channels, cone and translation
    # sdd = sid = 512
    model, geom = make_case(kind, views=64, rows=40, channels=128)
    rng = np.random.default_rng(2)
    recon = rng.random(geom.recon_shape).astype(np.float32)
    np.random.seed(5)
    sino = model.forward_project(recon).cpu().numpy()
    np.random.seed(5)
    sino_ref = O.forward_project(geom, recon)
    assert rel_l2(sino, sino_ref) <= TOL
    bp = model.back_project(sino).cpu().numpy()
    assert rel_l2(bp, O.back_project(geom, sino_ref)) <= TOL


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_saved_and_loaded_model_projects_the_same(cuda, kind, tmp_path):
    # tests/test_projectors.py:96-145: A^T A of one pixel cylinder before and after to_file / from_file
    model, geom = make_case(kind, views=16, rows=8, channels=32)
    nr, nc, ns = geom.recon_shape
    idx = np.arange(nr * nc, dtype=np.int32)
    x = np.zeros((nr * nc, ns), np.float32)
    x[(nr // 4) * nc + nc // 3, :] = 1
    aty = model.sparse_back_project(model.sparse_forward_project(x, idx), idx).cpu().numpy()
    fn = str(tmp_path / 'model.yaml')
    model.to_file(fn)
    new = type(model).from_file(fn)
    assert mb.ParameterHandler.compare_parameter_handlers(model, new)
    aty_new = new.sparse_back_project(new.sparse_forward_project(x, idx), idx).cpu().numpy()
    assert np.allclose(aty, aty_new, atol=1e-4)


def test_edge_cases(cuda):
    model, geom = make_case('parallel', views=6, rows=4, channels=16)
    ns = geom.recon_shape[2]
    # empty pixel set: the forward projection is all zeros, the back projection empty
    empty = np.zeros(0, dtype=np.int32)
    fp = model.sparse_forward_project(np.zeros((0, ns), np.float32), empty).cpu().numpy()
    assert fp.shape == geom.sinogram_shape and not fp.any()
    assert model.sparse_back_project(np.ones(geom.sinogram_shape, np.float32), empty).shape == (0, ns)
    # duplicated pixels accumulate
    idx = np.array([5, 5, 9], dtype=np.int32)
    x = np.ones((3, ns), np.float32)
    np.testing.assert_allclose(model.sparse_forward_project(x, idx).cpu().numpy(),
                               O.sparse_forward_project(geom, x, idx), rtol=1e-5, atol=1e-6)
    # shape errors raise before any launch
    with pytest.raises(ValueError):
        model.sparse_forward_project(np.zeros((2, ns + 1), np.float32), idx[:2])
    # an out-of-range pixel index is skipped by the kernels' own bounds checks and reported
    mb._capi.get_device_error()
    bad = np.array([3, 10 ** 6], dtype=np.int32)
    out = model.sparse_forward_project(np.ones((2, ns), np.float32), bad).cpu().numpy()
    assert mb._capi.get_device_error() & 1
    np.testing.assert_allclose(out, O.sparse_forward_project(geom, np.ones((1, ns), np.float32), bad[:1]),
                               rtol=1e-5, atol=1e-6)


def test_determinism_of_back_projection(cuda):
    model, geom = make_case('cone', views=16, rows=8, channels=32)
    idx = np.arange(geom.recon_shape[0] * geom.recon_shape[1], dtype=np.int32)
    y = np.random.default_rng(0).random(geom.sinogram_shape).astype(np.float32)
    a = model.sparse_back_project(y, idx).cpu().numpy()
    b = model.sparse_back_project(y, idx).cpu().numpy()
    np.testing.assert_array_equal(a, b)   # no float atomics on the back-projection side


def test_autotuned_plans_agree_with_default(cuda):
    """Every candidate plan the autotuner can pick (forced one at a time) computes the same projections as the
    default plan, up to float summation order, and the tuned choice is reproducible call after call."""
    from mbirjax_b200 import _capi
    for kind, (v, r, c) in (('parallel', (40, 12, 96)), ('cone', (32, 24, 64)), ('parallel', (24, 40, 64))):
        model, geom = make_case(kind, views=v, rows=r, channels=c)
        nr, nc, ns = geom.recon_shape
        np.random.seed(5)
        sub = mb.gen_pixel_partition(geom.recon_shape, 3)[0]
        vox = np.random.default_rng(1).random((sub.shape[0], ns)).astype(np.float32)
        sino = np.random.default_rng(2).random(geom.sinogram_shape).astype(np.float32)
        old = _capi.set_autotune(0)
        try:
            fp0 = model.sparse_forward_project(vox, sub).cpu().numpy()
            bp0 = model.sparse_back_project(sino, sub).cpu().numpy()
            for mode in (2, 3, 1):
                _capi.set_autotune(mode)
                fp = model.sparse_forward_project(vox, sub).cpu().numpy()
                bp = model.sparse_back_project(sino, sub).cpu().numpy()
                assert rel_l2(fp, fp0) <= 1e-6, (kind, mode)
                assert rel_l2(bp, bp0) <= 1e-6, (kind, mode)
            np.testing.assert_array_equal(model.sparse_forward_project(vox, sub).cpu().numpy(), fp)
        finally:
            _capi.set_autotune(old)
        np.testing.assert_allclose(fp0, O.sparse_forward_project(geom, vox, sub), rtol=2e-4,
                                   atol=2e-5 * np.abs(fp0).max())


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_one_view_plugin_functions(cuda, kind):
    """The reference's per-view plugin functions (forward_project_pixel_batch_to_one_view /
    back_project_one_view_to_pixel_batch, with projector_params as its Projectors builds them) on a one-view
    geometry: the same view as the model's projection restricted to that view, and the oracle's one-view
    projectors, for both coefficient powers."""
    model, geom = make_case(kind, views=9, rows=6, channels=28)
    nr, nc, ns = geom.recon_shape
    rng = np.random.default_rng(11)
    idx = rng.permutation(nr * nc)[: nr * nc // 2].astype(np.int32)
    x = rng.standard_normal((len(idx), ns)).astype(np.float32)
    view = rng.standard_normal(geom.sinogram_shape[1:]).astype(np.float32)
    pp = model.get_projector_params()
    cls = type(model)
    view_params = np.asarray(model.get_params(model.get_params('view_params_name')), dtype=np.float32)
    for j in (0, 4):
        fp = cls.forward_project_pixel_batch_to_one_view(x, idx, view_params[j], pp).cpu().numpy()
        assert fp.shape == geom.sinogram_shape[1:]
        sub = model.sparse_forward_project(x, idx, view_indices=np.array([j], np.int32)).cpu().numpy()[0]
        assert rel_l2(fp, sub) <= 1e-6
        assert rel_l2(fp, O.forward_project_one_view(geom, x, idx, geom.angles[j])) <= TOL
        for power in (1, 2):
            bp = cls.back_project_one_view_to_pixel_batch(view, idx, view_params[j], pp, coeff_power=power)
            bp = bp.cpu().numpy()
            assert bp.shape == (len(idx), ns)
            assert rel_l2(bp, O.back_project_one_view(geom, view, idx, geom.angles[j], coeff_power=power)) <= TOL
