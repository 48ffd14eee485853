"""CPU tests of the host side: the C-ABI library loads and exports every declared symbol, argument validation
returns error codes without touching a GPU, and the host logic (parameters, geometry radii, partitions,
auto-regularisation) matches the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

import mbirjax_b200 as mb
from mbirjax_b200 import _capi
import oracle as O
from cases import make_case, oracle_geometry

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, 'include', 'mbirjax_b200.h')).read()
    return sorted(set(re.findall(r'^MBX_API [^;(]*?\b(mbx_\w+)\s*\(', text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    lib = _capi.load_library()
    declared = _declared_symbols()
    assert len(declared) >= 14
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(_capi.exported_symbols()) == declared
    assert 'sm_100a' in _capi.version()


def test_invalid_arguments_return_error_codes():
    lib = _capi.load_library()
    g = _capi.MbxGeom()
    assert lib.mbx_sparse_forward_project(ctypes.byref(g), None, None, 0, None, 1, None, None, 0, None) == -1
    assert lib.mbx_sparse_back_project(None, None, None, None, 0, None, 1, 1, 1.0, None, None, 0, None) == -1
    assert lib.mbx_direct_filter(None, None, None, None) == -1
    assert lib.mbx_error_string(-4).decode().startswith('workspace')
    g.kind, g.num_views, g.num_det_rows, g.num_det_channels = 0, 4, 2, 8
    g.num_recon_rows = g.num_recon_cols = 8
    g.num_recon_slices = 2
    g.delta_det_channel = g.delta_det_row = g.delta_voxel = 1.0
    g.psf_radius = 7  # above MBX_MAX_PSF_RADIUS
    g.angles = 1
    assert lib.mbx_sparse_forward_project(ctypes.byref(g), None, None, 0, None, 1, 1, None, 0, None) == -2


def test_compute_without_gpu_fails_loudly(monkeypatch):
    import torch
    if torch.cuda.is_available():
        pytest.skip('GPU present')
    model, _ = make_case('parallel')
    with pytest.raises(mb.MbxError):
        model.forward_project(np.zeros(model.get_params('recon_shape'), dtype=np.float32))


@pytest.mark.parametrize('kind,kw', [('parallel', {}), ('cone', {}), ('cone', {'sid_factor': 2.0}),
                                     ('parallel', {'delta_voxel': 2.5}), ('cone', {'delta_voxel': 3.0}),
                                     ('translation', {}), ('translation', {'sid_factor': 2.0}),
                                     ('translation', {'y_spread': 4.0})])
def test_geometry_matches_oracle(kind, kw):
    model, geom = make_case(kind, views=8, rows=10, channels=40, **kw)
    gp = model.get_geometry_parameters()
    assert gp.psf_radius == geom.psf_radius
    if kind == 'cone':
        assert gp.bp_psf_radius == geom.bp_psf_radius
        assert model.get_magnification() == pytest.approx(geom.magnification)
    # default recon sizes (parallel_beam.py:125-136, cone_beam.py:174-187, translation_model.py:142-186)
    m2, g2 = make_case(kind, views=8, rows=10, channels=40)
    assert tuple(m2.get_params('recon_shape')) == tuple(g2.recon_shape)
    if kind == 'translation':  # the oracle derives recon size, row pitch and psf radius on its own
        g3 = O.translation_geometry(m2.get_params('sinogram_shape'), m2.get_params('translation_vectors'),
                                    m2.get_params('source_detector_dist'), m2.get_params('source_iso_dist'))
        assert tuple(g3.recon_shape) == tuple(m2.get_params('recon_shape'))
        assert g3.delta_recon_row == m2.get_params('delta_recon_row')
        assert g3.psf_radius == m2.get_geometry_parameters().psf_radius


@pytest.mark.parametrize('y_spread,sid_factor', [(0.0, None), (6.0, None), (3.0, 2.0)])
def test_translation_magnification_bound_covers_every_pixel_and_view(y_spread, sid_factor):
    # the fast back projector sizes its detector-row cache from this bound: it must hold for every pixel row and
    # every view's ty (mag = 1 / (1/M - y/D), y = delta_recon_row (row - (Nr-1)/2) - ty)
    model, geom = make_case('translation', views=14, rows=8, channels=32, y_spread=y_spread, sid_factor=sid_factor)
    bound = model._max_magnification()
    nr = geom.recon_shape[0]
    rows = np.arange(nr)
    for tv in geom.angles:
        y = geom.delta_recon_row * (rows - (nr - 1) / 2.0) - float(tv[1])
        mag = 1.0 / (1.0 / geom.magnification - y / geom.source_detector_dist)
        assert np.all(mag > 0) and np.all(mag <= bound)
    assert bound <= 1.01 * np.max(1.0 / (1.0 / geom.magnification - (geom.delta_recon_row * (nr - 1) / 2.0 -
                                                                      np.min(geom.angles[:, 1])) /
                                         geom.source_detector_dist))


def test_translation_model_reference_geometry():
    """The geometry TranslationModel derives for the reference's VCD test setup (tests/test_vcd.py:27-64:
    40 rows x 128 channels, source at 512 = detector distance, a 7 x 7 raster of translations 22 ALU apart,
    one view per translation), worked out by hand from translation_model.py:109-186: half cone angle
    atan(128 / 1024), row pitch sqrt(2) * 8, a box of (132 + 64) x (132 + 20) voxels,
    ceil(49 * 128 * 40 / (196 * 152)) = 9 rows."""
    from mbirjax_b200.utilities import gen_translation_vectors
    tv = gen_translation_vectors(7, 7, 22, 22)
    model = mb.TranslationModel((49, 40, 128), tv, source_detector_dist=512, source_iso_dist=512)
    assert model.get_params('delta_recon_row') == pytest.approx(np.sqrt(2) * 8, rel=1e-6)
    assert tuple(model.get_params('recon_shape')) == (9, 196, 152)
    assert model.get_geometry_parameters().psf_radius == 1
    assert list(model.get_params('qggmrf_nbr_wts')) == [0.5, 1, 1]
    assert model.use_ror_mask  # reset to True by the base constructor, as in the reference
    with pytest.raises(ValueError):
        mb.TranslationModel((48, 40, 128), tv, source_detector_dist=512, source_iso_dist=512)
    with pytest.raises(ValueError):
        mb.TranslationModel((49, 40, 128), tv, source_detector_dist=np.inf, source_iso_dist=512)


def test_set_params_semantics():
    model, _ = make_case('parallel')
    with pytest.raises(ValueError):
        model.set_params(not_a_param=1)
    with pytest.warns(UserWarning):
        model.set_params(sigma_x=0.5)
    assert model.get_params('auto_regularize_flag') is False
    with pytest.warns(UserWarning):
        model.set_params(sharpness=0.0)
    assert model.get_params('auto_regularize_flag') is True
    with pytest.raises(ValueError):
        model.set_params(recon_shape=(32, 32, 5))  # slices must equal det rows for parallel beam


def test_partitions_reproduce_oracle_stream():
    shape = (37, 37, 4)
    np.random.seed(11)
    a = mb.gen_set_of_pixel_partitions(shape, [1, 4, 7])
    a_perm = np.random.permutation(4)
    np.random.seed(11)
    b = O.gen_set_of_pixel_partitions(shape, [1, 4, 7])
    b_perm = np.random.permutation(4)
    for x, y in zip(a, b):
        np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(a_perm, b_perm)
    np.testing.assert_array_equal(mb.get_2d_ror_mask(shape), O.get_2d_ror_mask(shape))


def test_morton_sorted_partition_keeps_each_subset():
    """The processing order the projectors get is a per-subset permutation: same sets, Z-order within each."""
    from mbirjax_b200.vcd_utils import morton_sorted_partition
    np.random.seed(3)
    part = mb.gen_pixel_partition((61, 45, 2), 5)
    srt = morton_sorted_partition(part, 45)
    assert srt.shape == part.shape and srt.dtype == np.int32
    for a, b in zip(part, srt):
        np.testing.assert_array_equal(np.sort(a), np.sort(b))
    # consecutive entries are close in the image: mean step far below a row-major walk's
    r, c = np.divmod(srt[0].astype(np.int64), 45)
    assert np.mean(np.abs(np.diff(r)) + np.abs(np.diff(c))) < 6.0


def test_prefetched_regularisation_views_give_the_same_statistics():
    # the batched set-up hands auto_set_regularization_params the ~20 views it reads (copied to the host up
    # front); subsampling that subsample again selects every view of it, so the statistics are the same
    import torch
    from mbirjax_b200.batched import _view_subsample
    for views in (7, 20, 39, 40, 123, 720):
        model, _ = make_case('parallel', views=views, rows=4, channels=24)
        rng = np.random.default_rng(views)
        sino = rng.random(model.get_params('sinogram_shape')).astype(np.float32)
        w = rng.random(model.get_params('sinogram_shape')).astype(np.float32)
        full = model.auto_set_regularization_params(sino, weights=w)
        sub = model.auto_set_regularization_params(_view_subsample(torch.as_tensor(sino)),
                                                   weights=_view_subsample(w))
        assert sub == full


def test_zorder_sort_matches_sorting_by_code():
    # the cached rank-table sort gives the order of sorting each subset by its Morton code, repeats included
    from mbirjax_b200.vcd_utils import morton_order, morton_sorted_partition
    for shape, k in (((61, 45, 2), 5), ((96, 512, 1), 3), ((5, 7, 1), 2)):
        np.random.seed(4)
        part = mb.gen_pixel_partition(shape, k)
        want = np.stack([p[morton_order(p, shape[1])] for p in part])
        np.testing.assert_array_equal(morton_sorted_partition(part, shape[1]), want)
    rep = np.array([[3, 3, 1, 8], [2, 5, 7, 0]], dtype=np.int32)
    np.testing.assert_array_equal(morton_sorted_partition(rep, 4),
                                  np.stack([p[morton_order(p, 4)] for p in rep]))


def test_full_indices_draw_as_a_one_subset_partition():
    # repeated calls return the sorted region of reconstruction and leave np.random where the reference's
    # one-subset partition (a permutation of N) leaves it, so later partitions are the reference's
    for shape, mask in (((40, 40, 3), True), ((17, 23, 2), False)):
        for seed in (0, 1):
            np.random.seed(seed)
            a = [O.gen_full_indices(shape, mask) for _ in range(3)]
            after_oracle = np.random.permutation(10)
            np.random.seed(seed)
            b = [mb.gen_full_indices(shape, mask) for _ in range(3)]
            after = np.random.permutation(10)
            for x, y in zip(a, b):
                np.testing.assert_array_equal(x, y)
            np.testing.assert_array_equal(after, after_oracle)
    b[0][0] = -1  # results are copies: the kept set is not changed by a caller
    np.testing.assert_array_equal(mb.gen_full_indices((17, 23, 2), False), a[0])


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_auto_regularization_matches_oracle(kind):
    model, geom = make_case(kind, views=40, rows=6, channels=32)
    rng = np.random.default_rng(5)
    sino = rng.random(geom.sinogram_shape).astype(np.float32)
    sino[:, :, :4] = 0
    w = rng.random(geom.sinogram_shape).astype(np.float32)
    model.set_params(sharpness=0.0, snr_db=30.0)
    reg = model.auto_set_regularization_params(sino, weights=w)
    sy, sx, sp = O.auto_regularization(geom, sino, w, snr_db=30.0, sharpness=0.0)
    assert reg['sigma_y'] == pytest.approx(sy, rel=1e-7)
    assert reg['sigma_x'] == pytest.approx(sx, rel=1e-7)
    assert reg['sigma_prox'] == pytest.approx(sp, rel=1e-7)


def test_qggmrf_b_weights():
    assert mb.get_b_from_nbr_wts([1.0, 2.0, 3.0]) == pytest.approx(O.get_b_from_nbr_wts([1.0, 2.0, 3.0]))


def test_batched_scan_shapes_are_in_range():
    from mbirjax_b200.utilities import batched_scan_shapes
    shapes = batched_scan_shapes()
    assert len(shapes) == 24
    for v, r, c in shapes:
        assert 60 <= v <= 720 and 8 <= r <= 64 and 96 <= c <= 512


def _host_device(monkeypatch):
    """Point the models' device at the CPU, so the host logic up to the CUDA library runs here (the library
    refuses host tensors before any launch)."""
    import torch
    import mbirjax_b200.tomography_model as tm
    monkeypatch.setattr(tm, '_cuda_device', lambda: torch.device('cpu'))
    return tm


@pytest.mark.parametrize('kind', ['parallel', 'cone', 'translation'])
def test_one_view_geometry_matches_the_model_record(monkeypatch, kind):
    """The per-view plugin functions (forward_project_pixel_batch_to_one_view / back_project_one_view_to_pixel_batch)
    build, from the reference's projector_params and one view's angle or translation, the same geometry record as
    the model's own projections, with one view."""
    tm = _host_device(monkeypatch)
    extra = {'det_channel_offset': 0.25} if kind == 'parallel' else {'det_channel_offset': 0.25, 'det_row_offset': -0.5}
    model, _ = make_case(kind, views=6, rows=4, channels=20, y_spread=2.0 if kind == 'translation' else 0.0, **extra)
    full = model._geometry()
    view_params = np.asarray(model.get_params(model.get_params('view_params_name')), dtype=np.float32)
    g, view_dev = tm.one_view_geometry(model._kind(), model.get_projector_params(), view_params[2])
    for name, _ in _capi.MbxGeom._fields_:
        if name not in ('num_views', 'angles', 'translations', 'max_magnification'):
            assert getattr(g, name) == getattr(full, name), name
    assert g.num_views == 1
    assert (g.translations if kind == 'translation' else g.angles) == view_dev.data_ptr()
    np.testing.assert_array_equal(view_dev.numpy().reshape(-1), view_params[2].reshape(-1))
    if kind == 'translation':
        gp = model.get_geometry_parameters()
        assert g.max_magnification == pytest.approx(tm.translation_max_magnification(
            gp.delta_recon_row, model.get_params('recon_shape')[0], view_params[2, 1], gp.magnification,
            gp.source_detector_dist), rel=1e-6)
        assert 0 < g.max_magnification <= full.max_magnification   # one view's bound within all views'


def test_one_view_plugin_functions_check_their_arguments(monkeypatch):
    tm = _host_device(monkeypatch)
    model, _ = make_case('parallel', views=6, rows=4, channels=20)
    pp = model.get_projector_params()
    nr, nc, ns = model.get_params('recon_shape')
    fp = mb.ParallelBeamModel.forward_project_pixel_batch_to_one_view
    bp = mb.ParallelBeamModel.back_project_one_view_to_pixel_batch
    idx = np.arange(5, dtype=np.int32)
    with pytest.raises(ValueError):
        fp(np.zeros((5, ns + 1), np.float32), idx, 0.3, pp)              # slices do not match the recon
    with pytest.raises(ValueError):
        fp(np.zeros((4, ns), np.float32), idx, 0.3, pp)                  # one cylinder per index
    with pytest.raises(ValueError):
        fp(np.zeros((5, ns), np.float32), idx, np.zeros(2), pp)          # one angle per view
    with pytest.raises(ValueError):
        bp(np.zeros((4, 21), np.float32), idx, 0.3, pp)                  # (rows, channels) of the detector
    with pytest.raises(ValueError):
        bp(np.zeros((4, 20), np.float32), idx, 0.3, pp, coeff_power=3)
    tmodel, _ = make_case('translation', views=6, rows=4, channels=20)
    with pytest.raises(ValueError):
        mb.TranslationModel.forward_project_pixel_batch_to_one_view(
            np.zeros((5, tmodel.get_params('recon_shape')[2]), np.float32), idx, np.zeros(2),
            tmodel.get_projector_params())
    # valid arguments reach the CUDA library, which refuses host tensors before any launch
    with pytest.raises(mb.MbxError):
        fp(np.zeros((5, ns), np.float32), idx, 0.3, pp)
    with pytest.raises(mb.MbxError):
        bp(np.zeros((4, 20), np.float32), idx, 0.3, pp, coeff_power=2)
    # the base class has no projector: it warns and returns None, as the reference's
    with pytest.warns(UserWarning):
        assert mb.TomographyModel.forward_project_pixel_batch_to_one_view(None, None, None, pp) is None
    with pytest.warns(UserWarning):
        assert mb.TomographyModel.back_project_one_view_to_pixel_batch(None, None, None, pp) is None


def test_translation_phantoms(monkeypatch):
    """gen_translation_phantom (utilities.py:696-825 of the reference): 'dots' seeds np.random with 42 and fills
    the middle rows with exactly int(cols * slices * fill_rate) distinct ones each; 'text' needs a TrueType font
    and says so when there is none; other options are refused."""
    from mbirjax_b200.utilities import gen_translation_phantom
    shape = (12, 10, 8)
    p = gen_translation_phantom(shape, 'dots', None, fill_rate=0.25)
    assert p.dtype == np.float32 and p.shape == shape
    assert set(np.unique(p)) <= {0.0, 1.0}
    counts = p.reshape(12, -1).sum(axis=1)
    np.testing.assert_array_equal(counts, [0, 0] + [20] * 8 + [0, 0])       # pad 12 // 6 = 2 rows each side
    after = np.random.rand()
    np.testing.assert_array_equal(gen_translation_phantom(shape, 'dots', None, fill_rate=0.25), p)
    assert np.random.rand() == after                                          # same draws from seed 42 each call
    with pytest.raises(ValueError):
        gen_translation_phantom(shape, 'squares', None)
    try:
        t = gen_translation_phantom((40, 48, 48), 'text', ['ab', 'cd'], font_size=12)
    except FileNotFoundError as e:
        assert 'font' in str(e)                                                  # no TrueType font on this machine
    else:
        assert t.shape == (40, 48, 48) and set(np.unique(t)) <= {0.0, 1.0}
    # the rendering itself, with PIL's built-in scalable font standing in for a TrueType file
    from PIL import ImageFont
    builtin = ImageFont.load_default(size=12)
    monkeypatch.setattr(ImageFont, 'truetype', lambda *args, **kwargs: builtin)
    t = gen_translation_phantom((40, 48, 48), 'text', ['ab', 'cd'], font_size=12)
    assert t.shape == (40, 48, 48) and set(np.unique(t)) <= {0.0, 1.0}
    assert np.flatnonzero(t.reshape(40, -1).sum(axis=1)).tolist() == [13, 26]   # rows 40 // 3 * (1, 2)
    cols, slices = np.nonzero(t[13])
    assert 10 < cols.mean() < 38 and 10 < slices.mean() < 38                       # centred in the plane


def test_geometry_validation_as_the_reference():
    """verify_valid_params of the geometries (parallel_beam.py:72-92, cone_beam.py:82-108): one angle per view, a
    parallel recon with one slice per detector row, and a warning (not an error) for a cone angle over 45
    degrees."""
    with pytest.raises(ValueError, match='view dependent'):
        mb.ParallelBeamModel((8, 4, 16), np.zeros(7))
    with pytest.raises(ValueError, match='view dependent'):
        mb.ConeBeamModel((8, 4, 16), np.zeros(9), source_detector_dist=64, source_iso_dist=32)
    with pytest.warns(UserWarning, match='45 degrees'):
        mb.ConeBeamModel((8, 40, 16), np.zeros(8), source_detector_dist=10, source_iso_dist=5)
    model = mb.ParallelBeamModel((8, 4, 16), np.zeros(8))
    with pytest.raises(ValueError, match='slices'):
        model.set_params(recon_shape=(16, 16, 5))


def test_partition_draws_from_a_random_state_are_the_global_stream():
    """np.random.seed(s) followed by the global draws is the stream RandomState(s): partitions and region-of-
    reconstruction draws from an explicit RandomState equal the seeded global ones, and leave it in the same
    state."""
    shape = (37, 41, 3)
    for seed in (0, 5):
        np.random.seed(seed)
        want = mb.gen_pixel_partition(shape, 4)
        mb.gen_full_indices(shape)
        mb.gen_full_indices(shape)
        want_state = np.random.get_state()[1]
        rs = np.random.RandomState(seed)
        got = mb.gen_pixel_partition(shape, 4, rng=rs)
        mb.gen_full_indices(shape, rng=rs)
        mb.gen_full_indices(shape, rng=rs)
        np.testing.assert_array_equal(got, want)
        np.testing.assert_array_equal(rs.get_state()[1], want_state)


def test_batched_host_draws_on_threads_match_the_sequential_stream():
    """The batched path's host part with per-scan seeds (threads, one RandomState each) gives what the plain path
    draws scan after scan from the seeded global stream, and leaves the global stream where the plain path does."""
    from mbirjax_b200.batched import BatchedVCD, _view_subsample
    from mbirjax_b200.vcd_utils import morton_sorted_partition
    shapes = [(30, 6, 40), (24, 9, 36), (40, 4, 52)]
    models, sinos = [], []
    rng = np.random.default_rng(0)
    for v, r, c in shapes:
        m = mb.ParallelBeamModel((v, r, c), np.linspace(0, np.pi, v, endpoint=False).astype(np.float32))
        m.set_params(sharpness=0.0, granularity=[4], partition_sequence=[0], verbose=0)
        models.append(m)
        sinos.append(rng.random((v, r, c)).astype(np.float32))
    seeds = [3, 8, 5]
    b = BatchedVCD(models, sinos, seeds=seeds)
    small, small_w = b._host_subsamples()
    regs, parts, sched, fms, qps, sigmas = b._host_draws(4, small, small_w)
    end_state = np.random.get_state()[1].copy()
    for i, (m, sd) in enumerate(zip(models, seeds)):
        np.random.seed(sd)
        reg = m.auto_set_regularization_params(_view_subsample(sinos[i]))
        shape = m.get_params('recon_shape')
        part = mb.gen_set_of_pixel_partitions(shape, [4])[0]
        mb.gen_full_indices(shape)
        mb.gen_full_indices(shape)
        order = np.stack([np.random.permutation(4) for _ in range(4)])
        assert reg == regs[i]
        np.testing.assert_array_equal(parts[i], morton_sorted_partition(part, shape[1]))
        np.testing.assert_array_equal(sched.reshape(4, 4, len(models))[:, :, i], order)
        assert fms[i] == pytest.approx(1.0 / reg['sigma_y'] ** 2)
    np.testing.assert_array_equal(np.random.get_state()[1], end_state)
