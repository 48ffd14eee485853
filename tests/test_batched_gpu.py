"""Batched VCD (persistent work-list kernels over many scans, all iterations in one CUDA graph) against the
plain per-scan path and the oracle: same partitions, subset orders and qGGMRF parameters."""
import numpy as np
import pytest
import torch

import mbirjax_b200 as mb
from mbirjax_b200.batched import BatchedVCD, morton_order
from mbirjax_b200.utilities import gen_ellipsoid_phantom
import oracle as O
from cases import rel_l2

pytestmark = pytest.mark.gpu


def _scan(kind, views, rows, channels, seed):
    ang = np.linspace(0, np.pi if kind == 'parallel' else 2 * np.pi, views, endpoint=False).astype(np.float32)
    if kind == 'parallel':
        model = mb.ParallelBeamModel((views, rows, channels), ang)
        geom = O.parallel_geometry((views, rows, channels), ang)
    else:
        model = mb.ConeBeamModel((views, rows, channels), ang, 4.0 * channels, 4.0 * channels)
        geom = O.cone_geometry((views, rows, channels), ang, 4.0 * channels, 4.0 * channels)
    model.set_params(sharpness=0.0, granularity=[4], partition_sequence=[0], verbose=0)
    ph = gen_ellipsoid_phantom(geom.recon_shape, 5, seed).numpy()
    np.random.seed(seed)
    sino = O.forward_project(geom, ph)
    sino = (sino + np.random.default_rng(seed).normal(0, 0.01 * np.abs(sino).max(), sino.shape)).astype(np.float32)
    return model, geom, sino


def _plain(model, sino, seed, iters, w=None):
    np.random.seed(seed)
    rec, d = model.recon(sino, weights=w, max_iterations=iters, stop_threshold_change_pct=0, logfile_path=None,
                         print_logs=False)
    return rec.cpu().numpy(), d


@pytest.mark.parametrize('use_graph', [True, False])
def test_batched_matches_plain_and_oracle(cuda, use_graph):
    shapes = [(40, 6, 48), (23, 9, 37), (61, 4, 64)]
    seeds = [3, 4, 5]
    items = [_scan('parallel', v, r, c, sd) for (v, r, c), sd in zip(shapes, seeds)]
    models = [it[0] for it in items]
    sinos = [it[2] for it in items]
    recons, dicts = BatchedVCD(models, sinos, seeds=seeds).recon(max_iterations=4, use_graph=use_graph)
    for (model, geom, sino), rec, d, sd in zip(items, recons, dicts, seeds):
        plain, pd = _plain(model, sino, sd, 4)
        assert rel_l2(rec.cpu().numpy(), plain) <= 1e-5
        np.testing.assert_allclose(d['fm_rmse'], pd['recon_params']['fm_rmse'], rtol=1e-4)
        np.testing.assert_allclose(d['alpha_values'], pd['recon_params']['alpha_values'], rtol=1e-4)
    # one scan against the oracle
    model, geom, sino = items[0]
    np.random.seed(seeds[0])
    ref, _ = O.vcd.recon(geom, sino, granularity=[4], partition_sequence=[0], max_iterations=4, sharpness=0.0,
                         stop_threshold_change_pct=0)
    assert rel_l2(recons[0].cpu().numpy(), ref) <= 1e-4


def test_batched_cone_with_weights(cuda):
    items = [_scan('cone', 24, 6, 32, 7), _scan('cone', 30, 8, 28, 8)]
    models = [it[0] for it in items]
    sinos = [it[2] for it in items]
    ws = [np.exp(-s / s.max()).astype(np.float32) for s in sinos]
    recons, dicts = BatchedVCD(models, sinos, weights=ws, seeds=[7, 8]).recon(max_iterations=3)
    for (model, geom, sino), w, rec, sd in zip(items, ws, recons, [7, 8]):
        plain, _ = _plain(model, sino, sd, 3, w)
        assert rel_l2(rec.cpu().numpy(), plain) <= 1e-5


def test_batched_translation_matches_plain(cuda):
    """Translation scans in one batch: zero initialisation as TranslationModel.recon, the same partition and subset
    draws, and the translation kernels of the batched stages give the plain path's reconstructions."""
    from cases import translations_for
    items = []
    for views, rows, channels, seed in ((12, 6, 24, 2), (16, 8, 28, 3)):
        model = mb.TranslationModel((views, rows, channels), translations_for(views, seed=seed),
                                    source_detector_dist=4.0 * channels, source_iso_dist=4.0 * channels)
        model.set_params(sharpness=0.0, granularity=[4], partition_sequence=[0], verbose=0)
        shape = tuple(model.get_params('recon_shape'))
        ph = gen_ellipsoid_phantom(shape, 4, seed).numpy()
        sino = model.forward_project(torch.as_tensor(ph, device='cuda')).cpu().numpy()
        items.append((model, sino, seed))
    models, sinos, seeds = [it[0] for it in items], [it[1] for it in items], [it[2] for it in items]
    with pytest.warns(UserWarning):  # no direct recon for translation geometry: the init is zeros
        recons, _ = BatchedVCD(models, sinos, seeds=seeds).recon(max_iterations=3)
    for (model, sino, sd), rec in zip(items, recons):
        np.random.seed(sd)
        with pytest.warns(UserWarning):
            plain, _ = model.recon(sino, max_iterations=3, stop_threshold_change_pct=0, logfile_path=None,
                                   print_logs=False)
        assert rel_l2(rec.cpu().numpy(), plain.cpu().numpy()) <= 1e-5


def test_morton_order_is_a_permutation():
    idx = np.sort(np.random.default_rng(0).choice(64 * 64, 500, replace=False)).astype(np.int32)
    o = morton_order(idx, 64)
    assert sorted(o.tolist()) == list(range(500))


def test_batched_alternative_plans_match_default(cuda):
    """The batched stages with the alternative projector plans the autotuner can choose (forced) give the same
    reconstruction as with the default plans."""
    from mbirjax_b200 import _capi
    shapes, seeds = [(30, 6, 40), (26, 20, 48)], [7, 8]
    out = {}
    for mode in (0, 2):
        old = _capi.set_autotune(mode)
        try:
            items = [_scan('parallel', v, r, c, sd) for (v, r, c), sd in zip(shapes, seeds)]
            recons, _ = BatchedVCD([it[0] for it in items], [it[2] for it in items], seeds=seeds).recon(max_iterations=3)
            out[mode] = [x.cpu().numpy() for x in recons]
        finally:
            _capi.set_autotune(old)
    for a, b in zip(out[0], out[2]):
        assert rel_l2(b, a) <= 1e-5


def test_planned_forward_projections_match_the_walk(cuda):
    """The planned forward projections (each subset's sorted record passes stored once per reconstruction and
    replayed every iteration) reconstruct bit for bit what the walk (scan and sort every time) does, and a repeated
    planned recon is bit for bit the same."""
    from mbirjax_b200 import batched as B
    shapes, seeds = [(40, 6, 48), (23, 9, 37), (61, 4, 64)], [3, 4, 5]
    out = {}
    old = B.PLAN_FORWARD
    try:
        items = [_scan('parallel', v, r, c, sd) for (v, r, c), sd in zip(shapes, seeds)]
        for planned in (False, True):
            B.PLAN_FORWARD = planned
            B.release_batched_sessions()
            recons, _ = BatchedVCD([it[0] for it in items], [it[2] for it in items], seeds=seeds).recon(max_iterations=3)
            sess = next(iter(B._SESSIONS.values()))
            assert sess.planned_forward == planned
            out[planned] = [r.cpu() for r in recons]
        again, _ = BatchedVCD([it[0] for it in items], [it[2] for it in items], seeds=seeds).recon(max_iterations=3)
    finally:
        B.PLAN_FORWARD = old
        B.release_batched_sessions()
    for a, b, c in zip(out[False], out[True], again):
        assert torch.equal(a, b)
        assert torch.equal(b, c.cpu())


def test_unplanned_tiles_are_walked_by_the_replay(cuda):
    """A tile whose records need more stored passes than a plan holds (here every view of a 1280 x 1280 recon seen by a
    128-channel detector: about 166 000 pixels in its one channel block, over 80 passes) is walked by the replay
    kernel in the replay's shared memory with smaller passes; the recon matches the one without planned
    projections (to float summation order: the passes differ)."""
    from mbirjax_b200 import batched as B
    views, rows, channels = 12, 4, 128
    ang = np.linspace(0, np.pi, views, endpoint=False).astype(np.float32)
    model = mb.ParallelBeamModel((views, rows, channels), ang)
    model.set_params(recon_shape=(1280, 1280, rows), sharpness=0.0, granularity=[1], partition_sequence=[0],
                     verbose=0)
    rng = np.random.default_rng(9)
    sino = rng.random((views, rows, channels)).astype(np.float32)
    out = {}
    old = B.PLAN_FORWARD
    try:
        for planned in (False, True):
            B.PLAN_FORWARD = planned
            B.release_batched_sessions()
            recons, _ = BatchedVCD([model], [sino], seeds=[2]).recon(max_iterations=2)
            assert next(iter(B._SESSIONS.values())).planned_forward == planned
            out[planned] = recons[0].cpu().numpy()
    finally:
        B.PLAN_FORWARD = old
        B.release_batched_sessions()
    assert rel_l2(out[True], out[False]) <= 1e-6
    assert np.abs(out[False]).max() > 0


def test_graph_replays_count_their_kernels(cuda):
    """Every replay of the batched graphs adds the kernels its capture recorded to batched.replayed_launches(), so
    that a benchmark counting library launches sees the replayed ones too."""
    from mbirjax_b200 import batched as B
    items = [_scan('parallel', v, r, c, sd) for (v, r, c), sd in zip([(30, 6, 40), (26, 5, 44)], [1, 2])]
    args = ([it[0] for it in items], [it[2] for it in items])
    BatchedVCD(*args, seeds=[1, 2]).recon(max_iterations=2)  # builds the session and captures its graphs
    n0 = B.replayed_launches()
    BatchedVCD(*args, seeds=[1, 2]).recon(max_iterations=2)
    sess = next(s for s in B._SESSIONS.values() if s.max_iterations == 2)
    assert B.replayed_launches() - n0 == sess.setup_kernels + sess.iter_kernels > 2 * 8
