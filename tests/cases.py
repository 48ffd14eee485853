"""Geometry cases shared by the CPU and GPU tests: each builds a mbirjax_b200 model and the matching
oracle geometry from the same arguments."""
import json
import os

import numpy as np

import mbirjax_b200 as mb
import oracle as O


def angles_for(kind, num_views, num_det_channels, sdd):
    """Angle set of the reference's projector tests (tests/test_projectors.py:45-52)."""
    cone_angle = 2 * np.arctan2(num_det_channels / 2, sdd) if kind == 'cone' else 0.0
    start, end = -(np.pi + cone_angle) / 2, (np.pi + cone_angle) / 2
    return np.linspace(start, end, num_views, endpoint=False).astype(np.float32)


def translations_for(num_views, seed=0, y_spread=0.0):
    """Translation vectors of the reference's projector tests (tests/test_projectors.py:54-62): x and z uniform
    in [-10, 10], y = 0 (or uniform in [-y_spread, y_spread])."""
    rng = np.random.default_rng(seed)
    tv = np.zeros((num_views, 3))
    tv[:, 0] = rng.uniform(-10, 10, num_views)
    tv[:, 1] = rng.uniform(-y_spread, y_spread, num_views) if y_spread else 0.0
    tv[:, 2] = rng.uniform(-10, 10, num_views)
    return tv


def make_case(kind, views=16, rows=8, channels=32, sdd_factor=4.0, sid_factor=None, y_spread=0.0, **params):
    """Returns (model, oracle_geometry).  params are set on the model before the oracle geometry is derived."""
    sdd = sdd_factor * channels
    sid = sdd if sid_factor is None else sid_factor * channels
    ang = angles_for(kind, views, channels, sdd)
    if kind == 'parallel':
        model = mb.ParallelBeamModel((views, rows, channels), ang)
    elif kind == 'translation':
        model = mb.TranslationModel((views, rows, channels), translations_for(views, y_spread=y_spread),
                                    source_detector_dist=sdd, source_iso_dist=sid)
    else:
        model = mb.ConeBeamModel((views, rows, channels), ang, source_detector_dist=sdd, source_iso_dist=sid)
    if params:
        model.set_params(**params)
    return model, oracle_geometry(model)


def oracle_geometry(model):
    sino_shape, recon_shape = model.get_params(['sinogram_shape', 'recon_shape'])
    kw = dict(delta_det_channel=model.get_params('delta_det_channel'), delta_det_row=model.get_params('delta_det_row'),
              det_channel_offset=model.get_params('det_channel_offset'),
              det_row_offset=model.get_params('det_row_offset'), delta_voxel=model.get_params('delta_voxel'),
              recon_shape=recon_shape)
    if isinstance(model, mb.TranslationModel):
        return O.translation_geometry(sino_shape, model.get_params('translation_vectors'),
                                      model.get_params('source_detector_dist'), model.get_params('source_iso_dist'),
                                      delta_recon_row=model.get_params('delta_recon_row'), **kw)
    ang = np.asarray(model.get_params('angles'), dtype=np.float32)
    if isinstance(model, mb.ConeBeamModel):
        g = O.cone_geometry(sino_shape, ang, model.get_params('source_detector_dist'),
                            model.get_params('source_iso_dist'), recon_slice_offset=model.get_params('recon_slice_offset'),
                            **kw)
    else:
        g = O.parallel_geometry(sino_shape, ang, **kw)
    return g


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


# The error bounds of the reference's end-to-end tests, extracted from its test files by
# tests/golden/make_acceptance_bounds.py.
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'golden', 'acceptance_bounds.json')) as _f:
    ACCEPTANCE_BOUNDS = json.load(_f)


# The reference's FBP/FDK acceptance test (tests/test_fbp_fdk.py:14-47): 128 views of a 128 x 128 detector; parallel
# beam over [-pi/2, pi/2), cone beam over [-pi, pi) with sdd = 4 * 128 and sid = sdd / 2; the recon of the forward
# projection of the low-dynamic-range Shepp-Logan phantom must stay under these error bounds, which the reference
# sets just above its own deterministic results.
FBP_FDK_SIZE = 128
FBP_TOLERANCES = ACCEPTANCE_BOUNDS['fbp']
FDK_TOLERANCES = ACCEPTANCE_BOUNDS['fdk']


def fbp_fdk_model(kind):
    n = FBP_FDK_SIZE
    if kind == 'parallel':
        ang = np.linspace(-np.pi / 2, np.pi / 2, n, endpoint=False).astype(np.float32)
        return mb.ParallelBeamModel((n, n, n), ang)
    sdd = 4 * n
    ang = np.linspace(-np.pi, np.pi, n, endpoint=False).astype(np.float32)
    return mb.ConeBeamModel((n, n, n), ang, source_detector_dist=sdd, source_iso_dist=sdd / 2)


def recon_error_stats(recon, phantom):
    """max |x - x_true|, ||x - x_true|| / ||x_true|| and the 95th percentile of |x - x_true|, as the reference's
    test computes them."""
    recon, phantom = np.asarray(recon), np.asarray(phantom)
    err = np.abs(recon - phantom)
    return {'max_diff': float(np.amax(err)), 'nrmse': float(np.linalg.norm(recon - phantom) / np.linalg.norm(phantom)),
            'pct_95': float(np.percentile(err, 95))}


# The reference's VCD acceptance test (tests/test_vcd.py:16-45, 80-120): 64 views of a 40 x 128 detector, angles of
# the projector tests, cone beam with sdd = sid = 4 * 128, the model's default recon (sharpness 1, multi-granular
# partitions, at most 15 iterations, stop at 0.2%) of the forward projection of the Shepp-Logan phantom.
VCD_TOLERANCES = ACCEPTANCE_BOUNDS['vcd']


def vcd_acceptance_model(kind):
    views, rows, channels = 64, 40, 128
    sdd = 4 * channels
    ang = angles_for(kind, views, channels, sdd)
    if kind == 'parallel':
        return mb.ParallelBeamModel((views, rows, channels), ang)
    return mb.ConeBeamModel((views, rows, channels), ang, source_detector_dist=sdd, source_iso_dist=sdd)
