"""Geometry records for the oracle (test infrastructure only).

Restates how the reference derives the projector parameters from the model parameters:

* parallel beam: ``parallel_beam.py:94-136`` (geometry params, psf radius, auto recon size);
* cone beam: ``cone_beam.py:68-80`` (magnification), ``cone_beam.py:110-187`` (geometry params,
  psf / bp_psf radii, auto recon size);
* translation: ``translation_model.py:69-81`` (magnification), ``translation_model.py:83-186`` (geometry
  params, psf radius, auto recon size with the ``delta_recon_row`` heuristic);
* default ``delta_voxel = delta_det_channel / magnification``: ``tomography_model.py:59-64``.

Scalars that the reference computes with ``jnp`` on Python floats are float32 there (JAX x64 is off),
so they are computed in float32 here too.
"""
from dataclasses import dataclass, field
import math

import numpy as np

F32 = np.float32


@dataclass
class OracleGeometry:
    kind: str                      # 'parallel', 'cone' or 'translation'
    sinogram_shape: tuple          # (views, det_rows, det_channels)
    recon_shape: tuple             # (rows, cols, slices)
    angles: np.ndarray             # (views,) float32 angles, or (views, 3) float32 translation vectors
    delta_det_channel: float = 1.0
    delta_det_row: float = 1.0
    det_channel_offset: float = 0.0
    det_row_offset: float = 0.0
    delta_voxel: float = 1.0
    recon_slice_offset: float = 0.0
    source_detector_dist: float = math.inf
    source_iso_dist: float = math.inf
    magnification: float = 1.0
    psf_radius: int = 1
    bp_psf_radius: int = 1
    entries_per_cylinder_batch: int = 128
    extra: dict = field(default_factory=dict)
    delta_recon_row: float = 1.0   # translation only


def _parallel_psf_radius(delta_det_channel, delta_voxel):
    # parallel_beam.py:115-123
    return int(np.ceil(np.ceil(F32(delta_voxel) / F32(delta_det_channel)) / F32(2)))


def _cone_psf_radii(delta_det_row, delta_det_channel, source_detector_dist, magnification, recon_shape,
                    delta_voxel):
    # cone_beam.py:138-172
    delta_det = F32(min(delta_det_row, delta_det_channel))
    if math.isinf(source_detector_dist):
        max_mag = F32(1)
        min_mag = F32(1)
    else:
        sid = F32(source_detector_dist) / F32(magnification)
        rmax = F32(max(recon_shape[0], recon_shape[1])) * F32(delta_voxel)
        max_mag = F32(source_detector_dist) / (sid - rmax)
        min_mag = F32(source_detector_dist) / (sid + rmax)
    psf = int(np.ceil(np.ceil(F32(delta_voxel) * max_mag / delta_det) / F32(2)))
    max_voxels_per_detector = delta_det / (min_mag * F32(delta_voxel))
    bp_psf = int(np.ceil(np.ceil(max_voxels_per_detector) / F32(2)))
    return psf, bp_psf


def parallel_geometry(sinogram_shape, angles, *, delta_det_channel=1.0, delta_det_row=1.0,
                      det_channel_offset=0.0, det_row_offset=0.0, delta_voxel=None, recon_shape=None):
    views, rows, channels = sinogram_shape
    if delta_voxel is None:
        delta_voxel = delta_det_channel  # magnification 1, tomography_model.py:59-64
    if recon_shape is None:
        # parallel_beam.py:125-136
        nr = int(math.ceil(channels * delta_det_channel / (delta_voxel * 1.0)))
        ns = int(round(rows * ((delta_det_row / delta_voxel) / 1.0)))
        recon_shape = (nr, nr, ns)
    return OracleGeometry('parallel', tuple(sinogram_shape), tuple(recon_shape),
                          np.asarray(angles, dtype=F32), delta_det_channel, delta_det_row,
                          det_channel_offset, det_row_offset, delta_voxel, 0.0, math.inf, math.inf, 1.0,
                          _parallel_psf_radius(delta_det_channel, delta_voxel), 1)


def cone_geometry(sinogram_shape, angles, source_detector_dist, source_iso_dist, *, delta_det_channel=1.0,
                  delta_det_row=1.0, det_channel_offset=0.0, det_row_offset=0.0, delta_voxel=None,
                  recon_shape=None, recon_slice_offset=0.0):
    views, rows, channels = sinogram_shape
    if math.isinf(source_detector_dist):
        mag = 1.0
    else:
        mag = source_detector_dist / source_iso_dist  # cone_beam.py:68-80
    if delta_voxel is None:
        delta_voxel = delta_det_channel / mag
    if recon_shape is None:
        # cone_beam.py:174-187
        nr = int(round(channels * ((delta_det_channel / delta_voxel) / mag)))
        ns = int(round(rows * ((delta_det_row / delta_voxel) / mag)))
        recon_shape = (nr, nr, ns)
    psf, bp_psf = _cone_psf_radii(delta_det_row, delta_det_channel, source_detector_dist, mag, recon_shape,
                                  delta_voxel)
    return OracleGeometry('cone', tuple(sinogram_shape), tuple(recon_shape), np.asarray(angles, dtype=F32),
                          delta_det_channel, delta_det_row, det_channel_offset, det_row_offset, delta_voxel,
                          recon_slice_offset, source_detector_dist, source_iso_dist, mag, psf, bp_psf)


def translation_geometry(sinogram_shape, translation_vectors, source_detector_dist, source_iso_dist, *,
                         delta_det_channel=1.0, delta_det_row=1.0, det_channel_offset=0.0, det_row_offset=0.0,
                         delta_voxel=None, recon_shape=None, delta_recon_row=None):
    """Translation geometry as TranslationModel derives it (float32 where the reference's jnp scalars are)."""
    views, rows, channels = sinogram_shape
    tv = np.asarray(translation_vectors, dtype=F32)
    mag = source_detector_dist / source_iso_dist  # translation_model.py:69-81 (finite distances only)
    if delta_voxel is None:
        delta_voxel = delta_det_channel / mag
    detect_box = np.array([delta_det_channel * channels, delta_det_row * rows], dtype=F32)
    if delta_recon_row is None:
        # translation_model.py:155-161
        half_cone_angle = np.arctan2(np.max(detect_box), F32(2 * source_detector_dist))
        delta_recon_row = float(F32(np.sqrt(2)) * (F32(delta_voxel) / np.tan(half_cone_angle)))
    if recon_shape is None:
        # translation_model.py:163-186
        cube = np.amax(tv, axis=0) - np.amin(tv, axis=0)
        box = np.ceil((np.array([cube[0], cube[2]], dtype=F32) + detect_box / F32(mag) / F32(2)) / F32(delta_voxel))
        nr = np.ceil(F32(views * channels * rows) / (box[0] * box[1]))
        nr = np.minimum(nr, np.floor((F32(source_iso_dist) - cube[1]) / F32(delta_recon_row)))
        recon_shape = (int(nr), int(box[0]), int(box[1]))
    # translation_model.py:109-140
    delta_det = F32(min(delta_det_row, delta_det_channel))
    closest = F32(source_iso_dist - 0.5 * recon_shape[0] * delta_recon_row) - np.amax(tv, axis=0)[1]
    max_mag = F32(source_detector_dist) / closest
    psf = int(np.ceil(np.ceil(F32(delta_voxel) * max_mag / delta_det) / F32(2)))
    g = OracleGeometry('translation', tuple(sinogram_shape), tuple(recon_shape), tv, delta_det_channel,
                       delta_det_row, det_channel_offset, det_row_offset, delta_voxel, 0.0, source_detector_dist,
                       source_iso_dist, mag, psf, psf)
    g.delta_recon_row = float(delta_recon_row)
    return g
