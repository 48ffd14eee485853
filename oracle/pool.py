"""Multi-core driver for the oracle (test / CPU-baseline infrastructure only).

Splits the views of a sparse forward or back projection across worker processes (``spawn`` start method, so a
pool never inherits a CUDA context) and reassembles the result; each worker runs the single-view restatements
of ``oracle.projectors``.  ``vcd_subset_update_pooled`` is ``oracle.vcd.vcd_subset_update`` with its two
projections distributed this way.  Used to time the reference arithmetic on all host cores.
"""
import multiprocessing as mp
import os

import numpy as np

from . import projectors as P
from .qggmrf import qggmrf_gradient_and_hessian_at_indices

_G = {}


def _init(geom):
    _G['geom'] = geom


def _fp_chunk(args):
    views, vox, pix = args
    geom = _G['geom']
    return np.stack([P.forward_project_one_view(geom, vox, pix, geom.angles[v]) for v in views])


def _bp_chunk(args):
    views, rows, pix, coeff_power = args
    geom = _G['geom']
    out = None
    for v, row in zip(views, rows):
        b = P.back_project_one_view(geom, row, pix, geom.angles[v], coeff_power)
        out = b if out is None else out + b
    return out


class OraclePool:
    def __init__(self, geom, workers=None):
        self.geom = geom
        self.workers = workers or os.cpu_count() or 1
        self.pool = mp.get_context('spawn').Pool(self.workers, initializer=_init, initargs=(geom,))

    def close(self):
        self.pool.close()
        self.pool.join()

    def _chunks(self):
        v = np.arange(self.geom.sinogram_shape[0])
        return [c for c in np.array_split(v, self.workers) if len(c)]

    def forward(self, vox, pix):
        parts = self.pool.map(_fp_chunk, [(c, vox, pix) for c in self._chunks()])
        return np.concatenate(parts, axis=0)

    def back(self, sino, pix, coeff_power=1):
        parts = self.pool.map(_bp_chunk, [(c, sino[c], pix, coeff_power) for c in self._chunks()])
        out = parts[0].copy()
        for p in parts[1:]:
            out += p
        return out


def vcd_subset_update_pooled(pool, flat_recon, error_sinogram, weights, fm_hessian, pixel_indices, fm_constant,
                             qggmrf_params):
    """tomography_model.py:1343-1542 with pooled projections; returns (flat_recon, error_sinogram, ell1, alpha)."""
    f32 = np.float32
    geom = pool.geom
    eps = f32(np.finfo(np.float32).eps)
    g_p, h_p = qggmrf_gradient_and_hessian_at_indices(flat_recon, geom.recon_shape, pixel_indices, qggmrf_params)
    wes = error_sinogram if weights is None else (weights * error_sinogram).astype(f32)
    g_f = (-fm_constant * pool.back(wes, pixel_indices)).astype(f32)
    h_f = (fm_constant * fm_hessian[pixel_indices]).astype(f32)
    delta = (-((g_f + g_p) / (h_f + h_p))).astype(f32)
    pl = np.sum(g_p * delta, dtype=f32)
    pq = f32(0.5) * np.sum(h_p * delta ** 2, dtype=f32)
    dsino = pool.forward(delta, pixel_indices)
    w = 1 if weights is None else weights
    fl = f32(fm_constant) * np.sum(wes * dsino, dtype=f32)
    fq = f32(fm_constant) * np.sum(dsino * dsino * w, dtype=f32)
    alpha = f32(np.clip((fl - pl) / (fq + pq + eps), eps, 1.5))
    delta = (alpha * delta).astype(f32)
    flat_recon = flat_recon.copy()
    np.add.at(flat_recon, pixel_indices, delta)
    error_sinogram = (error_sinogram - alpha * dsino).astype(f32)
    return flat_recon, error_sinogram, float(np.sum(np.abs(delta), dtype=f32)), float(alpha)
