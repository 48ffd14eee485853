"""Multi-core driver for the oracle (test / CPU-baseline infrastructure only).

Splits the views of a sparse forward or back projection across worker processes (``spawn`` start method, so a
pool never inherits a CUDA context) and reassembles the result; each worker runs the single-view restatements
of ``oracle.projectors``.  An ``OraclePool`` has the projector functions of ``oracle.projectors``
(``sparse_forward_project``, ``sparse_back_project``, ``forward_project``, ``back_project``,
``compute_hessian_diagonal``) with the same arguments, so the VCD restatement (``oracle.vcd``, argument
``proj``) runs unchanged with its projections spread over the host cores.  The back projection sums the view
chunks in chunk order, so a pooled result is reproducible for a given number of workers.
"""
import multiprocessing as mp
import os

import numpy as np

from . import projectors as P
from .partitions import gen_full_indices

def _fp_chunk(args):
    geom, views, vox, pix, dt = args
    return np.stack([P.forward_project_one_view(geom, vox, pix, geom.angles[v], dt) for v in views])


def _bp_chunk(args):
    geom, views, rows, pix, coeff_power, dt = args
    out = None
    for v, row in zip(views, rows):
        b = P.back_project_one_view(geom, row, pix, geom.angles[v], coeff_power, dt)
        out = b if out is None else out + b
    return out


class OraclePool:
    """A pool of worker processes for the oracle's projections of any geometry (each task carries its geometry;
    ``geom`` is the one the older ``forward`` / ``back`` shorthands use)."""

    def __init__(self, geom=None, workers=None):
        self.geom = geom
        self.workers = workers or os.cpu_count() or 1
        self.pool = mp.get_context('spawn').Pool(self.workers)

    def close(self):
        self.pool.close()
        self.pool.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _chunks(self, views):
        return [c for c in np.array_split(views, self.workers) if len(c)]

    @staticmethod
    def _views(geom, view_indices):
        if view_indices is None:
            return np.arange(geom.sinogram_shape[0])
        return np.asarray(view_indices, dtype=np.int64)

    # the projector functions of oracle.projectors, with the views spread over the workers
    def sparse_forward_project(self, geom, voxel_values, pixel_indices, view_indices=None, dtype=np.float32):
        dt = np.dtype(dtype).type
        vox = np.asarray(voxel_values)
        pix = np.asarray(pixel_indices)
        parts = self.pool.map(_fp_chunk, [(geom, c, vox, pix, dt) for c in self._chunks(self._views(geom, view_indices))])
        return np.concatenate(parts, axis=0)

    def sparse_back_project(self, geom, sinogram, pixel_indices, view_indices=None, coeff_power=1, dtype=np.float32):
        dt = np.dtype(dtype).type
        pix = np.asarray(pixel_indices)
        parts = self.pool.map(_bp_chunk, [(geom, c, sinogram[c], pix, coeff_power, dt)
                                          for c in self._chunks(self._views(geom, view_indices))])
        out = parts[0].copy()
        for p in parts[1:]:
            out += p
        return out

    def forward_project(self, geom, recon, dtype=np.float32):
        idx = gen_full_indices(geom.recon_shape)  # the reference's np.random draws, as oracle.projectors
        flat = np.asarray(recon).reshape((-1, geom.recon_shape[2]))
        return self.sparse_forward_project(geom, flat[idx], idx, dtype=dtype)

    def back_project(self, geom, sinogram, dtype=np.float32):
        idx = gen_full_indices(geom.recon_shape)
        cyl = self.sparse_back_project(geom, sinogram, idx, dtype=dtype)
        out = np.zeros((geom.recon_shape[0] * geom.recon_shape[1], geom.recon_shape[2]), dtype=cyl.dtype)
        out[idx] = cyl
        return out.reshape(geom.recon_shape)

    def compute_hessian_diagonal(self, geom, weights=None, dtype=np.float32):
        if weights is None:
            weights = np.ones(geom.sinogram_shape, dtype=dtype)
        nr, nc, ns = geom.recon_shape
        idx = np.arange(nr * nc)
        return self.sparse_back_project(geom, weights, idx, coeff_power=2, dtype=dtype).reshape((nr, nc, ns))

    # the older name of one pooled forward / back projection over all views
    def forward(self, vox, pix):
        return self.sparse_forward_project(self.geom, vox, pix)

    def back(self, sino, pix, coeff_power=1):
        return self.sparse_back_project(self.geom, sino, pix, coeff_power=coeff_power)


def vcd_subset_update_pooled(pool, flat_recon, error_sinogram, weights, fm_hessian, pixel_indices, fm_constant,
                             qggmrf_params):
    """tomography_model.py:1343-1542 with pooled projections; returns (flat_recon, error_sinogram, ell1, alpha)."""
    from .vcd import vcd_subset_update
    return vcd_subset_update(pool.geom, flat_recon, error_sinogram, weights, fm_hessian, pixel_indices, fm_constant,
                             qggmrf_params, proj=pool)
