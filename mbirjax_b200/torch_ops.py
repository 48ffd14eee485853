"""The CUDA library's entry points as PyTorch dispatcher operators, ``torch.ops.mbirjax_b200.*``.

The operators (``csrc_torch/mbx_torch_ops.cpp``, built into ``_lib/libmbirjax_b200_torch.so`` by
``mbirjax_b200.build()``) check dtype, contiguity and device of their tensors, allocate outputs and workspace with
the caching allocator and run on the current CUDA stream.  They are registered for CUDA only.  This module loads
them and turns a model's geometry into their scalar-list arguments:

    ops = torch_ops.load()
    gi, gf, views = torch_ops.geometry_args(model)
    sino = ops.sparse_forward_project(gi, gf, views, voxel_values, pixel_indices)
"""
import os

import torch

from ._capi import MbxError

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(_HERE, '_lib', 'libmbirjax_b200_torch.so')
_loaded = False

OPS = ('sparse_forward_project', 'sparse_back_project', 'direct_filter', 'qggmrf_grad_hess', 'qggmrf_loss_grad',
       'vcd_subset_step')


def load():
    """Registers the operators (once per process) and returns the torch.ops.mbirjax_b200 namespace."""
    global _loaded
    if not _loaded:
        if not os.path.exists(LIB):
            raise MbxError('mbirjax_b200 torch operators not found at %s; run mbirjax_b200.build()' % LIB)
        torch.ops.load_library(LIB)
        _loaded = True
    return torch.ops.mbirjax_b200


def geometry_args_of(g, view_params):
    """(geom_ints, geom_floats, view_params) of an MbxGeom record and its device view-parameter tensor."""
    gi = [g.kind, g.num_views, g.num_det_rows, g.num_det_channels, g.num_recon_rows, g.num_recon_cols,
          g.num_recon_slices, g.psf_radius, g.bp_psf_radius, g.entries_per_cylinder_batch]
    gf = [g.delta_det_channel, g.delta_det_row, g.det_channel_offset, g.det_row_offset, g.delta_voxel,
          g.recon_slice_offset, g.source_detector_dist, g.magnification, g.delta_recon_row, g.max_magnification]
    return [int(v) for v in gi], [float(v) for v in gf], view_params


def geometry_args(model):
    """The operator geometry arguments of a TomographyModel (its angles or translations stay on the device)."""
    g = model._geometry()
    return geometry_args_of(g, model._angles_dev)


def qparams_args(b, sigma_x, p, q, T):
    """qGGMRF parameters as the operators take them: [b0..b5, sigma_x, p, q, T]."""
    return [float(v) for v in list(b)] + [float(sigma_x), float(p), float(q), float(T)]
