"""ParallelBeamModel: parallel-beam geometry on the mbirjax_b200 kernels.

Drop-in for ``mbirjax.ParallelBeamModel`` (``parallel_beam.py:13-373``): constructor
``ParallelBeamModel(sinogram_shape, angles)``, ``get_magnification`` (1), ``verify_valid_params``,
``get_geometry_parameters``, ``get_psf_radius``, ``auto_set_recon_size``, ``fbp_filter`` / ``fbp_recon``
(= ``direct_filter`` / ``direct_recon``).  The model's projections run the batched kernels behind
``mbx_sparse_forward_project`` / ``mbx_sparse_back_project`` over all views at once; the reference's per-view
plugin functions (``forward_project_pixel_batch_to_one_view`` / ``back_project_one_view_to_pixel_batch``) keep
their signatures and run the same kernels on a one-view geometry.
"""
from collections import namedtuple
import math

import numpy as np

from . import _capi
from .tomography_model import TomographyModel, back_project_one_view, forward_project_one_view


class ParallelBeamModel(TomographyModel):

    def __init__(self, sinogram_shape, angles):
        angles = np.asarray(_host(angles), dtype=np.float32)
        super().__init__(sinogram_shape, angles=angles, view_params_name='angles')

    def _kind(self):
        return _capi.MBX_GEOM_PARALLEL

    def get_magnification(self):
        return 1.0

    def verify_valid_params(self):
        super().verify_valid_params()
        sinogram_shape, angles = self.get_params(['sinogram_shape', 'angles'])
        if np.asarray(angles).shape[0] != sinogram_shape[0]:
            raise ValueError('Number view dependent parameter vectors must equal the number of views. \n'
                             'Got {} for length of view-dependent parameters and {} for number of views.'.format(
                                 np.asarray(angles).shape[0], sinogram_shape[0]))
        recon_shape = self.get_params('recon_shape')
        if recon_shape is not None and recon_shape[2] != sinogram_shape[1]:
            raise ValueError('Number of recon slices must match number of sinogram rows. \n'
                             'Got {} for recon_shape and {} for sinogram_shape'.format(recon_shape, sinogram_shape))

    def get_geometry_parameters(self):
        names = ['delta_det_channel', 'det_channel_offset', 'delta_voxel']
        values = self.get_params(names)
        names += ['psf_radius']
        values.append(self.get_psf_radius())
        return namedtuple('GeometryParams', names)(*values)

    def get_psf_radius(self):
        """parallel_beam.py:115-123."""
        delta_det_channel, delta_voxel = self.get_params(['delta_det_channel', 'delta_voxel'])
        return int(np.ceil(np.ceil(np.float32(delta_voxel) / np.float32(delta_det_channel)) / np.float32(2)))

    def auto_set_recon_size(self, sinogram_shape, no_compile=True, no_warning=False):
        """parallel_beam.py:125-136."""
        delta_det_row, delta_det_channel, delta_voxel = self.get_params(['delta_det_row', 'delta_det_channel',
                                                                         'delta_voxel'])
        num_det_rows, num_det_channels = sinogram_shape[1:3]
        mag = self.get_magnification()
        num_recon_rows = int(math.ceil(num_det_channels * delta_det_channel / (delta_voxel * mag)))
        num_recon_slices = int(round(num_det_rows * ((delta_det_row / delta_voxel) / mag)))
        self.set_params(no_compile=no_compile, no_warning=no_warning,
                        recon_shape=(num_recon_rows, num_recon_rows, num_recon_slices))

    @staticmethod
    def forward_project_pixel_batch_to_one_view(voxel_values, pixel_indices, angle, projector_params):
        """parallel_beam.py:138-178: (N, S) voxel cylinders at pixel_indices -> the (R, C) view at angle, on the
        CUDA projector (a one-view geometry)."""
        return forward_project_one_view(_capi.MBX_GEOM_PARALLEL, voxel_values, pixel_indices, angle,
                                        projector_params)

    @staticmethod
    def back_project_one_view_to_pixel_batch(sinogram_view, pixel_indices, angle, projector_params, coeff_power=1):
        """parallel_beam.py:180-221: the (R, C) view at angle -> (N, S) voxel cylinders at pixel_indices, with
        coefficients A ** coeff_power, on the CUDA projector (a one-view geometry)."""
        return back_project_one_view(_capi.MBX_GEOM_PARALLEL, sinogram_view, pixel_indices, angle, projector_params,
                                     coeff_power)

    def fbp_filter(self, sinogram, filter_name='ramp', view_batch_size=100):
        return self.direct_filter(sinogram, filter_name=filter_name, view_batch_size=view_batch_size)

    def fbp_recon(self, sinogram, filter_name='ramp', view_batch_size=100):
        return self.direct_recon(sinogram, filter_name=filter_name, view_batch_size=view_batch_size)


def _host(x):
    try:
        import torch
        if isinstance(x, torch.Tensor):
            return x.detach().cpu().numpy()
    except ImportError:  # pragma: no cover
        pass
    return x
