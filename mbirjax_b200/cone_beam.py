"""ConeBeamModel: cone-beam geometry on the mbirjax_b200 kernels.

Drop-in for ``mbirjax.ConeBeamModel`` (``cone_beam.py:16-871``): constructor
``ConeBeamModel(sinogram_shape, angles, source_detector_dist, source_iso_dist)``, ``get_magnification``
(``:68-80``), ``verify_valid_params`` (``:82-108``), ``get_geometry_parameters`` (``:110-136``),
``get_psf_radius`` with ``bp_psf_radius`` (``:138-172``), ``auto_set_recon_size`` (``:174-187``) and
``fdk_filter`` / ``fdk_recon`` (= ``direct_filter`` / ``direct_recon``, ``:762-871``).  The separable
vertical/horizontal fan projectors (``:189-707``) run in the CUDA library, for all views at once or, through
the reference's per-view plugin functions, on a one-view geometry.
"""
from collections import namedtuple
import math
import warnings

import numpy as np

from . import _capi
from .tomography_model import TomographyModel, back_project_one_view, forward_project_one_view
from .parallel_beam import _host


class ConeBeamModel(TomographyModel):

    def __init__(self, sinogram_shape, angles, source_detector_dist, source_iso_dist):
        self.bp_psf_radius = 1
        self.entries_per_cylinder_batch = 128
        self.slice_range_length = 0
        angles = np.asarray(_host(angles), dtype=np.float32)
        super().__init__(sinogram_shape, angles=angles, source_detector_dist=source_detector_dist,
                         source_iso_dist=source_iso_dist, view_params_name='angles', recon_slice_offset=0.0)

    def _kind(self):
        return _capi.MBX_GEOM_CONE

    def get_magnification(self):
        source_detector_dist, source_iso_dist = self.get_params(['source_detector_dist', 'source_iso_dist'])
        if math.isinf(source_detector_dist):
            return 1
        return source_detector_dist / source_iso_dist

    def verify_valid_params(self):
        super().verify_valid_params()
        sinogram_shape, angles = self.get_params(['sinogram_shape', 'angles'])
        if np.asarray(angles).shape[0] != sinogram_shape[0]:
            raise ValueError('Number view dependent parameter vectors must equal the number of views. \n'
                             'Got {} for length of view-dependent parameters and {} for number of views.'.format(
                                 np.asarray(angles).shape[0], sinogram_shape[0]))
        source_detector_dist, delta_det_row, det_row_offset = self.get_params(
            ['source_detector_dist', 'delta_det_row', 'det_row_offset'])
        half_detector_height = delta_det_row * sinogram_shape[1] / 2 + abs(det_row_offset)
        if half_detector_height > source_detector_dist:
            warnings.warn('Cone angle is more than 45 degrees.  This will likely produce recon artifacts.')

    def get_geometry_parameters(self):
        names = ['delta_det_row', 'delta_det_channel', 'det_row_offset', 'det_channel_offset',
                 'source_detector_dist', 'delta_voxel', 'recon_slice_offset']
        values = self.get_params(names)
        names += ['magnification', 'psf_radius', 'bp_psf_radius', 'entries_per_cylinder_batch', 'slice_range_length']
        values.append(self.get_magnification())
        values.append(self.get_psf_radius())
        values += [self.bp_psf_radius, self.entries_per_cylinder_batch, self.slice_range_length]
        return namedtuple('GeometryParams', names)(*values)

    def get_psf_radius(self):
        """cone_beam.py:138-172 (float32 as the reference's jnp scalars); also sets bp_psf_radius."""
        f32 = np.float32
        delta_det_row, delta_det_channel, source_detector_dist, recon_shape, delta_voxel = self.get_params(
            ['delta_det_row', 'delta_det_channel', 'source_detector_dist', 'recon_shape', 'delta_voxel'])
        magnification = self.get_magnification()
        delta_det = f32(min(delta_det_row, delta_det_channel))
        if math.isinf(source_detector_dist):
            max_mag = min_mag = f32(1)
        else:
            sid = f32(source_detector_dist) / f32(magnification)
            rmax = f32(max(recon_shape[0], recon_shape[1])) * f32(delta_voxel)
            max_mag = f32(source_detector_dist) / (sid - rmax)
            min_mag = f32(source_detector_dist) / (sid + rmax)
        psf_radius = int(np.ceil(np.ceil(f32(delta_voxel) * max_mag / delta_det) / f32(2)))
        max_voxels_per_detector = delta_det / (min_mag * f32(delta_voxel))
        self.bp_psf_radius = int(np.ceil(np.ceil(max_voxels_per_detector) / f32(2)))
        self.slice_range_length = int(1 + 2 * self.bp_psf_radius +
                                      np.ceil(self.entries_per_cylinder_batch * max_voxels_per_detector))
        return psf_radius

    def auto_set_recon_size(self, sinogram_shape, no_compile=True, no_warning=False):
        delta_det_row, delta_det_channel, delta_voxel = self.get_params(['delta_det_row', 'delta_det_channel',
                                                                         'delta_voxel'])
        num_det_rows, num_det_channels = sinogram_shape[1:3]
        mag = self.get_magnification()
        num_recon_rows = int(round(num_det_channels * ((delta_det_channel / delta_voxel) / mag)))
        num_recon_slices = int(round(num_det_rows * ((delta_det_row / delta_voxel) / mag)))
        self.set_params(no_compile=no_compile, no_warning=no_warning,
                        recon_shape=(num_recon_rows, num_recon_rows, num_recon_slices))

    @staticmethod
    def forward_project_pixel_batch_to_one_view(voxel_values, pixel_indices, angle, projector_params):
        """cone_beam.py:189-217: (N, S) voxel cylinders at pixel_indices -> the (R, C) view at angle (vertical
        then horizontal fan), on the CUDA projector (a one-view geometry)."""
        return forward_project_one_view(_capi.MBX_GEOM_CONE, voxel_values, pixel_indices, angle, projector_params)

    @staticmethod
    def back_project_one_view_to_pixel_batch(sinogram_view, pixel_indices, single_view_params, projector_params,
                                             coeff_power=1):
        """cone_beam.py:379-407: the (R, C) view at angle single_view_params -> (N, S) voxel cylinders at
        pixel_indices (horizontal then vertical fan), with coefficients A ** coeff_power, on the CUDA projector
        (a one-view geometry)."""
        return back_project_one_view(_capi.MBX_GEOM_CONE, sinogram_view, pixel_indices, single_view_params,
                                     projector_params, coeff_power)

    def fdk_filter(self, sinogram, filter_name='ramp', view_batch_size=100):
        return self.direct_filter(sinogram, filter_name=filter_name, view_batch_size=view_batch_size)

    def fdk_recon(self, sinogram, filter_name='ramp', view_batch_size=100):
        return self.direct_recon(sinogram, filter_name=filter_name, view_batch_size=view_batch_size)
