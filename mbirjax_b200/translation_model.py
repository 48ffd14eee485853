"""TranslationModel: translation tomography on the mbirjax_b200 kernels.

Drop-in for ``mbirjax.TranslationModel`` (``translation_model.py:13-706``): the object is translated by a vector
(tx, ty, tz) per view in front of a fixed cone-beam source and flat detector, with no rotation.  Constructor
``TranslationModel(sinogram_shape, translation_vectors, source_detector_dist, source_iso_dist)``,
``get_magnification`` (``:69-81``), ``get_geometry_parameters`` (``:83-107``), ``get_psf_radius``
(``:109-140``) and ``auto_set_recon_size`` (``:142-186``) with its ``delta_recon_row`` heuristic.  The separable
vertical/horizontal fan projectors (``:190-706``) run in the CUDA library as the ``MBX_GEOM_TRANSLATION``
geometry.

Behaviour kept from the reference:

* ``qggmrf_nbr_wts`` defaults to (0.5, 1, 1) (rows are ``delta_recon_row`` apart, farther than columns);
* the reference sets ``use_ror_mask = False`` before the base constructor, which resets it to True, so full
  projections and partitions use the region-of-reconstruction mask as for the other geometries;
* there is no direct reconstruction: ``direct_filter`` / ``direct_recon`` warn and return zeros (the base
  ``TomographyModel``, ``tomography_model.py:934-964``), so ``recon`` starts from zeros.

One deliberate difference: the number of translation vectors must equal ``sinogram_shape[0]`` (as the angles
of the rotating geometries must); the reference does not check it.
"""
from collections import namedtuple
import math
import warnings

import numpy as np
import torch

from . import _capi
from .tomography_model import (TomographyModel, back_project_one_view, forward_project_one_view,
                               translation_max_magnification)
from .parallel_beam import _host


class TranslationModel(TomographyModel):

    def __init__(self, sinogram_shape, translation_vectors, source_detector_dist, source_iso_dist):
        self.use_ror_mask = False
        self.entries_per_cylinder_batch = 128
        translation_vectors = np.asarray(_host(translation_vectors), dtype=np.float32)
        super().__init__(sinogram_shape, translation_vectors=translation_vectors,
                         source_detector_dist=source_detector_dist, source_iso_dist=source_iso_dist,
                         view_params_name='translation_vectors', qggmrf_nbr_wts=(0.5, 1, 1))

    def _kind(self):
        return _capi.MBX_GEOM_TRANSLATION

    def get_magnification(self):
        source_detector_dist, source_iso_dist = self.get_params(['source_detector_dist', 'source_iso_dist'])
        if math.isinf(source_detector_dist):
            raise ValueError('Distance from source to detector is infinite, which means all translated projections '
                             'have the same information.')
        return source_detector_dist / source_iso_dist

    def verify_valid_params(self):
        super().verify_valid_params()
        sinogram_shape, translation_vectors = self.get_params(['sinogram_shape', 'translation_vectors'])
        tv = np.asarray(translation_vectors)
        if tv.ndim != 2 or tv.shape[1] != 3:
            raise ValueError('translation_vectors must have shape (num_views, 3); got {}'.format(tv.shape))
        if tv.shape[0] != sinogram_shape[0]:
            raise ValueError('Number view dependent parameter vectors must equal the number of views. \n'
                             'Got {} for length of view-dependent parameters and {} for number of views.'.format(
                                 tv.shape[0], sinogram_shape[0]))

    def get_geometry_parameters(self):
        names = ['delta_det_row', 'delta_det_channel', 'det_row_offset', 'det_channel_offset',
                 'source_detector_dist', 'delta_voxel', 'delta_recon_row']
        values = self.get_params(names)
        names += ['magnification', 'psf_radius', 'entries_per_cylinder_batch']
        values.append(self.get_magnification())
        values.append(self.get_psf_radius())
        values.append(self.entries_per_cylinder_batch)
        return namedtuple('GeometryParams', names)(*values)

    def _max_magnification(self):
        """An upper bound of mag = 1 / (1/M - y/D) over every pixel row and view, y = delta_recon_row (row -
        (Nr-1)/2) - ty, with a small margin; 0 when some pixel reaches the source plane.  The fast back projector
        sizes its detector-row cache from it."""
        recon_shape, delta_recon_row, translation_vectors, sdd = self.get_params(
            ['recon_shape', 'delta_recon_row', 'translation_vectors', 'source_detector_dist'])
        ty = np.asarray(translation_vectors, dtype=np.float64)[:, 1]
        return translation_max_magnification(delta_recon_row, recon_shape[0], float(np.min(ty)),
                                             self.get_magnification(), sdd)

    @staticmethod
    def forward_project_pixel_batch_to_one_view(voxel_values, pixel_indices, translation_vector, projector_params):
        """translation_model.py:190-242: (N, S) voxel cylinders at pixel_indices -> the (R, C) view of the object
        translated by translation_vector, on the CUDA projector (a one-view geometry)."""
        return forward_project_one_view(_capi.MBX_GEOM_TRANSLATION, voxel_values, pixel_indices, translation_vector,
                                        projector_params)

    @staticmethod
    def back_project_one_view_to_pixel_batch(sinogram_view, pixel_indices, single_view_params, projector_params,
                                             coeff_power=1):
        """translation_model.py:382-410: the (R, C) view -> (N, S) voxel cylinders at pixel_indices, with
        coefficients A ** coeff_power, on the CUDA projector (a one-view geometry)."""
        return back_project_one_view(_capi.MBX_GEOM_TRANSLATION, sinogram_view, pixel_indices, single_view_params,
                                     projector_params, coeff_power)

    def get_psf_radius(self):
        """translation_model.py:109-140 in float32 as the reference's jnp scalars: detector elements on either
        side of the centre one that the closest voxel (largest magnification) can reach."""
        f32 = np.float32
        delta_det_row, delta_det_channel, source_iso_dist, source_detector_dist, recon_shape, delta_voxel, \
            delta_recon_row, translation_vectors = self.get_params(
                ['delta_det_row', 'delta_det_channel', 'source_iso_dist', 'source_detector_dist', 'recon_shape',
                 'delta_voxel', 'delta_recon_row', 'translation_vectors'])
        self.get_magnification()  # raises for an infinite source distance
        delta_det = f32(min(delta_det_row, delta_det_channel))
        max_translation = np.amax(np.asarray(translation_vectors, dtype=f32), axis=0)
        source_to_closest_pixel = f32(source_iso_dist - (0.5 * recon_shape[0] * delta_recon_row)) - max_translation[1]
        max_magnification = f32(source_detector_dist) / source_to_closest_pixel
        if source_to_closest_pixel < 0:
            raise ValueError('Reconstruction volume extends into source - no valid projection in this case.')
        psf_radius = int(np.ceil(np.ceil(f32(delta_voxel) * max_magnification / delta_det) / f32(2)))
        if psf_radius > 4:
            warnings.warn('A single voxel may project onto 100 or more detector elements, which may lead to '
                          'artifacts. Consider using smaller voxels.')
        return psf_radius

    def auto_set_recon_size(self, sinogram_shape, no_compile=True, no_warning=False):
        """translation_model.py:142-186: row pitch sqrt(2) delta_voxel / tan(half cone angle); columns and slices
        cover the translated region plus half the magnified detector; rows from the number of measurements, at
        most up to the source."""
        f32 = np.float32
        source_detector_dist, source_iso_dist = self.get_params(['source_detector_dist', 'source_iso_dist'])
        delta_det_row, delta_det_channel = self.get_params(['delta_det_row', 'delta_det_channel'])
        magnification = self.get_magnification()
        delta_voxel = self.get_params('delta_voxel')
        num_views, num_det_rows, num_det_channels = sinogram_shape
        translation_vectors = np.asarray(self.get_params('translation_vectors'), dtype=f32)

        detect_box = np.array([delta_det_channel * num_det_channels, delta_det_row * num_det_rows], dtype=f32)
        half_cone_angle = np.arctan2(np.max(detect_box), f32(2 * source_detector_dist))
        delta_recon_row = float(f32(np.sqrt(2)) * (f32(delta_voxel) / np.tan(half_cone_angle)))

        cube = np.amax(translation_vectors, axis=0) - np.amin(translation_vectors, axis=0)
        recon_box = np.ceil((np.array([cube[0], cube[2]], dtype=f32) + detect_box / f32(magnification) / f32(2)) /
                            f32(delta_voxel))
        num_recon_rows = np.ceil(f32(num_views * num_det_channels * num_det_rows) / (recon_box[0] * recon_box[1]))
        max_recon_rows = np.floor((f32(source_iso_dist) - cube[1]) / f32(delta_recon_row))
        if max_recon_rows < 1:
            print(f"[Error] Computed max_recon_rows = {max_recon_rows} < 1. This suggests the object extends beyond "
                  f"the source.")
        num_recon_rows = np.minimum(num_recon_rows, max_recon_rows)
        recon_shape = (int(num_recon_rows), int(recon_box[0]), int(recon_box[1]))
        self.set_params(no_compile=no_compile, no_warning=no_warning, recon_shape=recon_shape,
                        delta_recon_row=delta_recon_row)

    def direct_filter(self, sinogram, filter_name=None, view_batch_size=TomographyModel.DIRECT_RECON_VIEW_BATCH_SIZE):
        warnings.warn('direct_filter not implemented for TomographyModel.')
        return torch.zeros_like(self._dev(sinogram))

    def direct_recon(self, sinogram, filter_name=None, view_batch_size=TomographyModel.DIRECT_RECON_VIEW_BATCH_SIZE):
        warnings.warn('direct_recon not implemented for TomographyModel.')
        return torch.zeros(tuple(self.get_params('recon_shape')), dtype=torch.float32, device=self._device())
