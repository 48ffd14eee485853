"""FBP / FDK filtering restated in NumPy (test infrastructure only).

* ``generate_direct_recon_filter``: ``tomography_utils.py:4-35``
* ``fbp_filter``: ``parallel_beam.py:303-348`` (filter x 1/delta_voxel^2, 'valid' convolution, x pi/V)
* ``fdk_filter``: ``cone_beam.py:779-846`` with ``detector_mn_to_uv`` ``cone_beam.py:709-738``
  (pre-weight D/sqrt(D^2+u^2+v^2), filter x delta_det_row/(delta_voxel^3 M0), convolution, x pi/V)

The reference evaluates ``fftconvolve(row, filter, mode='valid')``; with a row of C samples and a filter
of 2C-1 taps the valid part is out[i] = sum_j row[j] * h[i - j + C - 1], evaluated here exactly as a
Toeplitz product in float64 and rounded to float32.
"""
import numpy as np


def generate_direct_recon_filter(num_channels, filter_name='ramp'):
    if filter_name not in ['ramp']:
        raise ValueError('Unsupported filter. Supported filters are: ramp.')
    n = np.arange(-num_channels + 1, num_channels)
    return 0.5 * np.sinc(n) - 0.25 * np.sinc(n / 2) ** 2


def _convolve_rows_valid(rows, recon_filter):
    num_channels = rows.shape[-1]
    i = np.arange(num_channels)
    toeplitz = recon_filter[(i[None, :] - i[:, None]) + num_channels - 1]      # [j, i] -> h[i - j + C - 1]
    flat = rows.reshape((-1, num_channels)).astype(np.float64)
    return (flat @ toeplitz).reshape(rows.shape)


def fbp_filter(sinogram, delta_voxel, filter_name='ramp'):
    num_views, _, num_channels = sinogram.shape
    recon_filter = generate_direct_recon_filter(num_channels, filter_name) * (1 / delta_voxel ** 2)
    out = _convolve_rows_valid(np.asarray(sinogram), recon_filter) * (np.pi / num_views)
    return out.astype(np.float32)


def fdk_weight_map(num_rows, num_channels, source_detector_dist, delta_det_channel, delta_det_row,
                   det_channel_offset, det_row_offset):
    m = np.arange(num_rows)
    n = np.arange(num_channels)
    m_grid, n_grid = np.meshgrid(m, n, indexing='ij')
    v = (m_grid - (num_rows - 1) / 2.0) * delta_det_row - det_row_offset
    u = (n_grid - (num_channels - 1) / 2.0) * delta_det_channel - det_channel_offset
    return source_detector_dist / np.sqrt(source_detector_dist ** 2 + u ** 2 + v ** 2)


def fdk_filter(sinogram, source_detector_dist, magnification, delta_voxel, delta_det_row, delta_det_channel,
               det_row_offset=0.0, det_channel_offset=0.0, filter_name='ramp'):
    num_views, num_rows, num_channels = sinogram.shape
    weight = fdk_weight_map(num_rows, num_channels, source_detector_dist, delta_det_channel, delta_det_row,
                            det_channel_offset, det_row_offset)
    weighted = np.asarray(sinogram, dtype=np.float64) * weight[None]
    alpha = delta_det_row / (delta_voxel ** 3 * magnification)
    recon_filter = alpha * generate_direct_recon_filter(num_channels, filter_name)
    out = _convolve_rows_valid(weighted, recon_filter) * (np.pi / num_views)
    return out.astype(np.float32)
