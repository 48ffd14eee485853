"""Pixel partitions and region-of-reconstruction mask (test infrastructure only).

Restates ``vcd_utils.py:66-124, 176-223, 284-318``.  The partition uses the legacy global
``np.random`` stream exactly as the reference does (``permutation`` then ``choice(..., replace=False)``,
which consumes the stream even when it draws nothing), so a seeded call sequence reproduces the
reference's partitions without JAX.
"""
import warnings

import numpy as np


def get_2d_ror_mask(recon_shape):
    """vcd_utils.py:66-102 (default crop radius 0)."""
    num_recon_rows, num_recon_cols = recon_shape[:2]
    row_center = (num_recon_rows - 1) / 2
    col_center = (num_recon_cols - 1) / 2
    radius = max(row_center, col_center)
    col_coords = np.arange(num_recon_cols) - col_center
    row_coords = np.arange(num_recon_rows) - row_center
    coords = np.meshgrid(col_coords, row_coords)
    return coords[0] ** 2 + coords[1] ** 2 <= radius ** 2


def gen_pixel_partition(recon_shape, num_subsets, use_ror_mask=True):
    """vcd_utils.py:176-223."""
    num_recon_rows, num_recon_cols = recon_shape[:2]
    indices = np.arange(num_recon_rows * num_recon_cols, dtype=np.int32)
    if use_ror_mask:
        mask = get_2d_ror_mask(recon_shape).flatten()
        indices = indices[mask == 1]
    if num_subsets > len(indices):
        num_subsets = len(indices)
        warnings.warn('The number of partition subsets is greater than the number of pixels in the region of '
                      'reconstruction.  Reducing the number of subsets to equal the number of indices.')
    num_indices_per_subset = int(np.ceil(len(indices) / num_subsets))
    array_size = num_subsets * num_indices_per_subset
    num_extra_indices = array_size - len(indices)
    indices = np.random.permutation(indices)
    num_non_final_indices = (num_subsets - 1) * num_indices_per_subset
    extra_indices = np.random.choice(indices[:num_non_final_indices], size=num_extra_indices, replace=False)
    indices = np.concatenate((indices, extra_indices))
    indices = indices.reshape(num_subsets, indices.size // num_subsets)
    return np.sort(indices, axis=1).astype(np.int32)


def gen_set_of_pixel_partitions(recon_shape, granularity, use_ror_mask=True):
    """vcd_utils.py:105-124."""
    return [gen_pixel_partition(recon_shape, k, use_ror_mask=use_ror_mask) for k in granularity]


def gen_partition_sequence(partition_sequence, max_iterations):
    """vcd_utils.py:284-307."""
    seq = np.array(partition_sequence)
    if max_iterations > seq.size:
        return np.concatenate((seq, np.full(max_iterations - seq.size, seq[-1])))
    return seq[:max_iterations]


def gen_full_indices(recon_shape, use_ror_mask=True):
    """vcd_utils.py:310-318 (draws from np.random like the reference)."""
    return gen_pixel_partition(recon_shape, num_subsets=1, use_ror_mask=use_ror_mask)[0]
