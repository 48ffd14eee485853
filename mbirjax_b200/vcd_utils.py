"""Pixel partitions, partition sequences and the region-of-reconstruction mask (host side, NumPy).

Same contract as ``vcd_utils.py:66-124, 176-223, 284-318`` of the reference, including its use of the legacy
global ``np.random`` stream (``permutation``, then ``choice(..., replace=False)``), so that a run seeded with
``np.random.seed`` draws the same partitions and subset orders as the reference does.
"""
import warnings

import numpy as np


def get_2d_ror_mask(recon_shape, *, crop_radius_pixels=0, crop_radius_fraction=0.0):
    """Boolean (rows, cols) disk inscribed on the longer edge, optionally shrunk (vcd_utils.py:66-102)."""
    if crop_radius_pixels != 0 and crop_radius_fraction != 0.0:
        raise ValueError('Only one of crop_radius_pixels and crop_radius_fraction can be nonzero.')
    num_rows, num_cols = recon_shape[:2]
    row_center, col_center = (num_rows - 1) / 2, (num_cols - 1) / 2
    radius = max(row_center, col_center)
    crop = max(int(radius * crop_radius_fraction), crop_radius_pixels, 0)
    radius -= crop
    cols = np.arange(num_cols) - col_center
    rows = np.arange(num_rows) - row_center
    return cols[None, :] ** 2 + rows[:, None] ** 2 <= radius ** 2


def gen_pixel_partition(recon_shape, num_subsets, use_ror_mask=True, rng=None):
    """(num_subsets, ceil(N/num_subsets)) int32 array of sorted flat pixel indices (vcd_utils.py:176-223).

    rng: a legacy np.random.RandomState to draw from instead of the global stream (np.random.seed(s) followed by
    the global draws is the same stream as RandomState(s))."""
    rng = np.random if rng is None else rng
    num_rows, num_cols = recon_shape[:2]
    indices = np.arange(num_rows * num_cols, dtype=np.int32)
    if use_ror_mask:
        indices = indices[get_2d_ror_mask(recon_shape).flatten()]
    if num_subsets > len(indices):
        num_subsets = len(indices)
        warnings.warn('\nThe number of partition subsets is greater than the number of pixels in the region of '
                      'reconstruction.  \nReducing the number of subsets to equal the number of indices.')
    per_subset = int(np.ceil(len(indices) / num_subsets))
    num_extra = num_subsets * per_subset - len(indices)
    indices = rng.permutation(indices)
    num_non_final = (num_subsets - 1) * per_subset
    extra = rng.choice(indices[:num_non_final], size=num_extra, replace=False)
    indices = np.concatenate((indices, extra)).reshape(num_subsets, -1)
    return np.sort(indices, axis=1).astype(np.int32)


def gen_set_of_pixel_partitions(recon_shape, granularity, output_device=None, use_ror_mask=True, rng=None):
    """One partition per entry of granularity (vcd_utils.py:105-124); output_device is accepted and ignored."""
    return [gen_pixel_partition(recon_shape, k, use_ror_mask=use_ror_mask, rng=rng) for k in granularity]


def gen_partition_sequence(partition_sequence, max_iterations):
    """Extend (or cut) the sequence to max_iterations by repeating its last entry (vcd_utils.py:284-307)."""
    seq = np.array(partition_sequence)
    if max_iterations > seq.size:
        return np.concatenate((seq, np.full(max_iterations - seq.size, seq[-1])))
    return seq[:max_iterations]


_FULL_INDICES = {}  # (rows, cols, use_ror_mask) -> sorted region of reconstruction
_CACHE_GRIDS = 64    # grid sizes each host cache keeps (the oldest entry goes first; a batch holds many)


def _cache_put(cache, key, value):
    if len(cache) >= _CACHE_GRIDS:
        cache.pop(next(iter(cache)))
    cache[key] = value
    return value


def gen_full_indices(recon_shape, use_ror_mask=True, rng=None):
    """All pixels of the region of reconstruction, sorted (vcd_utils.py:310-318).

    The reference draws them as a one-subset partition: a permutation of the N pixels (and an empty choice) from
    the global np.random stream, then a sort, so the result is always the same sorted set while the stream
    advances by one permutation of N.  After the first call for a grid, this returns a copy of the kept set and
    advances the stream by shuffling N scratch entries, which draws exactly what that permutation draws.
    rng: a legacy RandomState to draw from instead of the global stream (it shuffles scratch of its own, so calls
    from several threads with their own streams share nothing but the read-only kept set)."""
    key = (int(recon_shape[0]), int(recon_shape[1]), bool(use_ror_mask))
    hit = _FULL_INDICES.get(key)
    if hit is None:
        idx = gen_pixel_partition(recon_shape, num_subsets=1, use_ror_mask=use_ror_mask, rng=rng)[0]
        _cache_put(_FULL_INDICES, key, (idx, np.empty(len(idx), dtype=np.int32)))
        return idx.copy()
    idx, scratch = hit
    if rng is None:
        np.random.shuffle(scratch)
    else:
        rng.shuffle(np.empty(len(idx), dtype=np.int32))
    return idx.copy()


def morton_order(pixel_indices, num_cols):
    """Positions of pixel_indices sorted by the Z-order (Morton) code of (row, col): neighbouring positions are
    spatially close, so the channel gathers of a warp of the back projector stay within a few sectors."""
    idx = np.asarray(pixel_indices, dtype=np.int64)
    row, col = idx // num_cols, idx % num_cols

    def spread(v):
        v = v.astype(np.uint64) & np.uint64(0xFFFF)
        v = (v | (v << np.uint64(8))) & np.uint64(0x00FF00FF)
        v = (v | (v << np.uint64(4))) & np.uint64(0x0F0F0F0F)
        v = (v | (v << np.uint64(2))) & np.uint64(0x33333333)
        v = (v | (v << np.uint64(1))) & np.uint64(0x55555555)
        return v

    code = spread(row) | (spread(col) << np.uint64(1))
    return np.argsort(code, kind='stable').astype(np.int32)


_ZORDER_GRIDS = {}  # (rows rounded up to 64, cols) -> (every pixel of that grid in Z-order, its Z-order rank)


def _zorder_grid(num_rows, num_cols):
    key = (-(-num_rows // 64) * 64, num_cols)
    hit = _ZORDER_GRIDS.get(key)
    if hit is None:
        allpix = np.arange(key[0] * key[1], dtype=np.int32)
        z = allpix[morton_order(allpix, num_cols)]
        rank = np.empty(z.size, dtype=np.int32)
        rank[z] = np.arange(z.size, dtype=np.int32)
        hit = _cache_put(_ZORDER_GRIDS, key, (z, rank))
    return hit


def morton_sorted_partition(partition, num_cols):
    """Each subset (row) of a partition reordered by the Z-order code of its pixels.  A subset is a set: the
    VCD update does not depend on the order of its pixels, but the projectors run faster when consecutive
    pixels are close in the image (fewer sectors per gather, and whole chunks of the list can be skipped by
    the channel blocks of the forward projector they cannot reach).

    Every pixel's rank in the Z-order of its grid is computed once per grid size; a subset is then its sorted
    ranks mapped back to pixels (the codes are distinct, so this is the order of sorting by code)."""
    partition = np.asarray(partition)
    if partition.size == 0:
        return partition.astype(np.int32)
    if partition.min() < 0:
        return np.stack([p[morton_order(p, num_cols)] for p in partition]).astype(np.int32)
    z, rank = _zorder_grid(int(partition.max()) // num_cols + 1, num_cols)
    return z[np.sort(rank[partition], axis=1)].astype(np.int32)
