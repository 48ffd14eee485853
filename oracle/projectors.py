"""NumPy restatement of the reference's sparse projectors (test infrastructure only).

Each per-view function follows the reference formula for formula, in the same precision (float32 by
default, as JAX with x64 off computes them), and the same index rounding (``np.round`` is round-half-to-
even, as ``jnp.round``).  ``dtype=np.float64`` evaluates the same formulas in float64 for the adjointness
oracle.  The scatter/gather of one view is written as a sparse matrix product so that config-sized
cases stay tractable on CPU; the coefficients and index sets are exactly the reference's.

Reference functions restated here:

* parallel ``compute_proj_data`` / ``recon_ij_to_x``: ``parallel_beam.py:223-284``
* parallel FP one view: ``parallel_beam.py:138-178``; BP one view: ``parallel_beam.py:180-221``
* cone ``compute_horizontal_data``: ``cone_beam.py:593-644``; ``recon_ijk_to_xyz``: ``cone_beam.py:646-666``
* cone vertical FP one pixel: ``cone_beam.py:286-377`` (detector-row-centric, 128-row batches)
* cone horizontal FP: ``cone_beam.py:244-284``; horizontal BP: ``cone_beam.py:409-451``
* cone vertical BP one pixel: ``cone_beam.py:480-541`` with ``compute_vertical_data_single_pixel``
  ``cone_beam.py:543-591`` (voxel-centric, 128-slice batches)
* translation ``compute_horizontal_data``: ``translation_model.py:595-644``; ``recon_ijk_to_xyz``:
  ``translation_model.py:646-656``; ``compute_y_mag_for_pixel``: ``translation_model.py:694-706``
* translation horizontal FP / BP: ``translation_model.py:244-284`` / ``:412-453`` (coefficient L / cos(theta_p),
  no delta_voxel factor); vertical FP: ``translation_model.py:286-378`` and vertical BP:
  ``translation_model.py:482-593``, the cone's fans with the slice axis shifted by -tz and psf_radius taps
* batching over views / pixels: ``projectors.py:61-209``; ``tomography_model.py:531-708``

For translation geometry ``geom.angles`` holds the (views, 3) translation vectors and the per-view functions
take one translation vector where the rotating geometries take an angle.
"""
import numpy as np
import scipy.sparse as sp

from .partitions import gen_full_indices


def _c(dtype, v):
    return dtype.type(v) if hasattr(dtype, 'type') else np.dtype(dtype).type(v)


def _pixel_xy_tilde(geom, pixel_indices, dt):
    nr, nc = geom.recon_shape[:2]
    row, col = np.unravel_index(np.asarray(pixel_indices, dtype=np.int64), (nr, nc))
    dv = dt(geom.delta_voxel)
    y_tilde = dv * (row.astype(dt) - dt((nr - 1) / 2.0))
    x_tilde = dv * (col.astype(dt) - dt((nc - 1) / 2.0))
    return x_tilde, y_tilde


def parallel_proj_data(geom, pixel_indices, angle, dt=np.float32):
    """parallel_beam.py:223-284: returns n_p, n_p_center, W_p_c, cos_alpha_p_xy."""
    x_tilde, y_tilde = _pixel_xy_tilde(geom, pixel_indices, dt)
    angle = dt(angle)
    cosine, sine = dt(np.cos(angle)), dt(np.sin(angle))
    x = cosine * x_tilde - sine * y_tilde
    num_det_channels = geom.sinogram_shape[2]
    det_center_channel = dt((num_det_channels - 1) / 2.0)
    n_p = (x + dt(geom.det_channel_offset)) / dt(geom.delta_det_channel) + det_center_channel
    n_p_center = np.round(n_p).astype(np.int64)
    cos_alpha = dt(max(abs(cosine), abs(sine)))
    w_p_c = (dt(geom.delta_voxel) / dt(geom.delta_det_channel)) * cos_alpha
    return n_p, n_p_center, np.full(n_p.shape, w_p_c, dtype=dt), np.full(n_p.shape, cos_alpha, dtype=dt)


def cone_horizontal_data(geom, pixel_indices, angle, dt=np.float32):
    """cone_beam.py:593-644 (+ recon_ijk_to_xyz cone_beam.py:646-666)."""
    x_tilde, y_tilde = _pixel_xy_tilde(geom, pixel_indices, dt)
    angle = dt(angle)
    cosine, sine = dt(np.cos(angle)), dt(np.sin(angle))
    x_p = cosine * x_tilde - sine * y_tilde
    y_p = sine * x_tilde + cosine * y_tilde
    D = dt(geom.source_detector_dist)
    pixel_mag = dt(1) / (dt(1 / geom.magnification) - y_p / D)
    u_p = pixel_mag * x_p
    num_det_channels = geom.sinogram_shape[2]
    det_center_channel = dt((num_det_channels - 1) / 2.0)
    n_p = (u_p + dt(geom.det_channel_offset)) / dt(geom.delta_det_channel) + det_center_channel
    n_p_center = np.round(n_p).astype(np.int64)
    theta_p = np.arctan2(u_p, D).astype(dt)
    cos_alpha = np.maximum(np.abs(np.cos(angle - theta_p)), np.abs(np.sin(angle - theta_p))).astype(dt)
    w_p_c = pixel_mag * (dt(geom.delta_voxel) / dt(geom.delta_det_channel)) * (cos_alpha / np.cos(theta_p).astype(dt))
    return n_p, n_p_center, w_p_c.astype(dt), cos_alpha


def _translation_xy(geom, pixel_indices, tv, dt):
    """recon_ijk_to_xyz, translation_model.py:646-656: (x_p, y_p) of each pixel for translation vector tv."""
    nr, nc = geom.recon_shape[:2]
    row, col = np.unravel_index(np.asarray(pixel_indices, dtype=np.int64), (nr, nc))
    y_p = dt(geom.delta_recon_row) * (row.astype(dt) - dt((nr - 1) / 2.0)) - dt(tv[1])
    x_p = dt(geom.delta_voxel) * (col.astype(dt) - dt((nc - 1) / 2.0)) - dt(tv[0])
    return x_p, y_p


def _translation_pixel_mag(geom, pixel_indices, tv, dt):
    """compute_y_mag_for_pixel, translation_model.py:694-706."""
    _, y_p = _translation_xy(geom, pixel_indices, tv, dt)
    return dt(1) / (dt(1 / geom.magnification) - y_p / dt(geom.source_detector_dist))


def translation_horizontal_data(geom, pixel_indices, tv, dt=np.float32):
    """translation_model.py:595-644: returns n_p, n_p_center, W_p_c, cos_theta_p."""
    x_p, y_p = _translation_xy(geom, pixel_indices, tv, dt)
    D = dt(geom.source_detector_dist)
    pixel_mag = dt(1) / (dt(1 / geom.magnification) - y_p / D)
    u_p = pixel_mag * x_p
    det_center_channel = dt((geom.sinogram_shape[2] - 1) / 2.0)
    n_p = (u_p + dt(geom.det_channel_offset)) / dt(geom.delta_det_channel) + det_center_channel
    n_p_center = np.round(n_p).astype(np.int64)
    cos_theta = np.cos(np.arctan2(u_p, D).astype(dt)).astype(dt)
    w_p_c = pixel_mag * (dt(geom.delta_voxel) / dt(geom.delta_det_channel))
    return n_p, n_p_center, w_p_c.astype(dt), cos_theta


def _channel_matrix(geom, pixel_indices, angle, dt, coeff_power):
    """Sparse (C x N) matrix of channel coefficients A_chan_n for one view (raised to coeff_power).

    The coefficient is the reference's (parallel_beam.py:170-175 / cone_beam.py:276-281 / translation_model.py:
    275-281, where it has no delta_voxel factor); ``angle`` is the translation vector for translation geometry."""
    if geom.kind == 'parallel':
        n_p, n_c, w, cos_a = parallel_proj_data(geom, pixel_indices, angle, dt)
    elif geom.kind == 'cone':
        n_p, n_c, w, cos_a = cone_horizontal_data(geom, pixel_indices, angle, dt)
    else:
        n_p, n_c, w, cos_a = translation_horizontal_data(geom, pixel_indices, angle, dt)
    num_det_channels = geom.sinogram_shape[2]
    l_max = np.minimum(dt(1), w)
    num_pixels = n_p.shape[0]
    taps = 2 * geom.psf_radius + 1
    rows = np.empty((num_pixels, taps), dtype=np.int64)
    vals = np.empty((num_pixels, taps), dtype=dt)
    for t, n_offset in enumerate(range(-geom.psf_radius, geom.psf_radius + 1)):
        n = n_c + n_offset
        abs_delta = np.abs(n_p - n.astype(dt))
        l_pcn = np.clip((w + dt(1)) / dt(2) - abs_delta, dt(0), l_max)
        a = l_pcn / cos_a if geom.kind == 'translation' else dt(geom.delta_voxel) * l_pcn / cos_a
        valid = (n >= 0) & (n < num_det_channels)
        a = a * valid.astype(dt)
        if coeff_power != 1:
            a = a ** coeff_power
        rows[:, t] = np.clip(n, 0, num_det_channels - 1)  # a tap off the detector has coefficient 0
        vals[:, t] = a
    # one column per pixel holding its taps (rows ascending), built directly in compressed-column form
    indptr = np.arange(0, taps * num_pixels + 1, taps, dtype=np.int64)
    return sp.csc_matrix((vals.ravel(), rows.ravel(), indptr), shape=(num_det_channels, num_pixels), dtype=dt)


def _cone_pixel_mag(geom, pixel_indices, angle, dt):
    """compute_y_mag_for_pixel, cone_beam.py:740-760."""
    x_tilde, y_tilde = _pixel_xy_tilde(geom, pixel_indices, dt)
    angle = dt(angle)
    cosine, sine = dt(np.cos(angle)), dt(np.sin(angle))
    y = sine * x_tilde + cosine * y_tilde
    return dt(1) / (dt(1 / geom.magnification) - y / dt(geom.source_detector_dist))


def cone_forward_vertical(geom, voxel_values, pixel_indices, angle, dt=np.float32):
    """cone_beam.py:286-377, vectorised over pixels: (N, S) voxel cylinders -> (N, R) detector columns."""
    pixel_mag = _cone_pixel_mag(geom, pixel_indices, angle, dt)
    return _fan_forward_vertical(geom, voxel_values, pixel_mag, geom.recon_slice_offset, geom.bp_psf_radius, dt)


def translation_forward_vertical(geom, voxel_values, pixel_indices, tv, dt=np.float32):
    """translation_model.py:286-378: the cone's detector-row-centric fan with slice heights
    delta_voxel (k - (S-1)/2) - tz and psf_radius taps."""
    pixel_mag = _translation_pixel_mag(geom, pixel_indices, tv, dt)
    return _fan_forward_vertical(geom, voxel_values, pixel_mag, -dt(tv[2]), geom.psf_radius, dt)


def _fan_forward_vertical(geom, voxel_values, pixel_mag, zoff, radius, dt):
    num_views, num_det_rows, _ = geom.sinogram_shape
    num_slices = voxel_values.shape[1]
    dv = dt(geom.delta_voxel)
    pixel_mag = pixel_mag[:, None]                                             # (N, 1)
    k = np.arange(num_slices)
    z = dv * (k.astype(dt) - dt((num_slices - 1) / 2.0)) + dt(zoff)
    v = pixel_mag * z[None, :]
    D = dt(geom.source_detector_dist)
    cos_phi = np.cos(np.arctan2(v, D).astype(dt)).astype(dt)
    scaled = (voxel_values.astype(dt) / cos_phi).astype(dt)                   # (N, S)
    w_p_r = (pixel_mag * dv) / dt(geom.delta_det_row)                         # (N, 1)
    slope = w_p_r
    l_max = np.minimum(dt(1), w_p_r)
    rows_per_batch = min(geom.entries_per_cylinder_batch, num_det_rows)
    num_batches = (num_det_rows + rows_per_batch - 1) // rows_per_batch
    det_center_row = dt((num_det_rows - 1) / 2.0)
    row_batch = np.arange(rows_per_batch)
    columns = []
    for b in range(num_batches):
        start = rows_per_batch * b
        m_center = start + row_batch
        v_m = (m_center.astype(dt) - det_center_row) * dt(geom.delta_det_row) - dt(geom.det_row_offset)
        z_m = v_m[None, :] / pixel_mag                                          # (N, rpb)
        k_m = (z_m - dt(zoff)) / dv + dt((num_slices - 1) / 2.0)
        k_m_center = np.round(k_m).astype(np.int64)
        m_p = slope * (k_m_center.astype(dt) - k_m[:, :1]) + dt(m_center[0])
        new_col = np.zeros(k_m.shape, dtype=dt)
        for k_offset in range(-radius, radius + 1):
            k_ind = k_m_center + k_offset
            abs_delta = np.abs(m_p + slope * dt(k_offset) - m_center[None, :].astype(dt))
            a = np.clip((w_p_r + dt(1)) / dt(2) - abs_delta, dt(0), l_max)
            a = a * ((k_ind >= 0) & (k_ind < num_slices)).astype(dt)
            gathered = np.take_along_axis(scaled, np.clip(k_ind, 0, num_slices - 1), axis=1)
            new_col = new_col + a * gathered
        columns.append(new_col)
    return np.concatenate(columns, axis=1)[:, :num_det_rows].astype(dt)


def cone_back_vertical(geom, det_columns, pixel_indices, angle, coeff_power=1, dt=np.float32):
    """cone_beam.py:480-591, vectorised over pixels: (N, R) detector columns -> (N, S) voxel cylinders."""
    x_tilde, y_tilde = _pixel_xy_tilde(geom, pixel_indices, dt)
    angle = dt(angle)
    cosine, sine = dt(np.cos(angle)), dt(np.sin(angle))
    y_p = sine * x_tilde + cosine * y_tilde
    pixel_mag = dt(1) / (dt(1 / geom.magnification) - y_p / dt(geom.source_detector_dist))
    return _fan_back_vertical(geom, det_columns, pixel_mag, geom.recon_slice_offset, coeff_power, dt)


def translation_back_vertical(geom, det_columns, pixel_indices, tv, coeff_power=1, dt=np.float32):
    """translation_model.py:482-593: the cone's voxel-centric fan with slice heights
    delta_voxel (k - (S-1)/2) - tz."""
    pixel_mag = _translation_pixel_mag(geom, pixel_indices, tv, dt)
    return _fan_back_vertical(geom, det_columns, pixel_mag, -dt(tv[2]), coeff_power, dt)


def _fan_back_vertical(geom, det_columns, pixel_mag, zoff, coeff_power, dt):
    num_views, num_det_rows, _ = geom.sinogram_shape
    num_slices = geom.recon_shape[2]
    dv = dt(geom.delta_voxel)
    D = dt(geom.source_detector_dist)
    pixel_mag = pixel_mag[:, None]                                             # (N, 1)
    slices_per_batch = min(geom.entries_per_cylinder_batch, num_slices)
    num_batches = (num_slices + slices_per_batch - 1) // slices_per_batch
    det_center_row = dt((num_det_rows - 1) / 2.0)
    out = []
    for b in range(num_batches):
        cur = slices_per_batch * b + np.arange(slices_per_batch)
        z_p = dv * (cur.astype(dt) - dt((num_slices - 1) / 2.0)) + dt(zoff)
        v_p = pixel_mag * z_p[None, :]
        m_p = (v_p + dt(geom.det_row_offset)) / dt(geom.delta_det_row) + det_center_row
        m_c = np.round(m_p).astype(np.int64)
        cos_phi = np.cos(np.arctan2(v_p, D).astype(dt)).astype(dt)
        w_p_r = pixel_mag * (dv / dt(geom.delta_det_row))
        l_max = np.minimum(dt(1), w_p_r)
        new_cyl = np.zeros(m_p.shape, dtype=dt)
        for m_offset in range(-geom.psf_radius, geom.psf_radius + 1):
            m = m_c + m_offset
            abs_delta = np.abs(m_p - m.astype(dt))
            l_prm = np.clip((w_p_r + dt(1)) / dt(2) - abs_delta, dt(0), l_max)
            a = l_prm / cos_phi
            a = a * ((m >= 0) & (m < num_det_rows)).astype(dt)
            if coeff_power != 1:
                a = a ** coeff_power
            gathered = np.take_along_axis(det_columns, np.clip(m, 0, num_det_rows - 1), axis=1)
            new_cyl = new_cyl + a * gathered
        out.append(new_cyl)
    return np.concatenate(out, axis=1)[:, :num_slices].astype(dt)


def forward_project_one_view(geom, voxel_values, pixel_indices, angle, dt=np.float32):
    """(N, S) -> (R, C) for one view; parallel_beam.py:138-178 / cone_beam.py:189-217 /
    translation_model.py:190-217."""
    voxel_values = np.asarray(voxel_values, dtype=dt)
    if geom.kind == 'parallel':
        columns = voxel_values                                                  # slice k <-> row k
    elif geom.kind == 'cone':
        columns = cone_forward_vertical(geom, voxel_values, pixel_indices, angle, dt)
    else:
        columns = translation_forward_vertical(geom, voxel_values, pixel_indices, angle, dt)
    chan = _channel_matrix(geom, pixel_indices, angle, dt, 1)
    return np.asarray((chan @ columns).T, dtype=dt)


def back_project_one_view(geom, view, pixel_indices, angle, coeff_power=1, dt=np.float32):
    """(R, C) -> (N, S) for one view; parallel_beam.py:180-221 / cone_beam.py:379-407 /
    translation_model.py:382-410."""
    view = np.asarray(view, dtype=dt)
    chan = _channel_matrix(geom, pixel_indices, angle, dt, coeff_power)
    columns = np.asarray(chan.T @ view.T, dtype=dt)                             # (N, R)
    if geom.kind == 'parallel':
        return columns
    if geom.kind == 'cone':
        return cone_back_vertical(geom, columns, pixel_indices, angle, coeff_power, dt)
    return translation_back_vertical(geom, columns, pixel_indices, angle, coeff_power, dt)


def _view_list(geom, view_indices):
    if view_indices is None:
        return np.arange(geom.sinogram_shape[0])
    return np.asarray(view_indices, dtype=np.int64)


def sparse_forward_project(geom, voxel_values, pixel_indices, view_indices=None, dtype=np.float32):
    """tomography_model.py:576-622 / projectors.py:61-129: (N, S) -> (len(view_indices), R, C)."""
    dt = np.dtype(dtype).type
    views = _view_list(geom, view_indices)
    _, num_det_rows, num_det_channels = geom.sinogram_shape
    out = np.zeros((len(views), num_det_rows, num_det_channels), dtype=dt)
    for j, v in enumerate(views):
        out[j] = forward_project_one_view(geom, voxel_values, pixel_indices, geom.angles[v], dt)
    return out


def sparse_back_project(geom, sinogram, pixel_indices, view_indices=None, coeff_power=1, dtype=np.float32):
    """tomography_model.py:624-677 / projectors.py:131-209: full sinogram -> (N, S).

    ``view_indices`` index the first axis of ``sinogram`` and the angle table together."""
    dt = np.dtype(dtype).type
    views = _view_list(geom, view_indices)
    num_slices = geom.recon_shape[2]
    out = np.zeros((len(pixel_indices), num_slices), dtype=dt)
    for v in views:
        out += back_project_one_view(geom, sinogram[v], pixel_indices, geom.angles[v], coeff_power, dt)
    return out


def forward_project(geom, recon, dtype=np.float32):
    """tomography_model.py:531-551: full FP over the region of reconstruction."""
    idx = gen_full_indices(geom.recon_shape)
    flat = np.asarray(recon).reshape((-1, geom.recon_shape[2]))
    return sparse_forward_project(geom, flat[idx], idx, dtype=dtype)


def back_project(geom, sinogram, dtype=np.float32):
    """tomography_model.py:553-574: full BP, zero outside the region of reconstruction."""
    idx = gen_full_indices(geom.recon_shape)
    cyl = sparse_back_project(geom, sinogram, idx, dtype=dtype)
    out = np.zeros((geom.recon_shape[0] * geom.recon_shape[1], geom.recon_shape[2]), dtype=cyl.dtype)
    out[idx] = cyl
    return out.reshape(geom.recon_shape)


def compute_hessian_diagonal(geom, weights=None, dtype=np.float32):
    """tomography_model.py:679-708: BP of the weights with squared coefficients over every pixel."""
    if weights is None:
        weights = np.ones(geom.sinogram_shape, dtype=dtype)
    nr, nc, ns = geom.recon_shape
    idx = np.arange(nr * nc)
    return sparse_back_project(geom, weights, idx, coeff_power=2, dtype=dtype).reshape((nr, nc, ns))
