"""VCD reconstruction restated in NumPy (test infrastructure only).

* auto regularization: ``tomography_model.py:756-932``
* ``vcd_recon``: ``tomography_model.py:1086-1255`` (direct-recon init, alpha rescale, Hessian diagonal,
  iterations, ``fm_rmse`` ``:1633-1658``, NMAE, stop test)
* ``vcd_partition_iterator``: ``tomography_model.py:1257-1308`` (``np.random.permutation`` subset order)
* subset update: ``tomography_model.py:1343-1542`` and ``get_forward_lin_quad`` ``:1546-1631``

Everything is float32, as the reference computes it; reductions are float32 sums.  Every function takes the
projector implementation as ``proj`` (default: the single-process ``oracle.projectors``; an
``oracle.pool.OraclePool`` spreads the views over the host cores).
"""
import numpy as np

from . import projectors as P
from .filters import fbp_filter, fdk_filter
from .qggmrf import get_b_from_nbr_wts, qggmrf_gradient_and_hessian_at_indices
from .partitions import gen_set_of_pixel_partitions, gen_partition_sequence

EPS_F32 = np.float32(np.finfo(np.float32).eps)


def auto_regularization(geom, sinogram, weights=None, snr_db=30.0, sharpness=1.0):
    """Returns (sigma_y, sigma_x, sigma_prox) as the reference's auto_set_* compute them."""
    max_views_to_use = np.minimum(20, sinogram.shape[0])
    step_size = sinogram.shape[0] // max_views_to_use
    small_sino = np.array(sinogram[::step_size])
    small_w = 1 if weights is None else np.array(weights[::step_size])
    indicator = np.int8(small_sino > (0.01 * 5.0) * np.mean(np.fabs(small_sino)))
    mag = geom.magnification
    signal_rms = float(np.average(small_w * small_sino ** 2, None, indicator) ** 0.5)
    rel_noise_std = 10 ** (-snr_db / 20)
    pixel_pitch_rel = geom.delta_voxel / (geom.delta_det_channel / mag)
    sigma_y = np.float32(rel_noise_std * signal_rms * (pixel_pitch_rel ** 0.5))
    typical_sino = np.average(np.abs(small_sino), weights=indicator)
    rs = geom.recon_shape
    path_space = (2 * rs[0] * rs[1]) / (rs[0] + rs[1]) * geom.delta_voxel
    path_sino = small_sino.shape[-1] * geom.delta_det_channel / mag
    recon_std = typical_sino / np.minimum(path_space, path_sino)
    sigma_x = np.float32(0.2 * (2 ** sharpness) * recon_std)
    return float(sigma_y), float(sigma_x), float(sigma_x)


def direct_recon(geom, sinogram, proj=P):
    if geom.kind == 'translation':  # no direct recon: the base model's zeros (tomography_model.py:934-949)
        return np.zeros(geom.recon_shape, dtype=np.float32)
    if geom.kind == 'parallel':
        filtered = fbp_filter(sinogram, geom.delta_voxel)
    else:
        filtered = fdk_filter(sinogram, geom.source_detector_dist, geom.magnification, geom.delta_voxel,
                              geom.delta_det_row, geom.delta_det_channel, geom.det_row_offset,
                              geom.det_channel_offset)
    return proj.back_project(geom, filtered)


def forward_model_loss(error_sinogram, sigma_y, weights=None):
    if weights is None:
        return float(np.sqrt((1.0 / sigma_y ** 2) * np.mean(error_sinogram * error_sinogram)))
    avg = np.average(weights)
    return float(np.sqrt((1.0 / sigma_y ** 2) * np.mean((error_sinogram * error_sinogram) * (weights / avg))))


def vcd_subset_update(geom, flat_recon, error_sinogram, weights, fm_hessian, pixel_indices, fm_constant,
                      qggmrf_params, prox_input=None, sigma_prox=None, positivity=False, proj=P):
    """One subset step; returns (flat_recon, error_sinogram, ell1, alpha).

    prox_input (flat, like flat_recon): the proximal-map prior of tomography_model.py:1388-1391 instead of qGGMRF,
    gradient (x - v) / sigma_prox^2 (qggmrf.py:8-28) and Hessian sigma_prox^2, as the reference writes it.
    positivity: the clip of tomography_model.py:1497-1507, delta >= -x / (alpha + eps) after alpha is found, then
    the forward projection of the clipped delta; alpha is not recomputed."""
    f32 = np.float32
    if prox_input is None:
        prior_grad, prior_hess = qggmrf_gradient_and_hessian_at_indices(flat_recon, geom.recon_shape, pixel_indices,
                                                                        qggmrf_params)
    else:
        prior_grad = ((1.0 / (f32(sigma_prox) ** 2.0)) *
                      (flat_recon[pixel_indices] - prox_input[pixel_indices])).astype(f32)
        prior_hess = f32(sigma_prox) ** 2
    wes = error_sinogram if weights is None else (weights * error_sinogram).astype(f32)
    forward_grad = (-fm_constant * proj.sparse_back_project(geom, wes, pixel_indices)).astype(f32)
    forward_hess = (fm_constant * fm_hessian[pixel_indices]).astype(f32)
    delta = (-((forward_grad + prior_grad) / (forward_hess + prior_hess))).astype(f32)
    prior_linear = np.sum(prior_grad * delta, dtype=f32)
    prior_quad = f32(0.5) * np.sum(prior_hess * delta ** 2, dtype=f32)
    delta_sino = proj.sparse_forward_project(geom, delta, pixel_indices)
    forward_linear = f32(fm_constant) * np.sum(wes * delta_sino, dtype=f32)
    w = 1 if weights is None else weights
    forward_quad = f32(fm_constant) * np.sum(delta_sino * delta_sino * w, dtype=f32)
    alpha = (forward_linear - prior_linear) / (forward_quad + prior_quad + EPS_F32)
    alpha = f32(np.clip(alpha, EPS_F32, 1.5))
    if positivity:
        pos_constant = f32(1.0) / (alpha + EPS_F32)
        delta = np.maximum(-pos_constant * flat_recon[pixel_indices], delta).astype(f32)
        delta_sino = proj.sparse_forward_project(geom, delta, pixel_indices)
    delta = (alpha * delta).astype(f32)
    flat_recon = flat_recon.copy()
    np.add.at(flat_recon, pixel_indices, delta)
    error_sinogram = (error_sinogram - (alpha * delta_sino)).astype(f32)
    ell1 = float(np.sum(np.abs(delta), dtype=f32))
    return flat_recon, error_sinogram, ell1, float(alpha)


def vcd_recon(geom, sinogram, partitions, partition_sequence, *, sigma_y, sigma_x, p=2.0, q=1.2, T=1.0,
              qggmrf_nbr_wts=(1.0, 1.0, 1.0), weights=None, init_recon=None, stop_threshold_change_pct=0.0,
              prox_input=None, sigma_prox=None, positivity=False, proj=P):
    """Returns (recon, dict(fm_rmse, nmae_update, alpha_values))."""
    f32 = np.float32
    sinogram = np.asarray(sinogram, dtype=f32)
    if init_recon is None:
        init_recon = direct_recon(geom, sinogram, proj)
    elif isinstance(init_recon, int) and init_recon == 0:
        init_recon = np.zeros(geom.recon_shape, dtype=f32)
    init_recon = np.asarray(init_recon, dtype=f32)
    es = proj.forward_project(geom, init_recon)
    wes = es if weights is None else (weights * es).astype(f32)
    norm = np.sum(wes * es, dtype=f32)
    alpha = np.sum(wes * sinogram, dtype=f32) / norm if norm > 0 else f32(1)
    error_sinogram = (sinogram - alpha * es).astype(f32)
    recon = (alpha * init_recon).astype(f32)
    fm_hessian = proj.compute_hessian_diagonal(geom, weights).reshape((-1, geom.recon_shape[2]))
    fm_constant = 1.0 / (sigma_y ** 2.0)
    b = get_b_from_nbr_wts(list(qggmrf_nbr_wts))
    qparams = (b, sigma_x, p, q, T)
    flat_recon = recon.reshape((-1, geom.recon_shape[2]))
    prox_flat = None if prox_input is None else np.asarray(prox_input, dtype=f32).reshape((-1, geom.recon_shape[2]))
    fm_rmse, nmae, alphas = [], [], []
    for i in range(len(partition_sequence)):
        partition = partitions[partition_sequence[i]]
        ell1_sum, alpha_sum = 0.0, 0.0
        for index in np.random.permutation(partition.shape[0]):
            flat_recon, error_sinogram, ell1, a = vcd_subset_update(
                geom, flat_recon, error_sinogram, weights, fm_hessian, partition[index], fm_constant, qparams,
                prox_flat, sigma_prox, positivity, proj)
            ell1_sum += ell1
            alpha_sum += a
        fm_rmse.append(forward_model_loss(error_sinogram, sigma_y, weights))
        nmae.append(ell1_sum / float(np.sum(np.abs(flat_recon))))
        alphas.append(alpha_sum / partition.shape[0])
        if nmae[-1] < stop_threshold_change_pct / 100:
            break
    return flat_recon.reshape(geom.recon_shape), dict(fm_rmse=fm_rmse, nmae_update=nmae, alpha_values=alphas,
                                                     error_sinogram=error_sinogram)


def recon(geom, sinogram, *, granularity, partition_sequence, max_iterations, weights=None, init_recon=None,
          snr_db=30.0, sharpness=1.0, p=2.0, q=1.2, T=1.0, qggmrf_nbr_wts=(1.0, 1.0, 1.0),
          stop_threshold_change_pct=0.2, positivity=False, proj=P):
    """tomography_model.py:966-1084 with the reference's np.random call order."""
    sigma_y, sigma_x, _ = auto_regularization(geom, sinogram, weights, snr_db, sharpness)
    partitions = gen_set_of_pixel_partitions(geom.recon_shape, granularity)
    seq = gen_partition_sequence(partition_sequence, max_iterations)
    out, stats = vcd_recon(geom, sinogram, partitions, seq, sigma_y=sigma_y, sigma_x=sigma_x, p=p, q=q, T=T,
                           qggmrf_nbr_wts=qggmrf_nbr_wts, weights=weights, init_recon=init_recon,
                           stop_threshold_change_pct=stop_threshold_change_pct, positivity=positivity, proj=proj)
    stats['sigma_y'], stats['sigma_x'] = sigma_y, sigma_x
    return out, stats


def prox_map(geom, prox_input, sinogram, *, sigma_y, sigma_x, sigma_prox, granularity, partition_sequence,
             max_iterations, weights=None, init_recon=None, stop_threshold_change_pct=0.2, positivity=False):
    """tomography_model.py:1660-1697: partitions for every granularity entry, the partition sequence, then
    vcd_recon with the proximal prior (the regularisation parameters are the model's current ones)."""
    partitions = gen_set_of_pixel_partitions(geom.recon_shape, granularity)
    seq = gen_partition_sequence(partition_sequence, max_iterations)
    return vcd_recon(geom, sinogram, partitions, seq, sigma_y=sigma_y, sigma_x=sigma_x, weights=weights,
                     init_recon=init_recon, stop_threshold_change_pct=stop_threshold_change_pct,
                     prox_input=prox_input, sigma_prox=sigma_prox, positivity=positivity)
