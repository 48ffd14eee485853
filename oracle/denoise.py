"""NumPy restatement of the reference's qGGMRF denoiser and median filter (test infrastructure only).

* ``vcd_subset_denoiser``: denoising.py:366-411 (identity forward model, forward Hessian 1, prior quadratic term
  over-relaxed by 1.1, alpha clipped to [eps, 1.5])
* ``denoise``: the iteration of QGGMRFDenoiser.denoise (denoising.py:197-330): one partition, subsets in order,
  stop when the relative change drops below the threshold
* ``estimate_image_noise_std``: denoising.py:80-136
* ``median_filter3d``: denoising.py:414-490, the 27-point median with edge replication
"""
import numpy as np

from .qggmrf import qggmrf_gradient_and_hessian_at_indices

EPS_F32 = np.finfo(np.float32).eps


def vcd_subset_denoiser(flat_image, flat_error_image, pixel_indices, fm_constant, qggmrf_params, image_shape):
    f32 = np.float32
    prior_grad, prior_hess = qggmrf_gradient_and_hessian_at_indices(flat_image, image_shape, pixel_indices,
                                                                    qggmrf_params)
    cur_error = flat_error_image[pixel_indices]
    forward_grad = (-f32(fm_constant) * cur_error).astype(f32)
    delta = (-((forward_grad + prior_grad) / (f32(1) + prior_hess))).astype(f32)
    prior_linear = np.sum(prior_grad * delta, dtype=np.float64)
    prior_quad = (1 / 1.1) * np.sum(prior_hess * delta ** 2, dtype=np.float64)
    forward_linear = fm_constant * np.sum(cur_error * delta, dtype=np.float64)
    forward_quad = fm_constant * np.sum(delta * delta, dtype=np.float64)
    alpha = (forward_linear - prior_linear) / (forward_quad + prior_quad + EPS_F32)
    alpha = f32(np.clip(alpha, EPS_F32, 1.5))
    delta = (alpha * delta).astype(f32)
    flat_image = flat_image.copy()
    np.add.at(flat_image, pixel_indices, delta)
    flat_error_image = flat_error_image.copy()
    flat_error_image[pixel_indices] = (cur_error - delta).astype(f32)
    return flat_image, flat_error_image, float(np.sum(np.abs(delta), dtype=np.float64)), float(alpha)


def denoise(image, partition, sigma_y, qggmrf_params, max_iterations, stop_threshold_change_pct, init_image=None):
    """Returns (denoised image, nmae per iteration, mean alpha per iteration)."""
    image = np.asarray(image, dtype=np.float32)
    shape = image.shape
    init = image.copy() if init_image is None else np.asarray(init_image, dtype=np.float32)
    flat_error = (image - init).reshape((-1, shape[2]))
    flat_image = init.reshape((-1, shape[2])).copy()
    fm_constant = 1.0 / (sigma_y ** 2.0)
    nmae, alphas = [], []
    for _ in range(max_iterations):
        l1, asum = 0.0, 0.0
        for subset in partition:
            flat_image, flat_error, ell1, a = vcd_subset_denoiser(flat_image, flat_error, subset, fm_constant,
                                                                  qggmrf_params, shape)
            l1 += ell1
            asum += a
        nmae.append(l1 / float(np.sum(np.abs(flat_image), dtype=np.float64)))
        alphas.append(asum / len(partition))
        if nmae[-1] < stop_threshold_change_pct / 100.0:
            break
    return flat_image.reshape(shape), nmae, alphas


def _support(noisy_image, sigma_noise):
    threshold = 0.05 * np.mean(np.fabs(noisy_image)) + sigma_noise
    threshold = min(threshold, np.amax(noisy_image))
    return np.int8(noisy_image >= threshold)


def _neighbour_std(noisy_image, support):
    inds = [np.clip(i, 1, None) for i in np.where(support)]
    vals = np.stack([noisy_image[inds[0], inds[1], inds[2]], noisy_image[inds[0] - 1, inds[1], inds[2]],
                     noisy_image[inds[0], inds[1] - 1, inds[2]], noisy_image[inds[0], inds[1], inds[2] - 1]], axis=0)
    return np.mean(np.std(vals, axis=0))


def estimate_image_noise_std(image):
    image = np.asarray(image)
    s = _neighbour_std(image, _support(image, 0.0))
    return _neighbour_std(image, _support(image, s))


def median_filter3d(x):
    """Median of every 3x3x3 neighbourhood of the edge-padded volume (float32)."""
    x = np.asarray(x, dtype=np.float32)
    xp = np.pad(x, 1, mode='edge')
    d0, d1, d2 = x.shape
    stack = np.stack([xp[a:a + d0, b:b + d1, c:c + d2] for a in range(3) for b in range(3) for c in range(3)])
    return np.median(stack, axis=0).astype(np.float32)
