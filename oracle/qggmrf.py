"""qGGMRF prior restated in NumPy (test infrastructure only).

* ``get_b_from_nbr_wts``: ``qggmrf.py:388-395``
* ``get_2_b_tilde``: ``qggmrf.py:250-279``
* surrogate gradient / Hessian at indices: ``qggmrf.py:118-148`` with the per-cylinder pass
  ``qggmrf.py:151-188`` and the per-slice pass ``qggmrf.py:191-247`` (``mode='clip'`` neighbours)
* ``qggmrf_loss``: ``qggmrf.py:31-65``
* ``b_tilde_by_definition`` / ``compute_qggmrf_grad_and_hessian``: ``qggmrf.py:282-294, 344-385``
* ``qggmrf_loss_grad``: the analytic gradient of ``qggmrf_loss`` (the reference obtains it by autodiff);
  derived from rho(a) = a^p/(p sigma^p) u/(1+u), u = (a/(T sigma))^(q-p), a = max(|delta|, T sigma eps).
"""
import numpy as np

EPS_F32 = float(np.finfo(np.float32).eps)


def get_b_from_nbr_wts(qggmrf_nbr_wts):
    b = np.array([qggmrf_nbr_wts, qggmrf_nbr_wts]).T.flatten()
    b = b / np.sum(b)
    return tuple(float(v) for v in b)


def get_2_b_tilde(delta, b_for_delta, qggmrf_params, dt=np.float32):
    b, sigma_x, p, q, T = qggmrf_params
    delta = np.asarray(delta, dtype=dt)
    scaled_delta = np.abs(delta) / dt(T * sigma_x) + dt(EPS_F32)
    delta_q_minus_2 = scaled_delta ** dt(q - 2.0)
    delta_q_minus_p = scaled_delta ** dt(q - p)
    numerator = delta_q_minus_2 * (dt(q / p) + delta_q_minus_p)
    denominator = (dt(1) + delta_q_minus_p) ** 2
    scale = (T ** (p - 2)) / (sigma_x * sigma_x)
    rho_prime_over_delta = dt(scale) * numerator / denominator
    return (dt(b_for_delta) * rho_prime_over_delta).astype(dt)


def _per_cylinder(cylinders, qggmrf_params, dt):
    b = qggmrf_params[0]
    b_plus, b_minus = b[4], b[5]
    zero = np.zeros((cylinders.shape[0], 1), dtype=dt)
    delta = np.concatenate((zero, np.diff(cylinders, axis=1).astype(dt), zero), axis=1)
    b2 = get_2_b_tilde(delta, 1.0, qggmrf_params, dt)
    b2d = b2 * delta
    grad = -dt(b_plus) * b2d[:, 1:]
    hess = dt(b_plus) * b2[:, 1:]
    grad = grad + dt(b_minus) * b2d[:, :-1]
    hess = hess + dt(b_minus) * b2[:, :-1]
    return grad.astype(dt), hess.astype(dt)


def qggmrf_gradient_and_hessian_at_indices(flat_recon, recon_shape, pixel_indices, qggmrf_params,
                                           dt=np.float32):
    """Returns (gradient, hessian), each (len(pixel_indices), num_slices)."""
    flat_recon = np.asarray(flat_recon, dtype=dt)
    pixel_indices = np.asarray(pixel_indices, dtype=np.int64)
    b = qggmrf_params[0]
    grad, hess = _per_cylinder(flat_recon[pixel_indices], qggmrf_params, dt)
    num_rows, num_cols = recon_shape[:2]
    row, col = np.unravel_index(pixel_indices, (num_rows, num_cols))
    xs0 = flat_recon[pixel_indices]
    for (dr, dc), b_value in zip([(1, 0), (-1, 0), (0, 1), (0, -1)], [b[0], b[1], b[2], b[3]]):
        nbr = np.ravel_multi_index([row + dr, col + dc], (num_rows, num_cols), mode='clip')
        delta = xs0 - flat_recon[nbr]
        b2 = get_2_b_tilde(delta, b_value, qggmrf_params, dt)
        grad = grad + b2 * delta
        hess = hess + b2
    return grad.astype(dt), hess.astype(dt)


def _rho(delta, sigma_x, p, q, T, dt):
    a_min = dt(T * sigma_x * EPS_F32)
    abs_delta = np.maximum(np.abs(delta), a_min)
    delta_scale = abs_delta / dt(T * sigma_x)
    ds_q_minus_p = delta_scale ** dt(q - p)
    numerator = abs_delta ** dt(p) / dt(p * sigma_x ** p)
    numerator = numerator * ds_q_minus_p
    return numerator / (dt(1) + ds_q_minus_p)


def _rho_prime(delta, sigma_x, p, q, T, dt):
    a_min = dt(T * sigma_x * EPS_F32)
    a = np.abs(delta)
    clipped = a < a_min
    a = np.maximum(a, a_min)
    u = (a / dt(T * sigma_x)) ** dt(q - p)
    d = a ** dt(p - 1) / dt(sigma_x ** p) * u * (dt(q / p) + u) / (dt(1) + u) ** 2
    d = np.where(clipped, dt(0), d)
    return (np.sign(delta) * d).astype(dt)


def _b_per_axis(b):
    return [(b[j] + b[j + 1]) / (2 * sum(b)) for j in (0, 2, 4)]


def qggmrf_loss(full_recon, qggmrf_params, dt=np.float64):
    b, sigma_x, p, q, T = qggmrf_params
    full_recon = np.asarray(full_recon, dtype=dt)
    loss = 0.0
    for axis, b_axis in enumerate(_b_per_axis(b)):
        loss += b_axis * float(np.sum(_rho(np.diff(full_recon, axis=axis), sigma_x, p, q, T, dt), dtype=np.float64))
    return loss


def qggmrf_loss_grad(full_recon, qggmrf_params, dt=np.float64):
    b, sigma_x, p, q, T = qggmrf_params
    full_recon = np.asarray(full_recon, dtype=dt)
    grad = np.zeros_like(full_recon)
    for axis, b_axis in enumerate(_b_per_axis(b)):
        rp = dt(b_axis) * _rho_prime(np.diff(full_recon, axis=axis), sigma_x, p, q, T, dt)
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[axis] = slice(0, -1)
        hi[axis] = slice(1, None)
        grad[tuple(hi)] += rp
        grad[tuple(lo)] -= rp
    return grad


def b_tilde_by_definition(delta, sigma_x, p, q, T):
    a_min = T * sigma_x * EPS_F32
    abs_delta = np.maximum(np.abs(delta), a_min)
    delta_scale = abs_delta / (T * sigma_x)
    ds_q_minus_p = delta_scale ** (q - p)
    ds_p_minus_2 = abs_delta ** (p - 2)
    numerator = ds_p_minus_2 / (2 * sigma_x ** p)
    numerator = numerator * ds_q_minus_p * ((q / p) + ds_q_minus_p)
    return numerator / (1 + ds_q_minus_p) ** 2


def compute_qggmrf_grad_and_hessian(full_recon, qggmrf_params):
    """qggmrf.py:344-385, in float64."""
    b, sigma_x, p, q, T = qggmrf_params
    full_recon = np.asarray(full_recon, dtype=np.float64)
    hess = np.zeros_like(full_recon)
    grad = np.zeros_like(full_recon)
    for axis, b_axis in enumerate(_b_per_axis(b)):
        cur_delta = np.diff(full_recon, axis=axis)
        shape = list(full_recon.shape)
        shape[axis] = 1
        zero = np.zeros(shape)
        cur_delta = np.concatenate((zero, cur_delta, zero), axis=axis)
        bt = b_tilde_by_definition(cur_delta, sigma_x, p, q, T)
        n = bt.shape[axis]
        bt_plus = np.take(bt, np.arange(1, n), axis=axis)
        bt_minus = np.take(bt, np.arange(0, n - 1), axis=axis)
        d_plus = np.take(cur_delta, np.arange(1, n), axis=axis)
        d_minus = np.take(cur_delta, np.arange(0, n - 1), axis=axis)
        hess += 2 * b_axis * (bt_plus + bt_minus)
        grad += 2 * b_axis * (-bt_plus * d_plus + bt_minus * d_minus)
    return grad, hess
