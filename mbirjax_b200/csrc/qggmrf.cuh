// qGGMRF prior parameters and per-voxel surrogate gradient / Hessian, shared by qggmrf.cu and vcd.cu.
// Restates get_2_b_tilde (qggmrf.py:250-279) and the cylinder / in-slice neighbour passes of
// qggmrf_gradient_and_hessian_at_indices (qggmrf.py:151-247).
#pragma once

#include <cmath>

#include "mbx_common.cuh"

namespace mbx {

struct QParams {
    float b[6];
    float t_sigma;      // T * sigma_x
    float q_minus_2;
    float q_minus_p;
    float q_over_p;
    float scale;        // T^(p-2) / sigma_x^2
    float p;
    float p_minus_1;
    float inv_p_sigma_p;  // 1 / (p sigma_x^p)
    float inv_sigma_p;    // 1 / sigma_x^p
    float a_min;          // T sigma_x eps
    float b_axis[3];      // (b_j + b_{j+1}) / (2 sum b) for rows, cols, slices
};

inline QParams make_qparams(const mbx_qggmrf_params &qp) {
    QParams q;
    double bsum = 0.0;
    for (int i = 0; i < 6; ++i) {
        q.b[i] = qp.b[i];
        bsum += qp.b[i];
    }
    const double T = qp.T, s = qp.sigma_x, p = qp.p, qq = qp.q;
    q.t_sigma = (float)(T * s);
    q.q_minus_2 = (float)(qq - 2.0);
    q.q_minus_p = (float)(qq - p);
    q.q_over_p = (float)(qq / p);
    q.scale = (float)(std::pow(T, p - 2.0) / (s * s));
    q.p = (float)p;
    q.p_minus_1 = (float)(p - 1.0);
    q.inv_p_sigma_p = (float)(1.0 / (p * std::pow(s, p)));
    q.inv_sigma_p = (float)(1.0 / std::pow(s, p));
    q.a_min = (float)(T * s * 1.1920928955078125e-07);
    for (int a = 0; a < 3; ++a) q.b_axis[a] = (float)((qp.b[2 * a] + qp.b[2 * a + 1]) / (2.0 * bsum));
    return q;
}

// 2 * b_tilde(delta) for neighbour weight b (get_2_b_tilde, qggmrf.py:250-279).
__device__ __forceinline__ float two_b_tilde(float delta, float b, const QParams &q) {
    const float s = fabsf(delta) / q.t_sigma + 1.1920928955078125e-07f;
    const float d_q2 = powf(s, q.q_minus_2);
    // p = 2 (the default) makes the two exponents equal: one power, the same value
    const float d_qp = q.q_minus_p == q.q_minus_2 ? d_q2 : powf(s, q.q_minus_p);
    const float num = d_q2 * (q.q_over_p + d_qp);
    const float den = (1.0f + d_qp) * (1.0f + d_qp);
    return b * (q.scale * num / den);
}

// Surrogate gradient and Hessian of one voxel (pixel index idx, slice k) of a flat recon.
__device__ __forceinline__ void qggmrf_voxel(const float *__restrict__ recon, int nr, int nc, int ns, int idx, int k,
                                             const QParams &q, float &grad, float &hess) {
    const float *cyl = recon + (long long)idx * ns;
    const float x0 = __ldg(cyl + k);
    // cylinder neighbours: delta[k+1] = x[k+1] - x[k] (0 at the end), delta[k] = x[k] - x[k-1] (0 at the start)
    const float d_plus = (k + 1 < ns) ? __ldg(cyl + k + 1) - x0 : 0.0f;
    const float d_minus = (k > 0) ? x0 - __ldg(cyl + k - 1) : 0.0f;
    const float bt_plus = two_b_tilde(d_plus, 1.0f, q);
    const float bt_minus = two_b_tilde(d_minus, 1.0f, q);
    grad = -q.b[4] * (bt_plus * d_plus);
    hess = q.b[4] * bt_plus;
    grad += q.b[5] * (bt_minus * d_minus);
    hess += q.b[5] * bt_minus;
    // in-slice neighbours with clipped indices: row+1, row-1, col+1, col-1
    const int row = idx / nc;
    const int col = idx - row * nc;
    const int nbr[4] = {min(row + 1, nr - 1) * nc + col, max(row - 1, 0) * nc + col, row * nc + min(col + 1, nc - 1),
                        row * nc + max(col - 1, 0)};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const float delta = x0 - __ldg(recon + (long long)nbr[j] * ns + k);
        const float bt = two_b_tilde(delta, q.b[j], q);
        grad += bt * delta;
        hess += bt;
    }
}

}  // namespace mbx
