// qGGMRF prior kernels (sm_100a).
//
// mbx_qggmrf_grad_hess replaces qggmrf_gradient_and_hessian_at_indices (qggmrf.py:118-148): the
// per-cylinder pass (qggmrf.py:151-188, zero differences beyond both ends of the cylinder) and the
// per-slice pass over the four in-slice neighbours with clipped indices (qggmrf.py:191-247), both built on
// get_2_b_tilde (qggmrf.py:250-279).  One thread per (subset pixel, slice), lanes along the slice axis, so
// every read of the centre and of each neighbour cylinder is coalesced.
//
// mbx_qggmrf_loss_grad replaces qggmrf_loss (qggmrf.py:31-65) and adds its analytic gradient (the
// reference differentiates it with autodiff): rho(a) = a^p/(p sigma^p) u/(1+u), u = (a/(T sigma))^(q-p),
// a = max(|delta|, T sigma eps), and rho'(delta) = sign(delta) a^(p-1)/sigma^p u (q/p + u)/(1+u)^2 (0 where
// the clip is active).  Each voxel computes its own gradient from its up-to-six neighbour differences (no
// atomics); the loss is reduced in float64 with a fixed-order two-stage reduction.
#include "mbx_common.cuh"
#include "mbx_host.hpp"
#include "mbx_reduce.cuh"
#include "qggmrf.cuh"

namespace mbx {

__global__ void qggmrf_grad_hess_kernel(const float *__restrict__ recon, int nr, int nc, int ns,
                                        const int32_t *__restrict__ pix, long long num_pixels, const QParams q,
                                        float *__restrict__ grad_out, float *__restrict__ hess_out, int *err) {
    const long long total = num_pixels * ns;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long p = i / ns;
        const int k = (int)(i - p * ns);
        const int idx = pix[p];
        float g = 0.0f, h = 0.0f;
        if (idx < 0 || idx >= nr * nc) {
            flag_error(err, MBX_ERRFLAG_PIXEL);
        } else {
            qggmrf_voxel(recon, nr, nc, ns, idx, k, q, g, h);
        }
        grad_out[i] = g;
        hess_out[i] = h;
    }
}

__device__ __forceinline__ float qrho(float delta, const QParams &q) {
    const float a = fmaxf(fabsf(delta), q.a_min);
    const float u = powf(a / q.t_sigma, q.q_minus_p);
    return powf(a, q.p) * q.inv_p_sigma_p * u / (1.0f + u);
}

__device__ __forceinline__ float qrho_prime(float delta, const QParams &q) {
    const float a0 = fabsf(delta);
    if (a0 < q.a_min) return 0.0f;
    const float u = powf(a0 / q.t_sigma, q.q_minus_p);
    const float d = powf(a0, q.p_minus_1) * q.inv_sigma_p * u * (q.q_over_p + u) / ((1.0f + u) * (1.0f + u));
    return delta < 0.0f ? -d : d;
}

__global__ void qggmrf_loss_grad_kernel(const float *__restrict__ x, int nr, int nc, int ns, const QParams q,
                                        float *__restrict__ grad_out, double *__restrict__ partials) {
    const long long total = (long long)nr * nc * ns;
    const long long sr = (long long)nc * ns;  // row stride
    double loss = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(i % ns);
        const long long pc = i / ns;
        const int col = (int)(pc % nc);
        const int row = (int)(pc / nc);
        const float x0 = __ldg(x + i);
        float g = 0.0f;
        float l = 0.0f;
        // axis 0 (rows), axis 1 (cols), axis 2 (slices): forward difference owned by this voxel
        if (row + 1 < nr) {
            const float d = __ldg(x + i + sr) - x0;
            l += q.b_axis[0] * qrho(d, q);
            g -= q.b_axis[0] * qrho_prime(d, q);
        }
        if (row > 0) g += q.b_axis[0] * qrho_prime(x0 - __ldg(x + i - sr), q);
        if (col + 1 < nc) {
            const float d = __ldg(x + i + ns) - x0;
            l += q.b_axis[1] * qrho(d, q);
            g -= q.b_axis[1] * qrho_prime(d, q);
        }
        if (col > 0) g += q.b_axis[1] * qrho_prime(x0 - __ldg(x + i - ns), q);
        if (k + 1 < ns) {
            const float d = __ldg(x + i + 1) - x0;
            l += q.b_axis[2] * qrho(d, q);
            g -= q.b_axis[2] * qrho_prime(d, q);
        }
        if (k > 0) g += q.b_axis[2] * qrho_prime(x0 - __ldg(x + i - 1), q);
        if (grad_out) grad_out[i] = g;
        loss += (double)l;
    }
    block_reduce_store(loss, partials);
}

static unsigned loss_blocks(long long total) {
    long long b = (total + 255) / 256;
    const long long cap = 4LL * num_sms();
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (unsigned)b;
}

int qggmrf_grad_hess(const float *recon, int nr, int nc, int ns, const int32_t *pix, long long num_pixels,
                     const mbx_qggmrf_params &qp, float *grad, float *hess, cudaStream_t st) {
    if (num_pixels == 0) return MBX_OK;
    const QParams q = make_qparams(qp);
    const long long total = num_pixels * ns;
    qggmrf_grad_hess_kernel<<<grid_for(total, 256), 256, 0, st>>>(recon, nr, nc, ns, pix, num_pixels, q, grad, hess,
                                                                   device_error_ptr());
    mbx::note_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
}

}  // namespace mbx

extern "C" int mbx_qggmrf_grad_hess(const float *flat_recon, int32_t num_recon_rows, int32_t num_recon_cols,
                                    int32_t num_recon_slices, const int32_t *pixel_indices, int64_t num_pixels,
                                    const mbx_qggmrf_params *qp, float *grad_out, float *hess_out, void *stream) {
    if (!flat_recon || !qp || num_recon_rows <= 0 || num_recon_cols <= 0 || num_recon_slices <= 0 || num_pixels < 0)
        return MBX_ERR_INVALID_ARG;
    if (num_pixels > 0 && (!pixel_indices || !grad_out || !hess_out)) return MBX_ERR_INVALID_ARG;
    if (!(qp->sigma_x > 0.0f) || !(qp->T > 0.0f) || !(qp->p > 0.0f)) return MBX_ERR_INVALID_ARG;
    return mbx::qggmrf_grad_hess(flat_recon, num_recon_rows, num_recon_cols, num_recon_slices, pixel_indices,
                                 num_pixels, *qp, grad_out, hess_out, static_cast<cudaStream_t>(stream));
}

extern "C" size_t mbx_qggmrf_loss_grad_workspace_bytes(int32_t num_recon_rows, int32_t num_recon_cols,
                                                       int32_t num_recon_slices) {
    if (num_recon_rows <= 0 || num_recon_cols <= 0 || num_recon_slices <= 0) return 0;
    const long long total = (long long)num_recon_rows * num_recon_cols * num_recon_slices;
    return mbx::align256(mbx::loss_blocks(total) * sizeof(double));
}

extern "C" int mbx_qggmrf_loss_grad(const float *recon, int32_t num_recon_rows, int32_t num_recon_cols,
                                    int32_t num_recon_slices, const mbx_qggmrf_params *qp, double *loss_out,
                                    float *grad_out, void *workspace, size_t workspace_bytes, void *stream) {
    if (!recon || !qp || !loss_out || num_recon_rows <= 0 || num_recon_cols <= 0 || num_recon_slices <= 0)
        return MBX_ERR_INVALID_ARG;
    if (!(qp->sigma_x > 0.0f) || !(qp->T > 0.0f) || !(qp->p > 0.0f)) return MBX_ERR_INVALID_ARG;
    const long long total = (long long)num_recon_rows * num_recon_cols * num_recon_slices;
    const unsigned blocks = mbx::loss_blocks(total);
    if (!workspace || workspace_bytes < blocks * sizeof(double)) return MBX_ERR_WORKSPACE;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const mbx::QParams q = mbx::make_qparams(*qp);
    double *partials = static_cast<double *>(workspace);
    mbx::qggmrf_loss_grad_kernel<<<blocks, 256, 0, st>>>(recon, num_recon_rows, num_recon_cols, num_recon_slices, q,
                                                          grad_out, partials);
    mbx::note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return mbx::set_cuda_error(e);
    mbx::launch_sum_partials(partials, (int)blocks, 1, loss_out, st);
    e = cudaGetLastError();
    return e == cudaSuccess ? MBX_OK : mbx::set_cuda_error(e);
}
