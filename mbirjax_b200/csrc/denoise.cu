// qGGMRF denoiser subset update and the 3x3x3 median filter (sm_100a).
//
// mbx_qggmrf_denoise_step replaces vcd_subset_denoiser (denoising.py:366-411), the subset update of
// QGGMRFDenoiser.denoise: the forward model is the identity, so the "sinogram" is the error image
// e = noisy - image, the forward Hessian is 1, and the prior's quadratic term is over-relaxed by 1.1 instead of 2.
// Per subset, fully on the device, with the step size kept in device memory:
//   1. dn_delta_kernel: qGGMRF gradient/Hessian (g_p, h_p) per voxel, g_f = -fm e, delta = -(g_f + g_p)/(1 + h_p),
//      float64 block partials of <g_p, delta>, <h_p, delta^2>, <e, delta>, <delta, delta>
//   2. dn_alpha_kernel (one warp): fixed-order sums, alpha = clip((fm <e,d> - <g_p,d>) / (fm <d,d> +
//      <h_p,d^2>/1.1 + eps), eps, 1.5)
//   3. dn_apply_kernel: image[idx] += alpha delta, e[idx] -= alpha delta, float64 partials of |alpha delta|
//   4. the l1 partials are summed into stats[1]
// mbx_median_filter3d replaces median_filter3d (denoising.py:414-490): median of the 27 voxels of each 3x3x3
// neighbourhood with edge replication.
#include "mbx_common.cuh"
#include "mbx_host.hpp"
#include "mbx_reduce.cuh"
#include "qggmrf.cuh"

namespace mbx {

constexpr float DN_EPS_F32 = 1.1920928955078125e-07f;
constexpr int DN_THREADS = 256;

__global__ void dn_delta_kernel(const float *__restrict__ image, const float *__restrict__ err, int nr, int nc, int ns,
                                const int32_t *__restrict__ pix, long long num_pixels, float fm_constant,
                                const QParams q, float *__restrict__ delta, double *__restrict__ partials,
                                int *errw) {
    const long long total = num_pixels * ns;
    double pl = 0.0, pq = 0.0, fl = 0.0, fq = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long p = i / ns;
        const int k = (int)(i - p * ns);
        const int idx = pix[p];
        float d = 0.0f;
        if (idx < 0 || idx >= nr * nc) {
            flag_error(errw, MBX_ERRFLAG_PIXEL);
        } else {
            float gp, hp;
            qggmrf_voxel(image, nr, nc, ns, idx, k, q, gp, hp);
            const float e = err[(long long)idx * ns + k];
            const float gf = -fm_constant * e;
            d = -((gf + gp) / (1.0f + hp));
            pl += (double)(gp * d);
            pq += (double)(hp * (d * d));
            fl += (double)(e * d);
            fq += (double)(d * d);
        }
        delta[i] = d;
    }
    const double v[4] = {pl, pq, fl, fq};
    block_reduce_store_n<4>(v, partials);
}

// stats: [0] alpha, [1] l1 of the update (written by the l1 sum), [2] alpha numerator, [3] alpha denominator
__global__ void dn_alpha_kernel(const double *__restrict__ partials, int nblocks, double fm_constant,
                                float *__restrict__ alpha_out, double *__restrict__ stats) {
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    double s[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        double a = 0.0;
        for (int b = lane; b < nblocks; b += 32) a += partials[b * 4 + v];
        s[v] = __shfl_sync(0xffffffffu, warp_sum(a), 0);
    }
    if (lane == 0) {
        const double num = fm_constant * s[2] - s[0];
        const double den = fm_constant * s[3] + s[1] / 1.1 + (double)DN_EPS_F32;
        float a = (float)(num / den);
        a = fminf(fmaxf(a, DN_EPS_F32), 1.5f);  // jnp.clip(alpha, eps, 1.5)
        if (num != num || den != den) a = nanf("");
        *alpha_out = a;
        if (stats) {
            stats[0] = (double)a;
            stats[2] = num;
            stats[3] = den;
        }
    }
}

__global__ void dn_apply_kernel(float *__restrict__ image, float *__restrict__ err, int ns,
                                const int32_t *__restrict__ pix, long long num_pixels, int npix_grid,
                                const float *__restrict__ delta, const float *__restrict__ alpha_ptr,
                                double *__restrict__ partials) {
    const float alpha = *alpha_ptr;
    const long long total = num_pixels * ns;
    double l1 = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const long long p = i / ns;
        const int k = (int)(i - p * ns);
        const int idx = pix[p];
        if (idx < 0 || idx >= npix_grid) continue;
        const long long v = (long long)idx * ns + k;
        const float d = alpha * delta[i];
        atomicAdd(image + v, d);  // .at[idx].add
        err[v] = err[v] - d;      // .at[idx].set(e - alpha delta)
        l1 += (double)fabsf(d);
    }
    block_reduce_store(l1, partials);
}

// 3x3x3 median with edge replication: the 14th smallest of the 27 values (a partial selection sort).
__global__ void median3_kernel(const float *__restrict__ x, int d0, int d1, int d2, float *__restrict__ out) {
    const long long total = (long long)d0 * d1 * d2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % d2);
        const int b = (int)((i / d2) % d1);
        const int a = (int)(i / ((long long)d1 * d2));
        float v[27];
        int n = 0;
#pragma unroll
        for (int da = -1; da <= 1; ++da)
#pragma unroll
            for (int db = -1; db <= 1; ++db)
#pragma unroll
                for (int dc = -1; dc <= 1; ++dc) {
                    const int aa = min(max(a + da, 0), d0 - 1), bb = min(max(b + db, 0), d1 - 1),
                              cc = min(max(c + dc, 0), d2 - 1);
                    v[n++] = __ldg(x + ((long long)aa * d1 + bb) * d2 + cc);
                }
        // move the 14 smallest to the front in order; v[13] is then the median
#pragma unroll
        for (int s = 0; s < 14; ++s) {
#pragma unroll
            for (int t = s + 1; t < 27; ++t) {
                const float lo = fminf(v[s], v[t]), hi = fmaxf(v[s], v[t]);
                v[s] = lo;
                v[t] = hi;
            }
        }
        out[i] = v[13];
    }
}

struct DnLayout {
    size_t delta, partials, l1, alpha, total;
    int max_blocks;
};

static DnLayout dn_layout(long long num_pixels, int ns) {
    DnLayout L;
    L.max_blocks = 4 * num_sms();
    size_t off = 0;
    L.delta = off;
    off += align256((size_t)num_pixels * ns * 4);
    L.partials = off;
    off += align256((size_t)L.max_blocks * 4 * sizeof(double));
    L.l1 = off;
    off += align256((size_t)L.max_blocks * sizeof(double));
    L.alpha = off;
    off += 256;
    L.total = off;
    return L;
}

static unsigned dn_blocks(long long n, int max_blocks) {
    long long b = (n + DN_THREADS - 1) / DN_THREADS;
    if (b > max_blocks) b = max_blocks;
    if (b < 1) b = 1;
    return (unsigned)b;
}

}  // namespace mbx

extern "C" size_t mbx_qggmrf_denoise_step_workspace_bytes(int64_t num_pixels, int32_t num_slices) {
    if (num_pixels < 0 || num_slices <= 0) return 0;
    return mbx::dn_layout(num_pixels, num_slices).total;
}

extern "C" int mbx_qggmrf_denoise_step(float *flat_image, float *flat_error_image, int32_t num_rows, int32_t num_cols,
                                       int32_t num_slices, const int32_t *pixel_indices, int64_t num_pixels,
                                       float fm_constant, const mbx_qggmrf_params *qp, double *stats_out,
                                       void *workspace, size_t workspace_bytes, void *stream) {
    using namespace mbx;
    if (!flat_image || !flat_error_image || !pixel_indices || !qp || num_pixels <= 0 || num_rows <= 0 ||
        num_cols <= 0 || num_slices <= 0)
        return MBX_ERR_INVALID_ARG;
    if (!(qp->sigma_x > 0.0f) || !(qp->T > 0.0f) || !(qp->p > 0.0f)) return MBX_ERR_INVALID_ARG;
    const DnLayout L = dn_layout(num_pixels, num_slices);
    if (!workspace || workspace_bytes < L.total) return MBX_ERR_WORKSPACE;
    char *base = static_cast<char *>(workspace);
    float *delta = reinterpret_cast<float *>(base + L.delta);
    double *partials = reinterpret_cast<double *>(base + L.partials);
    double *l1 = reinterpret_cast<double *>(base + L.l1);
    float *alpha = reinterpret_cast<float *>(base + L.alpha);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long ncyl = num_pixels * num_slices;
    const unsigned nb = dn_blocks(ncyl, L.max_blocks);
    dn_delta_kernel<<<nb, DN_THREADS, 0, st>>>(flat_image, flat_error_image, num_rows, num_cols, num_slices,
                                               pixel_indices, num_pixels, fm_constant, make_qparams(*qp), delta,
                                               partials, device_error_ptr());
    note_launch();
    dn_alpha_kernel<<<1, 32, 0, st>>>(partials, (int)nb, (double)fm_constant, alpha, stats_out);
    note_launch();
    dn_apply_kernel<<<nb, DN_THREADS, 0, st>>>(flat_image, flat_error_image, num_slices, pixel_indices, num_pixels,
                                               num_rows * num_cols, delta, alpha, l1);
    note_launch();
    if (stats_out) launch_sum_partials(l1, (int)nb, 1, stats_out + 1, st);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
}

extern "C" int mbx_median_filter3d(const float *x, int32_t d0, int32_t d1, int32_t d2, float *out, void *stream) {
    using namespace mbx;
    if (!x || !out || d0 <= 0 || d1 <= 0 || d2 <= 0 || x == out) return MBX_ERR_INVALID_ARG;
    const long long total = (long long)d0 * d1 * d2;
    median3_kernel<<<grid_for(total, 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(x, d0, d1, d2, out);
    note_launch();
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
}
