// VCD subset update, fully device-resident (sm_100a).
//
// Replaces the vcd_subset_updater closure of TomographyModel.create_vcd_subset_updater
// (tomography_model.py:1343-1542), get_forward_lin_quad (tomography_model.py:1546-1631) and update_recon
// (tomography_model.py:1820-1823).  The reference runs ~15 XLA ops per subset with a host synchronisation
// (float(alpha), tomography_model.py:1528); here one subset is seven launches on one stream with the step
// size kept in device memory, so a whole iteration can be captured in a CUDA graph:
//
//   1. back projection of W*e at the subset (the weights are multiplied into the gathers)
//   2. vcd_delta_kernel: qGGMRF gradient/Hessian per voxel (inline), g_f = -fm*bp, h_f = fm*H[idx],
//      delta = -(g_f+g_p)/(h_f+h_p); float64 block partials of <g_p,delta> and <h_p,delta^2>
//   3. forward projection of delta -> delta_sino (full sinogram)
//   4. vcd_linquad_kernel: float64 block partials of <W e, delta_sino> and <W delta_sino, delta_sino>
//   5. vcd_alpha_kernel (one block): fixed-order sums, alpha = clip((fl-pl)/(fq+pq+eps), eps, 1.5)
//   6. vcd_apply_kernel: recon[idx] += alpha*delta, float64 partials of |alpha*delta|
//   7. vcd_error_kernel: e -= alpha*delta_sino, and the last block folds the l1 partials into stats
#include "mbx_common.cuh"
#include "mbx_host.hpp"
#include "mbx_reduce.cuh"
#include "qggmrf.cuh"

namespace mbx {

constexpr float EPS_F32 = 1.1920928955078125e-07f;

__global__ void sum_partials_kernel(const double *__restrict__ partials, int nblocks, int nv, double *__restrict__ out) {
    // one warp per value, fixed order: lane l sums blocks l, l+32, ...; then a fixed shuffle tree
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int v = warp; v < nv; v += blockDim.x >> 5) {
        double s = 0.0;
        for (int b = lane; b < nblocks; b += 32) s += partials[b * nv + v];
        s = warp_sum(s);
        if (lane == 0) out[v] = s;
    }
}

void launch_sum_partials(const double *partials, int nblocks, int nv, double *out, cudaStream_t st) {
    sum_partials_kernel<<<1, 256, 0, st>>>(partials, nblocks, nv, out);
    mbx::note_launch();
}

__device__ __forceinline__ double fixed_order_sum(const double *__restrict__ partials, int nblocks, int nv, int v) {
    // called by one full warp; returns the sum on all lanes
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += partials[b * nv + v];
    s = warp_sum(s);
    return __shfl_sync(0xffffffffu, s, 0);
}

// prox (optional, flat like recon): proximal-map prior instead of qGGMRF (tomography_model.py:1388-1391):
// g_p = (x - v) / sigma_prox^2 (qggmrf.py:8-28), h_p = sigma_prox^2 as the reference writes it.
__global__ void vcd_delta_kernel(const float *__restrict__ recon, int nr, int nc, int ns,
                                 const int32_t *__restrict__ pix, long long num_pixels, const float *__restrict__ bp,
                                 const float *__restrict__ fm_hessian, float fm_constant, const QParams q,
                                 const float *__restrict__ prox, float sigma_prox,
                                 float *__restrict__ delta, double *__restrict__ partials, int *err) {
    const long long total = num_pixels * ns;
    double pl = 0.0, pq = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int k;
        const long long p = div_rem(i, ns, k);
        const int idx = pix[p];
        float d = 0.0f;
        if (idx < 0 || idx >= nr * nc) {
            flag_error(err, MBX_ERRFLAG_PIXEL);
        } else {
            float gp, hp;
            if (prox) {
                const long long v = (long long)idx * ns + k;
                gp = (1.0f / (sigma_prox * sigma_prox)) * (recon[v] - __ldg(prox + v));
                hp = sigma_prox * sigma_prox;
            } else {
                qggmrf_voxel(recon, nr, nc, ns, idx, k, q, gp, hp);
            }
            const float gf = -fm_constant * bp[i];
            const float hf = fm_constant * __ldg(fm_hessian + (long long)idx * ns + k);
            d = -((gf + gp) / (hf + hp));
            pl += (double)(gp * d);
            pq += (double)(hp * (d * d));
        }
        delta[i] = d;
    }
    const double v[2] = {pl, pq};
    block_reduce_store_n<2>(v, partials);
}

// Positivity (tomography_model.py:1497-1507): delta = max(-x / (alpha + eps), delta) at the subset, with the
// alpha already found; the caller then forward-projects the clipped delta again.
__global__ void vcd_clip_kernel(const float *__restrict__ recon, int ns, const int32_t *__restrict__ pix,
                                long long num_pixels, int npix_grid, const float *__restrict__ alpha,
                                float *__restrict__ delta) {
    const long long total = num_pixels * ns;
    const float pc = 1.0f / (*alpha + EPS_F32);
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int k;
        const long long p = div_rem(i, ns, k);
        const int idx = pix[p];
        if (idx < 0 || idx >= npix_grid) continue;  // flagged by vcd_delta_kernel; its delta is 0
        delta[i] = fmaxf(-pc * recon[(long long)idx * ns + k], delta[i]);
    }
}

__global__ void vcd_linquad_kernel(const float *__restrict__ dsino, const float *__restrict__ err_sino,
                                   const float *__restrict__ wts, long long total, double *__restrict__ partials) {
    double fl = 0.0, fq = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x * 4;
    // float4 main body (all sinogram buffers come from 256-byte aligned allocations)
    const long long n4 = total / 4;
    for (long long i4 = blockIdx.x * (long long)blockDim.x + threadIdx.x; i4 < n4; i4 += stride / 4) {
        const float4 ds = reinterpret_cast<const float4 *>(dsino)[i4];
        const float4 e = reinterpret_cast<const float4 *>(err_sino)[i4];
        float4 w = make_float4(1.f, 1.f, 1.f, 1.f);
        if (wts) w = reinterpret_cast<const float4 *>(wts)[i4];
        fl += (double)((w.x * e.x) * ds.x) + (double)((w.y * e.y) * ds.y) + (double)((w.z * e.z) * ds.z) +
              (double)((w.w * e.w) * ds.w);
        fq += (double)(ds.x * ds.x * w.x) + (double)(ds.y * ds.y * w.y) + (double)(ds.z * ds.z * w.z) +
              (double)(ds.w * ds.w * w.w);
    }
    for (long long i = n4 * 4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const float w = wts ? wts[i] : 1.0f;
        fl += (double)((w * err_sino[i]) * dsino[i]);
        fq += (double)(dsino[i] * dsino[i] * w);
    }
    const double v[2] = {fl, fq};
    block_reduce_store_n<2>(v, partials);
}

// stats: [0] alpha, [1] l1 of the update, [2] alpha numerator, [3] alpha denominator
__global__ void vcd_alpha_kernel(const double *__restrict__ prior_partials, int nb_prior,
                                 const double *__restrict__ fwd_partials, int nb_fwd, double fm_constant,
                                 float *__restrict__ alpha_out, double *__restrict__ stats) {
    if (threadIdx.x >= 32) return;
    const double pl = fixed_order_sum(prior_partials, nb_prior, 2, 0);
    const double pq = 0.5 * fixed_order_sum(prior_partials, nb_prior, 2, 1);
    const double fl = fm_constant * fixed_order_sum(fwd_partials, nb_fwd, 2, 0);
    const double fq = fm_constant * fixed_order_sum(fwd_partials, nb_fwd, 2, 1);
    if (threadIdx.x == 0) {
        const double num = fl - pl;
        const double den = fq + pq + (double)EPS_F32;
        float a = (float)(num / den);
        a = fminf(fmaxf(a, EPS_F32), 1.5f);  // jnp.clip(alpha, eps, 1.5)
        if (num != num || den != den) a = nanf("");
        *alpha_out = a;
        if (stats) {
            stats[0] = (double)a;
            stats[2] = num;
            stats[3] = den;
        }
    }
}

__global__ void vcd_apply_kernel(float *__restrict__ recon, int ns, const int32_t *__restrict__ pix,
                                 long long num_pixels, int npix_grid, const float *__restrict__ delta,
                                 const float *__restrict__ alpha_ptr, double *__restrict__ partials) {
    const float alpha = *alpha_ptr;
    const long long total = num_pixels * ns;
    double l1 = 0.0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        int k;
        const long long p = div_rem(i, ns, k);
        const int idx = pix[p];
        if (idx < 0 || idx >= npix_grid) continue;
        const float d = alpha * delta[i];
        atomicAdd(recon + (long long)idx * ns + k, d);  // .at[idx].add: duplicates accumulate
        l1 += (double)fabsf(d);
    }
    block_reduce_store(l1, partials);
}

__global__ void vcd_error_kernel(float *__restrict__ err_sino, const float *__restrict__ dsino, long long total,
                                 const float *__restrict__ alpha_ptr, const double *__restrict__ l1_partials,
                                 int nb_l1, double *__restrict__ stats) {
    const float alpha = *alpha_ptr;
    const long long n4 = total / 4;
    for (long long i4 = blockIdx.x * (long long)blockDim.x + threadIdx.x; i4 < n4;
         i4 += (long long)gridDim.x * blockDim.x) {
        float4 e = reinterpret_cast<float4 *>(err_sino)[i4];
        const float4 d = reinterpret_cast<const float4 *>(dsino)[i4];
        e.x -= alpha * d.x;
        e.y -= alpha * d.y;
        e.z -= alpha * d.z;
        e.w -= alpha * d.w;
        reinterpret_cast<float4 *>(err_sino)[i4] = e;
    }
    for (long long i = n4 * 4 + blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x)
        err_sino[i] -= alpha * dsino[i];
    if (blockIdx.x == 0 && threadIdx.x < 32 && stats) {
        const double l1 = fixed_order_sum(l1_partials, nb_l1, 1, 0);
        if (threadIdx.x == 0) stats[1] = l1;
    }
}

struct VcdLayout {
    size_t bp, delta, dsino, fpws, bpws, partials, alpha, total;
    size_t fp_bytes, bp_bytes;
    int max_blocks;
};

static VcdLayout vcd_layout(const mbx_geom &g, long long num_pixels) {
    VcdLayout L;
    const size_t ncyl = (size_t)num_pixels * g.num_recon_slices * 4;
    const size_t nsino = (size_t)g.num_views * g.num_det_rows * g.num_det_channels * 4;
    L.fp_bytes = fp_workspace_bytes(g, num_pixels, g.num_views);
    L.bp_bytes = bp_workspace_bytes(g, num_pixels, g.num_views);
    L.max_blocks = 4 * num_sms();
    size_t off = 0;
    L.bp = off;
    off += align256(ncyl);
    L.delta = off;
    off += align256(ncyl);
    L.dsino = off;
    off += align256(nsino);
    L.fpws = off;
    off += align256(L.fp_bytes);
    L.bpws = off;
    off += align256(L.bp_bytes);
    L.partials = off;
    off += align256((size_t)3 * L.max_blocks * 2 * sizeof(double));
    L.alpha = off;
    off += 256;
    L.total = off;
    return L;
}

static unsigned red_blocks(long long n, int max_blocks) {
    long long b = (n + 255) / 256;
    if (b > max_blocks) b = max_blocks;
    if (b < 1) b = 1;
    return (unsigned)b;
}

int vcd_subset_step(const mbx_geom &g, float *recon, float *err_sino, const float *wts, const float *fm_hessian,
                    const int32_t *pix, long long num_pixels, float fm_constant, const mbx_qggmrf_params &qp,
                    const float *prox, float sigma_prox, int positivity, double *stats, void *ws, size_t ws_bytes,
                    cudaStream_t st) {
    const VcdLayout L = vcd_layout(g, num_pixels);
    if (!ws || ws_bytes < L.total) return MBX_ERR_WORKSPACE;
    char *base = static_cast<char *>(ws);
    float *bp = reinterpret_cast<float *>(base + L.bp);
    float *delta = reinterpret_cast<float *>(base + L.delta);
    float *dsino = reinterpret_cast<float *>(base + L.dsino);
    double *partials = reinterpret_cast<double *>(base + L.partials);
    double *prior_partials = partials;
    double *fwd_partials = partials + 2 * L.max_blocks;
    double *l1_partials = partials + 4 * L.max_blocks;
    float *alpha = reinterpret_cast<float *>(base + L.alpha);
    const int ns = g.num_recon_slices;
    const long long ncyl = num_pixels * ns;
    const long long nsino = (long long)g.num_views * g.num_det_rows * g.num_det_channels;
    int *err = device_error_ptr();

    int rc = back_project(g, err_sino, wts, pix, num_pixels, nullptr, g.num_views, 1, 1.0f, bp, base + L.bpws,
                          L.bp_bytes, st);
    if (rc != MBX_OK) return rc;
    const unsigned nb1 = red_blocks(ncyl, L.max_blocks);
    vcd_delta_kernel<<<nb1, 256, 0, st>>>(recon, g.num_recon_rows, g.num_recon_cols, ns, pix, num_pixels, bp,
                                          fm_hessian, fm_constant, make_qparams(qp), prox, sigma_prox, delta,
                                          prior_partials, err);
    mbx::note_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error(e);
    rc = forward_project(g, delta, pix, num_pixels, nullptr, g.num_views, dsino, base + L.fpws, L.fp_bytes, st);
    if (rc != MBX_OK) return rc;
    const unsigned nb2 = red_blocks(nsino / 4 + 1, L.max_blocks);
    vcd_linquad_kernel<<<nb2, 256, 0, st>>>(dsino, err_sino, wts, nsino, fwd_partials);
    mbx::note_launch();
    vcd_alpha_kernel<<<1, 32, 0, st>>>(prior_partials, (int)nb1, fwd_partials, (int)nb2, (double)fm_constant, alpha,
                                       stats);
    mbx::note_launch();
    if (positivity) {
        vcd_clip_kernel<<<red_blocks(ncyl, L.max_blocks), 256, 0, st>>>(recon, ns, pix, num_pixels,
                                                                       g.num_recon_rows * g.num_recon_cols, alpha,
                                                                       delta);
        mbx::note_launch();
        e = cudaGetLastError();
        if (e != cudaSuccess) return set_cuda_error(e);
        rc = forward_project(g, delta, pix, num_pixels, nullptr, g.num_views, dsino, base + L.fpws, L.fp_bytes, st);
        if (rc != MBX_OK) return rc;
    }
    const unsigned nb3 = red_blocks(ncyl, L.max_blocks);
    vcd_apply_kernel<<<nb3, 256, 0, st>>>(recon, ns, pix, num_pixels, g.num_recon_rows * g.num_recon_cols, delta,
                                          alpha, l1_partials);
    mbx::note_launch();
    vcd_error_kernel<<<grid_for(nsino / 4 + 1, 256), 256, 0, st>>>(err_sino, dsino, nsino, alpha, l1_partials,
                                                                  (int)nb3, stats);
    mbx::note_launch();
    e = cudaGetLastError();
    return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
}

size_t vcd_workspace_bytes(const mbx_geom &g, long long num_pixels) { return vcd_layout(g, num_pixels).total; }

}  // namespace mbx

extern "C" size_t mbx_vcd_subset_step_workspace_bytes(const mbx_geom *g, int64_t num_pixels) {
    if (mbx::validate_geom(g) != MBX_OK || num_pixels < 0) return 0;
    return mbx::vcd_workspace_bytes(*g, num_pixels);
}

extern "C" int mbx_vcd_subset_step(const mbx_geom *g, float *flat_recon, float *error_sinogram, const float *weights,
                                   const float *fm_hessian, const int32_t *pixel_indices, int64_t num_pixels,
                                   float fm_constant, const mbx_qggmrf_params *qp, double *stats_out, void *workspace,
                                   size_t workspace_bytes, void *stream) {
    int rc = mbx::validate_geom(g);
    if (rc != MBX_OK) return rc;
    if (!flat_recon || !error_sinogram || !fm_hessian || !pixel_indices || !qp || num_pixels <= 0)
        return MBX_ERR_INVALID_ARG;
    if (!(qp->sigma_x > 0.0f) || !(qp->T > 0.0f) || !(qp->p > 0.0f)) return MBX_ERR_INVALID_ARG;
    if ((reinterpret_cast<uintptr_t>(error_sinogram) & 15) || (weights && (reinterpret_cast<uintptr_t>(weights) & 15)))
        return MBX_ERR_INVALID_ARG;  // float4 passes over the sinogram need 16-byte alignment
    return mbx::vcd_subset_step(*g, flat_recon, error_sinogram, weights, fm_hessian, pixel_indices, num_pixels,
                                fm_constant, *qp, nullptr, 0.0f, 0, stats_out, workspace, workspace_bytes,
                                static_cast<cudaStream_t>(stream));
}

extern "C" int mbx_vcd_subset_step_ex(const mbx_geom *g, float *flat_recon, float *error_sinogram,
                                      const float *weights, const float *fm_hessian, const int32_t *pixel_indices,
                                      int64_t num_pixels, float fm_constant, const mbx_qggmrf_params *qp,
                                      const float *prox_input, float sigma_prox, int32_t positivity,
                                      double *stats_out, void *workspace, size_t workspace_bytes, void *stream) {
    int rc = mbx::validate_geom(g);
    if (rc != MBX_OK) return rc;
    if (!flat_recon || !error_sinogram || !fm_hessian || !pixel_indices || !qp || num_pixels <= 0)
        return MBX_ERR_INVALID_ARG;
    if (prox_input) {
        if (!(sigma_prox > 0.0f)) return MBX_ERR_INVALID_ARG;
    } else if (!(qp->sigma_x > 0.0f) || !(qp->T > 0.0f) || !(qp->p > 0.0f)) {
        return MBX_ERR_INVALID_ARG;
    }
    if ((reinterpret_cast<uintptr_t>(error_sinogram) & 15) || (weights && (reinterpret_cast<uintptr_t>(weights) & 15)))
        return MBX_ERR_INVALID_ARG;  // float4 passes over the sinogram need 16-byte alignment
    return mbx::vcd_subset_step(*g, flat_recon, error_sinogram, weights, fm_hessian, pixel_indices, num_pixels,
                                fm_constant, *qp, prox_input, sigma_prox, positivity ? 1 : 0, stats_out, workspace,
                                workspace_bytes, static_cast<cudaStream_t>(stream));
}
