// Cone-beam forward projector specialised for psf_radius == bp_psf_radius == 1 (the reference's default
// geometry).  Same contract and arithmetic as the general fp_kernel (forward_project.cu), organised to cut
// instructions per (pixel, detector row, view):
//
//  * CTA = one view x a band of MT detector rows held in shared memory (odd pitch, conflict-free), 256 threads;
//    pixels are walked in chunks of FPF_PB.
//  * Per chunk, one thread per pixel computes the trig-free channel footprint (centre channel + three
//    coefficients), 1/(mag*delta_voxel) and the slab of slices the row band can touch.
//  * The slab of every pixel's cylinder is loaded once, coalesced along the slice axis, already multiplied by
//    1/cos(phi_k) = sqrt(1 + (mag z_k / D)^2), into shared memory.
//  * Each (pixel, row) pair (lanes along rows) then evaluates the detector-row-centric vertical fan of the
//    reference (cone_beam.py:347-372: slice k_m hit by the row centre, round, three taps around it, with the
//    128-row batch anchor of the reference's lax.map) from the slab and scatters into the tile with shared
//    atomics; the lanes of a warp hit different tile rows.
#pragma once

#include <climits>
#include <cmath>

#include "mbx_common.cuh"
#include "mbx_host.hpp"

namespace mbx {

constexpr int FPF_THREADS = 256;
constexpr int FPF_PB = 64;      // pixels per chunk
constexpr int FPF_SLAB = 64;    // max slices per pixel slab

struct FpfPlan {
    int c_pad, mt, tiles, splits, bx, by;
    long long pixels_per_split;
    size_t smem, workspace;
    bool ok;
};

inline FpfPlan plan_fp_fast(const mbx_geom &g, long long num_pixels, int num_views_sel) {
    FpfPlan pl;
    pl.ok = g.kind == MBX_GEOM_CONE && g.psf_radius == 1 && g.bp_psf_radius == 1;
    const int C = g.num_det_channels, R = g.num_det_rows;
    pl.c_pad = (C % 2 == 0) ? C + 1 : C;
    int mt = 32;
    while (mt > 4 && (size_t)mt * pl.c_pad * 4 > 80 * 1024) mt >>= 1;
    if (mt > R) {
        mt = 1;
        while (mt * 2 <= R) mt <<= 1;
        if (mt < R) mt <<= 1;  // next power of two >= R, still <= 32
        if (mt > 32) mt = 32;
    }
    pl.mt = mt;
    pl.tiles = ceil_div(R, mt);
    pl.bx = mt < 32 ? mt : 32;
    pl.by = FPF_THREADS / pl.bx;
    // slab length bound: rows per tile / min slope + 4 (min slope = min_mag * delta_voxel / delta_det_row)
    const double half_r = 0.5 * (g.num_recon_rows - 1), half_c = 0.5 * (g.num_recon_cols - 1);
    const double rho = g.delta_voxel * std::sqrt(half_r * half_r + half_c * half_c);
    const double dinv = std::isinf(g.source_detector_dist) ? 0.0 : rho / g.source_detector_dist;
    const double min_mag = 1.0 / (1.0 / g.magnification + dinv);
    const double slope = min_mag * g.delta_voxel / g.delta_det_row;
    if ((double)mt / slope + 4.0 > FPF_SLAB) pl.ok = false;
    if (1.0 / g.magnification - dinv <= 1e-6) pl.ok = false;  // recon reaches the source
    pl.smem = (size_t)mt * pl.c_pad * 4 + (size_t)FPF_PB * (FPF_SLAB + 12) * 4 + (size_t)mt * 8;
    const long long base = (long long)num_views_sel * pl.tiles;
    const int sms = num_sms();
    long long splits = 1;
    if (base < 4LL * sms && num_pixels > 4LL * FPF_PB) {
        splits = (4LL * sms + base - 1) / base;
        long long maxs = num_pixels / (4LL * FPF_PB);
        if (maxs < 1) maxs = 1;
        if (splits > maxs) splits = maxs;
        if (splits > 64) splits = 64;
    }
    pl.splits = (int)splits;
    pl.pixels_per_split = (num_pixels + splits - 1) / splits;
    if (pl.pixels_per_split < 1) pl.pixels_per_split = 1;
    pl.workspace = pl.splits > 1 ? align256((size_t)pl.splits * num_views_sel * R * (size_t)C * 4) : 0;
    return pl;
}

__global__ void __launch_bounds__(FPF_THREADS, 3)
fp_cone_fast_kernel(const mbx_geom g, const float *__restrict__ vox, const int32_t *__restrict__ pix,
                    long long num_pixels, const int32_t *__restrict__ views, float *__restrict__ dst, int mt_cap,
                    int c_pad, long long pixels_per_split, long long split_stride, int *err) {
    extern __shared__ __align__(16) float sm[];
    float *tile = sm;                                         // [mt][c_pad]
    float *slab = tile + mt_cap * c_pad;                      // [FPF_PB][FPF_SLAB]
    int *h_nc = reinterpret_cast<int *>(slab + FPF_PB * FPF_SLAB);
    float *h_a0 = reinterpret_cast<float *>(h_nc + FPF_PB);
    float *h_a1 = h_a0 + FPF_PB, *h_a2 = h_a1 + FPF_PB;
    float *h_imd = h_a2 + FPF_PB;                             // 1 / (mag * delta_voxel)
    float *h_wr = h_imd + FPF_PB;                             // W_r = mag * delta_voxel / delta_det_row
    float *h_mdd = h_wr + FPF_PB;                             // (mag / D)
    int *h_klo = reinterpret_cast<int *>(h_mdd + FPF_PB);     // first slice of the slab
    int *h_kn = h_klo + FPF_PB;                               // slab length
    float *h_pad = reinterpret_cast<float *>(h_kn + FPF_PB);  // 3 spare words per pixel (alignment)
    float *s_vm = h_pad + 3 * FPF_PB;                         // [mt] detector height of each row centre
    float *s_vb = s_vm + mt_cap;                              // [mt] same for the row's 128-row batch start

    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int j = blockIdx.x;
    const int m0 = blockIdx.y * mt_cap;
    const int split = blockIdx.z;
    const int num_rows = g.num_det_rows, num_channels = g.num_det_channels, num_slices = g.num_recon_slices;
    const int mt = min(mt_cap, num_rows - m0);
    const int npix_grid = g.num_recon_rows * g.num_recon_cols;
    int rows_per_batch = g.entries_per_cylinder_batch;
    if (rows_per_batch > num_rows) rows_per_batch = num_rows;

    const int vi = views ? views[j] : j;
    const bool view_ok = vi >= 0 && vi < g.num_views;
    if (!view_ok && tid == 0) flag_error(err, MBX_ERRFLAG_VIEW);
    const float angle = view_ok ? g.angles[vi] : 0.0f;
    const float cs = cosf(angle), sn = sinf(angle);
    const float D = g.source_detector_dist;
    const float inv_d = isinf(D) ? 0.0f : 1.0f / D;
    const float inv_dc = 1.0f / g.delta_det_channel;
    const float det_center_row = 0.5f * (float)(num_rows - 1);
    const float center_slice = 0.5f * (float)(num_slices - 1);
    const float z0 = g.recon_slice_offset - g.delta_voxel * center_slice;
    // k_m(m) = (v_m / mag - offset) / delta_voxel + (S-1)/2 = v_m * h_imd + kconst
    const float kconst = center_slice - g.recon_slice_offset / g.delta_voxel;

    for (int i = tid; i < mt * c_pad; i += FPF_THREADS) tile[i] = 0.0f;
    for (int i = tid; i < mt; i += FPF_THREADS) {
        const int m = m0 + i;
        const int b0 = (m / rows_per_batch) * rows_per_batch;
        s_vm[i] = ((float)m - det_center_row) * g.delta_det_row - g.det_row_offset;
        s_vb[i] = ((float)b0 - det_center_row) * g.delta_det_row - g.det_row_offset;
    }

    const long long p_begin = (long long)split * pixels_per_split;
    long long p_end = p_begin + pixels_per_split;
    if (p_end > num_pixels) p_end = num_pixels;
    if (!view_ok) p_end = p_begin;

    for (long long pb = p_begin; pb < p_end; pb += FPF_PB) {
        __syncthreads();
        if (tid < FPF_PB) {
            const long long p = pb + tid;
            int nc = INT_MIN, klo = 0, kn = 0;
            if (p < p_end) {
                const int idx = pix[p];
                if (idx < 0 || idx >= npix_grid) {
                    flag_error(err, MBX_ERRFLAG_PIXEL);
                } else {
                    float xt, yt;
                    pixel_tilde(g, idx, xt, yt);
                    const float x_p = cs * xt - sn * yt;
                    const float y_p = sn * xt + cs * yt;
                    const float mag = 1.0f / (1.0f / g.magnification - y_p * inv_d);
                    const float u = mag * x_p;
                    const float n_p = (u + g.det_channel_offset) * inv_dc + 0.5f * (float)(num_channels - 1);
                    const float t = u * inv_d;
                    const float cos_tp = rsqrtf(fmaf(t, t, 1.0f));
                    const float sin_tp = t * cos_tp;
                    const float cd = cs * cos_tp + sn * sin_tp, sd = sn * cos_tp - cs * sin_tp;
                    const float cos_alpha = fmaxf(fabsf(cd), fabsf(sd));
                    const float w = mag * (g.delta_voxel * inv_dc) * (cos_alpha / cos_tp);
                    const float scale = g.delta_voxel / cos_alpha;
                    nc = (int)rintf(n_p);
                    const float half_w = (w + 1.0f) * 0.5f, l_max = fminf(1.0f, w), d = n_p - (float)nc;
                    float a[3];
#pragma unroll
                    for (int k = -1; k <= 1; ++k) {
                        const int n = nc + k;
                        a[k + 1] = (n < 0 || n >= num_channels)
                                       ? 0.0f
                                       : scale * fminf(fmaxf(half_w - fabsf(d - (float)k), 0.0f), l_max);
                    }
                    h_a0[tid] = a[0];
                    h_a1[tid] = a[1];
                    h_a2[tid] = a[2];
                    const float imd = 1.0f / (mag * g.delta_voxel);
                    h_imd[tid] = imd;
                    h_wr[tid] = (mag * g.delta_voxel) / g.delta_det_row;
                    h_mdd[tid] = mag * inv_d;
                    const float ka = fmaf(s_vm[0], imd, kconst), kb = fmaf(s_vm[mt - 1], imd, kconst);
                    klo = max((int)rintf(fminf(ka, kb)) - 1, 0);
                    const int khi = min((int)rintf(fmaxf(ka, kb)) + 1, num_slices - 1);
                    kn = max(khi - klo + 1, 0);
                    if (kn > FPF_SLAB) kn = FPF_SLAB;  // bounded by the plan; taps outside read as 0
                }
            }
            h_nc[tid] = nc;
            h_klo[tid] = klo;
            h_kn[tid] = kn;
        }
        __syncthreads();
        const int np = (int)min((long long)FPF_PB, p_end - pb);
        // slab of each cylinder, scaled by 1/cos(phi_k); lanes along slices (coalesced)
        for (int pl = threadIdx.y; pl < np; pl += blockDim.y) {
            const int kn = h_kn[pl];
            if (h_nc[pl] == INT_MIN) continue;
            const float *cyl = vox + (pb + pl) * (long long)num_slices + h_klo[pl];
            const float mdd = h_mdd[pl];
            const float mz0 = mdd * (z0 + g.delta_voxel * (float)h_klo[pl]);
            const float mdz = mdd * g.delta_voxel;
            for (int kk = threadIdx.x; kk < kn; kk += blockDim.x) {
                const float tt = fmaf((float)kk, mdz, mz0);
                const float q = fmaf(tt, tt, 1.0f);
                slab[pl * FPF_SLAB + kk] = __ldg(cyl + kk) * (q * rsqrtf(q));
            }
        }
        __syncthreads();
        for (int pl = threadIdx.y; pl < np; pl += blockDim.y) {
            const int nc = h_nc[pl];
            if (nc == INT_MIN) continue;
            const float a0 = h_a0[pl], a1 = h_a1[pl], a2 = h_a2[pl];
            const float imd = h_imd[pl], w_r = h_wr[pl];
            const int klo = h_klo[pl], kn = h_kn[pl];
            const float half_w = (w_r + 1.0f) * 0.5f, l_max = fminf(1.0f, w_r);
            const float *sp = slab + pl * FPF_SLAB;
            for (int ml = threadIdx.x; ml < mt; ml += blockDim.x) {
                const int m = m0 + ml;
                const float k_m = fmaf(s_vm[ml], imd, kconst);
                const float k_m0 = fmaf(s_vb[ml], imd, kconst);
                const int k_c = (int)rintf(k_m);
                const int b0 = (m / rows_per_batch) * rows_per_batch;
                const float m_p = fmaf(w_r, (float)k_c - k_m0, (float)b0);
                const float dm = m_p - (float)m;
                float col = 0.0f;
#pragma unroll
                for (int ko = -1; ko <= 1; ++ko) {
                    const int kk = k_c + ko - klo;
                    if (kk >= 0 && kk < kn) {
                        const float a = fminf(fmaxf(half_w - fabsf(fmaf(w_r, (float)ko, dm)), 0.0f), l_max);
                        col = fmaf(a, sp[kk], col);
                    }
                }
                if (col != 0.0f) {
                    float *trow = tile + ml * c_pad;
                    if (a0 != 0.0f) atomicAdd(trow + nc - 1, a0 * col);
                    if (a1 != 0.0f) atomicAdd(trow + nc, a1 * col);
                    if (a2 != 0.0f) atomicAdd(trow + nc + 1, a2 * col);
                }
            }
        }
    }
    __syncthreads();
    float *out = dst + (long long)split * split_stride + ((long long)j * num_rows + m0) * num_channels;
    for (int ml = threadIdx.y; ml < mt; ml += blockDim.y)
        for (int n = threadIdx.x; n < num_channels; n += blockDim.x)
            out[(long long)ml * num_channels + n] = tile[ml * c_pad + n];
}

}  // namespace mbx
