// Forward projector for psf_radius == 1 (and bp_psf_radius == 1 for cone beam), parallel and cone beam:
// channel-block gather, no atomics, deterministic.  Same contract and arithmetic as the general fp_kernel
// (forward_project.cu), which replaces Projectors.sparse_forward_project (projectors.py:61-129) over
// parallel_beam.py:138-178 and cone_beam.py:189-377.
//
// One CTA owns an output block: one view x CB_NB consecutive channels x all detector rows.
//  1. Scan: the 256 threads walk the pixel list 256 at a time, compute each pixel's channel footprint
//     (centre channel, three coefficients; trig-free for cone beam) and keep, by an ordered ballot/prefix
//     compaction into shared memory, the pixels with a tap inside the block (at most CB_CAP per pass).
//  2. Accumulate: threads are grouped into "lane groups" of RL lanes (RL = rows handled at once, lanes run
//     along detector rows, so each voxel-cylinder read is contiguous).  Every lane group owns a private copy
//     of the tile rows it handles and walks a strided share of the compacted pixels, adding the three
//     channel taps into its copy with plain shared-memory read-modify-writes: within a group lanes hold
//     distinct rows, and no two groups share a copy, so there are no races and no atomics.  For cone beam
//     each lane first evaluates the detector-row-centric vertical fan of the reference (cone_beam.py:347-372,
//     including the 128-row batch anchor) for its row, reading the cylinder directly (L1-resident).
//  3. Reduce: the private copies of each tile row are summed in a fixed order and written, coalesced.
#pragma once

#include <climits>
#include <cmath>

#include "mbx_common.cuh"
#include "mbx_host.hpp"

namespace mbx {

constexpr int CB_THREADS = 256;
constexpr int CB_NB = 32;          // channels per block
constexpr int CB_PITCH = CB_NB + 1;
constexpr int CB_CAP = 1024;       // compacted pixels per pass

struct CbPlan {
    int rl;        // rows per lane group (power of two <= 32)
    int lg_per_warp, groups;   // lane groups per warp, lane groups per CTA
    int row_groups;            // ceil(R / rl)
    int copies;                // private copies per row group (>= 1)
    int cblocks;               // channel blocks per view
    size_t smem;
    bool ok;
};

// Per compacted pixel record (structure of arrays in shared memory).
struct CbList {
    int *p;       // pixel position in the caller's list
    int *nc;      // centre channel
    float *a0, *a1, *a2;
    float *imd;   // cone: 1 / (mag * delta_voxel)
    float *wr;    // cone: W_r
    float *mdz;   // cone: (mag / D) * delta_voxel
    float *mz0;   // cone: (mag / D) * z_0
};

inline CbPlan plan_fp_cb(const mbx_geom &g) {
    CbPlan pl;
    pl.ok = g.psf_radius == 1 && (g.kind == MBX_GEOM_PARALLEL || g.bp_psf_radius == 1);
    const int R = g.num_det_rows;
    int rl = 1;
    while (rl < R && rl < 32) rl <<= 1;
    pl.rl = rl;
    pl.lg_per_warp = 32 / rl;
    pl.groups = 8 * pl.lg_per_warp;
    pl.row_groups = ceil_div(R, rl);
    pl.copies = pl.groups >= pl.row_groups ? pl.groups / pl.row_groups : 1;
    pl.cblocks = ceil_div(g.num_det_channels, CB_NB);
    const size_t tile_words = (size_t)pl.row_groups * pl.copies * rl * CB_PITCH;
    const size_t list_words = (size_t)CB_CAP * 9;
    const size_t table_words = (g.kind == MBX_GEOM_CONE) ? (size_t)3 * R : 0;
    pl.smem = (tile_words + list_words + table_words + 64) * 4;
    if (pl.smem > 200 * 1024) pl.ok = false;
    if (g.kind == MBX_GEOM_CONE) {
        const double half_r = 0.5 * (g.num_recon_rows - 1), half_c = 0.5 * (g.num_recon_cols - 1);
        const double rho = g.delta_voxel * std::sqrt(half_r * half_r + half_c * half_c);
        const double dinv = std::isinf(g.source_detector_dist) ? 0.0 : rho / g.source_detector_dist;
        if (1.0 / g.magnification - dinv <= 1e-6) pl.ok = false;  // recon reaches the source
    }
    return pl;
}

// Fractional centre channel n_p of one pixel (the same arithmetic as cb_footprint, so both agree on round(n_p)).
template <int KIND>
__device__ __forceinline__ float cb_channel(const mbx_geom &g, float cs, float sn, float xt, float yt, float inv_d,
                                            float &mag) {
    const float inv_dc = 1.0f / g.delta_det_channel;
    const float det_center_channel = 0.5f * (float)(g.num_det_channels - 1);
    const float x_p = cs * xt - sn * yt;
    if (KIND == MBX_GEOM_PARALLEL) {
        mag = 1.0f;
        return (x_p + g.det_channel_offset) * inv_dc + det_center_channel;
    }
    const float y_p = sn * xt + cs * yt;
    mag = 1.0f / (1.0f / g.magnification - y_p * inv_d);
    return (mag * x_p + g.det_channel_offset) * inv_dc + det_center_channel;
}

// Channel footprint of one pixel (trig-free for cone beam); also the cone vertical constants.
template <int KIND>
__device__ __forceinline__ void cb_footprint(const mbx_geom &g, float cs, float sn, float xt, float yt, int &nc,
                                             float &a0, float &a1, float &a2, float &imd, float &wr, float &mdz,
                                             float &mz0) {
    const float inv_dc = 1.0f / g.delta_det_channel;
    const float inv_d = isinf(g.source_detector_dist) ? 0.0f : 1.0f / g.source_detector_dist;
    float mag;
    const float n_p = cb_channel<KIND>(g, cs, sn, xt, yt, inv_d, mag);
    float w, scale;
    if (KIND == MBX_GEOM_PARALLEL) {
        const float cos_alpha = fmaxf(fabsf(cs), fabsf(sn));
        w = (g.delta_voxel * inv_dc) * cos_alpha;
        scale = g.delta_voxel / cos_alpha;
        imd = wr = mdz = mz0 = 0.0f;
    } else {
        const float u = mag * (cs * xt - sn * yt);
        const float t = u * inv_d;
        const float cos_tp = rsqrtf(fmaf(t, t, 1.0f));
        const float sin_tp = t * cos_tp;
        const float cd = cs * cos_tp + sn * sin_tp, sd = sn * cos_tp - cs * sin_tp;
        const float cos_alpha = fmaxf(fabsf(cd), fabsf(sd));
        w = mag * (g.delta_voxel * inv_dc) * (cos_alpha / cos_tp);
        scale = g.delta_voxel / cos_alpha;
        imd = 1.0f / (mag * g.delta_voxel);
        wr = (mag * g.delta_voxel) / g.delta_det_row;
        const float mdd = mag * inv_d;
        const float z0 = g.recon_slice_offset - g.delta_voxel * 0.5f * (float)(g.num_recon_slices - 1);
        mdz = mdd * g.delta_voxel;
        mz0 = mdd * z0;
    }
    nc = (int)rintf(n_p);
    const float half_w = (w + 1.0f) * 0.5f, l_max = fminf(1.0f, w), d = n_p - (float)nc;
    float c[3];
#pragma unroll
    for (int k = -1; k <= 1; ++k) {
        const int n = nc + k;
        c[k + 1] = (n < 0 || n >= g.num_det_channels) ? 0.0f
                                                       : scale * fminf(fmaxf(half_w - fabsf(d - (float)k), 0.0f), l_max);
    }
    a0 = c[0];
    a1 = c[1];
    a2 = c[2];
}

// Arguments of one forward projection (one scan).
struct FpArgs {
    mbx_geom g;
    const float *vox;          // (num_pixels, S)
    const int32_t *pix;        // (num_pixels,)
    long long num_pixels;
    const int32_t *views;      // (num_views_sel,) or NULL
    int num_views_sel;
    float *out;                // (num_views_sel, R, C)
    int vox_by_index;          // 0: vox is (num_pixels, S) in list order; 1: vox is a flat recon indexed by pixel
    CbPlan plan;
};

template <int KIND>
__device__ void fp_cb_tile(const FpArgs &A, int j, int cb, float *sm, int *err) {
    const mbx_geom &g = A.g;
    const CbPlan &pl = A.plan;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int num_rows = g.num_det_rows, num_channels = g.num_det_channels, num_slices = g.num_recon_slices;
    const int n0 = cb * CB_NB;
    const int rl = pl.rl;
    const int row_groups = pl.row_groups, copies = pl.copies;

    float *tile = sm;  // [row_group][copy][rl][CB_PITCH]
    const size_t tile_words = (size_t)row_groups * copies * rl * CB_PITCH;
    CbList L;
    L.p = reinterpret_cast<int *>(sm + tile_words);
    L.nc = L.p + CB_CAP;
    L.a0 = reinterpret_cast<float *>(L.nc + CB_CAP);
    L.a1 = L.a0 + CB_CAP;
    L.a2 = L.a1 + CB_CAP;
    L.imd = L.a2 + CB_CAP;
    L.wr = L.imd + CB_CAP;
    L.mdz = L.wr + CB_CAP;
    L.mz0 = L.mdz + CB_CAP;
    float *s_vm = L.mz0 + CB_CAP;             // cone: [R] detector height of each row centre
    float *s_vb = s_vm + num_rows;            // cone: [R] same at the row's 128-row batch start
    int *s_b0 = reinterpret_cast<int *>(s_vb + num_rows);  // cone: [R] batch start row
    int *s_misc = (KIND == MBX_GEOM_CONE) ? s_b0 + num_rows : reinterpret_cast<int *>(s_vm);
    // s_misc[0..7]: warp counts, [8]: list count

    const int vi = A.views ? A.views[j] : j;
    const bool view_ok = vi >= 0 && vi < g.num_views;
    if (!view_ok && tid == 0 && cb == 0) flag_error(err, MBX_ERRFLAG_VIEW);
    const float angle = view_ok ? g.angles[vi] : 0.0f;
    const float cs = cosf(angle), sn = sinf(angle);
    const float kconst = 0.5f * (float)(num_slices - 1) - g.recon_slice_offset / g.delta_voxel;
    const float inv_cols = 1.0f / (float)g.num_recon_cols;
    const float inv_d = isinf(g.source_detector_dist) ? 0.0f : 1.0f / g.source_detector_dist;

    __syncthreads();  // previous tile of this CTA (batched use) is finished with shared memory
    for (size_t i = tid; i < tile_words; i += CB_THREADS) tile[i] = 0.0f;
    if (KIND == MBX_GEOM_CONE) {
        int rows_per_batch = g.entries_per_cylinder_batch;
        if (rows_per_batch > num_rows) rows_per_batch = num_rows;
        const float det_center_row = 0.5f * (float)(num_rows - 1);
        for (int m = tid; m < num_rows; m += CB_THREADS) {
            const int b0 = (m / rows_per_batch) * rows_per_batch;
            s_vm[m] = ((float)m - det_center_row) * g.delta_det_row - g.det_row_offset;
            s_vb[m] = ((float)b0 - det_center_row) * g.delta_det_row - g.det_row_offset;
            s_b0[m] = b0;
        }
    }

    // lane group of this thread
    const int lg = warp * pl.lg_per_warp + lane / rl;   // 0 .. groups-1
    const int lr = lane % rl;                            // row within the group
    const int npix_grid = g.num_recon_rows * g.num_recon_cols;
    long long scan = 0;
    const long long num_pixels = view_ok ? A.num_pixels : 0;

    while (scan < num_pixels) {
        // ---- 1. compaction of the pixels that touch this channel block (ordered)
        int count = 0;
        __syncthreads();  // the previous pass is done with the list
        const int count0 = count;
        while (scan < num_pixels && count <= CB_CAP - CB_THREADS) {
            const long long p = scan + tid;
            bool take = false;
            if (p < num_pixels) {
                const int idx = A.pix[p];
                if (idx < 0 || idx >= npix_grid) {
                    if (cb == 0 && j == 0) flag_error(err, MBX_ERRFLAG_PIXEL);
                } else {
                    float xt, yt, mag;
                    pixel_tilde_fast(g, idx, inv_cols, xt, yt);
                    const int nc = (int)rintf(cb_channel<KIND>(g, cs, sn, xt, yt, inv_d, mag));
                    take = nc + 1 >= n0 && nc - 1 < n0 + CB_NB;
                }
            }
            const unsigned ballot = __ballot_sync(0xffffffffu, take);
            if (lane == 0) s_misc[warp] = __popc(ballot);
            __syncthreads();
            int base = count;
            for (int w = 0; w < warp; ++w) base += s_misc[w];
            int total = 0;
            for (int w = 0; w < 8; ++w) total += s_misc[w];
            if (take) L.p[base + __popc(ballot & ((1u << lane) - 1u))] = (int)p;
            count += total;
            scan += CB_THREADS;
            __syncthreads();
        }
        // footprints of the kept pixels only (dense, no divergence)
        for (int i = count0 + tid; i < count; i += CB_THREADS) {
            const int p = L.p[i];
            const int idx = A.pix[p];
            float xt, yt;
            pixel_tilde_fast(g, idx, inv_cols, xt, yt);
            int nc;
            float a0, a1, a2, imd, wr, mdz, mz0;
            cb_footprint<KIND>(g, cs, sn, xt, yt, nc, a0, a1, a2, imd, wr, mdz, mz0);
            L.p[i] = A.vox_by_index ? idx : p;  // row of vox holding this pixel's cylinder
            L.nc[i] = nc;
            L.a0[i] = a0;
            L.a1[i] = a1;
            L.a2[i] = a2;
            L.imd[i] = imd;
            L.wr[i] = wr;
            L.mdz[i] = mdz;
            L.mz0[i] = mz0;
        }
        __syncthreads();
        // ---- 2. accumulation into the private copy of each lane group
        for (int rg = lg / copies; rg < row_groups; rg += (pl.groups >= row_groups ? row_groups : pl.groups)) {
            // with copies > 1 the lane groups of a row group split the pixel list; else each group walks them all
            const int copy = (pl.groups >= row_groups) ? lg % copies : 0;
            if (pl.groups >= row_groups && lg >= row_groups * copies) break;
            const int m = rg * rl + lr;
            float *trow = tile + (((size_t)rg * copies + copy) * rl + lr) * CB_PITCH;
            if (m < num_rows) {
                float vm = 0.f, vb = 0.f;
                int b0 = 0;
                if (KIND == MBX_GEOM_CONE) {
                    vm = s_vm[m];
                    vb = s_vb[m];
                    b0 = s_b0[m];
                }
                for (int i = copy; i < count; i += copies) {
                    const int nc = L.nc[i];
                    const float *cyl = A.vox + (long long)L.p[i] * num_slices;
                    float val;
                    if (KIND == MBX_GEOM_PARALLEL) {
                        val = __ldg(cyl + m);
                    } else {
                        const float imd = L.imd[i], w_r = L.wr[i];
                        const float k_m = fmaf(vm, imd, kconst);
                        const float k_m0 = fmaf(vb, imd, kconst);
                        const int k_c = (int)rintf(k_m);
                        const float dm = fmaf(w_r, (float)k_c - k_m0, (float)(b0 - m));
                        const float half_w = (w_r + 1.0f) * 0.5f, l_max = fminf(1.0f, w_r);
                        const float mdz = L.mdz[i], mz0 = L.mz0[i];
                        val = 0.0f;
#pragma unroll
                        for (int ko = -1; ko <= 1; ++ko) {
                            const int k = k_c + ko;
                            if (k >= 0 && k < num_slices) {
                                const float a = fminf(fmaxf(half_w - fabsf(fmaf(w_r, (float)ko, dm)), 0.0f), l_max);
                                const float t = fmaf((float)k, mdz, mz0);
                                const float q = fmaf(t, t, 1.0f);
                                val = fmaf(a, __ldg(cyl + k) * (q * rsqrtf(q)), val);
                            }
                        }
                    }
                    const int c = nc - n0;  // column of the centre tap
                    if (c - 1 >= 0 && c - 1 < CB_NB) trow[c - 1] = fmaf(L.a0[i], val, trow[c - 1]);
                    if (c >= 0 && c < CB_NB) trow[c] = fmaf(L.a1[i], val, trow[c]);
                    if (c + 1 >= 0 && c + 1 < CB_NB) trow[c + 1] = fmaf(L.a2[i], val, trow[c + 1]);
                }
            }
            if (pl.groups >= row_groups) break;
        }
    }
    __syncthreads();
    // ---- 3. fixed-order sum of the private copies, coalesced write
    const int nch = min(CB_NB, num_channels - n0);
    float *out = A.out + (long long)j * num_rows * num_channels + n0;
    for (int e = tid; e < num_rows * CB_NB; e += CB_THREADS) {
        const int m = e / CB_NB, c = e - (e / CB_NB) * CB_NB;
        if (c >= nch) continue;
        const int rg = m / rl, lr2 = m - rg * rl;
        float s = 0.0f;
        for (int cp = 0; cp < copies; ++cp) s += tile[(((size_t)rg * copies + cp) * rl + lr2) * CB_PITCH + c];
        out[(long long)m * num_channels + c] = s;
    }
}

template <int KIND>
__global__ void __launch_bounds__(CB_THREADS, 2) fp_cb_kernel(const FpArgs A, int *err) {
    extern __shared__ __align__(16) float smcb[];
    fp_cb_tile<KIND>(A, blockIdx.x, blockIdx.y, smcb, err);
}

}  // namespace mbx
