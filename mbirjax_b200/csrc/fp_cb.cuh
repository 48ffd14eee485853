// Forward projector for psf_radius == 1 (and bp_psf_radius == 1 for cone beam), parallel and cone beam:
// channel-block gather with a per-block counting sort, register accumulation, no atomics on data, deterministic.
// Same contract and arithmetic as the general fp_kernel (forward_project.cu), which replaces
// Projectors.sparse_forward_project (projectors.py:61-129) over parallel_beam.py:138-178 and cone_beam.py:189-377.
//
// One CTA owns an output block: one view x nb consecutive channels (nb = 32, 64 or 128) x all detector rows.
// It walks the caller's pixel list in passes of at most `cap` kept pixels:
//  1. Scan: the 256 threads compute each pixel's centre channel n_c (trig-free for cone beam) and keep, by an
//     ordered ballot compaction, the pixels with a tap inside the block; bin = n_c - n0 + 1 in [0, nb + 1].
//  2. Sort: a stable counting sort by bin (shared-memory histogram, warp-aggregated ranks from
//     __match_any_sync), during which the kept pixels' footprints are computed and stored as sorted records
//     {cylinder offset, three channel coefficients} plus the bin.
//  3. Accumulate: the bins are split into 8 contiguous ranges of about equal record counts, one per warp (at
//     least two bins each).  A warp's lanes form ppw sub-groups of 32/ppw lanes; sub-group k walks records
//     k, k + ppw, ... of the warp's range (so the sub-groups stay in step), and each lane carries rpl detector
//     rows (contiguous voxel-cylinder reads, rows rl apart).  The walk is flat and software-pipelined (8 loads in flight per
//     lane); because the records are sorted by centre channel, a lane keeps three running channel sums per
//     row in registers and, when the bin changes, channel bin-2 is done and is added once to the sub-group's
//     private tile copy.  Channels at the ends of a warp's range also receive taps from the neighbouring
//     warp; those partial sums are added in two phases (even warps, barrier, odd warps), so no tile element
//     has two writers at once.
//  4. Write: the copies of each tile element are summed in a fixed order and written, coalesced.
// For cone beam each lane evaluates the detector-row-centric vertical fan of the reference
// (cone_beam.py:347-372, including the 128-row batch anchor) for its rows, reading the cylinder directly.
// Translation geometry (translation_model.py:190-378) is the cone's arithmetic with the view's translation in
// place of the rotation, rows spaced by delta_recon_row, no delta_voxel factor in the channel coefficient, and the
// slice heights shifted by -tz (a per-view constant of the tile).
#pragma once

#include <algorithm>
#include <climits>
#include <cmath>
#include <type_traits>

#include "mbx_common.cuh"
#include "mbx_host.hpp"

namespace mbx {

#ifndef MBX_FPCB_SMEM_TIER0
#define MBX_FPCB_SMEM_TIER0 (112 * 1024)  // shared memory a plan first tries to fit (2 CTAs per SM)
#endif

constexpr int CB_THREADS = 256;
constexpr int CB_WARPS = CB_THREADS / 32;
constexpr int CB_LOADS = 8;  // loads in flight per lane in the accumulation walk
constexpr int CB_PAD = 32;   // padding records after a pass's last record: the parallel walk reads U * PPW <= 32 ahead
constexpr int CB_MAX_PASSES = 64;  // passes of one tile a planned list can hold (more: the tile is not planned)

// Shared-memory layout of a channel-block tile for one pass size (offsets in 4-byte words).
struct CbLayout {
    int cap;   // records per pass
    int fill;  // the scan stops adding pixels once a pass holds more than this many
    int o_rec, o_rec2, o_sbin, o_ubin, o_bstart, o_run, o_wcnt, o_wstart, o_cone, o_hl, o_misc, o_win;
    size_t smem;
};

struct CbPlan {
    int nb;          // channels per block
    int ppw;         // sub-groups per warp (1, 2 or 4)
    int rl;          // lanes per sub-group = 32 / ppw
    int rpl;         // detector rows per lane per row pass (1..4)
    int row_passes;  // ceil(R / (rl * rpl))
    int rpad;        // row_passes * rl * rpl
    int pitch;       // tile row pitch (nb + 1)
    int nbins;       // nb + 2
    int cblocks;     // channel blocks per view
    int minb;        // resident CTAs per SM the kernel variant is compiled for (2 or 3)
    CbLayout walk;   // scan, sort and walk passes of walk.cap records (also the build of stored passes)
    CbLayout replay; // replay of stored passes (of walk.cap records): the tile, records, bins and bin starts only,
                     // which leaves the rest of the SM's shared memory to the L1 cache that serves the row loads
    CbLayout small;  // a walk that fits replay.smem: the tiles a build could not store, walked by the replay kernel
    bool ok;
};

// Cone / translation walk: records a lane prefetches, and the slice window of one record and sub-group (the
// secant-weighted voxels of the slices its rows of one row pass touch, for slopes of at least 2/3 row per slice;
// a record with a wider span is read tap by tap instead).
__host__ __device__ constexpr int cb_cone_records(int rpl) { return (CB_LOADS / rpl) > 0 ? (CB_LOADS / rpl) : 1; }
__host__ __device__ constexpr int cb_cone_window(int ppw, int rpl) { return (3 * rpl * (32 / ppw)) / 2 + 4; }

// Walk layout for passes of cap records: tile copies, sorted records (+ the cone's second words), bins, scan
// order, bin starts, histogram, per-warp counts and starts, cone row tables, chunk hit list, warp counts, cone
// slice windows.
inline CbLayout cb_layout(const CbPlan &pl, int kind, int R, int cap) {
    CbLayout lo = {};
    lo.cap = cap;
    lo.fill = cap - CB_THREADS;
    size_t o = (size_t)pl.ppw * pl.rpad * pl.pitch;
    o = (o + 3) & ~(size_t)3;
    lo.o_rec = (int)o;
    o += 4 * (size_t)(cap + CB_PAD);
    lo.o_rec2 = (int)o;
    if (kind != MBX_GEOM_PARALLEL) o += 4 * (size_t)cap;
    lo.o_sbin = (int)o;
    o += cap + CB_PAD;
    lo.o_ubin = (int)o;
    o += cap;
    lo.o_bstart = (int)o;
    o += pl.nbins + 1;
    lo.o_run = (int)o;
    o += pl.nbins;
    lo.o_wcnt = (int)o;
    o += (size_t)CB_WARPS * pl.nbins;
    lo.o_wstart = (int)o;
    o += (size_t)CB_WARPS * pl.nbins;
    lo.o_cone = (int)o;
    if (kind != MBX_GEOM_PARALLEL) o += 3 * (size_t)R;
    lo.o_hl = (int)o;
    o += CB_THREADS;
    lo.o_misc = (int)o;
    o += 3 * CB_WARPS;
    lo.o_win = (int)o;
    if (kind != MBX_GEOM_PARALLEL)
        o += (size_t)CB_WARPS * cb_cone_records(pl.rpl) * pl.ppw * cb_cone_window(pl.ppw, pl.rpl);
    lo.smem = o * 4;
    return lo;
}

// Replay layout for stored passes of cap records: what the walk of a pass reads (tile copies, records, bins, bin
// starts, cone row tables and slice windows), none of the scan and sort buffers.
inline CbLayout cb_layout_replay(const CbPlan &pl, int kind, int R, int cap) {
    CbLayout lo = {};
    lo.cap = cap;
    lo.fill = cap - CB_THREADS;
    size_t o = (size_t)pl.ppw * pl.rpad * pl.pitch;
    o = (o + 3) & ~(size_t)3;
    lo.o_rec = (int)o;
    o += 4 * (size_t)(cap + CB_PAD);
    lo.o_rec2 = (int)o;
    if (kind != MBX_GEOM_PARALLEL) o += 4 * (size_t)cap;
    lo.o_sbin = (int)o;
    o += cap + CB_PAD;
    lo.o_bstart = (int)o;
    o += pl.nbins + 1;
    lo.o_cone = (int)o;
    if (kind != MBX_GEOM_PARALLEL) o += 3 * (size_t)R;
    lo.o_win = (int)o;
    if (kind != MBX_GEOM_PARALLEL)
        o += (size_t)CB_WARPS * cb_cone_records(pl.rpl) * pl.ppw * cb_cone_window(pl.ppw, pl.rpl);
    lo.o_ubin = lo.o_run = lo.o_wcnt = lo.o_wstart = lo.o_hl = lo.o_misc = 0;  // scan and sort buffers: unused
    lo.smem = o * 4;
    return lo;
}

// The replay layout of a plan, and the walk that fits it (the largest pass size, down to 256 records; the replay
// layout grows to the 256-record walk when even that does not fit).
inline void cb_plan_replay(CbPlan &pl, int kind, int R) {
    pl.replay = cb_layout_replay(pl, kind, R, pl.walk.cap);
    for (int cap = pl.walk.cap / 2; cap >= CB_THREADS; cap >>= 1) {
        pl.small = cb_layout(pl, kind, R, cap);
        if (pl.small.smem <= pl.replay.smem) return;
    }
    pl.small = cb_layout(pl, kind, R, CB_THREADS);
    pl.replay.smem = std::max(pl.replay.smem, pl.small.smem);
}

// num_views_sel: views per call (0 = all); min_blocks: CTAs wanted per call (a narrower channel block is
// chosen to reach it); 0 = widest block.  minb: 2 (first shared-memory tier 112 KB) or 3 (74 KB, for the kernel
// variant compiled for three resident CTAs per SM); nb_max: widest channel block allowed.
// avoid_ppw: when nonzero, the best lane layout with a different number of sub-groups (an autotuner candidate).
// max_cap: most records per pass.
inline CbPlan plan_fp_cb(const mbx_geom &g, int num_views_sel = 0, long long min_blocks = 0, int minb = 2,
                         int nb_max = 128, int avoid_ppw = 0, int max_cap = 2048) {
    CbPlan pl = {};
    pl.minb = minb;
    // translation geometry: radius 1 in both fans, and a magnification bound from the host (which also says that
    // no pixel reaches the source plane, so the channel's denominator has one sign over the recon)
    pl.ok = g.psf_radius == 1 && (g.kind == MBX_GEOM_PARALLEL || (g.kind == MBX_GEOM_CONE && g.bp_psf_radius == 1) ||
                                  (g.kind == MBX_GEOM_TRANSLATION && g.max_magnification > 0.0f));
    const int R = g.num_det_rows, C = g.num_det_channels;
    // lane layout: padded rows weighted by the cost of ppw diverging sub-groups, plus a small cost per pass
    static const int combos[12][2] = {{1, 1}, {1, 2}, {1, 3}, {1, 4}, {2, 1}, {2, 2},
                                      {2, 3}, {2, 4}, {4, 1}, {4, 2}, {4, 3}, {4, 4}};
    double best = 1e300;
    for (const auto &cb : combos) {
        const int ppw = cb[0], rpl = cb[1], rows = (32 / ppw) * rpl;
        if (ppw == avoid_ppw) continue;
        const int passes = ceil_div(R, rows);
        const double f = ppw == 1 ? 1.0 : (ppw == 2 ? 1.15 : 1.35);
        const double cost = (double)passes * rows * f + 2.0 * passes;
        if (cost < best - 1e-9) {
            best = cost;
            pl.ppw = ppw;
            pl.rpl = rpl;
        }
    }
    pl.rl = 32 / pl.ppw;
    pl.row_passes = ceil_div(R, pl.rl * pl.rpl);
    pl.rpad = pl.row_passes * pl.rl * pl.rpl;
    // widest channel block, then largest pass, that fit the shared-memory tier (2, then 1 CTA per SM)
    const size_t tiers[2] = {minb >= 3 ? (size_t)74 * 1024 : (size_t)MBX_FPCB_SMEM_TIER0, (size_t)200 * 1024};
    bool found = false;
    for (int t = 0; t < 2 && !found; ++t) {
        for (int nb = nb_max; nb >= 32 && !found; nb >>= 1) {
            const long long nv = num_views_sel > 0 ? num_views_sel : g.num_views;
            if (nb > 32 && min_blocks > 0 && (long long)ceil_div(C, nb) * nv < min_blocks) continue;
            for (int cap = max_cap; cap >= 512 && !found; cap >>= 1) {
                CbPlan q = pl;
                q.nb = nb;
                q.pitch = nb + 1;
                q.nbins = nb + 2;
                q.cblocks = ceil_div(C, nb);
                q.walk = cb_layout(q, g.kind, R, cap);
                if (q.walk.smem <= tiers[t]) {
                    pl = q;
                    found = true;
                }
            }
        }
    }
    if (!found) pl.ok = false;
    if (found) cb_plan_replay(pl, g.kind, R);
    if ((long long)g.num_recon_rows * g.num_recon_cols > (1LL << 24)) pl.ok = false;  // bin and index share a word
    if (g.kind == MBX_GEOM_CONE) {
        const double half_r = 0.5 * (g.num_recon_rows - 1), half_c = 0.5 * (g.num_recon_cols - 1);
        const double rho = g.delta_voxel * std::sqrt(half_r * half_r + half_c * half_c);
        const double dinv = std::isinf(g.source_detector_dist) ? 0.0 : rho / g.source_detector_dist;
        if (1.0 / g.magnification - dinv <= 1e-6) pl.ok = false;  // recon reaches the source
    }
    return pl;
}

// The plans an autotuner times for one call shape: the default, the variant compiled for three resident CTAs
// per SM (smaller passes), narrower channel blocks (more CTAs, shorter bins), and the best lane layout with a
// different number of sub-groups per warp.  Returns how many are usable.
constexpr int CB_MAX_CANDIDATES = 4;
inline int fp_cb_candidates(const mbx_geom &g, int num_views_sel, long long min_blocks,
                            CbPlan out[CB_MAX_CANDIDATES]) {
    int n = 0;
    const CbPlan c0 = plan_fp_cb(g, num_views_sel, min_blocks, 2, 128);
    if (!c0.ok) return 0;
    out[n++] = c0;
    const CbPlan c1 = plan_fp_cb(g, num_views_sel, min_blocks, 3, 128);
    if (c1.ok) out[n++] = c1;
    if (c0.nb > 32) {
        const CbPlan c2 = plan_fp_cb(g, num_views_sel, min_blocks, 2, c0.nb / 2);
        if (c2.ok) out[n++] = c2;
    }
    const CbPlan c3 = plan_fp_cb(g, num_views_sel, min_blocks, 2, 128, c0.ppw);
    if (c3.ok) out[n++] = c3;
    return n;
}

// Fractional centre channel n_p of one pixel.
template <int KIND>
__device__ __forceinline__ float cb_channel(const mbx_geom &g, float cs, float sn, float xt, float yt, float inv_d,
                                            float &mag) {
    const float inv_dc = 1.0f / g.delta_det_channel;
    const float det_center_channel = 0.5f * (float)(g.num_det_channels - 1);
    if (KIND == MBX_GEOM_TRANSLATION) {  // (cs, sn) carry the view's (tx, ty): no rotation
        const float xp = xt - cs, yp = yt - sn;
        mag = 1.0f / (1.0f / g.magnification - yp * inv_d);
        return (mag * xp + g.det_channel_offset) * inv_dc + det_center_channel;
    }
    const float x_p = cs * xt - sn * yt;
    if (KIND == MBX_GEOM_PARALLEL) {
        mag = 1.0f;
        return (x_p + g.det_channel_offset) * inv_dc + det_center_channel;
    }
    const float y_p = sn * xt + cs * yt;
    mag = 1.0f / (1.0f / g.magnification - y_p * inv_d);
    return (mag * x_p + g.det_channel_offset) * inv_dc + det_center_channel;
}

// Channel footprint of one pixel whose centre channel nc was fixed by the scan (trig-free for cone beam);
// also the cone vertical constants.
template <int KIND>
__device__ __forceinline__ void cb_footprint(const mbx_geom &g, float cs, float sn, float xt, float yt, int nc,
                                             float &a0, float &a1, float &a2, float &imd, float &wr, float &mdz,
                                             float &mz0, float tz = 0.0f) {
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
    } else if (KIND == MBX_GEOM_TRANSLATION) {
        // coefficient L / cos(theta_p) with no delta_voxel factor (translation_model.py:244-284); the vertical fan
        // is the cone's with slice heights delta_voxel k + z0, z0 = -tz - delta_voxel (S-1)/2
        const float u = mag * (xt - cs);
        const float t = u * inv_d;
        const float cos_tp = rsqrtf(fmaf(t, t, 1.0f));
        w = mag * (g.delta_voxel * inv_dc);
        scale = 1.0f / cos_tp;
        imd = 1.0f / (mag * g.delta_voxel);
        wr = (mag * g.delta_voxel) / g.delta_det_row;
        const float mdd = mag * inv_d;
        const float z0 = -tz - g.delta_voxel * 0.5f * (float)(g.num_recon_slices - 1);
        mdz = mdd * g.delta_voxel;
        mz0 = mdd * z0;
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
    const int4 *chunk_box;     // optional: per 256 list entries {row min, row max, col min, col max}, or
                               // row min -1 when the chunk holds an index off the grid (never skipped)
    CbPlan plan;
};

constexpr int CB_CHUNK = 256;  // list entries per chunk of chunk_box (= the scan step)
static_assert(CB_CHUNK == CB_THREADS, "the scan walks the list one chunk per step");

inline size_t fp_chunk_box_bytes(long long num_pixels) {
    return align256((size_t)((num_pixels + CB_CHUNK - 1) / CB_CHUNK) * sizeof(int4));
}

// Bounding box of the grid pixels of list entries chunk * CB_CHUNK .. + CB_CHUNK - 1, by a block of CB_CHUNK
// threads, into box[chunk].
__device__ __forceinline__ void fp_chunk_bounds_block(const int32_t *__restrict__ pix, long long num_pixels,
                                                      int num_rows, int num_cols, int4 *__restrict__ box,
                                                      long long chunk) {
    __shared__ int red[4][CB_CHUNK / 32];
    const long long p = chunk * CB_CHUNK + threadIdx.x;
    int rmin = INT_MAX, rmax = INT_MIN, cmin = INT_MAX, cmax = INT_MIN, bad = 0;
    if (p < num_pixels) {
        const int idx = pix[p];
        if (idx < 0 || idx >= num_rows * num_cols) {
            bad = 1;
        } else {
            const int r = idx / num_cols, c = idx - (idx / num_cols) * num_cols;
            rmin = rmax = r;
            cmin = cmax = c;
        }
    }
    rmin = min(rmin, bad ? -1 : rmin);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        rmin = min(rmin, __shfl_xor_sync(0xffffffffu, rmin, off));
        rmax = max(rmax, __shfl_xor_sync(0xffffffffu, rmax, off));
        cmin = min(cmin, __shfl_xor_sync(0xffffffffu, cmin, off));
        cmax = max(cmax, __shfl_xor_sync(0xffffffffu, cmax, off));
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        red[0][warp] = rmin;
        red[1][warp] = rmax;
        red[2][warp] = cmin;
        red[3][warp] = cmax;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < CB_CHUNK / 32; ++w) {
            rmin = min(rmin, red[0][w]);
            rmax = max(rmax, red[1][w]);
            cmin = min(cmin, red[2][w]);
            cmax = max(cmax, red[3][w]);
        }
        if (rmin < 0) rmin = -1;  // an off-grid index: the projector must see every entry to flag it
        box[chunk] = make_int4(rmin, rmax, cmin, cmax);
    }
    __syncthreads();  // red may be reused by the block's next chunk
}

// Bounding box of the grid pixels of each CB_CHUNK list entries (one CTA of CB_CHUNK threads per chunk).
static __global__ void __launch_bounds__(CB_CHUNK) fp_chunk_bounds_kernel(const int32_t *__restrict__ pix,
                                                                    long long num_pixels, int num_rows, int num_cols,
                                                                    int4 *__restrict__ box) {
    fp_chunk_bounds_block(pix, num_pixels, num_rows, num_cols, box, blockIdx.x);
}

// Pixel position relative to the recon centre (ALU); translation geometry spaces rows by delta_recon_row.
template <int KIND>
__device__ __forceinline__ void cb_pixel(const mbx_geom &g, int idx, float inv_cols, float &xt, float &yt) {
    pixel_tilde_fast(g, idx, inv_cols, xt, yt, KIND == MBX_GEOM_TRANSLATION ? g.delta_recon_row : 0.0f);
}

// True when no pixel of the box can have a centre channel in [n0 - 1, n0 + nb] (one rounding step of slack
// on each side).  The channel is a linear (parallel) or linear-fractional (cone, denominator of one sign) function
// of the pixel position, so its extremes over the box are at the corners.
template <int KIND>
__device__ __forceinline__ bool cb_box_misses(const mbx_geom &g, int4 bx, float cs, float sn, float inv_d, int n0,
                                              int nb) {
    if (bx.x < 0) return false;
    float lo = 3.0e38f, hi = -3.0e38f;
#pragma unroll
    for (int corner = 0; corner < 4; ++corner) {
        const int r = (corner & 1) ? bx.y : bx.x;
        const int c = (corner & 2) ? bx.w : bx.z;
        const float dy = KIND == MBX_GEOM_TRANSLATION ? g.delta_recon_row : g.delta_voxel;
        const float yt = dy * ((float)r - 0.5f * (float)(g.num_recon_rows - 1));
        const float xt = g.delta_voxel * ((float)c - 0.5f * (float)(g.num_recon_cols - 1));
        float mag;
        const float np = cb_channel<KIND>(g, cs, sn, xt, yt, inv_d, mag);
        lo = fminf(lo, np);
        hi = fmaxf(hi, np);
    }
    const float nlo = rintf(lo) - 1.0f, nhi = rintf(hi) + 1.0f;  // centre channels of the box lie in [nlo, nhi]
    return nhi < (float)(n0 - 1) || nlo > (float)(n0 + nb);
}

// Detector-row constants of the cone vertical fan (one per lane and row).
struct CbRow {
    float vm, vb;
    int b0;
};

// Value of one record for detector row m: the voxel itself (parallel: cyl already points at slice m) or the
// cone vertical fan (cyl points at the start of the cylinder).
template <int KIND>
__device__ __forceinline__ float cb_value(const float *cyl, int m, int num_slices, const float4 &cv,
                                          const CbRow &rw, float kconst) {
    if (KIND == MBX_GEOM_PARALLEL) return __ldg(cyl);
    const float w_r = cv.y;
    const float k_m = fmaf(rw.vm, cv.x, kconst);
    const float k_m0 = fmaf(rw.vb, cv.x, kconst);
    const int k_c = (int)rintf(k_m);
    const float dm = fmaf(w_r, (float)k_c - k_m0, (float)(rw.b0 - m));
    const float half_w = (w_r + 1.0f) * 0.5f, l_max = fminf(1.0f, w_r);
    float val = 0.0f;
#pragma unroll
    for (int ko = -1; ko <= 1; ++ko) {
        const int k = k_c + ko;
        if (k >= 0 && k < num_slices) {
            const float a = fminf(fmaxf(half_w - fabsf(fmaf(w_r, (float)ko, dm)), 0.0f), l_max);
            const float t = fmaf((float)k, cv.z, cv.w);
            const float q = fmaf(t, t, 1.0f);
            val = fmaf(a, __ldg(cyl + k) * (q * rsqrtf(q)), val);
        }
    }
    return val;
}

// The same value for a cone / translation record from its slice window: wp points at slice k_c of the window,
// which holds voxel k times its secant (the product cb_value forms), so the taps, their order and their rounding
// are cb_value's.
__device__ __forceinline__ float cb_value_win(const float *wp, int k_c, int m, int num_slices, const float4 &cv,
                                              const CbRow &rw, float kconst) {
    const float w_r = cv.y;
    const float k_m0 = fmaf(rw.vb, cv.x, kconst);
    const float dm = fmaf(w_r, (float)k_c - k_m0, (float)(rw.b0 - m));
    const float half_w = (w_r + 1.0f) * 0.5f, l_max = fminf(1.0f, w_r);
    float val = 0.0f;
#pragma unroll
    for (int ko = -1; ko <= 1; ++ko) {
        const int k = k_c + ko;
        if (k >= 0 && k < num_slices) {
            const float a = fminf(fmaxf(half_w - fabsf(fmaf(w_r, (float)ko, dm)), 0.0f), l_max);
            val = fmaf(a, wp[ko], val);
        }
    }
    return val;
}

// What one warp needs to accumulate one pass.
struct CbPass {
    const float4 *rec, *rec2;  // sorted records (rec2: cone only)
    const int *sbin;           // bin of each sorted record
    const int *bstart;         // bin starts
    float *tile;
    const float *s_vm, *s_vb;  // cone row tables
    const int *s_b0;
    float *win;                // cone: slice windows [warps][records][sub-groups][window]
    int b_lo, b_hi;            // this warp's bins
};

// Accumulation of one pass by one warp: PPW sub-groups, RPL rows per lane; then the edge writes.
// Cone and translation records: per loop iteration the warp stages, for each of its U records per sub-group,
// the slices the sub-group's rows of the row pass touch (a window of voxel x secant, one coalesced load per
// slice) in shared memory, and each row reads its three taps from there; a record whose slice span exceeds the
// window (slopes under 2/3 row per slice) makes the warp read tap by tap for that iteration (cb_value).  Both
// ways give a record's row value with the same operations in the same order.  Against three scattered loads and
// three secants per row, the window made the cone subset projection 1.57x faster (256 views x 128 x 256).
template <int KIND, int PPW, int RPL>
__device__ __forceinline__ void cb_accumulate(const FpArgs &A, const CbPass &P, int warp, int lane, float kconst) {
    const mbx_geom &g = A.g;
    const CbPlan &pl = A.plan;
    constexpr int RL = 32 / PPW;
    constexpr int U = cb_cone_records(RPL);          // records prefetched per lane
    constexpr int WIN = cb_cone_window(PPW, RPL);    // window floats per record and sub-group
    const int sub = lane / RL, lr = lane % RL;
    const int num_rows = g.num_det_rows, num_slices = g.num_recon_slices, nb = pl.nb;
    // this sub-group's records: every PPW-th of the warp's range, so the sub-groups walk the same bins in step
    const int w_lo = P.bstart[P.b_lo], w_hi = P.bstart[P.b_hi];
    const int r_a = w_lo + sub, r_b = w_hi;
    // edge channels of the warp's range: E0, E1 (shared with the warp below), E2, E3 (with the warp above)
    const int E0 = P.b_lo - 2, E1 = P.b_lo - 1, E2 = P.b_hi - 2, E3 = P.b_hi - 1;
    for (int rp = 0; rp < pl.row_passes; ++rp) {
        int m[RPL], mcl[RPL];
        const float *vb[RPL];
        float *trow[RPL];
        CbRow rw[RPL];
#pragma unroll
        for (int j = 0; j < RPL; ++j) {
            m[j] = (rp * RPL + j) * RL + lr;
            const int mc = min(m[j], num_rows - 1);  // rows past R read a valid row; never written out
            mcl[j] = mc;
            vb[j] = A.vox + (KIND == MBX_GEOM_PARALLEL ? mc : 0);
            trow[j] = P.tile + ((size_t)sub * pl.rpad + m[j]) * pl.pitch;
            rw[j].vm = rw[j].vb = 0.f;
            rw[j].b0 = 0;
            if (KIND != MBX_GEOM_PARALLEL) {
                rw[j].vm = P.s_vm[mc];
                rw[j].vb = P.s_vb[mc];
                rw[j].b0 = P.s_b0[mc];
            }
        }
        // before bin bc: x = sum for channel bc-2, y = sum for channel bc-1; bin bc adds s0/s1/s2 to them and bc
        float x[RPL], y[RPL], s0[RPL], s1[RPL], s2[RPL], e0[RPL], e1[RPL], e2[RPL], e3[RPL];
#pragma unroll
        for (int j = 0; j < RPL; ++j) x[j] = y[j] = s0[j] = s1[j] = s2[j] = e0[j] = e1[j] = e2[j] = e3[j] = 0.0f;
        int bc = (r_a < r_b) ? P.sbin[r_a] : 0;
        // bin bc is complete: channel bc-2 receives its sum
        auto finish = [&]() {
            const int c = bc - 2;
            const bool interior = c >= P.b_lo && c <= P.b_hi - 3;
#pragma unroll
            for (int j = 0; j < RPL; ++j) {
                const float v = x[j] + s0[j];
                x[j] = y[j] + s1[j];
                y[j] = s2[j];
                s0[j] = s1[j] = s2[j] = 0.0f;
                if (interior) {
                    trow[j][c] += v;
                } else {
                    e0[j] += (c == E0) ? v : 0.0f;
                    e1[j] += (c == E1) ? v : 0.0f;
                    e2[j] += (c == E2) ? v : 0.0f;
                    e3[j] += (c == E3) ? v : 0.0f;
                }
            }
            ++bc;
        };
        float *wbase = P.win + (size_t)warp * U * PPW * WIN;
        // detector heights of the sub-group's first and last rows of this row pass: their centre slices bound
        // those of all its rows (k_c is monotone in the row)
        const float vm_first = __shfl_sync(0xffffffffu, rw[0].vm, sub * RL);
        const float vm_last = __shfl_sync(0xffffffffu, rw[RPL - 1].vm, sub * RL + RL - 1);
        // first slice of a record's window and the window's length
        auto window_of = [&](const float4 &cv, int &lo, int &len) {
            const int kf = (int)rintf(fmaf(vm_first, cv.x, kconst));
            const int kl = (int)rintf(fmaf(vm_last, cv.x, kconst));
            lo = min(kf, kl) - 1;
            len = max(kf, kl) - lo + 2;
        };
        // the loop runs over the warp's range (the same trip count in every sub-group, for the warp-wide window
        // exchange); a sub-group's records past its own range are read but contribute nothing
        for (int i = r_a; i - sub < w_hi; i += U * PPW) {
            float4 rq[U], cq[U];
            int bq[U];
            float vq[U][RPL];
            int fits = 1;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                // past the end: reread the last record of the warp's range, contribute nothing
                const int ii = min(i + u * PPW, w_hi - 1);
                rq[u] = P.rec[ii];
                bq[u] = P.sbin[ii];
                cq[u] = P.rec2[ii];
                int lo, len;
                window_of(cq[u], lo, len);
                if (len > WIN) fits = 0;
            }
            if (__all_sync(0xffffffffu, fits)) {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    int lo, len;
                    window_of(cq[u], lo, len);
                    float *w = wbase + (u * PPW + sub) * WIN;
                    const float *cyl = A.vox + __float_as_int(rq[u].x);
                    for (int t = lr; t < len; t += RL) {
                        const int k = lo + t;
                        float y = 0.0f;
                        if (k >= 0 && k < num_slices) {
                            const float tt = fmaf((float)k, cq[u].z, cq[u].w);
                            const float q = fmaf(tt, tt, 1.0f);
                            y = __ldg(cyl + k) * (q * rsqrtf(q));
                        }
                        w[t] = y;
                    }
                }
                __syncwarp();
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    int lo, len;
                    window_of(cq[u], lo, len);
                    const float *w = wbase + (u * PPW + sub) * WIN;
#pragma unroll
                    for (int j = 0; j < RPL; ++j) {
                        const int k_c = (int)rintf(fmaf(rw[j].vm, cq[u].x, kconst));
                        vq[u][j] = cb_value_win(w + (k_c - lo), k_c, mcl[j], num_slices, cq[u], rw[j], kconst);
                    }
                }
                __syncwarp();  // the next iteration's windows overwrite these
            } else {
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int off = __float_as_int(rq[u].x);  // 32-bit element offset of the cylinder
#pragma unroll
                    for (int j = 0; j < RPL; ++j)
                        vq[u][j] = cb_value<KIND>(vb[j] + off, mcl[j], num_slices, cq[u], rw[j], kconst);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                if (i + u * PPW < r_b) {
                    while (bc < bq[u]) finish();
#pragma unroll
                    for (int j = 0; j < RPL; ++j) {
                        s0[j] = fmaf(rq[u].y, vq[u][j], s0[j]);
                        s1[j] = fmaf(rq[u].z, vq[u][j], s1[j]);
                        s2[j] = fmaf(rq[u].w, vq[u][j], s2[j]);
                    }
                }
            }
        }
        if (r_a < r_b) {  // the last bin and the two channels above it
            finish();
            finish();
            finish();
        }
        // edge channels: even warps first, then odd warps
#pragma unroll
        for (int ph = 0; ph < 2; ++ph) {
            if (ph == 1) __syncthreads();
            if ((warp & 1) == ph) {
#pragma unroll
                for (int j = 0; j < RPL; ++j) {
                    if (E0 >= 0) trow[j][E0] += e0[j];
                    if (E1 >= 0) trow[j][E1] += e1[j];
                    if (E2 < nb) trow[j][E2] += e2[j];
                    if (E3 < nb) trow[j][E3] += e3[j];
                }
            }
        }
    }
}

// Read-only load of *p into v when ok; v keeps its value otherwise (a predicated load, no select).
__device__ __forceinline__ void ldg_if(float &v, const float *p, int ok) {
    asm("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q ld.global.nc.f32 %0, [%1];\n\t}"
        : "+f"(v)
        : "l"(p), "r"(ok));
}

#ifndef MBX_FPCB_LOADS2
#define MBX_FPCB_LOADS2 12  // parallel walk: row loads in flight per lane, variant for 2 CTAs per SM
#endif
#ifndef MBX_FPCB_LOADS3
#define MBX_FPCB_LOADS3 16  // the same, variant for 3 CTAs per SM (85 registers)
#endif

// Parallel-beam accumulation of one pass by one warp (same contract and record interleaving as cb_accumulate).
// Slice m of a cylinder is detector row m, so a lane's rows are one base pointer plus fixed strides and each
// record costs one address computation; rows past the last detector row are predicated off.  Running sums:
// before bin bc completes, ca[] / cbb[] / cc[] hold channels bc-2, bc-1, bc; completing bin bc finishes channel
// bc-2.  Only the first two channels finished in the walk can be shared with the warp below (E0, E1), and only
// the last two of the final flush with the warp above (E2, E3).
// The walk is bound by the latency of the row loads.  Each loop iteration first issues the row loads of U records
// (reading only the cylinder offset of each record), then, as the values arrive, reads each record's coefficients
// and bin from shared memory again and accumulates, so only the loaded values stay in registers across the load
// latency (4% faster on the batched replay stage than keeping the records live).  Full iterations run unguarded;
// the last one of a sub-group clamps its record positions to the warp's range and skips the clamped ones.
// Row loads in flight per lane, measured on the batched replay stage: 8, 10, 12, 16 -> 11.90, 11.39, 11.21, 11.40 ms
// (24 and 32, in an earlier build: 15.0 and 19.5 ms against 11.6 for 16; more lines in flight thrash the L1 that
// two CTAs' shared memory leaves).
// Measured and dropped: the row loads without L1 allocation or cached in L2 only (37% and 4%
// slower), one guarded loop instead of the unguarded loop and a tail (10% slower), sub-groups walking whole bins
// of their own (they diverge at every bin end).
template <int PPW, int RPL, int MINB>
__device__ __forceinline__ void cb_accumulate_par(const FpArgs &A, const CbPass &P, int warp, int lane) {
    const mbx_geom &g = A.g;
    const CbPlan &pl = A.plan;
    constexpr int RL = 32 / PPW;
    constexpr int LOADS = MINB >= 3 ? MBX_FPCB_LOADS3 : MBX_FPCB_LOADS2;
    constexpr int U = (LOADS / RPL) < 1 ? 1 : ((LOADS / RPL) > 32 ? 32 : (LOADS / RPL));
    const int sub = lane / RL, lr = lane % RL;
    const int num_rows = g.num_det_rows, nb = pl.nb, pitch = pl.pitch;
    const int w_lo = P.bstart[P.b_lo], w_hi = P.bstart[P.b_hi];
    const int r_a = w_lo + sub, r_b = w_hi;  // this sub-group: records sub, sub + PPW, ... of the warp's range
    const int E0 = P.b_lo - 2, E1 = P.b_lo - 1, E2 = P.b_hi - 2, E3 = P.b_hi - 1;
    for (int rp = 0; rp < pl.row_passes; ++rp) {
        const int m0 = rp * RPL * RL + lr;  // row of slot 0; slot j is row m0 + j * RL
        const float *base = A.vox + m0;
        int ok[RPL];
#pragma unroll
        for (int j = 0; j < RPL; ++j) ok[j] = (m0 + j * RL) < num_rows;
        float *trow0 = P.tile + ((size_t)sub * pl.rpad + m0) * pitch;
        float ca[RPL], cbb[RPL], cc[RPL], e0[RPL], e1[RPL];
#pragma unroll
        for (int j = 0; j < RPL; ++j) ca[j] = cbb[j] = cc[j] = e0[j] = e1[j] = 0.0f;
        int bc = (r_a < r_b) ? P.sbin[r_a] : 0;
        // bin bc is complete: channel bc-2 is done
        auto finish = [&]() {
            const int c = bc - 2;
            const bool interior = c >= P.b_lo;  // in the walk c <= b_hi - 4 always
            const bool is0 = c == E0, is1 = c == E1;
#pragma unroll
            for (int j = 0; j < RPL; ++j) {
                if (interior) trow0[j * RL * pitch + c] += ca[j];
                e0[j] = is0 ? ca[j] : e0[j];
                e1[j] = is1 ? ca[j] : e1[j];
                ca[j] = cbb[j];
                cbb[j] = cc[j];
                cc[j] = 0.0f;
            }
            ++bc;
        };
        float vq[U][RPL];
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int j = 0; j < RPL; ++j) vq[u][j] = 0.0f;  // rows past R keep a finite value (never written out)
        // one iteration: records i, i + PPW, ..., i + (U-1) PPW of the sub-group (CLAMP: the last, partial one)
        auto iteration = [&](int i, auto clamp) {
            constexpr bool CLAMP = decltype(clamp)::value;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int ii = CLAMP ? min(i + u * PPW, r_b - 1) : i + u * PPW;
                const float *cyl = base + __float_as_int(P.rec[ii].x);  // 32-bit element offset of the cylinder
#pragma unroll
                for (int j = 0; j < RPL; ++j) ldg_if(vq[u][j], cyl + j * RL, ok[j]);
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int ii = i + u * PPW;
                if (!CLAMP || ii < r_b) {
                    const float4 rq = P.rec[ii];
                    const int bq = P.sbin[ii];
                    while (bc < bq) finish();
#pragma unroll
                    for (int j = 0; j < RPL; ++j) {
                        ca[j] = fmaf(rq.y, vq[u][j], ca[j]);
                        cbb[j] = fmaf(rq.z, vq[u][j], cbb[j]);
                        cc[j] = fmaf(rq.w, vq[u][j], cc[j]);
                    }
                }
            }
        };
        int i = r_a;
        for (; i + (U - 1) * PPW < r_b; i += U * PPW) iteration(i, std::false_type{});
        if (i < r_b) iteration(i, std::true_type{});
        // final flush: channels bc-2, bc-1, bc; the ones above b_hi - 3 are shared with the warp above
        float e2[RPL], e3[RPL];
#pragma unroll
        for (int j = 0; j < RPL; ++j) e2[j] = e3[j] = 0.0f;
        if (r_a < r_b) {
#pragma unroll
            for (int t = 0; t < 3; ++t) {
                const int c = bc - 2 + t;
#pragma unroll
                for (int j = 0; j < RPL; ++j) {
                    const float v = (t == 0) ? ca[j] : (t == 1 ? cbb[j] : cc[j]);
                    if (c == E0)
                        e0[j] = v;
                    else if (c == E1)
                        e1[j] = v;
                    else if (c == E2)
                        e2[j] = v;
                    else if (c == E3)
                        e3[j] = v;
                    else
                        trow0[j * RL * pitch + c] += v;
                }
            }
        }
        // edge channels: even warps first, then odd warps
#pragma unroll
        for (int ph = 0; ph < 2; ++ph) {
            if (ph == 1) __syncthreads();
            if ((warp & 1) == ph) {
#pragma unroll
                for (int j = 0; j < RPL; ++j) {
                    float *tr = trow0 + j * RL * pitch;
                    if (E0 >= 0) tr[E0] += e0[j];
                    if (E1 >= 0) tr[E1] += e1[j];
                    if (E2 < nb) tr[E2] += e2[j];
                    if (E3 < nb) tr[E3] += e3[j];
                }
            }
        }
    }
}

// Modes of a channel-block tile: scan, sort and walk its pixels (the forward projection); build, which scans and
// sorts them and stores the sorted record passes in a CbPlanned list instead of walking them; replay, which walks
// the stored passes (no scan, no sort).  A planned list is built once for a pixel list and replayed as often as
// the same list is projected again with new voxel values (every iteration of a VCD reconstruction).
// CB_WALK_SMALL is the walk in the replay layout's shared memory (plan.small), for the tiles a build could not store.
enum { CB_WALK = 0, CB_BUILD = 1, CB_REPLAY = 2, CB_WALK_SMALL = 3 };

// Stored sorted record passes of every tile of one pixel list (device storage carved by the caller).  Records and
// pass slots are taken from bump cursors (reset before a build), so their placement depends on scheduling, but
// each tile replays its own passes in order: the result is deterministic.  A tile whose passes did not fit has
// tile_npass = -1 and must be projected by the walk instead.
struct CbPlanned {
    float4 *rec;                      // [rec_cap] sorted records of every pass
    float4 *rec2;                     // [rec_cap] second record word (cone / translation) or NULL
    uint8_t *sbin;                    // [rec_cap] bin of each record
    unsigned long long *rec_cursor;   // next free record
    int *pass_cursor;                 // next free pass slot
    long long *pass_rec;              // [pass_cap] first record of each pass
    int *pass_count;                  // [pass_cap] records of each pass
    int *pass_bstart;                 // [pass_cap][nbins + 1] bin starts of each pass
    int *tile_npass;                  // [tiles] passes of each tile (-1: not planned)
    int *tile_pass;                   // [tiles][CB_MAX_PASSES] pass slots of each tile
    long long rec_cap;
    int pass_cap;
};

template <int KIND, int MINB, int MODE = CB_WALK>
__device__ void fp_cb_tile(const FpArgs &A, int j, int cb, float *sm, int *err, const CbPlanned *PL = nullptr,
                           long long ptile = 0) {
    const mbx_geom &g = A.g;
    const CbPlan &pl = A.plan;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int num_rows = g.num_det_rows, num_channels = g.num_det_channels, num_slices = g.num_recon_slices;
    const int nb = pl.nb, nbins = pl.nbins, n0 = cb * nb;
    const CbLayout &Lo = MODE == CB_REPLAY ? pl.replay : (MODE == CB_WALK_SMALL ? pl.small : pl.walk);

    float *tile = sm;  // [ppw][rpad][pitch]
    float4 *rec = reinterpret_cast<float4 *>(sm + Lo.o_rec);    // sorted {cylinder offset (int bits), a0, a1, a2}
    float4 *rec2 = reinterpret_cast<float4 *>(sm + Lo.o_rec2);  // cone: sorted {imd, W_r, mdz, mz0}
    int *sbin = reinterpret_cast<int *>(sm + Lo.o_sbin);        // bin of each sorted record
    int *ubin = reinterpret_cast<int *>(sm + Lo.o_ubin);        // kept pixels, scan order: bin << 24 | key
                                                                // (key: pixel index when vox is indexed by pixel,
                                                                // else list position; both < 2^24)
    int *bstart = reinterpret_cast<int *>(sm + Lo.o_bstart);    // [nbins + 1] padded start of each bin
    int *run = reinterpret_cast<int *>(sm + Lo.o_run);          // [nbins] histogram, then placement cursor
    int *wcnt = reinterpret_cast<int *>(sm + Lo.o_wcnt);        // [warps][nbins] per-warp counts of a chunk
    int *wstart = reinterpret_cast<int *>(sm + Lo.o_wstart);    // [warps][nbins] per-warp start positions
    float *s_vm = sm + Lo.o_cone;                               // cone: [R] detector height of each row centre
    float *s_vb = s_vm + num_rows;                              // cone: [R] same at the row's 128-row batch start
    int *s_b0 = reinterpret_cast<int *>(s_vb + num_rows);       // cone: [R] batch start row
    int *hl = reinterpret_cast<int *>(sm + Lo.o_hl);            // chunks of the current segment that can hit
    int *s_misc = reinterpret_cast<int *>(sm + Lo.o_misc);      // [2][warps]: warp counts, double-buffered;
                                                                // [2][warps]: hit counts of a segment

    const int vi = A.views ? A.views[j] : j;
    const bool view_ok = vi >= 0 && vi < g.num_views;
    if (!view_ok && tid == 0 && cb == 0) flag_error(err, MBX_ERRFLAG_VIEW);
    float cs, sn, tz = 0.0f;  // translation: (cs, sn, tz) = the view's (tx, ty, tz)
    if (KIND == MBX_GEOM_TRANSLATION) {
        cs = view_ok ? g.translations[3 * vi] : 0.0f;
        sn = view_ok ? g.translations[3 * vi + 1] : 0.0f;
        tz = view_ok ? g.translations[3 * vi + 2] : 0.0f;
    } else {
        const float angle = view_ok ? g.angles[vi] : 0.0f;
        cs = cosf(angle);
        sn = sinf(angle);
    }
    // slice coordinate of detector height 0: (S-1)/2 - recon_slice_offset / delta_voxel (the translation view's
    // slice heights are shifted by -tz instead)
    const float zoff = KIND == MBX_GEOM_TRANSLATION ? -tz : g.recon_slice_offset;
    const float kconst = 0.5f * (float)(num_slices - 1) - zoff / g.delta_voxel;
    const float inv_cols = 1.0f / (float)g.num_recon_cols;
    const float inv_d = isinf(g.source_detector_dist) ? 0.0f : 1.0f / g.source_detector_dist;

    __syncthreads();  // previous tile of this CTA (batched use) is finished with shared memory
    const int tile_words = pl.ppw * pl.rpad * pl.pitch;
    for (int i = tid; i < tile_words; i += CB_THREADS) tile[i] = 0.0f;
    if (MODE != CB_REPLAY)
        for (int i = tid; i < CB_WARPS * nbins; i += CB_THREADS) wcnt[i] = 0;
    if (KIND != MBX_GEOM_PARALLEL) {
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

    // phase 3 of a pass whose sorted records (rec, rec2, sbin) and bin starts (bstart) are in shared memory
    auto walk = [&]() {
        // ---- 3. warp ranges of bins with about equal record counts, at least two bins each:
        //         B_v = 2v + max_{u<=v}(lb_u - 2u), then B_v <= nbins - 2(8 - v); lb_v = first bin starting at or
        //         after v/8 of the records
        CbPass P;
        {
            const int tot = bstart[nbins];
            int lb = 0;
            if (lane <= CB_WARPS) {
                const int target = (int)(((long long)lane * tot) / CB_WARPS);
                int lo = 0, hi = nbins;
                while (lo < hi) {
                    const int mid = (lo + hi) >> 1;
                    if (bstart[mid] >= target)
                        hi = mid;
                    else
                        lo = mid + 1;
                }
                lb = lo;
            }
            int t = (lane <= CB_WARPS) ? lb - 2 * lane : INT_MIN / 2;
    #pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, t, off);
                if (lane >= off) t = max(t, u);
            }
            int bv = min(2 * lane + t, nbins - 2 * (CB_WARPS - lane));
            if (lane == CB_WARPS) bv = nbins;
            P.b_lo = __shfl_sync(0xffffffffu, bv, warp);
            P.b_hi = __shfl_sync(0xffffffffu, bv, warp + 1);
        }
        P.rec = rec;
        P.rec2 = rec2;
        P.sbin = sbin;
        P.bstart = bstart;
        P.tile = tile;
        P.s_vm = s_vm;
        P.s_vb = s_vb;
        P.s_b0 = s_b0;
        P.win = sm + Lo.o_win;
        if (KIND == MBX_GEOM_PARALLEL) {
            switch (pl.ppw * 8 + pl.rpl) {  // the lane layouts plan_fp_cb chooses from
                case 9: cb_accumulate_par<1, 1, MINB>(A, P, warp, lane); break;
                case 10: cb_accumulate_par<1, 2, MINB>(A, P, warp, lane); break;
                case 11: cb_accumulate_par<1, 3, MINB>(A, P, warp, lane); break;
                case 12: cb_accumulate_par<1, 4, MINB>(A, P, warp, lane); break;
                case 17: cb_accumulate_par<2, 1, MINB>(A, P, warp, lane); break;
                case 18: cb_accumulate_par<2, 2, MINB>(A, P, warp, lane); break;
                case 19: cb_accumulate_par<2, 3, MINB>(A, P, warp, lane); break;
                case 20: cb_accumulate_par<2, 4, MINB>(A, P, warp, lane); break;
                case 33: cb_accumulate_par<4, 1, MINB>(A, P, warp, lane); break;
                case 34: cb_accumulate_par<4, 2, MINB>(A, P, warp, lane); break;
                case 35: cb_accumulate_par<4, 3, MINB>(A, P, warp, lane); break;
                default: cb_accumulate_par<4, 4, MINB>(A, P, warp, lane); break;
            }
        } else switch (pl.ppw * 8 + pl.rpl) {  // the lane layouts plan_fp_cb chooses from
            case 9: cb_accumulate<KIND, 1, 1>(A, P, warp, lane, kconst); break;
            case 10: cb_accumulate<KIND, 1, 2>(A, P, warp, lane, kconst); break;
            case 11: cb_accumulate<KIND, 1, 3>(A, P, warp, lane, kconst); break;
            case 12: cb_accumulate<KIND, 1, 4>(A, P, warp, lane, kconst); break;
            case 17: cb_accumulate<KIND, 2, 1>(A, P, warp, lane, kconst); break;
            case 18: cb_accumulate<KIND, 2, 2>(A, P, warp, lane, kconst); break;
            case 19: cb_accumulate<KIND, 2, 3>(A, P, warp, lane, kconst); break;
            case 20: cb_accumulate<KIND, 2, 4>(A, P, warp, lane, kconst); break;
            case 33: cb_accumulate<KIND, 4, 1>(A, P, warp, lane, kconst); break;
            case 34: cb_accumulate<KIND, 4, 2>(A, P, warp, lane, kconst); break;
            case 35: cb_accumulate<KIND, 4, 3>(A, P, warp, lane, kconst); break;
            default: cb_accumulate<KIND, 4, 4>(A, P, warp, lane, kconst); break;
        }
    };

    if constexpr (MODE == CB_REPLAY) {  // the stored passes of this tile, walked in order
        const int npass = min(PL->tile_npass[ptile], CB_MAX_PASSES);
        // the tile's pass table (slot, first record, count; count -1: not usable) read once into shared memory,
        // so that a pass's loads start without a chain of dependent global reads, and the records of the next
        // pass prefetched into L2 while the current one is walked (7.6% faster on the batched bench stage than
        // reading each pass's table entry and records when the pass starts)
        __shared__ long long s_prec[CB_MAX_PASSES];
        __shared__ int s_pslot[CB_MAX_PASSES], s_pcnt[CB_MAX_PASSES];
        for (int q = tid; q < npass; q += CB_THREADS) {
            const int ps = PL->tile_pass[ptile * CB_MAX_PASSES + q];
            int cnt = -1;
            long long rs = 0;
            if (ps >= 0 && ps < PL->pass_cap) {  // never written by a build otherwise
                cnt = PL->pass_count[ps];
                rs = PL->pass_rec[ps];
                if (cnt < 0 || cnt > Lo.cap || rs < 0 || rs + cnt > PL->rec_cap) cnt = -1;
            }
            s_pslot[q] = ps;
            s_pcnt[q] = cnt;
            s_prec[q] = rs;
        }
        __syncthreads();
        // L2 prefetch of pass q's records, bins and bin starts (addresses inside the pass's own ranges)
        auto prefetch_pass = [&](int q) {
            const int cnt = s_pcnt[q];
            if (cnt <= 0) return;
            const long long rs = s_prec[q];
            const char *r0 = reinterpret_cast<const char *>(PL->rec + rs);
            const char *r2 = KIND != MBX_GEOM_PARALLEL ? reinterpret_cast<const char *>(PL->rec2 + rs) : nullptr;
            for (long long o = (long long)tid * 128; o < (long long)cnt * 16; o += (long long)CB_THREADS * 128) {
                asm volatile("prefetch.global.L2 [%0];" ::"l"(r0 + o));
                if (KIND != MBX_GEOM_PARALLEL) asm volatile("prefetch.global.L2 [%0];" ::"l"(r2 + o));
            }
            const char *b0 = reinterpret_cast<const char *>(PL->sbin + rs);
            for (int o = tid * 128; o < cnt; o += CB_THREADS * 128) asm volatile("prefetch.global.L2 [%0];" ::"l"(b0 + o));
            const char *bs = reinterpret_cast<const char *>(PL->pass_bstart + (long long)s_pslot[q] * (nbins + 1));
            for (int o = tid * 128; o < (nbins + 1) * 4; o += CB_THREADS * 128)
                asm volatile("prefetch.global.L2 [%0];" ::"l"(bs + o));
        };
        if (npass > 0) prefetch_pass(0);
        for (int q = 0; q < npass; ++q) {
            const int ps = s_pslot[q], count = s_pcnt[q];
            const long long rs = s_prec[q];
            if (count < 0) {  // skip, and say so
                if (tid == 0) flag_error(err, MBX_ERRFLAG_CACHE);
                continue;
            }
            // no barrier before overwriting the lists: every warp read its last record, bin and bin start of the
            // previous pass before the edge-phase barrier that ends each walk, and after it only the tile is
            // written (0.7% faster on the batched replay stage than with a barrier per pass here)
            for (int b = tid; b <= nbins; b += CB_THREADS) bstart[b] = PL->pass_bstart[(long long)ps * (nbins + 1) + b];
            for (int i = tid; i < count; i += CB_THREADS) {
                rec[i] = PL->rec[rs + i];
                if (KIND != MBX_GEOM_PARALLEL) rec2[i] = PL->rec2[rs + i];
                sbin[i] = PL->sbin[rs + i];
            }
            if (tid < CB_PAD) {  // padding read (never used) by the walk past the last record
                rec[count + tid] = make_float4(0.f, 0.f, 0.f, 0.f);
                sbin[count + tid] = nbins - 1;
            }
            __syncthreads();
            if (q + 1 < npass) prefetch_pass(q + 1);
            walk();
        }
    }
    bool build_ok = true;  // build: every pass so far found room in the planned list
    int build_np = 0;      // build: passes stored so far

    const int npix_grid = g.num_recon_rows * g.num_recon_cols;
    const long long num_pixels = view_ok ? A.num_pixels : 0;
    const long long nchunks = (num_pixels + CB_CHUNK - 1) / CB_CHUNK;
    long long seg = 0;    // first chunk of the next segment of CB_THREADS chunks to test
    int nh = 0, hp = 0;   // chunks of the current segment that can reach the block (in hl), next one to scan
    int idx_next = -1;    // prefetched pixel index of entry tid of chunk hl[hp]
    bool more = MODE != CB_REPLAY && num_pixels > 0;

    while (more) {
        __syncthreads();  // the previous pass is done with every list
        for (int b = tid; b < nbins; b += CB_THREADS) run[b] = 0;
        __syncthreads();
        // ---- 1. ordered compaction of the pixels that touch this channel block
        int count = 0, par = 0;
        while (count <= Lo.fill) {
            if (hp == nh) {
                if (seg >= nchunks) {
                    more = false;
                    break;
                }
                // next segment: ordered list of its chunks whose bounding box can reach the block
                __syncthreads();  // everyone is done with hl
                const long long c = seg + tid;
                bool hit = false;
                if (c < nchunks)
                    hit = !A.chunk_box || !cb_box_misses<KIND>(g, __ldg(A.chunk_box + c), cs, sn, inv_d, n0, nb);
                const unsigned hb = __ballot_sync(0xffffffffu, hit);
                int *hw = s_misc + 2 * CB_WARPS;
                if (lane == 0) hw[warp] = __popc(hb);
                __syncthreads();
                int hbase = 0, htot = 0;
#pragma unroll
                for (int w = 0; w < CB_WARPS; ++w) {
                    const int k = hw[w];
                    hbase += (w < warp) ? k : 0;
                    htot += k;
                }
                if (hit) hl[hbase + __popc(hb & ((1u << lane) - 1u))] = (int)c;
                __syncthreads();
                nh = htot;
                hp = 0;
                seg += CB_THREADS;
                if (nh > 0) {
                    const long long p0 = (long long)hl[0] * CB_CHUNK + tid;
                    idx_next = p0 < num_pixels ? A.pix[p0] : -1;
                }
                continue;
            }
            const long long p = (long long)hl[hp] * CB_CHUNK + tid;
            const int idx = idx_next;
            ++hp;
            if (hp < nh) {  // prefetch the next chunk's entry while this one is compacted
                const long long pn = (long long)hl[hp] * CB_CHUNK + tid;
                idx_next = pn < num_pixels ? A.pix[pn] : -1;
            }
            bool take = false;
            int bin = 0;
            if (p < num_pixels) {
                if (idx < 0 || idx >= npix_grid) {
                    if (cb == 0 && j == 0) flag_error(err, MBX_ERRFLAG_PIXEL);
                } else {
                    float xt, yt, mag;
                    cb_pixel<KIND>(g, idx, inv_cols, xt, yt);
                    const int nc = (int)rintf(cb_channel<KIND>(g, cs, sn, xt, yt, inv_d, mag));
                    bin = nc - n0 + 1;
                    take = bin >= 0 && bin < nbins;
                }
            }
            const unsigned ballot = __ballot_sync(0xffffffffu, take);
            int *wc = s_misc + par * CB_WARPS;  // the other buffer is still being read by slower warps
            if (lane == 0) wc[warp] = __popc(ballot);
            __syncthreads();
            int base = count, total = 0;
#pragma unroll
            for (int w = 0; w < CB_WARPS; ++w) {
                const int c = wc[w];
                base += (w < warp) ? c : 0;
                total += c;
            }
            if (take) {
                const int pos = base + __popc(ballot & ((1u << lane) - 1u));
                ubin[pos] = (int)(((unsigned)bin << 24) | (unsigned)(A.vox_by_index ? idx : (int)p));
                atomicAdd(run + bin, 1);  // integer histogram: order-independent
            }
            count += total;
            par ^= 1;
        }
        __syncthreads();
        if (count == 0) continue;
        // ---- 2a. bin starts: exclusive scan of the histogram (warp 0); run[] becomes the placement cursor
        if (warp == 0) {
            const int per = (nbins + 31) / 32;
            int loc = 0;
            for (int k = 0; k < per; ++k) {
                const int b = lane * per + k;
                if (b < nbins) loc += run[b];
            }
            int incl = loc;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, incl, off);
                if (lane >= off) incl += t;
            }
            int acc = incl - loc;
            for (int k = 0; k < per; ++k) {
                const int b = lane * per + k;
                if (b < nbins) {
                    const int h = run[b];
                    bstart[b] = acc;
                    run[b] = acc;
                    acc += h;
                }
            }
            if (lane == 31) bstart[nbins] = incl;
        }
        __syncthreads();
        // ---- 2b. stable placement by bin, computing the footprints on the way.  Per chunk of 256 kept pixels:
        //          per-warp bin counts (ranks from __match_any_sync), then each bin's per-warp start positions
        //          (cursor + counts of the warps before), then the records.
        for (int base = 0; base < count; base += CB_THREADS) {
            const int i = base + tid;
            const bool valid = i < count;
            const unsigned ub = valid ? (unsigned)ubin[i] : 0u;
            const int b = valid ? (int)(ub >> 24) : -1;  // bins reach nb + 1 = 129: unsigned unpacking
            const unsigned peers = __match_any_sync(0xffffffffu, b);
            const int rank = __popc(peers & ((1u << lane) - 1u));
            if (valid && rank == 0) wcnt[warp * nbins + b] = __popc(peers);
            __syncthreads();
            for (int bb = tid; bb < nbins; bb += CB_THREADS) {
                int acc = run[bb];
                for (int w = 0; w < CB_WARPS; ++w) {
                    const int c = wcnt[w * nbins + bb];
                    wstart[w * nbins + bb] = acc;
                    wcnt[w * nbins + bb] = 0;
                    acc += c;
                }
                run[bb] = acc;
            }
            __syncthreads();
            if (valid) {
                const int pos = wstart[warp * nbins + b] + rank;
                const int key = (int)(ub & 0xFFFFFFu);
                const int idx = A.vox_by_index ? key : __ldg(A.pix + key);  // checked in the scan
                float xt, yt;
                cb_pixel<KIND>(g, idx, inv_cols, xt, yt);
                float a0, a1, a2, imd, wr, mdz, mz0;
                cb_footprint<KIND>(g, cs, sn, xt, yt, n0 + b - 1, a0, a1, a2, imd, wr, mdz, mz0, tz);
                // element offset of the pixel's cylinder (the host admits vox buffers of < 2^31 elements)
                rec[pos] = make_float4(__int_as_float(key * num_slices), a0, a1, a2);
                if (KIND != MBX_GEOM_PARALLEL) rec2[pos] = make_float4(imd, wr, mdz, mz0);
                sbin[pos] = b;
            }
            // the next chunk's counts go to wcnt (cleared above); its starts overwrite wstart only after the
            // barrier that follows, which every thread reaches after reading its start here
        }
        if (tid < CB_PAD) {  // padding read (never used) by the walk past the last record
            rec[count + tid] = make_float4(0.f, 0.f, 0.f, 0.f);
            sbin[count + tid] = nbins - 1;
        }
        __syncthreads();
        if (MODE == CB_BUILD) {  // store the pass instead of walking it
            __shared__ long long s_rs;
            __shared__ int s_ps;
            if (tid == 0) {
                long long rsv = -1;
                int psv = -1;
                if (build_ok && build_np < CB_MAX_PASSES) {
                    rsv = (long long)atomicAdd(PL->rec_cursor, (unsigned long long)count);
                    psv = atomicAdd(PL->pass_cursor, 1);
                    if (rsv + count > PL->rec_cap || psv >= PL->pass_cap) rsv = -1;
                }
                s_rs = rsv;
                s_ps = psv;
            }
            __syncthreads();
            const long long rsv = s_rs;
            const int psv = s_ps;
            if (rsv < 0) build_ok = false;
            if (build_ok) {
                for (int i = tid; i < count; i += CB_THREADS) {
                    PL->rec[rsv + i] = rec[i];
                    if (KIND != MBX_GEOM_PARALLEL) PL->rec2[rsv + i] = rec2[i];
                    PL->sbin[rsv + i] = (uint8_t)sbin[i];
                }
                for (int b = tid; b <= nbins; b += CB_THREADS) PL->pass_bstart[(long long)psv * (nbins + 1) + b] = bstart[b];
                if (tid == 0) {
                    PL->pass_rec[psv] = rsv;
                    PL->pass_count[psv] = count;
                    PL->tile_pass[ptile * CB_MAX_PASSES + build_np] = psv;
                }
            }
            ++build_np;
        } else {
            walk();
        }
    }
    if (MODE == CB_BUILD) {
        if (tid == 0) PL->tile_npass[ptile] = build_ok ? build_np : -1;
        return;
    }
    __syncthreads();
    // ---- 4. fixed-order sum of the sub-group copies, coalesced write
    const int nch = min(nb, num_channels - n0);
    const int ppw = pl.ppw;
    float *out = A.out + (long long)j * num_rows * num_channels + n0;
    for (int e = tid; e < num_rows * nb; e += CB_THREADS) {
        const int m = e / nb, c = e - (e / nb) * nb;
        if (c >= nch) continue;
        float s = 0.0f;
        for (int k = 0; k < ppw; ++k) s += tile[((size_t)k * pl.rpad + m) * pl.pitch + c];
        out[(long long)m * num_channels + c] = s;
    }
}

// MINB = plan.minb: the variant compiled for 2 resident CTAs per SM (up to 128 registers) or 3 (up to 85).
template <int KIND, int MINB>
__global__ void __launch_bounds__(CB_THREADS, MINB) fp_cb_kernel(const FpArgs A, int *err) {
    extern __shared__ __align__(16) float smcb[];
    fp_cb_tile<KIND, MINB>(A, blockIdx.x, blockIdx.y, smcb, err);
}

}  // namespace mbx
