// Batched VCD: many independent scans of uneven geometry reconstructed together (sm_100a).
//
// The per-scan reconstruction is the reference's VCD subset update (tomography_model.py:1343-1542, as in
// vcd.cu).  Batching replaces one launch per scan per stage with ONE persistent launch per stage for all scans:
// each stage kernel walks a packed work list -- the concatenation of every scan's tiles, described by
// per-stage prefix offsets over scans -- with a grid sized to the resident CTAs of the device, and decodes each
// tile into (scan, local tile) by binary search.  The two projection stages hand tiles out dynamically (an
// atomic counter reset by a memset before each launch) over a work list ordered by decreasing per-tile cost,
// so scans of very different size finish together.  Stages of one subset step:
//   b_bp      back projection of W*e at each scan's current subset (bp_fast tiles)
//   b_delta   qGGMRF gradient/Hessian + delta; float64 partials of the prior terms, one per tile
//   b_fp      forward projection of delta (channel-block tiles of fp_cb)
//   b_linquad float64 partials of <We, dA> and <W dA, dA> per sinogram tile
//   b_alpha   one warp per scan: fixed-order sums of that scan's partials -> alpha
//   b_apply   recon[idx] += alpha*delta, l1 partials
//   b_error   e -= alpha*dA, then b_l1 folds the l1 partials per scan
// The subset each scan updates at each step comes from a schedule table in device memory, and every per-(scan,
// subset) argument record is built once in mbx_vcd_batched_prepare, so the launches of a step depend only on
// the step number: the whole multi-iteration reconstruction can be captured once in a CUDA graph and replayed.
#include <algorithm>
#include <cstring>
#include <vector>

#include "back_project.cuh"
#include "bp_fast.cuh"
#include "fp_cb.cuh"
#include "mbx_common.cuh"
#include "mbx_host.hpp"
#include "mbx_reduce.cuh"
#include "qggmrf.cuh"

namespace mbx {

constexpr int BT_THREADS = 256;
constexpr int BT_ELEM_TILE = 2048;   // cylinder elements per tile (delta, apply)
constexpr int BT_SINO_TILE = 4096;   // sinogram / recon elements per tile (linquad, error, stats)
constexpr float BT_EPS_F32 = 1.1920928955078125e-07f;

struct VcdScan {
    float *recon;               // flat (Nr*Nc, S)
    float *err;                 // (V, R, C)
    const float *wts;           // (V, R, C) or NULL
    const float *hess;          // flat (Nr*Nc, S)
    const int32_t *partition;   // (K, M)
    float *bp, *delta, *dsino;  // workspace slices
    long long nsino, nrecon;
    int K, M, nr, nc, ns;
    float fm_constant;
    QParams q;
};

struct BatchedTables {
    VcdScan *scans;
    BpArgs *bpargs;     // [scan][subset]
    FpArgs *fpargs;     // [scan][subset]
    int *bp_off, *fp_off, *el_off, *sn_off, *rc_off;  // [num_scans + 1] tile prefix offsets
    int *fp_cblocks;    // [num_scans]
    int *bp_gx;         // [num_scans]
    int *bp_scan, *fp_scan;  // [num_scans]: scan at each position of the (cost-sorted) bp / fp work lists
    int *counters;      // [2]: next bp / fp tile to hand out (reset before each launch)
    int *schedule;      // [num_steps][num_scans]
    double *p_prior, *p_fwd, *p_l1, *p_iter;
    float *alpha;       // [num_scans]
    double *step_stats; // [num_steps][num_scans][4]
    double *iter_stats; // [num_iterations][num_scans][4]
};

struct BatchedPlanHost {
    BatchedTables t;
    int num_scans, kind, num_steps, num_iterations;
    int bp_total, fp_total, el_total, sn_total, rc_total;
    int bp_grid, fp_grid, el_grid, sn_grid, rc_grid;
    size_t bp_smem, fp_smem;
    int fp_minb;  // b_fp variant: 2 or 3 resident CTAs per SM
    int magic;
};
static_assert(sizeof(BatchedPlanHost) <= sizeof(mbx_batched_plan), "plan record too large");
constexpr int BT_MAGIC = 0x6d627862;

__device__ __forceinline__ int find_scan(const int *__restrict__ off, int num_scans, int t) {
    int lo = 0, hi = num_scans;  // off[lo] <= t < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(off + mid) <= t) lo = mid; else hi = mid;
    }
    return lo;
}

// Sum of NV values over the block into slot[NV * t + i] (fixed order).
template <int NV>
__device__ __forceinline__ void tile_reduce(const double (&v)[NV], double *slot) {
    __shared__ double sh[32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const double a = warp_sum(v[i]);
        if (lane == 0) sh[warp][i] = a;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double a = lane < BT_THREADS / 32 ? sh[lane][i] : 0.0;
            a = warp_sum(a);
            if (lane == 0) slot[i] = a;
        }
    }
    __syncthreads();
}

// Next tile of a dynamically scheduled work list (one atomic per CTA per tile).
__device__ __forceinline__ int fetch_tile(int *counter) {
    __shared__ int s_next;
    __syncthreads();  // every thread is done with the previous tile index
    if (threadIdx.x == 0) s_next = atomicAdd(counter, 1);
    __syncthreads();
    return s_next;
}

template <int KIND>
#ifndef MBX_BBP_MIN_BLOCKS
#define MBX_BBP_MIN_BLOCKS 3  // resident CTAs per SM the batched back projection is compiled for
#endif
__global__ void __launch_bounds__(BPF_THREADS, MBX_BBP_MIN_BLOCKS) b_bp(BatchedTables T, int num_scans, int step, int first, int total, int *err) {
    extern __shared__ __align__(16) float smb[];
    for (int t = first + fetch_tile(T.counters); t < total; t = first + fetch_tile(T.counters)) {
        const int k = find_scan(T.bp_off, num_scans, t);
        const int s = __ldg(T.bp_scan + k);
        const int local = t - __ldg(T.bp_off + k);
        const int sub = __ldg(T.schedule + step * num_scans + s);
        const int K = T.scans[s].K;
        const int gx = __ldg(T.bp_gx + s);
        bp_fast_tile<KIND>(T.bpargs[s * K + sub], local % gx, local / gx, 0, smb, err);
    }
}

// MINB: resident CTAs per SM the variant is compiled for (2 or 3, matching the plans' fp_cb minb).
template <int KIND, int MINB>
__global__ void __launch_bounds__(CB_THREADS, MINB) b_fp(BatchedTables T, int num_scans, int step, int first, int total, int *err) {
    extern __shared__ __align__(16) float smf2[];
    for (int t = first + fetch_tile(T.counters + 1); t < total; t = first + fetch_tile(T.counters + 1)) {
        const int k = find_scan(T.fp_off, num_scans, t);
        const int s = __ldg(T.fp_scan + k);
        const int local = t - __ldg(T.fp_off + k);
        const int sub = __ldg(T.schedule + step * num_scans + s);
        const int K = T.scans[s].K;
        const int cbs = __ldg(T.fp_cblocks + s);
        fp_cb_tile<KIND, MINB>(T.fpargs[s * K + sub], local / cbs, local % cbs, smf2, err);
    }
}

__global__ void __launch_bounds__(BT_THREADS) b_delta(BatchedTables T, int num_scans, int step, int total, int *err) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int s = find_scan(T.el_off, num_scans, t);
        const int local = t - __ldg(T.el_off + s);
        const VcdScan &sc = T.scans[s];
        const int sub = __ldg(T.schedule + step * num_scans + s);
        const int32_t *pix = sc.partition + (long long)sub * sc.M;
        const long long n = (long long)sc.M * sc.ns;
        const long long e0 = (long long)local * BT_ELEM_TILE;
        const long long e1 = min(n, e0 + BT_ELEM_TILE);
        const int npix = sc.nr * sc.nc;
        double pl = 0.0, pq = 0.0;
        for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) {
            const long long p = i / sc.ns;
            const int k = (int)(i - p * sc.ns);
            const int idx = pix[p];
            float d = 0.0f;
            if (idx < 0 || idx >= npix) {
                flag_error(err, MBX_ERRFLAG_PIXEL);
            } else {
                float gp, hp;
                qggmrf_voxel(sc.recon, sc.nr, sc.nc, sc.ns, idx, k, sc.q, gp, hp);
                const float gf = -sc.fm_constant * sc.bp[i];
                const float hf = sc.fm_constant * __ldg(sc.hess + (long long)idx * sc.ns + k);
                d = -((gf + gp) / (hf + hp));
                pl += (double)(gp * d);
                pq += (double)(hp * (d * d));
            }
            sc.delta[i] = d;
        }
        const double v[2] = {pl, pq};
        tile_reduce<2>(v, T.p_prior + 2 * t);
    }
}

__global__ void __launch_bounds__(BT_THREADS) b_linquad(BatchedTables T, int num_scans, int total) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int s = find_scan(T.sn_off, num_scans, t);
        const int local = t - __ldg(T.sn_off + s);
        const VcdScan &sc = T.scans[s];
        const long long e0 = (long long)local * BT_SINO_TILE;
        const long long e1 = min(sc.nsino, e0 + BT_SINO_TILE);
        double fl = 0.0, fq = 0.0;
        for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) {
            const float ds = sc.dsino[i], e = sc.err[i];
            const float w = sc.wts ? sc.wts[i] : 1.0f;
            fl += (double)((w * e) * ds);
            fq += (double)(ds * ds * w);
        }
        const double v[2] = {fl, fq};
        tile_reduce<2>(v, T.p_fwd + 2 * t);
    }
}

__device__ __forceinline__ double warp_range_sum(const double *__restrict__ p, int b, int e, int nv, int v) {
    const int lane = threadIdx.x & 31;
    double s = 0.0;
    for (int i = b + lane; i < e; i += 32) s += p[(long long)i * nv + v];
    s = warp_sum(s);
    return __shfl_sync(0xffffffffu, s, 0);
}

__global__ void b_alpha(BatchedTables T, int num_scans, int step) {
    const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (s >= num_scans) return;
    const VcdScan &sc = T.scans[s];
    const int eb = __ldg(T.el_off + s), ee = __ldg(T.el_off + s + 1);
    const int sb = __ldg(T.sn_off + s), se = __ldg(T.sn_off + s + 1);
    const double pl = warp_range_sum(T.p_prior, eb, ee, 2, 0);
    const double pq = 0.5 * warp_range_sum(T.p_prior, eb, ee, 2, 1);
    const double fm = (double)sc.fm_constant;
    const double fl = fm * warp_range_sum(T.p_fwd, sb, se, 2, 0);
    const double fq = fm * warp_range_sum(T.p_fwd, sb, se, 2, 1);
    if ((threadIdx.x & 31) == 0) {
        const double num = fl - pl, den = fq + pq + (double)BT_EPS_F32;
        float a = (float)(num / den);
        a = fminf(fmaxf(a, BT_EPS_F32), 1.5f);
        if (num != num || den != den) a = nanf("");
        T.alpha[s] = a;
        double *st = T.step_stats + ((long long)step * num_scans + s) * 4;
        st[0] = (double)a;
        st[2] = num;
        st[3] = den;
    }
}

__global__ void __launch_bounds__(BT_THREADS) b_apply(BatchedTables T, int num_scans, int step, int total) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int s = find_scan(T.el_off, num_scans, t);
        const int local = t - __ldg(T.el_off + s);
        const VcdScan &sc = T.scans[s];
        const int sub = __ldg(T.schedule + step * num_scans + s);
        const int32_t *pix = sc.partition + (long long)sub * sc.M;
        const float alpha = T.alpha[s];
        const long long n = (long long)sc.M * sc.ns;
        const long long e0 = (long long)local * BT_ELEM_TILE;
        const long long e1 = min(n, e0 + BT_ELEM_TILE);
        const int npix = sc.nr * sc.nc;
        double l1 = 0.0;
        for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) {
            const long long p = i / sc.ns;
            const int k = (int)(i - p * sc.ns);
            const int idx = pix[p];
            if (idx < 0 || idx >= npix) continue;
            const float d = alpha * sc.delta[i];
            atomicAdd(sc.recon + (long long)idx * sc.ns + k, d);
            l1 += (double)fabsf(d);
        }
        const double v[1] = {l1};
        tile_reduce<1>(v, T.p_l1 + t);
    }
}

__global__ void __launch_bounds__(BT_THREADS) b_error(BatchedTables T, int num_scans, int total) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int s = find_scan(T.sn_off, num_scans, t);
        const int local = t - __ldg(T.sn_off + s);
        const VcdScan &sc = T.scans[s];
        const float alpha = T.alpha[s];
        const long long e0 = (long long)local * BT_SINO_TILE;
        const long long e1 = min(sc.nsino, e0 + BT_SINO_TILE);
        for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) sc.err[i] -= alpha * sc.dsino[i];
    }
}

__global__ void b_l1(BatchedTables T, int num_scans, int step) {
    const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (s >= num_scans) return;
    const double l1 = warp_range_sum(T.p_l1, __ldg(T.el_off + s), __ldg(T.el_off + s + 1), 1, 0);
    if ((threadIdx.x & 31) == 0) T.step_stats[((long long)step * num_scans + s) * 4 + 1] = l1;
}

// Per-iteration statistics: sum of w e^2, sum of |recon| (the reference's fm_rmse and NMAE inputs).
__global__ void __launch_bounds__(BT_THREADS) b_iter_partials(BatchedTables T, int num_scans, int total_sn,
                                                             int total_rc) {
    for (int t = blockIdx.x; t < total_sn + total_rc; t += gridDim.x) {
        double a = 0.0;
        if (t < total_sn) {
            const int s = find_scan(T.sn_off, num_scans, t);
            const int local = t - __ldg(T.sn_off + s);
            const VcdScan &sc = T.scans[s];
            const long long e0 = (long long)local * BT_SINO_TILE, e1 = min(sc.nsino, e0 + BT_SINO_TILE);
            for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) {
                const float e = sc.err[i];
                const float w = sc.wts ? sc.wts[i] : 1.0f;
                a += (double)(e * e) * (double)w;
            }
        } else {
            const int tr = t - total_sn;
            const int s = find_scan(T.rc_off, num_scans, tr);
            const int local = tr - __ldg(T.rc_off + s);
            const VcdScan &sc = T.scans[s];
            const long long e0 = (long long)local * BT_SINO_TILE, e1 = min(sc.nrecon, e0 + BT_SINO_TILE);
            for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) a += (double)fabsf(sc.recon[i]);
        }
        const double v[1] = {a};
        tile_reduce<1>(v, T.p_iter + t);
    }
}

__global__ void b_iter_final(BatchedTables T, int num_scans, int iteration, int total_sn) {
    const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (s >= num_scans) return;
    const double e2 = warp_range_sum(T.p_iter, __ldg(T.sn_off + s), __ldg(T.sn_off + s + 1), 1, 0);
    const double ax = warp_range_sum(T.p_iter + total_sn, __ldg(T.rc_off + s), __ldg(T.rc_off + s + 1), 1, 0);
    if ((threadIdx.x & 31) == 0) {
        double *st = T.iter_stats + ((long long)iteration * num_scans + s) * 4;
        st[0] = e2;
        st[1] = ax;
        st[2] = 0.0;
        st[3] = 0.0;
    }
}

// ------------------------------------------------------------------------------------------------ host side
struct ScanSizes {
    long long ncyl, nsino, nrecon;
    int bp_tiles, bp_gx, fp_tiles, el_tiles, sn_tiles, rc_tiles;
    BpfPlan bpp;
    CbPlan fpp;
};

static int scan_sizes(const mbx_scan &sc, ScanSizes &z) {
    const mbx_geom &g = sc.geom;
    int rc = validate_geom(&g);
    if (rc != MBX_OK) return rc;
    if (!sc.flat_recon || !sc.error_sinogram || !sc.fm_hessian || !sc.partition) return MBX_ERR_INVALID_ARG;
    if (sc.num_subsets <= 0 || sc.subset_size <= 0) return MBX_ERR_INVALID_ARG;
    if (!(sc.qp.sigma_x > 0.0f) || !(sc.qp.T > 0.0f) || !(sc.qp.p > 0.0f)) return MBX_ERR_INVALID_ARG;
    z.bpp = plan_bp_fast(g, sc.subset_size, g.num_views);
    z.fpp = plan_fp_cb(g);
    if (!z.bpp.ok || !z.fpp.ok) return MBX_ERR_UNSUPPORTED;  // batched path needs the radius-1 kernels
    if ((long long)sc.subset_size * g.num_recon_slices >= (1LL << 31)) return MBX_ERR_UNSUPPORTED;
    if (sc.subset_size > (1 << 24)) return MBX_ERR_UNSUPPORTED;  // list positions share a word with the bin
    z.ncyl = (long long)sc.subset_size * g.num_recon_slices;
    z.nsino = (long long)g.num_views * g.num_det_rows * g.num_det_channels;
    z.nrecon = (long long)g.num_recon_rows * g.num_recon_cols * g.num_recon_slices;
    z.bp_gx = z.bpp.gx;
    z.bp_tiles = z.bpp.gx * z.bpp.gy;
    z.fp_tiles = g.num_views * z.fpp.cblocks;
    z.el_tiles = (int)((z.ncyl + BT_ELEM_TILE - 1) / BT_ELEM_TILE);
    z.sn_tiles = (int)((z.nsino + BT_SINO_TILE - 1) / BT_SINO_TILE);
    z.rc_tiles = (int)((z.nrecon + BT_SINO_TILE - 1) / BT_SINO_TILE);
    return MBX_OK;
}

struct Layout {
    size_t scans, bpargs, fpargs, offs, cblocks, gx, scan_of, counters, sched, p_prior, p_fwd, p_l1, p_iter, alpha,
        bufs, total;
    int bp_total, fp_total, el_total, sn_total, rc_total;
    std::vector<size_t> buf_off;  // per scan: bp, delta, dsino
    std::vector<size_t> box_off;  // per scan: chunk bounding boxes of its subsets, [K][chunks]
};

static int layout(const mbx_scan *scans, int n, int num_steps, Layout &L, std::vector<ScanSizes> &zs) {
    zs.resize(n);
    L.bp_total = L.fp_total = L.el_total = L.sn_total = L.rc_total = 0;
    int kind = -1, ksum = 0;
    for (int s = 0; s < n; ++s) {
        int rc = scan_sizes(scans[s], zs[s]);
        if (rc != MBX_OK) return rc;
        if (kind >= 0 && scans[s].geom.kind != kind) return MBX_ERR_UNSUPPORTED;  // one geometry kind per batch
        if (scans[s].num_subsets != scans[0].num_subsets) return MBX_ERR_UNSUPPORTED;  // argument table is [scan][K]
        kind = scans[s].geom.kind;
        L.bp_total += zs[s].bp_tiles;
        L.fp_total += zs[s].fp_tiles;
        L.el_total += zs[s].el_tiles;
        L.sn_total += zs[s].sn_tiles;
        L.rc_total += zs[s].rc_tiles;
        ksum += scans[s].num_subsets;
    }
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += align256(bytes); return o; };
    L.scans = take(sizeof(VcdScan) * n);
    L.bpargs = take(sizeof(BpArgs) * ksum);
    L.fpargs = take(sizeof(FpArgs) * ksum);
    L.offs = take(sizeof(int) * 5 * (n + 1));
    L.cblocks = take(sizeof(int) * n);
    L.gx = take(sizeof(int) * n);
    L.scan_of = take(sizeof(int) * 2 * n);
    L.counters = take(sizeof(int) * 2);
    L.sched = take(sizeof(int) * (size_t)num_steps * n);
    L.p_prior = take(sizeof(double) * 2 * (size_t)L.el_total);
    L.p_fwd = take(sizeof(double) * 2 * (size_t)L.sn_total);
    L.p_l1 = take(sizeof(double) * (size_t)L.el_total);
    L.p_iter = take(sizeof(double) * ((size_t)L.sn_total + L.rc_total));
    L.alpha = take(sizeof(float) * n);
    L.buf_off.resize(3 * (size_t)n);
    for (int s = 0; s < n; ++s) {
        L.buf_off[3 * s] = take(4 * (size_t)zs[s].ncyl);
        L.buf_off[3 * s + 1] = take(4 * (size_t)zs[s].ncyl);
        L.buf_off[3 * s + 2] = take(4 * (size_t)zs[s].nsino);
    }
    L.box_off.resize(n);
    for (int s = 0; s < n; ++s)
        L.box_off[s] = take((size_t)scans[s].num_subsets * fp_chunk_box_bytes(scans[s].subset_size));
    L.total = off;
    return MBX_OK;
}

template <typename K>
static int occupancy_grid(K kern, size_t smem, int total) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, BT_THREADS, smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const long long g = (long long)per_sm * num_sms();
    return (int)std::max(1LL, std::min<long long>(g, total));
}

}  // namespace mbx

using namespace mbx;

extern "C" size_t mbx_vcd_batched_workspace_bytes(const mbx_scan *scans, int32_t num_scans, int32_t num_steps) {
    if (!scans || num_scans <= 0 || num_steps <= 0) return 0;
    Layout L;
    std::vector<ScanSizes> zs;
    if (layout(scans, num_scans, num_steps, L, zs) != MBX_OK) return 0;
    return L.total;
}

static int launch_stage(const BatchedPlanHost *P, int step, int stage, cudaStream_t st);

// Autotuning of the forward-projection stage: the plans of every scan with the kernel variant compiled for 2
// resident CTAs per SM (the tables as built) against the same channel blocks with smaller passes and the variant
// compiled for 3.  Each is timed on step 0 (the stage only writes the scans' projection scratch, whose input is
// zeroed first); the faster one's argument table stays on the device, and the choice is remembered for the
// batch shape, so later plans of the same batch do not time again.
static int tune_batched_fp(BatchedPlanHost &P, const Layout &L, const std::vector<ScanSizes> &zs,
                           const mbx_scan *scans, int num_scans, const FpArgs *hf2, cudaStream_t st) {
    int ksum = 0;
    for (int s = 0; s < num_scans; ++s) ksum += scans[s].num_subsets;
    std::vector<FpArgs> f3(hf2, hf2 + ksum);
    size_t smem3 = 0;
    int ki = 0;
    for (int s = 0; s < num_scans; ++s) {
        const CbPlan c3 = plan_fp_cb(scans[s].geom, 0, 0, 3, zs[s].fpp.nb);
        if (!c3.ok || c3.nb != zs[s].fpp.nb || c3.cblocks != zs[s].fpp.cblocks) return MBX_OK;  // same work list only
        smem3 = std::max(smem3, c3.smem);
        for (int k = 0; k < scans[s].num_subsets; ++k, ++ki) f3[ki].plan = c3;
    }
    char *base = reinterpret_cast<char *>(P.t.scans) - L.scans;
    // the choice is cached per batch shape (every scan's sizes, subsets and pixels per subset)
    std::vector<long long> key = {2, P.kind, num_scans};
    for (int s = 0; s < num_scans; ++s) {
        const mbx_geom &g = scans[s].geom;
        key.insert(key.end(), {g.num_views, g.num_det_rows, g.num_det_channels, g.num_recon_rows, g.num_recon_cols,
                               g.num_recon_slices, scans[s].num_subsets, scans[s].subset_size});
    }
    auto use3 = [&]() -> int {
        cudaError_t e3 = cudaMemcpyAsync(base + L.fpargs, f3.data(), sizeof(FpArgs) * ksum, cudaMemcpyHostToDevice, st);
        if (e3 == cudaSuccess) e3 = cudaStreamSynchronize(st);
        if (e3 != cudaSuccess) return set_cuda_error(e3);
        P.fp_minb = 3;
        P.fp_smem = smem3;
        P.fp_grid = (P.kind == MBX_GEOM_PARALLEL) ? occupancy_grid(b_fp<MBX_GEOM_PARALLEL, 3>, smem3, P.fp_total)
                                                  : occupancy_grid(b_fp<MBX_GEOM_CONE, 3>, smem3, P.fp_total);
        return MBX_OK;
    };
    const int cached = autotune_forced() >= 0 ? (autotune_forced() >= 1 ? 3 : 2)
                                              : autotune_lookup(key.data(), (int)key.size());
    if (cached == 2) return MBX_OK;
    if (cached == 3) return use3();
    if (stream_is_capturing(st)) return MBX_OK;
    cudaError_t e = cudaSuccess;
    for (int s = 0; s < num_scans && e == cudaSuccess; ++s)
        e = cudaMemsetAsync(base + L.buf_off[3 * s + 1], 0, 4 * (size_t)zs[s].ncyl, st);
    if (e != cudaSuccess) return set_cuda_error(e);
    int rc = MBX_OK;
    auto run = [&]() {
        rc = launch_stage(&P, 0, 2, st);
        return rc == MBX_OK ? cudaSuccess : cudaErrorLaunchFailure;
    };
    float t2 = 0.0f, t3 = 0.0f;
    e = time_on_stream(run, st, t2);
    if (rc != MBX_OK) return rc;
    if (e != cudaSuccess) return set_cuda_error(e);
    const BatchedPlanHost keep = P;
    rc = use3();
    if (rc != MBX_OK) return rc;
    e = time_on_stream(run, st, t3);
    if (rc != MBX_OK) return rc;
    if (e != cudaSuccess) return set_cuda_error(e);
    autotune_store(key.data(), (int)key.size(), t2 <= t3 ? 2 : 3);
    if (t2 <= t3) {  // back to the tables as built
        P = keep;
        e = cudaMemcpyAsync(base + L.fpargs, hf2, sizeof(FpArgs) * ksum, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return set_cuda_error(e);
    }
    return MBX_OK;
}

// Per-scan lane layout of the forward-projection stage, after the kernel variant is chosen: each scan is timed
// alone on step 0 with its plan and with the best layout that has another number of sub-groups per warp (same
// channel blocks, so the same tiles), and keeps the faster.  Cached per batch shape.
static int tune_batched_fp_layouts(BatchedPlanHost &P, const Layout &L, const mbx_scan *scans, int num_scans,
                                   const int *o_fp, const int *scan_of, cudaStream_t st) {
    const int K = scans[0].num_subsets;  // every scan of a batch has the same number of subsets
    const int ksum = K * num_scans;
    char *base = reinterpret_cast<char *>(P.t.scans) - L.scans;
    std::vector<FpArgs> cur(ksum);
    cudaError_t e = cudaMemcpyAsync(cur.data(), base + L.fpargs, sizeof(FpArgs) * ksum, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_cuda_error(e);
    const std::vector<FpArgs> orig = cur;
    std::vector<FpArgs> alt = cur;
    std::vector<char> can(num_scans, 0);
    size_t smem_alt = 0;
    for (int sc = 0; sc < num_scans; ++sc) {
        const CbPlan &c0 = orig[sc * K].plan;
        const CbPlan q = plan_fp_cb(scans[sc].geom, 0, 0, c0.minb, c0.nb, c0.ppw);
        if (!q.ok || q.nb != c0.nb || q.cblocks != c0.cblocks || q.minb != c0.minb) continue;
        can[sc] = 1;
        for (int j = 0; j < K; ++j) alt[sc * K + j].plan = q;
        smem_alt = std::max(smem_alt, q.smem);
    }
    std::vector<long long> key = {5, P.kind, num_scans, P.fp_minb, -1};
    for (int sc = 0; sc < num_scans; ++sc) {
        const mbx_geom &g = scans[sc].geom;
        key.insert(key.end(), {g.num_views, g.num_det_rows, g.num_det_channels, g.num_recon_rows, g.num_recon_cols,
                               g.num_recon_slices, scans[sc].num_subsets, scans[sc].subset_size});
    }
    auto use = [&](int sc, int c) {
        for (int j = 0; j < K; ++j) cur[sc * K + j] = c ? alt[sc * K + j] : orig[sc * K + j];
    };
    auto upload = [&]() -> cudaError_t {
        cudaError_t e2 = cudaMemcpyAsync(base + L.fpargs, cur.data(), sizeof(FpArgs) * ksum, cudaMemcpyHostToDevice, st);
        return e2 == cudaSuccess ? cudaStreamSynchronize(st) : e2;
    };
    auto apply_smem = [&]() {
        size_t sm = 0;
        for (int k = 0; k < ksum; ++k) sm = std::max(sm, cur[k].plan.smem);
        P.fp_smem = sm;
        if (P.kind == MBX_GEOM_PARALLEL)
            P.fp_grid = P.fp_minb >= 3 ? occupancy_grid(b_fp<MBX_GEOM_PARALLEL, 3>, sm, P.fp_total)
                                       : occupancy_grid(b_fp<MBX_GEOM_PARALLEL, 2>, sm, P.fp_total);
        else
            P.fp_grid = P.fp_minb >= 3 ? occupancy_grid(b_fp<MBX_GEOM_CONE, 3>, sm, P.fp_total)
                                       : occupancy_grid(b_fp<MBX_GEOM_CONE, 2>, sm, P.fp_total);
    };
    bool all_cached = true;
    std::vector<int> choice(num_scans, 0);
    for (int sc = 0; sc < num_scans; ++sc) {
        if (!can[sc]) continue;
        if (autotune_forced() >= 0) {
            choice[sc] = autotune_forced() >= 1 ? 1 : 0;
        } else {
            key[4] = sc;
            const int c = autotune_lookup(key.data(), (int)key.size());
            if (c < 0) all_cached = false;
            choice[sc] = c == 1 ? 1 : 0;
        }
    }
    if (all_cached || autotune_forced() >= 0 || stream_is_capturing(st)) {
        for (int sc = 0; sc < num_scans; ++sc) use(sc, choice[sc]);
        e = upload();
        if (e != cudaSuccess) return set_cuda_error(e);
        apply_smem();
        return MBX_OK;
    }
    P.fp_smem = std::max(P.fp_smem, smem_alt);  // tuning launches fit either plan
    int *err = device_error_ptr();
    for (int k = 0; k < num_scans; ++k) {
        const int sc = scan_of[num_scans + k];
        if (!can[sc]) continue;
        const int first = o_fp[k], last = o_fp[k + 1];
        const int grid = std::min(P.fp_grid, last - first);
        auto run = [&]() -> cudaError_t {
            cudaError_t e2 = cudaMemsetAsync(P.t.counters + 1, 0, sizeof(int), st);
            if (e2 != cudaSuccess) return e2;
            if (P.kind == MBX_GEOM_PARALLEL) {
                if (P.fp_minb >= 3)
                    b_fp<MBX_GEOM_PARALLEL, 3><<<grid, CB_THREADS, P.fp_smem, st>>>(P.t, num_scans, 0, first, last, err);
                else
                    b_fp<MBX_GEOM_PARALLEL, 2><<<grid, CB_THREADS, P.fp_smem, st>>>(P.t, num_scans, 0, first, last, err);
            } else {
                if (P.fp_minb >= 3)
                    b_fp<MBX_GEOM_CONE, 3><<<grid, CB_THREADS, P.fp_smem, st>>>(P.t, num_scans, 0, first, last, err);
                else
                    b_fp<MBX_GEOM_CONE, 2><<<grid, CB_THREADS, P.fp_smem, st>>>(P.t, num_scans, 0, first, last, err);
            }
            note_launch();
            return cudaGetLastError();
        };
        float t[2] = {0.0f, 0.0f};
        for (int c = 0; c < 2; ++c) {
            use(sc, c);
            e = upload();
            if (e == cudaSuccess) e = time_on_stream(run, st, t[c]);
            if (e != cudaSuccess) return set_cuda_error(e);
        }
        choice[sc] = t[1] < t[0] ? 1 : 0;
        use(sc, choice[sc]);
        key[4] = sc;
        autotune_store(key.data(), (int)key.size(), choice[sc]);
    }
    e = upload();
    if (e != cudaSuccess) return set_cuda_error(e);
    apply_smem();
    return MBX_OK;
}

// Autotuning of the back-projection stage, per scan: staged (shared-memory) footprints, the tables as built,
// against per-thread footprints computed in registers (same tiles).  Each scan is timed alone on step 0 (the
// launch walks only that scan's tiles; the stage only writes the scans' back-projection scratch), so that every
// scan keeps the plan that suits its shape, as the plain path's per-call tuner would choose.  The choices are
// cached per batch shape.
static int tune_batched_bp(BatchedPlanHost &P, const Layout &L, const mbx_scan *scans, int num_scans,
                           const BpArgs *hb1, const int *o_bp, const int *scan_of, cudaStream_t st) {
    const int K = scans[0].num_subsets;  // every scan of a batch has the same number of subsets
    const int ksum = K * num_scans;
    std::vector<BpArgs> cur(hb1, hb1 + ksum), alt(hb1, hb1 + ksum);
    std::vector<char> can(num_scans, 1);
    size_t smem_alt = 0;
    for (int k = 0; k < ksum; ++k) {
        const BpfPlan q = plan_bp_fast(alt[k].g, alt[k].num_pixels, alt[k].g.num_views, 1);
        if (!q.ok || q.gx != alt[k].plan.gx || q.gy != alt[k].plan.gy || q.splits != 1) {
            can[k / K] = 0;
            continue;
        }
        alt[k].plan = q;
        smem_alt = std::max(smem_alt, q.smem);
    }
    char *base = reinterpret_cast<char *>(P.t.scans) - L.scans;
    std::vector<long long> key = {4, P.kind, num_scans, -1};
    for (int s = 0; s < num_scans; ++s) {
        const mbx_geom &g = scans[s].geom;
        key.insert(key.end(), {g.num_views, g.num_det_rows, g.num_det_channels, g.num_recon_rows, g.num_recon_cols,
                               g.num_recon_slices, scans[s].num_subsets, scans[s].subset_size,
                               scans[s].weights ? 1 : 0});
    }
    auto upload = [&]() -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(base + L.bpargs, cur.data(), sizeof(BpArgs) * ksum, cudaMemcpyHostToDevice, st);
        return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
    };
    auto apply_smem = [&]() {
        size_t sm = 0;
        for (int k = 0; k < ksum; ++k) sm = std::max(sm, cur[k].plan.smem);
        P.bp_smem = sm;
        P.bp_grid = (P.kind == MBX_GEOM_PARALLEL) ? occupancy_grid(b_bp<MBX_GEOM_PARALLEL>, sm, P.bp_total)
                                                  : occupancy_grid(b_bp<MBX_GEOM_CONE>, sm, P.bp_total);
    };
    auto use = [&](int s, int c) {
        for (int j = 0; j < K; ++j) cur[s * K + j] = c ? alt[s * K + j] : hb1[s * K + j];
    };
    bool all_cached = true;
    std::vector<int> choice(num_scans, 0);
    for (int s = 0; s < num_scans; ++s) {
        if (!can[s]) continue;
        if (autotune_forced() >= 0) {
            choice[s] = autotune_forced() >= 1 ? 1 : 0;
        } else {
            key[3] = s;
            const int c = autotune_lookup(key.data(), (int)key.size());
            if (c < 0) all_cached = false;
            choice[s] = c == 1 ? 1 : 0;
        }
    }
    if (all_cached || autotune_forced() >= 0 || stream_is_capturing(st)) {
        for (int s = 0; s < num_scans; ++s) use(s, can[s] ? choice[s] : 0);
        cudaError_t e = upload();
        if (e != cudaSuccess) return set_cuda_error(e);
        apply_smem();
        return MBX_OK;
    }
    P.bp_smem = std::max(P.bp_smem, smem_alt);  // tuning launches fit either plan
    int *err = device_error_ptr();
    for (int k = 0; k < num_scans; ++k) {
        const int s = scan_of[k];
        if (!can[s]) continue;
        const int first = o_bp[k], last = o_bp[k + 1];
        const int grid = std::min(P.bp_grid, last - first);
        auto run = [&]() -> cudaError_t {
            cudaError_t e = cudaMemsetAsync(P.t.counters, 0, sizeof(int), st);
            if (e != cudaSuccess) return e;
            if (P.kind == MBX_GEOM_PARALLEL)
                b_bp<MBX_GEOM_PARALLEL><<<grid, BPF_THREADS, P.bp_smem, st>>>(P.t, num_scans, 0, first, last, err);
            else
                b_bp<MBX_GEOM_CONE><<<grid, BPF_THREADS, P.bp_smem, st>>>(P.t, num_scans, 0, first, last, err);
            note_launch();
            return cudaGetLastError();
        };
        float t[2] = {0.0f, 0.0f};
        for (int c = 0; c < 2; ++c) {
            use(s, c);
            cudaError_t e = upload();
            if (e == cudaSuccess) e = time_on_stream(run, st, t[c]);
            if (e != cudaSuccess) return set_cuda_error(e);
        }
        choice[s] = t[1] < t[0] ? 1 : 0;
        use(s, choice[s]);
        key[3] = s;
        autotune_store(key.data(), (int)key.size(), choice[s]);
    }
    cudaError_t e = upload();
    if (e != cudaSuccess) return set_cuda_error(e);
    apply_smem();
    return MBX_OK;
}

extern "C" int mbx_vcd_batched_prepare(const mbx_scan *scans, int32_t num_scans, const int32_t *schedule,
                                       int32_t num_steps, int32_t num_iterations, double *step_stats,
                                       double *iter_stats, void *workspace, size_t workspace_bytes,
                                       mbx_batched_plan *plan_out, void *stream) {
    if (!scans || num_scans <= 0 || !schedule || num_steps <= 0 || num_iterations < 0 || !plan_out || !step_stats ||
        (num_iterations > 0 && !iter_stats))
        return MBX_ERR_INVALID_ARG;
    Layout L;
    std::vector<ScanSizes> zs;
    int rc = layout(scans, num_scans, num_steps, L, zs);
    if (rc != MBX_OK) return rc;
    if (!workspace || workspace_bytes < L.total) return MBX_ERR_WORKSPACE;
    for (int st = 0; st < num_steps; ++st)
        for (int s = 0; s < num_scans; ++s) {
            const int v = schedule[(size_t)st * num_scans + s];
            if (v < 0 || v >= scans[s].num_subsets) return MBX_ERR_INVALID_ARG;
        }
    char *base = static_cast<char *>(workspace);
    std::vector<char> host(L.sched + sizeof(int) * (size_t)num_steps * num_scans, 0);
    int *hscan_of = reinterpret_cast<int *>(host.data() + L.scan_of);
    VcdScan *hs = reinterpret_cast<VcdScan *>(host.data() + L.scans);
    BpArgs *hb = reinterpret_cast<BpArgs *>(host.data() + L.bpargs);
    FpArgs *hf = reinterpret_cast<FpArgs *>(host.data() + L.fpargs);
    int *hoff = reinterpret_cast<int *>(host.data() + L.offs);
    int *hcb = reinterpret_cast<int *>(host.data() + L.cblocks);
    int *hgx = reinterpret_cast<int *>(host.data() + L.gx);
    int *hsched = reinterpret_cast<int *>(host.data() + L.sched);
    const int n1 = num_scans + 1;
    int *o_bp = hoff, *o_fp = hoff + n1, *o_el = hoff + 2 * n1, *o_sn = hoff + 3 * n1, *o_rc = hoff + 4 * n1;
    o_bp[0] = o_fp[0] = o_el[0] = o_sn[0] = o_rc[0] = 0;
    size_t smem_bp = 0, smem_fp = 0;
    int ki = 0;
    for (int s = 0; s < num_scans; ++s) {
        const mbx_scan &sc = scans[s];
        const ScanSizes &z = zs[s];
        VcdScan &v = hs[s];
        v.recon = sc.flat_recon;
        v.err = sc.error_sinogram;
        v.wts = sc.weights;
        v.hess = sc.fm_hessian;
        v.partition = sc.partition;
        v.bp = reinterpret_cast<float *>(base + L.buf_off[3 * s]);
        v.delta = reinterpret_cast<float *>(base + L.buf_off[3 * s + 1]);
        v.dsino = reinterpret_cast<float *>(base + L.buf_off[3 * s + 2]);
        v.nsino = z.nsino;
        v.nrecon = z.nrecon;
        v.K = sc.num_subsets;
        v.M = sc.subset_size;
        v.nr = sc.geom.num_recon_rows;
        v.nc = sc.geom.num_recon_cols;
        v.ns = sc.geom.num_recon_slices;
        v.fm_constant = sc.fm_constant;
        v.q = make_qparams(sc.qp);
        for (int k = 0; k < sc.num_subsets; ++k, ++ki) {
            BpArgs &a = hb[ki];
            a.g = sc.geom;
            a.sino = sc.error_sinogram;
            a.wts = sc.weights;
            a.pix = sc.partition + (size_t)k * sc.subset_size;
            a.num_pixels = sc.subset_size;
            a.order = sc.partition_order ? sc.partition_order + (size_t)k * sc.subset_size : nullptr;
            a.views = nullptr;
            a.num_views_sel = sc.geom.num_views;
            a.views_per_split = sc.geom.num_views;
            a.coeff_power = 1;
            a.scale = 1.0f;
            a.out = v.bp;
            a.split_stride = 0;
            a.out_by_index = 0;
            a.plan = z.bpp;
            FpArgs &f = hf[ki];
            f.g = sc.geom;
            f.vox = v.delta;
            f.pix = a.pix;
            f.num_pixels = sc.subset_size;
            f.views = nullptr;
            f.num_views_sel = sc.geom.num_views;
            f.out = v.dsino;
            f.vox_by_index = 0;
            f.plan = z.fpp;
            f.chunk_box = reinterpret_cast<const int4 *>(base + L.box_off[s] + (size_t)k * fp_chunk_box_bytes(sc.subset_size));
        }
        // bp_fast smem without view splits
        smem_bp = std::max(smem_bp, z.bpp.smem);
        smem_fp = std::max(smem_fp, z.fpp.smem);
        hcb[s] = z.fpp.cblocks;
        hgx[s] = z.bp_gx;
        o_el[s + 1] = o_el[s] + z.el_tiles;
        o_sn[s + 1] = o_sn[s] + z.sn_tiles;
        o_rc[s + 1] = o_rc[s] + z.rc_tiles;
    }
    // bp / fp work lists: scans in decreasing order of per-tile cost, so that the dynamically scheduled tail of
    // a launch is made of the cheapest tiles
    {
        std::vector<int> ord(num_scans);
        std::vector<double> cost(num_scans);
        for (int s = 0; s < num_scans; ++s) {
            const mbx_geom &g = scans[s].geom;
            cost[s] = (double)g.num_views * std::min(g.num_recon_slices, zs[s].bpp.ts * zs[s].bpp.nsl) * 32.0 * zs[s].bpp.npg;
            ord[s] = s;
        }
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
        for (int k = 0; k < num_scans; ++k) {
            hscan_of[k] = ord[k];
            o_bp[k + 1] = o_bp[k] + zs[ord[k]].bp_tiles;
        }
        for (int s = 0; s < num_scans; ++s) {
            const mbx_geom &g = scans[s].geom;
            cost[s] = (double)scans[s].subset_size *
                      (2.0 + (double)(zs[s].fpp.nb + 2) * zs[s].fpp.rpad / g.num_det_channels);
            ord[s] = s;
        }
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
        for (int k = 0; k < num_scans; ++k) {
            hscan_of[num_scans + k] = ord[k];
            o_fp[k + 1] = o_fp[k] + zs[ord[k]].fp_tiles;
        }
    }
    std::memcpy(hsched, schedule, sizeof(int) * (size_t)num_steps * num_scans);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(base, host.data(), host.size(), cudaMemcpyHostToDevice, st);
    // chunk bounding boxes of every subset (the forward projection skips chunks that miss its channel block)
    for (int s = 0; s < num_scans && e == cudaSuccess; ++s) {
        const mbx_scan &sc = scans[s];
        const unsigned nch = (unsigned)((sc.subset_size + CB_CHUNK - 1) / CB_CHUNK);
        for (int k = 0; k < sc.num_subsets && e == cudaSuccess; ++k) {
            int4 *box = reinterpret_cast<int4 *>(base + L.box_off[s] + (size_t)k * fp_chunk_box_bytes(sc.subset_size));
            fp_chunk_bounds_kernel<<<nch, CB_CHUNK, 0, st>>>(sc.partition + (size_t)k * sc.subset_size, sc.subset_size,
                                                             sc.geom.num_recon_rows, sc.geom.num_recon_cols, box);
            note_launch();
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_cuda_error(e);

    BatchedPlanHost P;
    std::memset(&P, 0, sizeof(P));
    P.t.scans = reinterpret_cast<VcdScan *>(base + L.scans);
    P.t.bpargs = reinterpret_cast<BpArgs *>(base + L.bpargs);
    P.t.fpargs = reinterpret_cast<FpArgs *>(base + L.fpargs);
    int *doff = reinterpret_cast<int *>(base + L.offs);
    P.t.bp_off = doff;
    P.t.fp_off = doff + n1;
    P.t.el_off = doff + 2 * n1;
    P.t.sn_off = doff + 3 * n1;
    P.t.rc_off = doff + 4 * n1;
    P.t.fp_cblocks = reinterpret_cast<int *>(base + L.cblocks);
    P.t.bp_gx = reinterpret_cast<int *>(base + L.gx);
    P.t.bp_scan = reinterpret_cast<int *>(base + L.scan_of);
    P.t.fp_scan = P.t.bp_scan + num_scans;
    P.t.counters = reinterpret_cast<int *>(base + L.counters);
    P.t.schedule = reinterpret_cast<int *>(base + L.sched);
    P.t.p_prior = reinterpret_cast<double *>(base + L.p_prior);
    P.t.p_fwd = reinterpret_cast<double *>(base + L.p_fwd);
    P.t.p_l1 = reinterpret_cast<double *>(base + L.p_l1);
    P.t.p_iter = reinterpret_cast<double *>(base + L.p_iter);
    P.t.alpha = reinterpret_cast<float *>(base + L.alpha);
    P.t.step_stats = step_stats;
    P.t.iter_stats = iter_stats;
    P.num_scans = num_scans;
    P.kind = scans[0].geom.kind;
    P.num_steps = num_steps;
    P.num_iterations = num_iterations;
    P.bp_total = L.bp_total;
    P.fp_total = L.fp_total;
    P.el_total = L.el_total;
    P.sn_total = L.sn_total;
    P.rc_total = L.rc_total;
    P.bp_smem = smem_bp;
    P.fp_smem = smem_fp;
    P.fp_minb = 2;
    // kernel attributes and resident-CTA grids
    if (P.kind == MBX_GEOM_PARALLEL) {
        set_max_dynamic_smem(reinterpret_cast<const void *>(b_bp<MBX_GEOM_PARALLEL>), 100 * 1024);
        set_max_dynamic_smem(reinterpret_cast<const void *>(b_fp<MBX_GEOM_PARALLEL, 2>), 200 * 1024);
        set_max_dynamic_smem(reinterpret_cast<const void *>(b_fp<MBX_GEOM_PARALLEL, 3>), 200 * 1024);
        P.bp_grid = occupancy_grid(b_bp<MBX_GEOM_PARALLEL>, smem_bp, L.bp_total);
        P.fp_grid = occupancy_grid(b_fp<MBX_GEOM_PARALLEL, 2>, smem_fp, L.fp_total);
    } else {
        set_max_dynamic_smem(reinterpret_cast<const void *>(b_bp<MBX_GEOM_CONE>), 100 * 1024);
        set_max_dynamic_smem(reinterpret_cast<const void *>(b_fp<MBX_GEOM_CONE, 2>), 200 * 1024);
        set_max_dynamic_smem(reinterpret_cast<const void *>(b_fp<MBX_GEOM_CONE, 3>), 200 * 1024);
        P.bp_grid = occupancy_grid(b_bp<MBX_GEOM_CONE>, smem_bp, L.bp_total);
        P.fp_grid = occupancy_grid(b_fp<MBX_GEOM_CONE, 2>, smem_fp, L.fp_total);
    }
    {   // load every stage kernel now (lazy module loading must not happen inside a stream capture)
        cudaFuncAttributes fa;
        cudaFuncGetAttributes(&fa, b_delta);
        cudaFuncGetAttributes(&fa, b_linquad);
        cudaFuncGetAttributes(&fa, b_alpha);
        cudaFuncGetAttributes(&fa, b_apply);
        cudaFuncGetAttributes(&fa, b_error);
        cudaFuncGetAttributes(&fa, b_l1);
        cudaFuncGetAttributes(&fa, b_iter_partials);
        cudaFuncGetAttributes(&fa, b_iter_final);
        device_error_ptr();
    }
    P.el_grid = occupancy_grid(b_delta, 0, L.el_total);
    P.sn_grid = occupancy_grid(b_linquad, 0, L.sn_total);
    P.rc_grid = occupancy_grid(b_iter_partials, 0, L.sn_total + L.rc_total);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error(e);
    if (autotune_enabled()) {  // (also in forced mode: the tune functions then apply the forced choice)
        int rc2 = tune_batched_fp(P, L, zs, scans, num_scans, hf, st);
        if (rc2 == MBX_OK) rc2 = tune_batched_fp_layouts(P, L, scans, num_scans, o_fp, hscan_of, st);
        if (rc2 == MBX_OK) rc2 = tune_batched_bp(P, L, scans, num_scans, hb, o_bp, hscan_of, st);
        if (rc2 != MBX_OK) return rc2;
    }
    P.magic = BT_MAGIC;
    std::memset(plan_out, 0, sizeof(*plan_out));
    std::memcpy(plan_out, &P, sizeof(P));
    return MBX_OK;
}

static const BatchedPlanHost *plan_of(const mbx_batched_plan *p) {
    if (!p) return nullptr;
    const BatchedPlanHost *P = reinterpret_cast<const BatchedPlanHost *>(p);
    return P->magic == BT_MAGIC ? P : nullptr;
}

static int launch_stage(const BatchedPlanHost *P, int step, int stage, cudaStream_t st) {
    int *err = device_error_ptr();
    const BatchedTables &T = P->t;
    const int n = P->num_scans;
    const int warp_blocks = (n + 7) / 8;
    switch (stage) {
        case 0:
            {
                const cudaError_t me = cudaMemsetAsync(T.counters, 0, sizeof(int), st);
                if (me != cudaSuccess) return set_cuda_error(me);
            }
            if (P->kind == MBX_GEOM_PARALLEL)
                b_bp<MBX_GEOM_PARALLEL><<<P->bp_grid, BPF_THREADS, P->bp_smem, st>>>(T, n, step, 0, P->bp_total, err);
            else
                b_bp<MBX_GEOM_CONE><<<P->bp_grid, BPF_THREADS, P->bp_smem, st>>>(T, n, step, 0, P->bp_total, err);
            break;
        case 1: b_delta<<<P->el_grid, BT_THREADS, 0, st>>>(T, n, step, P->el_total, err); break;
        case 2:
            {
                const cudaError_t me = cudaMemsetAsync(T.counters + 1, 0, sizeof(int), st);
                if (me != cudaSuccess) return set_cuda_error(me);
            }
            if (P->kind == MBX_GEOM_PARALLEL) {
                if (P->fp_minb >= 3)
                    b_fp<MBX_GEOM_PARALLEL, 3><<<P->fp_grid, CB_THREADS, P->fp_smem, st>>>(T, n, step, 0, P->fp_total, err);
                else
                    b_fp<MBX_GEOM_PARALLEL, 2><<<P->fp_grid, CB_THREADS, P->fp_smem, st>>>(T, n, step, 0, P->fp_total, err);
            } else {
                if (P->fp_minb >= 3)
                    b_fp<MBX_GEOM_CONE, 3><<<P->fp_grid, CB_THREADS, P->fp_smem, st>>>(T, n, step, 0, P->fp_total, err);
                else
                    b_fp<MBX_GEOM_CONE, 2><<<P->fp_grid, CB_THREADS, P->fp_smem, st>>>(T, n, step, 0, P->fp_total, err);
            }
            break;
        case 3: b_linquad<<<P->sn_grid, BT_THREADS, 0, st>>>(T, n, P->sn_total); break;
        case 4: b_alpha<<<warp_blocks, 256, 0, st>>>(T, n, step); break;
        case 5: b_apply<<<P->el_grid, BT_THREADS, 0, st>>>(T, n, step, P->el_total); break;
        case 6: b_error<<<P->sn_grid, BT_THREADS, 0, st>>>(T, n, P->sn_total); break;
        case 7: b_l1<<<warp_blocks, 256, 0, st>>>(T, n, step); break;
        default: return MBX_ERR_INVALID_ARG;
    }
    note_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
}

extern "C" int mbx_vcd_batched_step(const mbx_batched_plan *plan, int32_t step, void *stream) {
    const BatchedPlanHost *P = plan_of(plan);
    if (!P || step < 0 || step >= P->num_steps) return MBX_ERR_INVALID_ARG;
    for (int stage = 0; stage < MBX_BATCHED_STAGES; ++stage) {
        const int rc = launch_stage(P, step, stage, static_cast<cudaStream_t>(stream));
        if (rc != MBX_OK) return rc;
    }
    return MBX_OK;
}

extern "C" int mbx_vcd_batched_stage(const mbx_batched_plan *plan, int32_t step, int32_t stage, void *stream) {
    const BatchedPlanHost *P = plan_of(plan);
    if (!P || step < 0 || step >= P->num_steps || stage < 0 || stage >= MBX_BATCHED_STAGES) return MBX_ERR_INVALID_ARG;
    return launch_stage(P, step, stage, static_cast<cudaStream_t>(stream));
}

extern "C" int mbx_vcd_batched_iteration_stats(const mbx_batched_plan *plan, int32_t iteration, void *stream) {
    const BatchedPlanHost *P = plan_of(plan);
    if (!P || iteration < 0 || iteration >= P->num_iterations) return MBX_ERR_INVALID_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n = P->num_scans;
    b_iter_partials<<<P->rc_grid, BT_THREADS, 0, st>>>(P->t, n, P->sn_total, P->rc_total);
    note_launch();
    b_iter_final<<<(n + 7) / 8, 256, 0, st>>>(P->t, n, iteration, P->sn_total);
    note_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
}
