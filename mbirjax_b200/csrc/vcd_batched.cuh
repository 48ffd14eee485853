// Batched VCD: the types and device helpers shared by the batched stages (vcd_batched.cu) and the forward-
// projection stage kernels, which are compiled per geometry kind in their own translation units
// (b_fp_parallel.cu, b_fp_cone.cu, b_fp_translation.cu) for build parallelism.
#pragma once

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
    float *hess;                // flat (Nr*Nc, S)
    const int32_t *partition;   // (K, M)
    float *bp, *delta, *dsino;  // workspace slices
    const float *y;             // measured sinogram (set-up input) or NULL
    long long nsino, nrecon;
    int K, M, nr, nc, ns;
};

// Direct-recon filtering of one scan in the set-up: rows of y into err.
struct FiltScan {
    const float *in;
    float *out;
    long long rows;
    int R, C, fdk;
    double filter_scale, out_scale, D, ddc, ddr, dco, dro;
};

// A work list of projection tiles over the scans of a batch: per scan, its argument record(s) and tile count.
// Tiles are numbered over the scans in `order` (decreasing per-tile cost) and handed out dynamically.
struct ProjList {
    const BpArgs *bp;      // back-projection records (or NULL)
    const FpArgs *fp;      // forward-projection records (or NULL)
    const int *off;        // [num_scans + 1] tile prefix over the positions of `order`
    const int *dim;        // [num_scans] per scan: gx (back projection) or channel blocks (forward)
    const int *order;      // [num_scans] scan at each position
    const int *schedule;   // [num_steps][num_scans] record of each scan at each step, or NULL (record 0)
    int stride;            // records per scan
    int *counter;          // next tile (reset by a memset before each launch)
    const CbPlanned *planned;  // forward lists: stored record passes of each record, or NULL (walk every tile)
};

// Projection work lists of a batch.  PL_BUILD covers every (scan, subset, view, channel block) tile: the builds
// of the planned forward projections.
enum { PL_BP = 0, PL_FP, PL_INIT_BP, PL_INIT_FP, PL_HESS, PL_BUILD, PL_COUNT };

struct BatchedTables {
    VcdScan *scans;
    float *fm;          // [scan] 1 / sigma_y^2 (per call)
    QParams *qp;        // [scan] qGGMRF parameters (per call)
    BpArgs *bpargs;     // [scan][subset]
    FpArgs *fpargs;     // [scan][subset]
    BpArgs *init_bp;    // [scan]: filtered sinogram -> recon over the region of reconstruction
    FpArgs *init_fp;    // [scan]: recon -> dsino over the region of reconstruction
    BpArgs *hess_bp;    // [scan]: weights (or ones) -> Hessian over every pixel, squared coefficients
    FiltScan *filt;     // [scan]
    CbPlanned *planned; // [scan][subset] stored record passes of the subset forward projections (planned batches)
    int *pl_off;        // [PL_COUNT][num_scans + 1]
    int *pl_dim;        // [PL_COUNT][num_scans]
    int *pl_order;      // [PL_COUNT][num_scans]
    int *el_off, *sn_off, *rc_off, *flt_off;  // [num_scans + 1] tile prefix offsets (scan order)
    int *box_first;     // [num_scans * K + 1] chunk prefix over (scan, subset) records
    int *counters;      // [PL_COUNT]
    int *schedule;      // [num_steps][num_scans]
    double *p_prior, *p_fwd, *p_l1, *p_iter, *p_init;
    float *alpha;       // [num_scans]
    float *alpha_init;  // [num_scans]
    double *step_stats; // [num_steps][num_scans][4]
    double *iter_stats; // [num_iterations][num_scans][4]
};

struct BatchedPlanHost {
    BatchedTables t;
    int num_scans, kind, num_steps, num_iterations, ksum, has_setup;
    int planned_fp;                 // subset forward projections replay stored record passes
    int pl_grid_replay, pl_grid_build;  // grids of the replay and build kernels (variant fp_minb)
    void *plan_cursors;             // [ksum] bump cursors of the planned lists (one memset resets them)
    size_t plan_cursor_bytes;
    int pl_total[PL_COUNT], pl_grid[PL_COUNT];
    size_t pl_smem[PL_COUNT];
    int el_total, sn_total, rc_total, flt_total, box_total;
    int el_grid, sn_grid, rc_grid, flt_grid, box_grid;
    size_t flt_smem;
    int fp_minb;  // b_fp variant of the subset stage: 2 or 3 resident CTAs per SM
    size_t fp_smem_replay;  // shared memory of the replay kernel (the replay layouts of the subset plans)
    int magic;
};
static_assert(sizeof(BatchedPlanHost) <= sizeof(mbx_batched_plan), "plan record too large");
constexpr int BT_MAGIC = 0x6d627863;

inline ProjList proj_list(const BatchedTables &T, int which, int num_scans) {
    ProjList L;
    L.bp = which == PL_BP ? T.bpargs : which == PL_INIT_BP ? T.init_bp : which == PL_HESS ? T.hess_bp : nullptr;
    L.fp = which == PL_FP ? T.fpargs : which == PL_INIT_FP ? T.init_fp : nullptr;
    L.off = T.pl_off + which * (num_scans + 1);
    L.dim = T.pl_dim + which * num_scans;
    L.order = T.pl_order + which * num_scans;
    const bool subsets = which == PL_BP || which == PL_FP;
    L.schedule = subsets ? T.schedule : nullptr;
    L.stride = 0;  // set by the caller (the number of subsets for the subset lists)
    L.counter = T.counters + which;
    L.planned = nullptr;
    return L;
}

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

#ifndef MBX_BATCHED_FP_CAP
#define MBX_BATCHED_FP_CAP 2048  // most records per pass of the batched forward projections (and their stored passes)
#endif

#ifndef MBX_BBP_MIN_BLOCKS
#define MBX_BBP_MIN_BLOCKS 3  // resident CTAs per SM the batched back projection is compiled for
#endif

// Record of scan s in a work list at a step.
template <class A>
__device__ __forceinline__ const A &list_record(const A *recs, const ProjList &L, int num_scans, int step, int s) {
    const int r = L.schedule ? __ldg(L.schedule + step * num_scans + s) : 0;
    return recs[s * L.stride + r];
}

// The forward-projection stage kernels of one geometry kind: b_fp (walk), b_fp_replay (stored passes) and
// b_fp_build (store the passes), each compiled for 2 or 3 resident CTAs per SM (minb).  fp_stage_kernel returns
// the kernel of (minb, mode) for occupancy queries and attributes; launch_fp_stage launches it over a work list.
const void *fp_stage_kernel(int kind, int minb, int mode);
void launch_fp_stage(int kind, int minb, int mode, int grid, size_t smem, cudaStream_t st, const ProjList &L, int n,
                     int step, int first, int total, int *err);

}  // namespace mbx
