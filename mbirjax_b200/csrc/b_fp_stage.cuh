// Batched forward-projection stage kernels, as templates over the geometry kind; each per-kind translation unit
// (b_fp_parallel.cu, b_fp_cone.cu, b_fp_translation.cu) instantiates them for its kind.
#pragma once

#include "vcd_batched.cuh"

namespace mbx {

// MINB: resident CTAs per SM the variant is compiled for (2 or 3, matching the plans' fp_cb minb).
template <int KIND, int MINB>
__global__ void __launch_bounds__(CB_THREADS, MINB) b_fp(ProjList L, int num_scans, int step, int first, int total, int *err) {
    extern __shared__ __align__(16) float smf2[];
    for (int t = first + fetch_tile(L.counter); t < total; t = first + fetch_tile(L.counter)) {
        const int k = find_scan(L.off, num_scans, t);
        const int s = __ldg(L.order + k);
        const int local = t - __ldg(L.off + k);
        const int cbs = __ldg(L.dim + s);
        fp_cb_tile<KIND, MINB>(list_record(L.fp, L, num_scans, step, s), local / cbs, local % cbs, smf2, err);
    }
}

// Subset forward projection from stored record passes: the tile's passes are walked as stored (no scan, no
// sort); a tile the build could not store is projected by the walk in the replay layout's shared memory (plan.small).
template <int KIND, int MINB>
__global__ void __launch_bounds__(CB_THREADS, MINB) b_fp_replay(ProjList L, int num_scans, int step, int first, int total, int *err) {
    extern __shared__ __align__(16) float smf3[];
    for (int t = first + fetch_tile(L.counter); t < total; t = first + fetch_tile(L.counter)) {
        const int k = find_scan(L.off, num_scans, t);
        const int s = __ldg(L.order + k);
        const int local = t - __ldg(L.off + k);
        const int cbs = __ldg(L.dim + s);
        const int r = L.schedule ? __ldg(L.schedule + step * num_scans + s) : 0;
        const FpArgs &A = L.fp[s * L.stride + r];
        const CbPlanned &pc = L.planned[s * L.stride + r];
        const int view = local / cbs, cb = local % cbs;
        const long long ptile = local;  // view * cbs + cb
        if (pc.tile_npass[ptile] >= 0)
            fp_cb_tile<KIND, MINB, CB_REPLAY>(A, view, cb, smf3, err, &pc, ptile);
        else
            fp_cb_tile<KIND, MINB, CB_WALK_SMALL>(A, view, cb, smf3, err);
    }
}

// Builds of the planned forward projections: every (scan, subset, view, channel block) tile scans and sorts its
// pixels and stores the sorted passes.
template <int KIND, int MINB>
__global__ void __launch_bounds__(CB_THREADS, MINB) b_fp_build(ProjList L, int num_scans, int first, int total, int *err) {
    extern __shared__ __align__(16) float smf4[];
    for (int t = first + fetch_tile(L.counter); t < total; t = first + fetch_tile(L.counter)) {
        const int k = find_scan(L.off, num_scans, t);
        const int s = __ldg(L.order + k);
        const int local = t - __ldg(L.off + k);
        const int cbs = __ldg(L.dim + s);
        const int per_subset = L.fp[s * L.stride].num_views_sel * cbs;
        const int sub = local / per_subset, r = local - sub * per_subset;
        fp_cb_tile<KIND, MINB, CB_BUILD>(L.fp[s * L.stride + sub], r / cbs, r % cbs, smf4, err,
                                         L.planned + s * L.stride + sub, r);
    }
}


// Kernel of (minb, mode) for geometry kind KIND.
template <int KIND>
const void *fp_stage_kernel_kind(int minb, int mode) {
    if (mode == CB_REPLAY)
        return minb >= 3 ? reinterpret_cast<const void *>(b_fp_replay<KIND, 3>)
                         : reinterpret_cast<const void *>(b_fp_replay<KIND, 2>);
    if (mode == CB_BUILD)
        return minb >= 3 ? reinterpret_cast<const void *>(b_fp_build<KIND, 3>)
                         : reinterpret_cast<const void *>(b_fp_build<KIND, 2>);
    return minb >= 3 ? reinterpret_cast<const void *>(b_fp<KIND, 3>) : reinterpret_cast<const void *>(b_fp<KIND, 2>);
}

template <int KIND, int MINB>
void launch_fp_stage_minb(int mode, int grid, size_t smem, cudaStream_t st, const ProjList &L, int n, int step,
                          int first, int total, int *err) {
    if (mode == CB_REPLAY)
        b_fp_replay<KIND, MINB><<<grid, CB_THREADS, smem, st>>>(L, n, step, first, total, err);
    else if (mode == CB_BUILD)
        b_fp_build<KIND, MINB><<<grid, CB_THREADS, smem, st>>>(L, n, first, total, err);
    else
        b_fp<KIND, MINB><<<grid, CB_THREADS, smem, st>>>(L, n, step, first, total, err);
}

// One launch of a forward-projection work list with the kernel of (minb, mode) for geometry kind KIND.
template <int KIND>
void launch_fp_stage_kind(int minb, int mode, int grid, size_t smem, cudaStream_t st, const ProjList &L, int n,
                          int step, int first, int total, int *err) {
    if (minb >= 3)
        launch_fp_stage_minb<KIND, 3>(mode, grid, smem, st, L, n, step, first, total, err);
    else
        launch_fp_stage_minb<KIND, 2>(mode, grid, smem, st, L, n, step, first, total, err);
}

}  // namespace mbx
