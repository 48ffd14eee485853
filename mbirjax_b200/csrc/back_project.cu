// Sparse back projector for parallel-beam, cone-beam and translation geometry (sm_100a).
//
// Replaces Projectors.sparse_back_project (projectors.py:131-209) over the geometry plugins
// ParallelBeamModel.back_project_one_view_to_pixel_batch (parallel_beam.py:180-221),
// ConeBeamModel.back_project_one_view_to_pixel_batch (cone_beam.py:379-541) and
// TranslationModel.back_project_one_view_to_pixel_batch (translation_model.py:382-542); coeff_power = 2 gives
// the Hessian diagonal of TomographyModel.compute_hessian_diagonal (tomography_model.py:679-708).  Radius-1
// geometries run bp_fast.cuh when its plan fits (translation geometry when the caller gives a magnification
// bound); the other cases run the general kernel of back_project.cuh, described here.
//
// One thread owns one pixel and a tile of ST slices.  Its ST accumulators stay in registers across all
// views, so there are no global atomics and no per-view partial cylinders.  Lanes run along pixels, so the
// channel gathers of a warp fall in a narrow channel range of one detector row.  Per-view angle, cos and
// sin are staged in shared memory.  For cone beam each thread first gathers, for every detector row its
// slice tile touches in this view, the horizontal fan sum sum_k A_chan_k * sino[m, n_c + k] into its own
// column of a shared-memory buffer (row-major across threads, so conflict-free), then applies the
// voxel-centric vertical fan from that buffer; each detector row is therefore gathered once per view
// instead of once per vertical tap.  The optional weights are multiplied into every gathered value
// (a fused W * e).  Views may be split over CTAs with a fixed-order second-stage sum when there are too
// few pixels to fill the GPU (caller workspace).
#include "back_project.cuh"
#include "bp_fast.cuh"

namespace mbx {

size_t bp_workspace_bytes(const mbx_geom &g, long long num_pixels, int num_views_sel) {
    const BpfPlan fp = plan_bp_fast(g, num_pixels, num_views_sel);
    if (fp.ok) return fp.workspace;
    return plan_bp(g, num_pixels, num_views_sel).workspace;
}

template <int KIND>
static cudaError_t launch_bp_fast(const mbx_geom &g, const BpfPlan &pl, const float *sino, const float *w,
                                  const int32_t *pix, long long n, const int32_t *views, int nv, int cp, float scale,
                                  float *dst, long long ss, cudaStream_t st, int out_slices = 0) {
    auto kern = bp_fast_kernel<KIND>;
    cudaError_t ea = set_max_dynamic_smem(reinterpret_cast<const void *>(kern), 100 * 1024);
    if (ea != cudaSuccess) return ea;
    BpArgs A;
    A.g = g;
    A.sino = sino;
    A.wts = w;
    A.pix = pix;
    A.num_pixels = n;
    A.order = nullptr;
    A.views = views;
    A.num_views_sel = nv;
    A.views_per_split = pl.views_per_split;
    A.coeff_power = cp;
    A.scale = scale;
    A.out = dst;
    A.split_stride = ss;
    A.out_by_index = 0;
    A.out_slices = out_slices;
    A.plan = pl;
    dim3 grid(pl.gx, pl.gy, pl.splits);
    kern<<<grid, BPF_THREADS, pl.smem, st>>>(A, device_error_ptr());
    note_launch();
    return cudaGetLastError();
}

int back_project(const mbx_geom &g, const float *sino, const float *w, const int32_t *pix, long long num_pixels,
                 const int32_t *views, int num_views_sel, int coeff_power, float scale, float *out, void *ws,
                 size_t ws_bytes, cudaStream_t st) {
    if (num_pixels == 0) return MBX_OK;
    if (bp_unit_broadcast(g, sino, w)) {  // unit-weight parallel Hessian: one slice, written to every slice
        const mbx_geom g1 = one_slice_geometry(g);
        const BpfPlan p1 = plan_bp_fast(g1, num_pixels, num_views_sel);
        if (p1.ok && p1.splits == 1) {
            const cudaError_t e = launch_bp_fast<MBX_GEOM_PARALLEL>(g1, p1, nullptr, nullptr, pix, num_pixels, views,
                                                                   num_views_sel, coeff_power, scale, out, 0, st,
                                                                   g.num_recon_slices);
            return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
        }
    }
    const BpfPlan fpl = plan_bp_fast(g, num_pixels, num_views_sel);
    if (fpl.ok) {
        if (fpl.workspace > 0 && (ws == nullptr || ws_bytes < fpl.workspace)) return MBX_ERR_WORKSPACE;
        float *dst = fpl.splits > 1 ? static_cast<float *>(ws) : out;
        const long long stride = num_pixels * (long long)g.num_recon_slices;
        const long long ss = fpl.splits > 1 ? stride : 0;
        auto run = [&](const BpfPlan &pl) -> cudaError_t {
            cudaError_t e;
            if (g.kind == MBX_GEOM_PARALLEL)
                e = launch_bp_fast<MBX_GEOM_PARALLEL>(g, pl, sino, w, pix, num_pixels, views, num_views_sel,
                                                      coeff_power, scale, dst, ss, st);
            else if (g.kind == MBX_GEOM_CONE)
                e = launch_bp_fast<MBX_GEOM_CONE>(g, pl, sino, w, pix, num_pixels, views, num_views_sel, coeff_power,
                                                  scale, dst, ss, st);
            else
                e = launch_bp_fast<MBX_GEOM_TRANSLATION>(g, pl, sino, w, pix, num_pixels, views, num_views_sel,
                                                         coeff_power, scale, dst, ss, st);
            if (e != cudaSuccess) return e;
            if (pl.splits > 1) {
                launch_split_sum(dst, stride, pl.splits, scale, out, stride, st);
                e = cudaGetLastError();
            }
            return e;
        };
        // staged (shared-memory) or per-thread (inline) footprints: cached per call shape, or timed now (each
        // candidate overwrites the whole output); both have the same grid, splits and workspace
        BpfPlan cand[2] = {fpl, plan_bp_fast(g, num_pixels, num_views_sel, 1)};
        int choice = 0;
        if (autotune_forced() >= 0) {
            choice = autotune_forced() >= 1 ? 1 : 0;
        } else if (autotune_enabled()) {
            long long n2 = 1;
            while (n2 < num_pixels) n2 <<= 1;
            const long long key[11] = {3, g.kind, num_views_sel, g.num_det_rows, g.num_det_channels, g.num_recon_slices,
                                       g.num_recon_rows, g.num_recon_cols, n2, views ? 1 : 0, w ? 1 : 0};
            choice = autotune_lookup(key, 11);
            if (choice < 0 || choice > 1) {
                choice = 0;
                if (!stream_is_capturing(st)) {
                    float t0 = 0.0f;  // the default first: a long call is not tuned (its output is complete)
                    cudaError_t e = time_once([&]() { return run(cand[0]); }, st, t0);
                    if (e != cudaSuccess) return set_cuda_error(e);
                    if (t0 > MBX_TUNE_BUDGET_MS) {
                        autotune_store(key, 11, 0);
                        return MBX_OK;
                    }
                    float t[2] = {0.0f, 0.0f};
                    e = time_candidates(2, [&](int c) { return run(cand[c]); }, st, t);
                    if (e != cudaSuccess) return set_cuda_error(e);
                    choice = t[1] < t[0] ? 1 : 0;
                    autotune_store(key, 11, choice);
                }
            }
        }
        const cudaError_t e = run(cand[choice]);
        return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
    }
    const BpPlan pl = plan_bp(g, num_pixels, num_views_sel);
    if (pl.workspace > 0 && (ws == nullptr || ws_bytes < pl.workspace)) return MBX_ERR_WORKSPACE;
    float *dst = pl.splits > 1 ? static_cast<float *>(ws) : out;
    const long long stride = num_pixels * (long long)g.num_recon_slices;
    const long long ss = pl.splits > 1 ? stride : 0;
    cudaError_t e;
    if (g.kind == MBX_GEOM_PARALLEL)
        e = launch_bp_parallel(g, pl, sino, w, pix, num_pixels, views, num_views_sel, coeff_power, scale, dst, ss, st);
    else if (g.kind == MBX_GEOM_CONE)
        e = launch_bp_cone(g, pl, sino, w, pix, num_pixels, views, num_views_sel, coeff_power, scale, dst, ss, st);
    else
        e = launch_bp_translation(g, pl, sino, w, pix, num_pixels, views, num_views_sel, coeff_power, scale, dst, ss,
                                  st);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (pl.splits > 1) {
        launch_split_sum(dst, stride, pl.splits, scale, out, stride, st);
        e = cudaGetLastError();
        if (e != cudaSuccess) return set_cuda_error(e);
    }
    return MBX_OK;
}

}  // namespace mbx

extern "C" size_t mbx_back_project_workspace_bytes(const mbx_geom *g, int64_t num_pixels, int32_t num_views_sel) {
    if (mbx::validate_geom(g) != MBX_OK || num_pixels < 0 || num_views_sel <= 0) return 0;
    return mbx::bp_workspace_bytes(*g, num_pixels, num_views_sel);
}

extern "C" int mbx_sparse_back_project(const mbx_geom *g, const float *sinogram, const float *weights,
                                       const int32_t *pixel_indices, int64_t num_pixels, const int32_t *view_indices,
                                       int32_t num_views_sel, int32_t coeff_power, float scale, float *out,
                                       void *workspace, size_t workspace_bytes, void *stream) {
    int rc = mbx::validate_geom(g);
    if (rc != MBX_OK) return rc;
    if (num_pixels < 0 || num_views_sel <= 0) return MBX_ERR_INVALID_ARG;
    if (num_pixels > 0 && (!pixel_indices || !out)) return MBX_ERR_INVALID_ARG;
    if (coeff_power != 1 && coeff_power != 2) return MBX_ERR_UNSUPPORTED;
    if (!view_indices && num_views_sel > g->num_views) return MBX_ERR_INVALID_ARG;
    if (!sinogram) {  // no sinogram: the values are the weights, or 1 everywhere when there are none either
        sinogram = weights;
        weights = nullptr;
    }
    return mbx::back_project(*g, sinogram, weights, pixel_indices, num_pixels, view_indices, num_views_sel,
                             coeff_power, scale, out, workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}
