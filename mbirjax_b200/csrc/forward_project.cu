// Sparse forward projector for parallel-beam, cone-beam and translation geometry (sm_100a).
//
// Replaces Projectors.sparse_forward_project (projectors.py:61-129) over the geometry plugins
// ParallelBeamModel.forward_project_pixel_batch_to_one_view (parallel_beam.py:138-178),
// ConeBeamModel.forward_project_pixel_batch_to_one_view (cone_beam.py:189-377) and
// TranslationModel.forward_project_pixel_batch_to_one_view (translation_model.py:190-378).
// Radius-1 geometries run the channel-block kernel of fp_cb.cuh when its plan fits (translation geometry when the
// caller gives a magnification bound); the other cases run the general kernel below.
//
// One CTA owns an output tile (one view x a band of detector rows x all channels) held in shared memory,
// walks every pixel of its pixel range in chunks of FP_PB, and scatters into the tile with shared-memory
// atomics.  Per chunk, FP_PB threads first compute the channel footprint of each pixel (centre channel +
// 2r+1 coefficients) into shared memory; then the threads walk (pixel, row) pairs with lanes along detector
// rows, so the voxel-cylinder reads are contiguous and the lanes of a warp hit different tile rows (the
// padded row pitch is odd, so there are no bank conflicts).  For cone beam each lane first evaluates the
// vertical fan (detector-row-centric, 2*bp_psf_radius+1 slices) for its row.  The finished tile is written
// once, coalesced.  When there are too few (view, row-band) tiles to fill the GPU, the pixel range is split
// over CTAs whose partial tiles are summed by split_sum_kernel in a fixed order (caller workspace).
#include <algorithm>
#include <climits>

#include "mbx_common.cuh"
#include "mbx_host.hpp"
#include "fp_cb.cuh"

namespace mbx {

constexpr int FP_PB = 64;  // pixels per footprint chunk
constexpr int FP_THREADS = 256;

template <int KIND, int MAXR, int MAXRBP>
__global__ void __launch_bounds__(FP_THREADS)
fp_kernel(const mbx_geom g, const float *__restrict__ vox, const int32_t *__restrict__ pix, long long num_pixels,
          const int32_t *__restrict__ views, float *__restrict__ dst, int row_tile, int c_pad,
          long long pixels_per_split, long long split_stride, int *err) {
    constexpr int NT = 2 * MAXR + 1;
    extern __shared__ __align__(16) float smem[];
    float *tile = smem;
    float *h_a = tile + row_tile * c_pad;
    int *h_nc = reinterpret_cast<int *>(h_a + FP_PB * NT);
    float *h_mag = reinterpret_cast<float *>(h_nc + FP_PB);

    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    const int nthreads = blockDim.x * blockDim.y;
    const int j = blockIdx.x;
    const int m0 = blockIdx.y * row_tile;
    const int split = blockIdx.z;
    const int num_rows = g.num_det_rows;
    const int num_channels = g.num_det_channels;
    const int num_slices = g.num_recon_slices;
    const int mt = min(row_tile, num_rows - m0);
    const int npix_grid = g.num_recon_rows * g.num_recon_cols;

    const int vi = views ? views[j] : j;
    const bool view_ok = vi >= 0 && vi < g.num_views;
    if (!view_ok && tid == 0) flag_error(err, MBX_ERRFLAG_VIEW);
    float angle = 0.0f, tx = 0.0f, ty = 0.0f, zoff = 0.0f;
    if (view_ok) {
        if (KIND == MBX_GEOM_TRANSLATION) {
            tx = g.translations[3 * vi];
            ty = g.translations[3 * vi + 1];
            zoff = -g.translations[3 * vi + 2];
        } else {
            angle = g.angles[vi];
        }
    }
    const float cs = cosf(angle);
    const float sn = sinf(angle);

    for (int i = tid; i < mt * c_pad; i += nthreads) tile[i] = 0.0f;

    const long long p_begin = (long long)split * pixels_per_split;
    long long p_end = p_begin + pixels_per_split;
    if (p_end > num_pixels) p_end = num_pixels;
    if (!view_ok) p_end = p_begin;

    for (long long pb = p_begin; pb < p_end; pb += FP_PB) {
        __syncthreads();
        if (tid < FP_PB) {
            const long long p = pb + tid;
            int nc = INT_MIN;
            if (p < p_end) {
                const int idx = pix[p];
                if (idx < 0 || idx >= npix_grid) {
                    flag_error(err, MBX_ERRFLAG_PIXEL);
                } else {
                    ChannelFootprint f;
                    if (KIND == MBX_GEOM_TRANSLATION) {
                        f = translation_footprint(g, idx, tx, ty);
                    } else {
                        float xt, yt;
                        pixel_tilde(g, idx, xt, yt);
                        f = (KIND == MBX_GEOM_PARALLEL) ? parallel_footprint(g, cs, sn, xt, yt)
                                                        : cone_footprint(g, angle, cs, sn, xt, yt);
                    }
                    nc = f.n_c;
#pragma unroll
                    for (int k = -MAXR; k <= MAXR; ++k)
                        h_a[tid * NT + k + MAXR] =
                            (k < -g.psf_radius || k > g.psf_radius)
                                ? 0.0f
                                : (KIND == MBX_GEOM_TRANSLATION ? translation_channel_coeff(g, f, k)
                                                                : channel_coeff(g, f, k));
                    h_mag[tid] = f.mag;
                }
            }
            h_nc[tid] = nc;
        }
        __syncthreads();
        const int np = (int)min((long long)FP_PB, p_end - pb);
        for (int pl = threadIdx.y; pl < np; pl += blockDim.y) {
            const int nc = h_nc[pl];
            if (nc == INT_MIN) continue;
            const float *cyl = vox + (pb + pl) * (long long)num_slices;
            float a[NT];
#pragma unroll
            for (int k = 0; k < NT; ++k) a[k] = h_a[pl * NT + k];
            const float mag = h_mag[pl];
            for (int ml = threadIdx.x; ml < mt; ml += blockDim.x) {
                float val;
                if (KIND == MBX_GEOM_PARALLEL)
                    val = __ldg(cyl + m0 + ml);
                else if (KIND == MBX_GEOM_CONE)
                    val = cone_fp_vertical<MAXRBP>(g, cyl, mag, m0 + ml);
                else
                    val = fan_fp_vertical<MAXRBP>(g, cyl, mag, m0 + ml, zoff, g.psf_radius);
                float *trow = tile + ml * c_pad;
#pragma unroll
                for (int k = -MAXR; k <= MAXR; ++k) {
                    const int n = nc + k;
                    if (n >= 0 && n < num_channels && a[k + MAXR] != 0.0f) atomicAdd(trow + n, a[k + MAXR] * val);
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

// out[i] = scale * sum_s ws[s * stride + i], s = 0..splits-1 in order.
__global__ void split_sum_kernel(const float *__restrict__ ws, long long stride, int splits, float scale,
                                 float *__restrict__ out, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int k = 0; k < splits; ++k) s += ws[k * stride + i];
        out[i] = scale * s;
    }
}

void launch_split_sum(const float *ws, long long stride, int splits, float scale, float *out, long long n,
                      cudaStream_t st) {
    split_sum_kernel<<<grid_for(n, 256), 256, 0, st>>>(ws, stride, splits, scale, out, n);
    mbx::note_launch();
}

struct FpPlan {
    int c_pad, row_tile, tiles, splits, bx, by;
    long long pixels_per_split;
    size_t smem, workspace;
};

static FpPlan plan_fp(const mbx_geom &g, long long num_pixels, int num_views_sel) {
    FpPlan pl;
    const int C = g.num_det_channels, R = g.num_det_rows;
    pl.c_pad = (C % 2 == 0) ? C + 1 : C;
    const size_t budget = 64 * 1024;
    long long rt = (long long)(budget / ((size_t)pl.c_pad * 4));
    if (rt > 64) rt = 64;
    if (rt < 1) rt = 1;
    if (rt > R) rt = R;
    pl.row_tile = (int)rt;
    pl.tiles = ceil_div(R, pl.row_tile);
    int bx = 1;
    while (bx < pl.row_tile && bx < 32) bx <<= 1;
    pl.bx = bx;
    pl.by = FP_THREADS / bx;
    // footprint header sized for the largest instantiation (launch_fp_kind may pick MAXR above the bucket of r)
    const int nmax = 2 * MBX_MAX_PSF_RADIUS + 1;
    pl.smem = (size_t)pl.row_tile * pl.c_pad * 4 + (size_t)FP_PB * (nmax * 4 + 8);
    const long long base = (long long)num_views_sel * pl.tiles;
    const int sms = num_sms();
    long long splits = 1;
    if (base < 4LL * sms && num_pixels > 4LL * FP_PB) {
        splits = (4LL * sms + base - 1) / base;
        long long maxs = num_pixels / (4LL * FP_PB);
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

template <int KIND, int MAXR, int MAXRBP>
static cudaError_t launch_fp_t(const mbx_geom &g, const FpPlan &pl, const float *vox, const int32_t *pix,
                               long long num_pixels, const int32_t *views, int num_views_sel, float *dst,
                               long long split_stride, cudaStream_t st) {
    auto kern = fp_kernel<KIND, MAXR, MAXRBP>;
    cudaError_t ea = set_max_dynamic_smem(reinterpret_cast<const void *>(kern), 200 * 1024);
    if (ea != cudaSuccess) return ea;
    dim3 grid(num_views_sel, pl.tiles, pl.splits), block(pl.bx, pl.by);
    kern<<<grid, block, pl.smem, st>>>(g, vox, pix, num_pixels, views, dst, pl.row_tile, pl.c_pad,
                                       pl.pixels_per_split, split_stride, device_error_ptr());
    mbx::note_launch();
    return cudaGetLastError();
}

template <int KIND>
static cudaError_t launch_fp_kind(const mbx_geom &g, const FpPlan &pl, const float *vox, const int32_t *pix,
                                  long long n, const int32_t *views, int nv, float *dst, long long ss,
                                  cudaStream_t st) {
    const int r = psf_bucket(g.psf_radius);
    // vertical taps: bp_psf_radius for the cone, psf_radius for translation (translation_model.py:364)
    const int rb = (KIND == MBX_GEOM_CONE)          ? psf_bucket(g.bp_psf_radius)
                   : (KIND == MBX_GEOM_TRANSLATION) ? psf_bucket(g.psf_radius)
                                                    : 1;
    if (r == 1 && rb == 1) return launch_fp_t<KIND, 1, 1>(g, pl, vox, pix, n, views, nv, dst, ss, st);
    if (r == 2 && rb <= 2) return launch_fp_t<KIND, 2, 2>(g, pl, vox, pix, n, views, nv, dst, ss, st);
    if (r == 1 && rb == 2) return launch_fp_t<KIND, 2, 2>(g, pl, vox, pix, n, views, nv, dst, ss, st);
    return launch_fp_t<KIND, MBX_MAX_PSF_RADIUS, MBX_MAX_PSF_RADIUS>(g, pl, vox, pix, n, views, nv, dst, ss, st);
}

size_t fp_workspace_bytes(const mbx_geom &g, long long num_pixels, int num_views_sel) {
    if (plan_fp_cb(g).ok && num_pixels * g.num_recon_slices < (1LL << 31) && num_pixels <= (1LL << 24))
        return fp_chunk_box_bytes(num_pixels);
    return plan_fp(g, num_pixels, num_views_sel).workspace;
}

template <int KIND, int MINB>
static cudaError_t launch_fp_cb_v(const FpArgs &A, cudaStream_t st) {
    cudaError_t ea = set_max_dynamic_smem(reinterpret_cast<const void *>(fp_cb_kernel<KIND, MINB>), 200 * 1024);
    if (ea != cudaSuccess) return ea;
    dim3 grid(A.num_views_sel, A.plan.cblocks);
    fp_cb_kernel<KIND, MINB><<<grid, CB_THREADS, A.plan.walk.smem, st>>>(A, device_error_ptr());
    note_launch();
    return cudaGetLastError();
}

static cudaError_t launch_fp_cb(const FpArgs &A, cudaStream_t st) {
    const bool three = A.plan.minb >= 3;
    switch (A.g.kind) {
        case MBX_GEOM_PARALLEL:
            return three ? launch_fp_cb_v<MBX_GEOM_PARALLEL, 3>(A, st) : launch_fp_cb_v<MBX_GEOM_PARALLEL, 2>(A, st);
        case MBX_GEOM_CONE:
            return three ? launch_fp_cb_v<MBX_GEOM_CONE, 3>(A, st) : launch_fp_cb_v<MBX_GEOM_CONE, 2>(A, st);
        default:
            return three ? launch_fp_cb_v<MBX_GEOM_TRANSLATION, 3>(A, st)
                         : launch_fp_cb_v<MBX_GEOM_TRANSLATION, 2>(A, st);
    }
}

int forward_project(const mbx_geom &g, const float *vox, const int32_t *pix, long long num_pixels,
                    const int32_t *views, int num_views_sel, float *out, void *ws, size_t ws_bytes,
                    cudaStream_t st) {
    CbPlan cand[CB_MAX_CANDIDATES];
    const int ncand = fp_cb_candidates(g, num_views_sel, 4LL * num_sms(), cand);
    // 32-bit cylinder offsets; list positions share a word with the bin
    if (ncand > 0 && num_pixels * g.num_recon_slices < (1LL << 31) && num_pixels <= (1LL << 24)) {
        FpArgs A;
        A.g = g;
        A.vox = vox;
        A.pix = pix;
        A.num_pixels = num_pixels;
        A.views = views;
        A.num_views_sel = num_views_sel;
        A.out = out;
        A.vox_by_index = 0;
        A.plan = cand[0];
        // bounding boxes of the list's chunks, so that each channel block skips the chunks that miss it
        const size_t need = fp_chunk_box_bytes(num_pixels);
        if (need > 0 && (ws == nullptr || ws_bytes < need)) return MBX_ERR_WORKSPACE;
        A.chunk_box = num_pixels > 0 ? static_cast<const int4 *>(ws) : nullptr;
        if (num_pixels > 0) {
            fp_chunk_bounds_kernel<<<(unsigned)((num_pixels + CB_CHUNK - 1) / CB_CHUNK), CB_CHUNK, 0, st>>>(
                pix, num_pixels, g.num_recon_rows, g.num_recon_cols, static_cast<int4 *>(ws));
            note_launch();
            cudaError_t e0 = cudaGetLastError();
            if (e0 != cudaSuccess) return set_cuda_error(e0);
        }
        // plan choice: cached per call shape, or timed now (each candidate overwrites the whole output)
        int choice = 0;
        if (autotune_forced() >= 0) {
            choice = std::min(autotune_forced(), ncand - 1);
        } else if (ncand > 1 && num_pixels > 0 && autotune_enabled()) {
            long long n2 = 1;
            while (n2 < num_pixels) n2 <<= 1;
            const long long key[10] = {1, g.kind, num_views_sel, g.num_det_rows, g.num_det_channels,
                                       g.num_recon_slices, g.num_recon_rows, g.num_recon_cols, n2, views ? 1 : 0};
            choice = autotune_lookup(key, 10);
            if (choice < 0 || choice >= ncand) {
                choice = 0;
                if (!stream_is_capturing(st)) {
                    // the default first, timed once: a long call is not tuned, and its output is already complete
                    A.plan = cand[0];
                    float t0 = 0.0f;
                    cudaError_t e = time_once([&]() { return launch_fp_cb(A, st); }, st, t0);
                    if (e != cudaSuccess) return set_cuda_error(e);
                    if (t0 > MBX_TUNE_BUDGET_MS) {
                        autotune_store(key, 10, 0);
                        return MBX_OK;
                    }
                    float t[CB_MAX_CANDIDATES];
                    e = time_candidates(
                        ncand, [&](int c) { A.plan = cand[c]; return launch_fp_cb(A, st); }, st, t);
                    if (e != cudaSuccess) return set_cuda_error(e);
                    for (int c = 1; c < ncand; ++c)
                        if (t[c] < t[choice]) choice = c;
                    autotune_store(key, 10, choice);
                }
            }
        }
        A.plan = cand[choice];
        cudaError_t e = launch_fp_cb(A, st);
        return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
    }
    const FpPlan pl = plan_fp(g, num_pixels, num_views_sel);
    if (pl.workspace > 0 && (ws == nullptr || ws_bytes < pl.workspace)) return MBX_ERR_WORKSPACE;
    float *dst = pl.splits > 1 ? static_cast<float *>(ws) : out;
    const long long stride = (long long)num_views_sel * g.num_det_rows * g.num_det_channels;
    const long long ss = pl.splits > 1 ? stride : 0;
    cudaError_t e;
    if (g.kind == MBX_GEOM_PARALLEL)
        e = launch_fp_kind<MBX_GEOM_PARALLEL>(g, pl, vox, pix, num_pixels, views, num_views_sel, dst, ss, st);
    else if (g.kind == MBX_GEOM_CONE)
        e = launch_fp_kind<MBX_GEOM_CONE>(g, pl, vox, pix, num_pixels, views, num_views_sel, dst, ss, st);
    else
        e = launch_fp_kind<MBX_GEOM_TRANSLATION>(g, pl, vox, pix, num_pixels, views, num_views_sel, dst, ss, st);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (pl.splits > 1) {
        launch_split_sum(dst, stride, pl.splits, 1.0f, out, stride, st);
        e = cudaGetLastError();
        if (e != cudaSuccess) return set_cuda_error(e);
    }
    return MBX_OK;
}

}  // namespace mbx

extern "C" size_t mbx_forward_project_workspace_bytes(const mbx_geom *g, int64_t num_pixels, int32_t num_views_sel) {
    if (mbx::validate_geom(g) != MBX_OK || num_pixels < 0 || num_views_sel <= 0) return 0;
    return mbx::fp_workspace_bytes(*g, num_pixels, num_views_sel);
}

extern "C" int mbx_sparse_forward_project(const mbx_geom *g, const float *voxel_values, const int32_t *pixel_indices,
                                          int64_t num_pixels, const int32_t *view_indices, int32_t num_views_sel,
                                          float *sinogram_out, void *workspace, size_t workspace_bytes, void *stream) {
    int rc = mbx::validate_geom(g);
    if (rc != MBX_OK) return rc;
    if (num_pixels < 0 || num_views_sel <= 0 || !sinogram_out) return MBX_ERR_INVALID_ARG;
    if (num_pixels > 0 && (!voxel_values || !pixel_indices)) return MBX_ERR_INVALID_ARG;
    if (!view_indices && num_views_sel > g->num_views) return MBX_ERR_INVALID_ARG;
    return mbx::forward_project(*g, voxel_values, pixel_indices, num_pixels, view_indices, num_views_sel,
                                sinogram_out, workspace, workspace_bytes, static_cast<cudaStream_t>(stream));
}
