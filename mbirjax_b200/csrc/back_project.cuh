// Back-projection kernel template and launch plan, shared by the per-geometry translation units
// bp_parallel.cu, bp_cone.cu and bp_translation.cu (see back_project.cu for the design notes).
#pragma once
#include <climits>
#include <cmath>

#include "mbx_common.cuh"
#include "mbx_host.hpp"

namespace mbx {

constexpr int BP_THREADS = 128;
constexpr int BP_VIEW_CHUNK = 128;
constexpr int BP_MAX_CACHE_ROWS = 96;

__device__ __forceinline__ float gather_row(const float *__restrict__ row, const float *__restrict__ wrow, int n,
                                            int num_channels) {
    const int nn = min(max(n, 0), num_channels - 1);  // clamped gather, as the reference's jnp indexing
    float v = row ? __ldg(row + nn) : 1.0f;            // no sinogram: every value is 1 (unit-weight Hessian)
    if (wrow) v *= __ldg(wrow + nn);
    return v;
}

template <int MAXR>
__device__ __forceinline__ float horizontal_row_sum(const float *__restrict__ view, const float *__restrict__ wview,
                                                    int m, int num_channels, int n_c, const float (&a)[2 * MAXR + 1]) {
    const long long off = (long long)m * num_channels;
    const float *row = view ? view + off : nullptr;
    const float *wrow = wview ? wview + off : nullptr;
    float c = 0.0f;
#pragma unroll
    for (int k = 0; k < 2 * MAXR + 1; ++k)
        if (a[k] != 0.0f) c += a[k] * gather_row(row, wrow, n_c + k - MAXR, num_channels);
    return c;
}

template <int MAXR>
__device__ __noinline__ float horizontal_row_sum_uncached(const float *__restrict__ view,
                                                          const float *__restrict__ wview, int m, int num_channels,
                                                          int n_c, const float *a) {
    float aa[2 * MAXR + 1];
#pragma unroll
    for (int k = 0; k < 2 * MAXR + 1; ++k) aa[k] = a[k];
    return horizontal_row_sum<MAXR>(view, wview, m, num_channels, n_c, aa);
}

template <int KIND, int MAXR, int ST>
__global__ void __launch_bounds__(BP_THREADS)
bp_kernel(const mbx_geom g, const float *__restrict__ sino, const float *__restrict__ wts,
          const int32_t *__restrict__ pix, long long num_pixels, const int32_t *__restrict__ views, int num_views_sel,
          int views_per_split, int coeff_power, float scale, float *__restrict__ dst, long long split_stride,
          int cache_rows, int *err) {
    constexpr int NT = 2 * MAXR + 1;
    __shared__ float s_ang[BP_VIEW_CHUNK], s_cs[BP_VIEW_CHUNK], s_sn[BP_VIEW_CHUNK];
    __shared__ int s_vi[BP_VIEW_CHUNK];
    extern __shared__ float colbuf[];  // [cache_rows][BP_THREADS], cone only

    const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    const int s0 = blockIdx.y * ST;
    const int split = blockIdx.z;
    const int num_rows = g.num_det_rows;
    const int num_channels = g.num_det_channels;
    const int num_slices = g.num_recon_slices;
    const int ns = min(ST, num_slices - s0);
    const int r = g.psf_radius;
    const int v_begin = split * views_per_split;
    const int v_end = min(num_views_sel, v_begin + views_per_split);

    bool active = p < num_pixels;
    int idx = 0;
    if (active) {
        idx = pix[p];
        if (idx < 0 || idx >= g.num_recon_rows * g.num_recon_cols) {
            if (blockIdx.y == 0 && split == 0) flag_error(err, MBX_ERRFLAG_PIXEL);
            active = false;
        }
    }
    float xt = 0.0f, yt = 0.0f;
    if (active && KIND != MBX_GEOM_TRANSLATION) pixel_tilde(g, idx, xt, yt);

    float acc[ST];
#pragma unroll
    for (int s = 0; s < ST; ++s) acc[s] = 0.0f;

    const float det_center_row = 0.5f * (float)(num_rows - 1);
    const float center_slice = 0.5f * (float)(num_slices - 1);
    float *mycol = colbuf + threadIdx.x;

    for (int vb = v_begin; vb < v_end; vb += BP_VIEW_CHUNK) {
        const int nv = min(BP_VIEW_CHUNK, v_end - vb);
        __syncthreads();
        for (int t = threadIdx.x; t < nv; t += blockDim.x) {
            const int vi = views ? views[vb + t] : vb + t;
            const bool ok = vi >= 0 && vi < g.num_views;
            if (!ok && blockIdx.x == 0 && blockIdx.y == 0) flag_error(err, MBX_ERRFLAG_VIEW);
            s_vi[t] = ok ? vi : -1;
            if (KIND == MBX_GEOM_TRANSLATION) {  // (zoff = -tz, tx, ty) in the (angle, cos, sin) slots
                s_ang[t] = ok ? -g.translations[3 * vi + 2] : 0.0f;
                s_cs[t] = ok ? g.translations[3 * vi] : 0.0f;
                s_sn[t] = ok ? g.translations[3 * vi + 1] : 0.0f;
            } else {
                const float ang = ok ? g.angles[vi] : 0.0f;
                s_ang[t] = ang;
                s_cs[t] = cosf(ang);
                s_sn[t] = sinf(ang);
            }
        }
        __syncthreads();
        if (!active) continue;
        for (int t = 0; t < nv; ++t) {
            const int vi = s_vi[t];
            if (vi < 0) continue;
            const ChannelFootprint f = (KIND == MBX_GEOM_PARALLEL) ? parallel_footprint(g, s_cs[t], s_sn[t], xt, yt)
                                       : (KIND == MBX_GEOM_CONE) ? cone_footprint(g, s_ang[t], s_cs[t], s_sn[t], xt, yt)
                                                                 : translation_footprint(g, idx, s_cs[t], s_sn[t]);
            float a[NT];
#pragma unroll
            for (int k = -MAXR; k <= MAXR; ++k) {
                const float c = (k < -r || k > r) ? 0.0f
                                : (KIND == MBX_GEOM_TRANSLATION) ? translation_channel_coeff(g, f, k)
                                                                 : channel_coeff(g, f, k);
                a[k + MAXR] = (coeff_power == 2) ? c * c : c;
            }
            const float *view = sino ? sino + (long long)vi * num_rows * num_channels : nullptr;
            const float *wview = wts ? wts + (long long)vi * num_rows * num_channels : nullptr;
            if (KIND == MBX_GEOM_PARALLEL) {
#pragma unroll
                for (int s = 0; s < ST; ++s)
                    if (s < ns) acc[s] += horizontal_row_sum<MAXR>(view, wview, s0 + s, num_channels, f.n_c, a);
            } else {
                // slice k sits at height delta_voxel (k - (S-1)/2) + zoff: recon_slice_offset for the cone,
                // -tz for a translation view (translation_model.py:654)
                const float zoff = (KIND == MBX_GEOM_TRANSLATION) ? s_ang[t] : g.recon_slice_offset;
                const float mag = f.mag;
                const float w_r = mag * (g.delta_voxel / g.delta_det_row);
                const float l_max = fminf(1.0f, w_r);
                const float half_w = (w_r + 1.0f) * 0.5f;
                // Detector rows touched by this slice tile: between the centre rows of its end slices +- r.
                const float z_first = g.delta_voxel * ((float)s0 - center_slice) + zoff;
                const float z_last = g.delta_voxel * ((float)(s0 + ns - 1) - center_slice) + zoff;
                const int mc_first = (int)rintf((mag * z_first + g.det_row_offset) / g.delta_det_row + det_center_row);
                const int mc_last = (int)rintf((mag * z_last + g.det_row_offset) / g.delta_det_row + det_center_row);
                const int m_lo = max(min(mc_first, mc_last) - r, 0);
                const int m_hi = min(max(mc_first, mc_last) + r, num_rows - 1);
                const bool cached = (m_hi - m_lo + 1) <= cache_rows;
                if (cached)
                    for (int m = m_lo; m <= m_hi; ++m)
                        mycol[(m - m_lo) * BP_THREADS] = horizontal_row_sum<MAXR>(view, wview, m, num_channels, f.n_c, a);
#pragma unroll
                for (int s = 0; s < ST; ++s) {
                    if (s < ns) {
                        const float z = g.delta_voxel * ((float)(s0 + s) - center_slice) + zoff;
                        const float v = mag * z;
                        const float m_p = (v + g.det_row_offset) / g.delta_det_row + det_center_row;
                        const int m_c = (int)rintf(m_p);
                        const float sec = sec_phi(v, g.source_detector_dist);
                        float sum = 0.0f;
#pragma unroll
                        for (int mo = -MAXR; mo <= MAXR; ++mo) {
                            if (mo < -r || mo > r) continue;
                            const int m = m_c + mo;
                            if (m < 0 || m >= num_rows) continue;
                            float aa = fminf(fmaxf(half_w - fabsf(m_p - (float)m), 0.0f), l_max) * sec;
                            if (coeff_power == 2) aa *= aa;
                            const float col = (cached && m >= m_lo && m <= m_hi)
                                                  ? mycol[(m - m_lo) * BP_THREADS]
                                                  : horizontal_row_sum_uncached<MAXR>(view, wview, m, num_channels, f.n_c, a);
                            sum += aa * col;
                        }
                        acc[s] += sum;
                    }
                }
            }
        }
    }
    if (p >= num_pixels) return;
    float *out = dst + (long long)split * split_stride + p * (long long)num_slices + s0;
    const float sc = (split_stride == 0) ? scale : 1.0f;
#pragma unroll
    for (int s = 0; s < ST; ++s)
        if (s < ns) out[s] = active ? sc * acc[s] : 0.0f;
}

struct BpPlan {
    int st, gx, gy, splits, views_per_split, cache_rows;
    size_t smem, workspace;
};

// Rows a slice tile of ST slices can touch in one view (for sizing the per-thread row cache).
inline int cone_cache_rows(const mbx_geom &g, int st) {
    const double half_r = 0.5 * (g.num_recon_rows - 1), half_c = 0.5 * (g.num_recon_cols - 1);
    const double rho = g.delta_voxel * std::sqrt(half_r * half_r + half_c * half_c);
    double inv = 1.0 / g.magnification - (std::isinf(g.source_detector_dist) ? 0.0 : rho / g.source_detector_dist);
    double max_mag = inv > 1e-6 ? 1.0 / inv : 1e6;
    const double w = max_mag * g.delta_voxel / g.delta_det_row;
    double rows = st * std::ceil(w) + 2.0 * g.psf_radius + 2.0;
    if (rows > BP_MAX_CACHE_ROWS) rows = BP_MAX_CACHE_ROWS;
    return (int)rows;
}

// Translation geometry: the host does not see the translations, so the cache is sized from psf_radius, which the
// model derives from the largest magnification (translation_model.py:134-172): a slice spans at most
// ceil(W) <= 2 psf_radius rows.  A view whose rows do not fit takes the uncached path.
inline int translation_cache_rows(const mbx_geom &g, int st) {
    const int r = g.psf_radius > 0 ? g.psf_radius : 1;
    const int rows = st * 2 * r + 2 * g.psf_radius + 2;
    return rows > BP_MAX_CACHE_ROWS ? BP_MAX_CACHE_ROWS : rows;
}

inline BpPlan plan_bp(const mbx_geom &g, long long num_pixels, int num_views_sel) {
    BpPlan pl;
    const int S = g.num_recon_slices;
    // the radius-4 instantiation exists only with ST = 8 (launch_bp_kind)
    pl.st = (S >= 16 && psf_bucket(g.psf_radius) <= 2) ? 16 : 8;
    pl.gx = ceil_div(num_pixels > 0 ? num_pixels : 1, BP_THREADS);
    pl.gy = ceil_div(S, pl.st);
    pl.cache_rows = (g.kind == MBX_GEOM_CONE)          ? cone_cache_rows(g, pl.st)
                    : (g.kind == MBX_GEOM_TRANSLATION) ? translation_cache_rows(g, pl.st)
                                                       : 0;
    pl.smem = (size_t)pl.cache_rows * BP_THREADS * 4;
    const long long base = (long long)pl.gx * pl.gy;
    const int sms = num_sms();
    long long splits = 1;
    if (base < 4LL * sms && num_views_sel >= 8) {
        splits = (4LL * sms + base - 1) / base;
        long long maxs = num_views_sel / 4;
        if (splits > maxs) splits = maxs;
        if (splits > 64) splits = 64;
        if (splits < 1) splits = 1;
    }
    pl.views_per_split = ceil_div(num_views_sel, splits);
    pl.splits = ceil_div(num_views_sel, pl.views_per_split);
    if (pl.splits < 1) pl.splits = 1;
    pl.workspace = pl.splits > 1 ? align256((size_t)pl.splits * num_pixels * S * 4) : 0;
    return pl;
}

template <int KIND, int MAXR, int ST>
static cudaError_t launch_bp_t(const mbx_geom &g, const BpPlan &pl, const float *sino, const float *w,
                               const int32_t *pix, long long n, const int32_t *views, int nv, int cp, float scale,
                               float *dst, long long ss, cudaStream_t st) {
    auto kern = bp_kernel<KIND, MAXR, ST>;
    cudaError_t ea = set_max_dynamic_smem(reinterpret_cast<const void *>(kern), BP_MAX_CACHE_ROWS * BP_THREADS * 4);
    if (ea != cudaSuccess) return ea;
    dim3 grid(pl.gx, pl.gy, pl.splits);
    kern<<<grid, BP_THREADS, pl.smem, st>>>(g, sino, w, pix, n, views, nv, pl.views_per_split, cp, scale, dst, ss,
                                            pl.cache_rows, device_error_ptr());
    mbx::note_launch();
    return cudaGetLastError();
}

template <int KIND, int MAXR>
static cudaError_t launch_bp_r(const mbx_geom &g, const BpPlan &pl, const float *sino, const float *w,
                               const int32_t *pix, long long n, const int32_t *views, int nv, int cp, float scale,
                               float *dst, long long ss, cudaStream_t st) {
    if (pl.st == 16) return launch_bp_t<KIND, MAXR, 16>(g, pl, sino, w, pix, n, views, nv, cp, scale, dst, ss, st);
    return launch_bp_t<KIND, MAXR, 8>(g, pl, sino, w, pix, n, views, nv, cp, scale, dst, ss, st);
}

template <int KIND>
cudaError_t launch_bp_kind(const mbx_geom &g, const BpPlan &pl, const float *sino, const float *w,
                                  const int32_t *pix, long long n, const int32_t *views, int nv, int cp, float scale,
                                  float *dst, long long ss, cudaStream_t st) {
    switch (psf_bucket(g.psf_radius)) {
        case 1: return launch_bp_r<KIND, 1>(g, pl, sino, w, pix, n, views, nv, cp, scale, dst, ss, st);
        case 2: return launch_bp_r<KIND, 2>(g, pl, sino, w, pix, n, views, nv, cp, scale, dst, ss, st);
        default: return launch_bp_t<KIND, MBX_MAX_PSF_RADIUS, 8>(g, pl, sino, w, pix, n, views, nv, cp, scale, dst, ss, st);
    }
}


// Defined in bp_parallel.cu / bp_cone.cu / bp_translation.cu.
cudaError_t launch_bp_parallel(const mbx_geom &g, const BpPlan &pl, const float *sino, const float *w,
                               const int32_t *pix, long long n, const int32_t *views, int nv, int cp, float scale,
                               float *dst, long long ss, cudaStream_t st);
cudaError_t launch_bp_cone(const mbx_geom &g, const BpPlan &pl, const float *sino, const float *w,
                           const int32_t *pix, long long n, const int32_t *views, int nv, int cp, float scale,
                           float *dst, long long ss, cudaStream_t st);
cudaError_t launch_bp_translation(const mbx_geom &g, const BpPlan &pl, const float *sino, const float *w,
                                  const int32_t *pix, long long n, const int32_t *views, int nv, int cp, float scale,
                                  float *dst, long long ss, cudaStream_t st);

}  // namespace mbx
