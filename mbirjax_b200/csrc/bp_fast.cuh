// Back projector specialised for psf_radius == 1 (the reference's default geometry: delta_voxel equal to the
// detector pitch at the magnification), for parallel and cone beam.  Same contract and arithmetic as the
// general bp_kernel (back_project.cuh); organised to minimise instructions per (pixel, slice, view):
//
//  * CTA = 256 threads = 8 warps; lanes run along 32 pixels, warps along slice tiles (or along further pixel
//    groups when the cylinder has fewer than 8 tiles).  The tile height ts <= 16 is chosen so that the tiles
//    split the slices evenly over a power-of-two number of warps; accumulators stay in registers.
//  * Per chunk of views, each (pixel, view) footprint is computed once, by one thread, into shared memory as
//    one float4 and read by every warp of that pixel: the first of three consecutive detector channels that
//    hold every nonzero tap and their coefficients (already raised to coeff_power; at the detector edges the
//    taps are shifted onto in-range channels with a zero coefficient, so every gather is three loads at
//    constant offsets from one pointer), plus for cone beam the affine map slice -> detector row
//    m_p(k) = A0 + k*A1 and the vertical-angle factor c2 = (mag/D)^2 so that 1/cos(phi_k) = sqrt(1 + c2 z_k^2).
//    The cone footprint is trig-free: cos/sin(theta - theta_p) and 1/cos(theta_p) come from the per-view
//    cos/sin and rsqrt(D^2 + u^2) instead of atan2/cos/sin per pixel.
//  * Cone: every detector row a warp's slice tile touches is gathered once per view into the thread's column
//    of a shared-memory row cache ([row][thread], conflict-free), rows outside the detector cached as 0; the
//    vertical fan then reads three cached rows per slice with no bounds tests.  plan_bp_fast admits a geometry
//    only when the rows of a slice tile (ts * max |dm/dk| + 4) fit the cache.
#pragma once

#include "back_project.cuh"

namespace mbx {

constexpr int BPF_THREADS = 256;
#ifndef MBX_BPF_ST
#define MBX_BPF_ST 16
#endif
constexpr int BPF_ST = MBX_BPF_ST;  // most slices per thread
constexpr int BPF_CACHE_ROWS = 48;  // row-cache depth per thread (cone): ts * max|dm/dk| + 4 must fit
#ifndef MBX_BPF_CHUNK_PARALLEL
#define MBX_BPF_CHUNK_PARALLEL 1024     // footprints staged per view chunk, parallel beam
#endif
#ifndef MBX_BPF_CHUNK_CONE
#define MBX_BPF_CHUNK_CONE 512          // same, cone beam (its row cache takes most of the shared memory)
#endif
#ifndef MBX_BPF_PREFETCH
#define MBX_BPF_PREFETCH 2              // parallel beam, staged footprints: views ahead whose rows are prefetched
#endif                                  // into L1 while the current view is gathered (0: none; 1, 2 and 4 measure
                                        // the same, 8.5% faster than none on the batched bench stage)

struct BpfPlan {
    int nsl;      // slice tiles per CTA (warps per pixel group)
    int npg;      // pixel groups of 32 per CTA
    int lg_pcta;  // log2(32 * npg)
    int chunk;    // footprints staged per view chunk (a multiple of BPF_THREADS); 0 with inline footprints
    int vc;       // views per chunk = chunk / (32 * npg); with inline footprints, views per table refill
    int inline_fp;  // 1: each thread computes its own pixel's footprints in registers (no staging, no barriers
                    // inside a view table); pays off when few warps share a pixel (short cylinders)
    int ts;       // slices per tile (<= BPF_ST)
    int tiles;    // ceil(S / ts)
    int gx, gy, splits, views_per_split;
    size_t smem, workspace;
    bool ok;
};

// Footprint of one (pixel, view): fa = {first channel (int bits; -1: no tap), c0, c1, c2} for the channels
// first, first+1, first+2; fb (cone) = {A0, A1, c2 = (mag/D)^2, 0}.
template <int KIND>
__device__ __forceinline__ void bpf_footprint(const mbx_geom &g, float cs, float sn, float x_tilde, float y_tilde,
                                              int coeff_power, float4 &fa, float4 &fb, float tz = 0.0f) {
    const float inv_dc = 1.0f / g.delta_det_channel;
    const int num_channels = g.num_det_channels;
    const float det_center_channel = 0.5f * (float)(num_channels - 1);
    float n_p, w, scale;  // scale = delta_voxel / cos_alpha
    fb = make_float4(0.f, 0.f, 0.f, 0.f);
    if (KIND == MBX_GEOM_TRANSLATION) {
        // (cs, sn) carry the view's (tx, ty); no rotation (translation_model.py:595-656).  Coefficient
        // L / cos(theta_p), no delta_voxel factor; the vertical fan is the cone's with slice heights
        // delta_voxel k + z0v, z0v = -tz - delta_voxel (S-1)/2, which fb.w carries.
        const float x_p = x_tilde - cs;
        const float y_p = y_tilde - sn;
        const float inv_d = 1.0f / g.source_detector_dist;
        const float mag = 1.0f / (1.0f / g.magnification - y_p * inv_d);
        const float u = mag * x_p;
        n_p = (u + g.det_channel_offset) * inv_dc + det_center_channel;
        const float t = u * inv_d;
        const float cos_tp = rsqrtf(fmaf(t, t, 1.0f));
        w = mag * (g.delta_voxel * inv_dc);
        scale = 1.0f / cos_tp;
        const float inv_dr = 1.0f / g.delta_det_row;
        const float z0v = -tz - g.delta_voxel * (0.5f * (float)(g.num_recon_slices - 1));
        const float mr = mag * inv_d;
        fb.x = (mag * z0v + g.det_row_offset) * inv_dr + 0.5f * (float)(g.num_det_rows - 1);
        fb.y = mag * g.delta_voxel * inv_dr;
        fb.z = mr * mr;
        fb.w = z0v;
    } else if (KIND == MBX_GEOM_PARALLEL) {
        const float x = cs * x_tilde - sn * y_tilde;
        n_p = (x + g.det_channel_offset) * inv_dc + det_center_channel;
        const float cos_alpha = fmaxf(fabsf(cs), fabsf(sn));
        w = (g.delta_voxel * inv_dc) * cos_alpha;
        scale = g.delta_voxel / cos_alpha;
    } else {
        const float x_p = cs * x_tilde - sn * y_tilde;
        const float y_p = sn * x_tilde + cs * y_tilde;
        const float inv_d = isinf(g.source_detector_dist) ? 0.0f : 1.0f / g.source_detector_dist;
        const float mag = 1.0f / (1.0f / g.magnification - y_p * inv_d);
        const float u = mag * x_p;
        n_p = (u + g.det_channel_offset) * inv_dc + det_center_channel;
        // theta_p = atan2(u, D): cos = D / h, sin = u / h with h = sqrt(D^2 + u^2)  (D = inf: cos 1, sin 0)
        const float t = u * inv_d;
        const float inv_h = rsqrtf(fmaf(t, t, 1.0f));                    // cos(theta_p)
        const float cos_tp = inv_h, sin_tp = t * inv_h;
        const float cd = cs * cos_tp + sn * sin_tp;                       // cos(theta - theta_p)
        const float sd = sn * cos_tp - cs * sin_tp;                       // sin(theta - theta_p)
        const float cos_alpha = fmaxf(fabsf(cd), fabsf(sd));
        w = mag * (g.delta_voxel * inv_dc) * (cos_alpha / cos_tp);
        scale = g.delta_voxel / cos_alpha;
        const float inv_dr = 1.0f / g.delta_det_row;
        const float center_slice = 0.5f * (float)(g.num_recon_slices - 1);
        const float z0 = g.recon_slice_offset - g.delta_voxel * center_slice;
        const float mr = mag * inv_d;
        fb.x = (mag * z0 + g.det_row_offset) * inv_dr + 0.5f * (float)(g.num_det_rows - 1);
        fb.y = mag * g.delta_voxel * inv_dr;
        fb.z = mr * mr;
    }
    const int nc = (int)rintf(n_p);
    const float half_w = (w + 1.0f) * 0.5f;
    const float l_max = fminf(1.0f, w);
    const float d = n_p - (float)nc;
    float a[3];
#pragma unroll
    for (int k = -1; k <= 1; ++k) {
        const int n = nc + k;
        float v = scale * fminf(fmaxf(half_w - fabsf(d - (float)k), 0.0f), l_max);
        if (n < 0 || n >= num_channels) v = 0.0f;
        a[k + 1] = (coeff_power == 2) ? v * v : v;
    }
    // channels first..first+2 on the detector; tap k of the pixel sits at position k - (first - (nc - 1))
    const int lo = nc - 1;
    const int first = min(max(lo, 0), num_channels - 3);
    const int sh = first - lo;
    float c[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const int j = k + sh;
        c[k] = (j == 0) ? a[0] : ((j == 1) ? a[1] : ((j == 2) ? a[2] : 0.0f));
    }
    const bool any = c[0] != 0.0f || c[1] != 0.0f || c[2] != 0.0f;
    fa = make_float4(__int_as_float(any ? first : -1), c[0], c[1], c[2]);
}

// Pixel position relative to the recon centre (ALU): x from the column, y from the row (translation geometry
// spaces rows by delta_recon_row).
template <int KIND>
__device__ __forceinline__ void bpf_pixel(const mbx_geom &g, int idx, float &x_tilde, float &y_tilde) {
    if (KIND == MBX_GEOM_TRANSLATION) {
        const int row = idx / g.num_recon_cols;
        const int col = idx - row * g.num_recon_cols;
        x_tilde = g.delta_voxel * ((float)col - 0.5f * (float)(g.num_recon_cols - 1));
        y_tilde = g.delta_recon_row * ((float)row - 0.5f * (float)(g.num_recon_rows - 1));
    } else {
        pixel_tilde(g, idx, x_tilde, y_tilde);
    }
}

// Arguments of one back projection (one scan).
struct BpArgs {
    mbx_geom g;
    const float *sino;         // full sinogram (num_views, R, C)
    const float *wts;          // optional weights, same shape (NULL: ones)
    const int32_t *pix;        // (num_pixels,) flat pixel indices
    long long num_pixels;
    const int32_t *order;      // optional permutation of [0, num_pixels): processing order (locality)
    const int32_t *views;      // (num_views_sel,) or NULL
    int num_views_sel, views_per_split, coeff_power;
    float scale;
    float *out;                // (num_pixels, S) in list order, or a flat recon when out_by_index
    long long split_stride;    // 0: final output; else partial-sum workspace stride
    int out_by_index;
    int out_slices;            // > 0: g has one slice and its value is written to all out_slices slices of the
                               // output cylinder (the unit-weight Hessian of parallel beam, equal in every slice)
    BpfPlan plan;
};

// Parallel beam with neither sinogram nor weights (the unit-weight Hessian diagonal): every detector row holds the
// same ones and every slice the same footprints, so all slices of a pixel receive the same sum of the same terms
// in the same order.  The back projection is then planned on one slice (one_slice_geometry) and that value is
// written to every slice.
inline bool bp_unit_broadcast(const mbx_geom &g, const float *sino, const float *wts) {
    return g.kind == MBX_GEOM_PARALLEL && !sino && !wts && g.num_recon_slices > 1;
}

inline mbx_geom one_slice_geometry(const mbx_geom &g) {
    mbx_geom g1 = g;
    g1.num_recon_slices = 1;
    return g1;
}

// Parallel-beam gather of one view into the first TS accumulators: three taps at constant offsets from one
// 32-bit element offset, one detector row per slice (TS = the tile's slice count, so no slot is predicated off).
template <int TS>
__device__ __forceinline__ void bpf_gather_rows(float (&acc)[BPF_ST], const float *__restrict__ sino, int o,
                                                int num_channels, const float4 &fa) {
#pragma unroll
    for (int s = 0; s < TS; ++s) {
        const float *q = sino + o;
        acc[s] = fmaf(fa.y, __ldg(q), fmaf(fa.z, __ldg(q + 1), fmaf(fa.w, __ldg(q + 2), acc[s])));
        o += num_channels;
    }
}

// The same for a tile of TS slices when TS fits the accumulators (other TS never occur: ns <= ts <= BPF_ST).
template <int TS>
__device__ __forceinline__ void bpf_gather_ts(float (&acc)[BPF_ST], const float *__restrict__ sino, int o,
                                              int num_channels, const float4 &fa) {
    if constexpr (TS <= BPF_ST) bpf_gather_rows<TS>(acc, sino, o, num_channels, fa);
}

template <int KIND>
__device__ void bp_fast_tile(const BpArgs &A, int bx, int by, int bz, float *smf, int *err) {
    const mbx_geom &g = A.g;
    const BpfPlan &P = A.plan;
    const float *__restrict__ sino = A.sino;
    const float *__restrict__ wts = A.wts;
    const int32_t *__restrict__ pix = A.pix;
    const long long num_pixels = A.num_pixels;
    const int32_t *__restrict__ views = A.views;
    const int num_views_sel = A.num_views_sel, views_per_split = A.views_per_split, coeff_power = A.coeff_power;
    const int nsl = P.nsl, vc = P.vc, lg_pcta = P.lg_pcta, chunk = P.chunk;
    const int pcta = 1 << lg_pcta;                  // pixels per CTA
    float4 *s_fa = reinterpret_cast<float4 *>(smf);  // [chunk] = [view in chunk][pixel]
    float4 *s_fb = s_fa + chunk;                     // cone: [chunk]
    float *s_cs = reinterpret_cast<float *>(s_fa + (KIND != MBX_GEOM_PARALLEL ? 2 : 1) * chunk);
    float *s_sn = s_cs + vc;
    int *s_voff = reinterpret_cast<int *>(s_sn + vc);      // element offset of each view (-1: invalid view)
    float *s_tz = reinterpret_cast<float *>(s_voff + vc);   // translation: tz of each view
    float *cache = s_tz + (KIND == MBX_GEOM_TRANSLATION ? vc : 0);  // [BPF_CACHE_ROWS][BPF_THREADS] (cone, transl.)

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int pg = warp / nsl, stl = warp - pg * nsl;
    const int pl = pg * 32 + lane;                                   // pixel within CTA
    const long long slot = (long long)bx * pcta + pl;
    const long long p = (A.order && slot < num_pixels) ? A.order[slot] : slot;  // list entry of this thread
    const int s0 = (by * nsl + stl) * P.ts;
    const int num_rows = g.num_det_rows, num_channels = g.num_det_channels, num_slices = g.num_recon_slices;
    const int ns = min(P.ts, num_slices - s0);
    const int split = bz;
    const int v_begin = split * views_per_split;
    const int v_end = min(num_views_sel, v_begin + views_per_split);
    const int npix_grid = g.num_recon_rows * g.num_recon_cols;
    const int view_stride = num_rows * num_channels;  // plan_bp_fast admits sinograms of < 2^31 elements
    const int s0c = s0 * num_channels;

    // pixel geometry of the pixel this thread computes footprints for (pixel tid % pcta of every view)
    const int fpl = tid & (pcta - 1);
    const long long fp_slot = (long long)bx * pcta + fpl;
    const long long fp_pixel = (A.order && fp_slot < num_pixels) ? A.order[fp_slot] : fp_slot;
    float fxt = 0.0f, fyt = 0.0f;
    bool fvalid = false;
    if (fp_pixel < num_pixels) {
        const int idx = pix[fp_pixel];
        if (idx >= 0 && idx < npix_grid) {
            bpf_pixel<KIND>(g, idx, fxt, fyt);
            fvalid = true;
        } else if (by == 0 && split == 0 && tid < pcta) {
            flag_error(err, MBX_ERRFLAG_PIXEL);
        }
    }
    bool active = p < num_pixels && ns > 0;
    float oxt = 0.0f, oyt = 0.0f;  // this thread's own pixel (inline footprints)
    if (active) {
        const int idx = pix[p];
        active = idx >= 0 && idx < npix_grid;
        if (active) bpf_pixel<KIND>(g, idx, oxt, oyt);
    }

    float acc[BPF_ST];
#pragma unroll
    for (int s = 0; s < BPF_ST; ++s) acc[s] = 0.0f;

    const float z0 = g.recon_slice_offset - g.delta_voxel * 0.5f * (float)(num_slices - 1);
    float *mycache = cache + tid;

    // gather of one view into the accumulators, from the footprint fa (+ fb for cone) at view offset voff
    auto gather = [&](const float4 &fa, const float4 &fb, int voff) {
        const int first = __float_as_int(fa.x);
        if (KIND == MBX_GEOM_PARALLEL) {
            // three taps at constant offsets from one 32-bit element offset, one detector row per slice
            int o = voff + s0c + first;
            if (!sino) {  // unit sinogram: the same additions as gathering ones (unit-weight Hessian)
#pragma unroll
                for (int s = 0; s < BPF_ST; ++s)
                    if (s < ns) acc[s] = fa.y + (fa.z + (fa.w + acc[s]));
            } else if (wts) {
#pragma unroll
                for (int s = 0; s < BPF_ST; ++s) {
                    if (s < ns) {
                        const float *q = sino + o, *qw = wts + o;
                        acc[s] = fmaf(fa.y, __ldg(q) * __ldg(qw),
                                      fmaf(fa.z, __ldg(q + 1) * __ldg(qw + 1), fmaf(fa.w, __ldg(q + 2) * __ldg(qw + 2), acc[s])));
                    }
                    o += num_channels;
                }
            } else {
                switch (ns) {  // the same for every lane of the warp (a warp holds one slice tile)
                    case 1: bpf_gather_ts<1>(acc, sino, o, num_channels, fa); break;
                    case 2: bpf_gather_ts<2>(acc, sino, o, num_channels, fa); break;
                    case 3: bpf_gather_ts<3>(acc, sino, o, num_channels, fa); break;
                    case 4: bpf_gather_ts<4>(acc, sino, o, num_channels, fa); break;
                    case 5: bpf_gather_ts<5>(acc, sino, o, num_channels, fa); break;
                    case 6: bpf_gather_ts<6>(acc, sino, o, num_channels, fa); break;
                    case 7: bpf_gather_ts<7>(acc, sino, o, num_channels, fa); break;
                    case 8: bpf_gather_ts<8>(acc, sino, o, num_channels, fa); break;
                    case 9: bpf_gather_ts<9>(acc, sino, o, num_channels, fa); break;
                    case 10: bpf_gather_ts<10>(acc, sino, o, num_channels, fa); break;
                    case 11: bpf_gather_ts<11>(acc, sino, o, num_channels, fa); break;
                    case 12: bpf_gather_ts<12>(acc, sino, o, num_channels, fa); break;
                    case 13: bpf_gather_ts<13>(acc, sino, o, num_channels, fa); break;
                    case 14: bpf_gather_ts<14>(acc, sino, o, num_channels, fa); break;
                    case 15: bpf_gather_ts<15>(acc, sino, o, num_channels, fa); break;
                    default: bpf_gather_rows<BPF_ST>(acc, sino, o, num_channels, fa); break;
                }
            }
        } else {
            const float A0 = fb.x, A1 = fb.y, c2 = fb.z;
            const float half_w = (A1 + 1.0f) * 0.5f;
            const float l_max = fminf(1.0f, A1);
            const int mc_first = (int)rintf(fmaf((float)s0, A1, A0));
            const int mc_last = (int)rintf(fmaf((float)(s0 + ns - 1), A1, A0));
            const int m_lo = min(mc_first, mc_last) - 1;
            const int m_hi = max(mc_first, mc_last) + 1;
            if (m_hi - m_lo + 1 > BPF_CACHE_ROWS) {  // excluded by plan_bp_fast; never read past the cache
                flag_error(err, MBX_ERRFLAG_CACHE);
                return;
            }
            for (int m = m_lo; m <= m_hi; ++m) {
                float c = 0.0f;
                if (m >= 0 && m < num_rows) {
                    const int o = voff + m * num_channels + first;
                    const float *q = sino + o;
                    if (!sino) {  // unit sinogram
                        c = fa.y + (fa.z + fa.w);
                    } else if (wts) {
                        const float *qw = wts + o;
                        c = fmaf(fa.y, __ldg(q) * __ldg(qw), fmaf(fa.z, __ldg(q + 1) * __ldg(qw + 1), fa.w * (__ldg(q + 2) * __ldg(qw + 2))));
                    } else {
                        c = fmaf(fa.y, __ldg(q), fmaf(fa.z, __ldg(q + 1), fa.w * __ldg(q + 2)));
                    }
                }
                mycache[(m - m_lo) * BPF_THREADS] = c;
            }
#pragma unroll
            for (int s = 0; s < BPF_ST; ++s) {
                if (s < ns) {
                    const float k = (float)(s0 + s);
                    const float m_p = fmaf(k, A1, A0);
                    const int m_c = (int)rintf(m_p);
                    const float d = m_p - (float)m_c;
                    const float z = fmaf(k, g.delta_voxel, KIND == MBX_GEOM_TRANSLATION ? fb.w : z0);
                    const float q = fmaf(c2, z * z, 1.0f);
                    float sec = q * rsqrtf(q);                       // 1 / cos(phi_k)
                    const float l_m = fminf(fmaxf(half_w - fabsf(d + 1.0f), 0.0f), l_max);
                    const float l_0 = fminf(fmaxf(half_w - fabsf(d), 0.0f), l_max);
                    const float l_p = fminf(fmaxf(half_w - fabsf(d - 1.0f), 0.0f), l_max);
                    const float *cc = mycache + (m_c - m_lo) * BPF_THREADS;
                    const float cm = cc[-BPF_THREADS], c0 = cc[0], cp = cc[BPF_THREADS];
                    if (coeff_power == 2) {
                        sec *= sec;
                        acc[s] = fmaf(sec, fmaf(l_m * l_m, cm, fmaf(l_0 * l_0, c0, (l_p * l_p) * cp)), acc[s]);
                    } else {
                        acc[s] = fmaf(sec, fmaf(l_m, cm, fmaf(l_0, c0, l_p * cp)), acc[s]);
                    }
                }
            }
        }
    };

    // per-view table of a chunk of views: angle cos/sin and element offset (-1: invalid view)
    auto fill_views = [&](int vb, int nv) {
        for (int t = tid; t < nv; t += BPF_THREADS) {
            const int vi = views ? views[vb + t] : vb + t;
            const bool ok = vi >= 0 && vi < g.num_views;
            if (!ok && bx == 0 && by == 0) flag_error(err, MBX_ERRFLAG_VIEW);
            s_voff[t] = ok ? vi * view_stride : -1;
            if (KIND == MBX_GEOM_TRANSLATION) {  // (tx, ty) in the (cos, sin) slots, tz in its own table
                s_cs[t] = ok ? g.translations[3 * vi] : 0.0f;
                s_sn[t] = ok ? g.translations[3 * vi + 1] : 0.0f;
                s_tz[t] = ok ? g.translations[3 * vi + 2] : 0.0f;
            } else {
                const float ang = ok ? g.angles[vi] : 0.0f;
                s_cs[t] = cosf(ang);
                s_sn[t] = sinf(ang);
            }
        }
    };

    if (P.inline_fp) {
        for (int vb = v_begin; vb < v_end; vb += vc) {
            const int nv = min(vc, v_end - vb);
            __syncthreads();
            fill_views(vb, nv);
            __syncthreads();
            if (!active) continue;
            for (int t = 0; t < nv; ++t) {
                const int voff = s_voff[t];
                if (voff < 0) continue;
                float4 fa, fb;
                bpf_footprint<KIND>(g, s_cs[t], s_sn[t], oxt, oyt, coeff_power, fa, fb,
                                    KIND == MBX_GEOM_TRANSLATION ? s_tz[t] : 0.0f);
                if (__float_as_int(fa.x) >= 0) gather(fa, fb, voff);
            }
        }
    } else {
        for (int vb = v_begin; vb < v_end; vb += vc) {
            const int nv = min(vc, v_end - vb);
            __syncthreads();
            fill_views(vb, nv);
            __syncthreads();
            for (int f = tid; f < chunk; f += BPF_THREADS) {
                const int t = f >> lg_pcta;
                if (t < nv) {
                    float4 fa = make_float4(__int_as_float(-1), 0.f, 0.f, 0.f), fb = make_float4(0.f, 0.f, 0.f, 0.f);
                    if (fvalid && s_voff[t] >= 0)
                        bpf_footprint<KIND>(g, s_cs[t], s_sn[t], fxt, fyt, coeff_power, fa, fb,
                                            KIND == MBX_GEOM_TRANSLATION ? s_tz[t] : 0.0f);
                    s_fa[f] = fa;
                    if (KIND != MBX_GEOM_PARALLEL) s_fb[f] = fb;
                }
            }
            __syncthreads();
            if (!active) continue;
            for (int t = 0; t < nv; ++t) {
                const int f = (t << lg_pcta) + pl;
                if (MBX_BPF_PREFETCH > 0 && KIND == MBX_GEOM_PARALLEL && sino && t + MBX_BPF_PREFETCH < nv) {
                    // the rows of a later view of the chunk: start their L2 -> L1 fills now, so that its gathers
                    // hit L1 (a prefetch writes no register and faults on no address; the view and channel are
                    // checked as for the gather).  (One prefetch per lane and view, of the warp's lowest and
                    // highest tap line per row, was 7% slower on the batched stage than this one per slice.)
                    const int tn = t + MBX_BPF_PREFETCH;
                    const int first_n = __float_as_int(s_fa[(tn << lg_pcta) + pl].x);
                    const int voff_n = s_voff[tn];
                    if (first_n >= 0 && voff_n >= 0) {
                        const float *q = sino + (voff_n + s0c + first_n);
                        for (int s = 0; s < ns; ++s, q += num_channels)
                            asm volatile("prefetch.global.L1 [%0];" ::"l"(q));
                    }
                }
                const float4 fa = s_fa[f];
                if (__float_as_int(fa.x) < 0) continue;
                gather(fa, KIND != MBX_GEOM_PARALLEL ? s_fb[f] : make_float4(0.f, 0.f, 0.f, 0.f), s_voff[t]);
            }
        }
    }
    if (p >= num_pixels || ns <= 0) return;
    long long row_of_out = p;
    if (A.out_by_index) {  // write into a flat recon at the pixel's index (skipped for invalid indices)
        if (!active) return;
        row_of_out = pix[p];
    }
    const float sc = (A.split_stride == 0) ? A.scale : 1.0f;
    if (A.out_slices > 0) {  // the one slice's value in every slice of the cylinder
        float *out = A.out + row_of_out * (long long)A.out_slices;
        const float v = active ? sc * acc[0] : 0.0f;
        for (int s = 0; s < A.out_slices; ++s) out[s] = v;
        return;
    }
    float *out = A.out + (long long)split * A.split_stride + row_of_out * (long long)num_slices + s0;
#pragma unroll
    for (int s = 0; s < BPF_ST; ++s)
        if (s < ns) out[s] = active ? sc * acc[s] : 0.0f;
}

template <int KIND>
__global__ void __launch_bounds__(BPF_THREADS, 3) bp_fast_kernel(const BpArgs A, int *err) {
    extern __shared__ __align__(16) float smf[];
    bp_fast_tile<KIND>(A, blockIdx.x, blockIdx.y, blockIdx.z, smf, err);
}

// inline_fp: 1 for the variant that computes footprints per thread in registers (see BpfPlan::inline_fp).
inline BpfPlan plan_bp_fast(const mbx_geom &g, long long num_pixels, int num_views_sel, int inline_fp = 0) {
    BpfPlan pl;
    pl.inline_fp = inline_fp;
    // 32-bit element offsets address the sinogram
    pl.ok = (g.kind == MBX_GEOM_PARALLEL || g.kind == MBX_GEOM_CONE ||
             (g.kind == MBX_GEOM_TRANSLATION && g.max_magnification > 0.0f)) &&
            (g.psf_radius == 1) && g.num_det_channels >= 3 &&
            (long long)g.num_views * g.num_det_rows * g.num_det_channels < (1LL << 31);
    const int S = g.num_recon_slices;
    // tile height: the fewest tiles of <= BPF_ST slices, rounded up to a power of two (<= 8) or a multiple of 8,
    // then the slices spread evenly over them
    const int t0 = ceil_div(S, BPF_ST);
    int T = 1;
    if (t0 <= 8) {
        while (T < t0) T <<= 1;
    } else {
        T = ceil_div(t0, 8) * 8;
    }
    pl.ts = ceil_div(S, T);
    pl.tiles = ceil_div(S, pl.ts);
    pl.nsl = 1;
    while (pl.nsl < pl.tiles && pl.nsl < 8) pl.nsl <<= 1;
    pl.npg = 8 / pl.nsl;
    pl.lg_pcta = 5;
    while ((1 << pl.lg_pcta) < 32 * pl.npg) ++pl.lg_pcta;
    const int pcta = 32 * pl.npg;
    pl.chunk = (g.kind != MBX_GEOM_PARALLEL) ? MBX_BPF_CHUNK_CONE : MBX_BPF_CHUNK_PARALLEL;
    if (pl.chunk < pcta) pl.chunk = pcta;
    pl.vc = pl.chunk / pcta;
    if (inline_fp) {  // no staged footprints; a view table of up to 1024 views per refill
        pl.chunk = 0;
        pl.vc = 1024;
    }
    pl.gx = ceil_div(num_pixels > 0 ? num_pixels : 1, pcta);
    pl.gy = ceil_div(pl.tiles, pl.nsl);
    if (g.kind == MBX_GEOM_CONE) {
        // the row cache must hold the rows of a slice tile: ts * max |dm/dk| + 4
        const double half_r = 0.5 * (g.num_recon_rows - 1), half_c = 0.5 * (g.num_recon_cols - 1);
        const double rho = g.delta_voxel * std::sqrt(half_r * half_r + half_c * half_c);
        const double inv = 1.0 / g.magnification - (std::isinf(g.source_detector_dist) ? 0.0 : rho / g.source_detector_dist);
        const double max_mag = inv > 1e-6 ? 1.0 / inv : 1e6;
        const double slope = max_mag * g.delta_voxel / g.delta_det_row;
        if (pl.ts * slope + 4 > BPF_CACHE_ROWS) pl.ok = false;
    } else if (g.kind == MBX_GEOM_TRANSLATION) {  // same bound from the host's magnification bound
        const double slope = (double)g.max_magnification * g.delta_voxel / g.delta_det_row;
        if (pl.ts * slope + 4 > BPF_CACHE_ROWS) pl.ok = false;
    }
    const long long base = (long long)pl.gx * pl.gy;
    const int sms = num_sms();
    long long splits = 1;
    if (base < 2LL * sms && num_views_sel >= 16) {
        splits = (2LL * sms + base - 1) / base;
        long long maxs = num_views_sel / 8;
        if (splits > maxs) splits = maxs;
        if (splits > 64) splits = 64;
        if (splits < 1) splits = 1;
    }
    pl.views_per_split = ceil_div(num_views_sel, splits);
    pl.splits = ceil_div(num_views_sel, pl.views_per_split);
    pl.smem = (size_t)pl.chunk * 16 * (g.kind != MBX_GEOM_PARALLEL ? 2 : 1) +
              (size_t)pl.vc * (g.kind == MBX_GEOM_TRANSLATION ? 16 : 12) +
              (g.kind != MBX_GEOM_PARALLEL ? (size_t)BPF_CACHE_ROWS * BPF_THREADS * 4 : 0);
    pl.workspace = pl.splits > 1 ? align256((size_t)pl.splits * num_pixels * S * 4) : 0;
    return pl;
}

}  // namespace mbx
