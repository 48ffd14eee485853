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
// The set-up of every scan (direct-recon initialisation, alpha rescale, Hessian diagonal) runs as batched stages
// too (mbx_vcd_batched_setup), over three more projection work lists (initial back and forward projection over
// each scan's region of reconstruction, Hessian back projection over every pixel).  The per-call parameters
// (regularisation, schedule, partitions) live in device tables that mbx_vcd_batched_update and
// mbx_vcd_batched_refresh rewrite, so a prepared plan, and graphs captured from it, serve every call of a batch
// shape.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "direct_filter.cuh"
#include "vcd_batched.cuh"

namespace mbx {

template <int KIND>
__global__ void __launch_bounds__(BPF_THREADS, MBX_BBP_MIN_BLOCKS) b_bp(ProjList L, int num_scans, int step, int first, int total, int *err) {
    extern __shared__ __align__(16) float smb[];
    for (int t = first + fetch_tile(L.counter); t < total; t = first + fetch_tile(L.counter)) {
        const int k = find_scan(L.off, num_scans, t);
        const int s = __ldg(L.order + k);
        const int local = t - __ldg(L.off + k);
        const int gx = __ldg(L.dim + s);
        bp_fast_tile<KIND>(list_record(L.bp, L, num_scans, step, s), local % gx, local / gx, 0, smb, err);
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
        const QParams q = T.qp[s];
        const float fm = T.fm[s];
        double pl = 0.0, pq = 0.0;
        for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) {
            int k;
            const long long p = div_rem(i, sc.ns, k);
            const int idx = pix[p];
            float d = 0.0f;
            if (idx < 0 || idx >= npix) {
                flag_error(err, MBX_ERRFLAG_PIXEL);
            } else {
                float gp, hp;
                qggmrf_voxel(sc.recon, sc.nr, sc.nc, sc.ns, idx, k, q, gp, hp);
                const float gf = -fm * sc.bp[i];
                const float hf = fm * __ldg(sc.hess + (long long)idx * sc.ns + k);
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
        // four elements per load when the scan's buffers are 16-byte aligned (tile starts are), the rest one by one
        const bool vec = (((uintptr_t)sc.dsino | (uintptr_t)sc.err | (uintptr_t)sc.wts) & 15) == 0;
        const long long full = vec ? e0 + ((e1 - e0) & ~3LL) : e0;
        const float4 *ds4 = reinterpret_cast<const float4 *>(sc.dsino), *e4 = reinterpret_cast<const float4 *>(sc.err);
        const float4 *w4 = reinterpret_cast<const float4 *>(sc.wts);
        for (long long j = e0 / 4 + threadIdx.x; j < full / 4; j += BT_THREADS) {
            const float4 ds = __ldg(ds4 + j), e = __ldg(e4 + j);
            const float4 w = sc.wts ? __ldg(w4 + j) : make_float4(1.0f, 1.0f, 1.0f, 1.0f);
            fl += (double)((w.x * e.x) * ds.x);
            fq += (double)(ds.x * ds.x * w.x);
            fl += (double)((w.y * e.y) * ds.y);
            fq += (double)(ds.y * ds.y * w.y);
            fl += (double)((w.z * e.z) * ds.z);
            fq += (double)(ds.z * ds.z * w.z);
            fl += (double)((w.w * e.w) * ds.w);
            fq += (double)(ds.w * ds.w * w.w);
        }
        for (long long i = full + threadIdx.x; i < e1; i += BT_THREADS) {
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
    const int eb = __ldg(T.el_off + s), ee = __ldg(T.el_off + s + 1);
    const int sb = __ldg(T.sn_off + s), se = __ldg(T.sn_off + s + 1);
    const double pl = warp_range_sum(T.p_prior, eb, ee, 2, 0);
    const double pq = 0.5 * warp_range_sum(T.p_prior, eb, ee, 2, 1);
    const double fm = (double)T.fm[s];
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
            int k;
            const long long p = div_rem(i, sc.ns, k);
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
        // four elements per load when the scan's buffers are 16-byte aligned (tile starts are), the rest one by one
        const bool vec = (((uintptr_t)sc.dsino | (uintptr_t)sc.err) & 15) == 0;
        const long long full = vec ? e0 + ((e1 - e0) & ~3LL) : e0;
        float4 *e4 = reinterpret_cast<float4 *>(sc.err);
        const float4 *ds4 = reinterpret_cast<const float4 *>(sc.dsino);
        for (long long j = e0 / 4 + threadIdx.x; j < full / 4; j += BT_THREADS) {
            float4 e = e4[j];
            const float4 d = __ldg(ds4 + j);
            e.x -= alpha * d.x;
            e.y -= alpha * d.y;
            e.z -= alpha * d.z;
            e.w -= alpha * d.w;
            e4[j] = e;
        }
        for (long long i = full + threadIdx.x; i < e1; i += BT_THREADS) sc.err[i] -= alpha * sc.dsino[i];
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

// ------------------------------------------------------------------------------------------------ set-up stages
// The reference's vcd_recon set-up (tomography_model.py:1110-1152) for every scan: x0 = direct recon, then
// alpha = <W A x0, y> / <W A x0, A x0> (1 when the denominator is 0), e = y - alpha A x0, x = alpha x0, and the
// Hessian diagonal.  The float32 products match TomographyModel._vcd_setup (W A x0 rounded to float32, sums in
// float64, alpha rounded to float32, then y - (alpha A x0) and alpha x0 each rounded once, without contraction).

// Zero every scan's flat recon (the direct recon is zero outside the region of reconstruction).
__global__ void __launch_bounds__(BT_THREADS) b_zero_recon(BatchedTables T, int num_scans, int total) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int s = find_scan(T.rc_off, num_scans, t);
        const int local = t - __ldg(T.rc_off + s);
        const VcdScan &sc = T.scans[s];
        const long long e0 = (long long)local * BT_SINO_TILE, e1 = min(sc.nrecon, e0 + BT_SINO_TILE);
        for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) sc.recon[i] = 0.0f;
    }
}

// FBP / FDK filtering of every scan's sinogram, FILT_ROWS detector rows per tile (direct_filter_rows).
__global__ void __launch_bounds__(FILT_THREADS) b_filter(BatchedTables T, int num_scans, int total) {
    extern __shared__ __align__(16) float smflt[];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int s = find_scan(T.flt_off, num_scans, t);
        const int local = t - __ldg(T.flt_off + s);
        const FiltScan &f = T.filt[s];
        direct_filter_rows(f.in, f.out, (long long)local * FILT_ROWS, f.rows, f.R, f.C, f.filter_scale, f.out_scale,
                           f.fdk, f.D, f.ddc, f.ddr, f.dco, f.dro, smflt);
    }
}

// float64 partials of <W A x0, A x0> and <W A x0, y> per sinogram tile (A x0 is in dsino).
__global__ void __launch_bounds__(BT_THREADS) b_init_partials(BatchedTables T, int num_scans, int total) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int s = find_scan(T.sn_off, num_scans, t);
        const int local = t - __ldg(T.sn_off + s);
        const VcdScan &sc = T.scans[s];
        const long long e0 = (long long)local * BT_SINO_TILE, e1 = min(sc.nsino, e0 + BT_SINO_TILE);
        double den = 0.0, num = 0.0;
        for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) {
            const float ax = sc.dsino[i];
            const float wes = sc.wts ? __fmul_rn(sc.wts[i], ax) : ax;
            den += (double)wes * (double)ax;
            num += (double)wes * (double)sc.y[i];
        }
        const double v[2] = {den, num};
        tile_reduce<2>(v, T.p_init + 2 * t);
    }
}

__global__ void b_init_alpha(BatchedTables T, int num_scans) {
    const int s = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (s >= num_scans) return;
    const int sb = __ldg(T.sn_off + s), se = __ldg(T.sn_off + s + 1);
    const double den = warp_range_sum(T.p_init, sb, se, 2, 0);
    const double num = warp_range_sum(T.p_init, sb, se, 2, 1);
    if ((threadIdx.x & 31) == 0) T.alpha_init[s] = den > 0.0 ? (float)(num / den) : 1.0f;
}

// e = y - alpha A x0 over the sinogram tiles, then x = alpha x0 over the recon tiles.
__global__ void __launch_bounds__(BT_THREADS) b_init_apply(BatchedTables T, int num_scans, int total_sn,
                                                           int total_rc) {
    for (int t = blockIdx.x; t < total_sn + total_rc; t += gridDim.x) {
        if (t < total_sn) {
            const int s = find_scan(T.sn_off, num_scans, t);
            const int local = t - __ldg(T.sn_off + s);
            const VcdScan &sc = T.scans[s];
            const float a = T.alpha_init[s];
            const long long e0 = (long long)local * BT_SINO_TILE, e1 = min(sc.nsino, e0 + BT_SINO_TILE);
            for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS)
                sc.err[i] = __fsub_rn(sc.y[i], __fmul_rn(a, sc.dsino[i]));
        } else {
            const int tr = t - total_sn;
            const int s = find_scan(T.rc_off, num_scans, tr);
            const int local = tr - __ldg(T.rc_off + s);
            const VcdScan &sc = T.scans[s];
            const float a = T.alpha_init[s];
            const long long e0 = (long long)local * BT_SINO_TILE, e1 = min(sc.nrecon, e0 + BT_SINO_TILE);
            for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) sc.recon[i] = __fmul_rn(a, sc.recon[i]);
        }
    }
}

// Translation geometry has no direct recon: x0 = 0, so A x0 = 0, alpha = 1 and e = y (the reference's base-class
// direct_recon returns zeros, tomography_model.py:934-949).
__global__ void __launch_bounds__(BT_THREADS) b_copy_sino(BatchedTables T, int num_scans, int total) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int s = find_scan(T.sn_off, num_scans, t);
        const int local = t - __ldg(T.sn_off + s);
        const VcdScan &sc = T.scans[s];
        const long long e0 = (long long)local * BT_SINO_TILE, e1 = min(sc.nsino, e0 + BT_SINO_TILE);
        for (long long i = e0 + threadIdx.x; i < e1; i += BT_THREADS) sc.err[i] = sc.y[i];
    }
}

// Chunk bounding boxes of every (scan, subset) record's pixel list (after new partitions are written).
__global__ void __launch_bounds__(CB_CHUNK) b_chunk_bounds(BatchedTables T, int ksum, int total) {
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const int k = find_scan(T.box_first, ksum, t);
        const FpArgs &f = T.fpargs[k];
        fp_chunk_bounds_block(f.pix, f.num_pixels, f.g.num_recon_rows, f.g.num_recon_cols,
                              const_cast<int4 *>(f.chunk_box), t - __ldg(T.box_first + k));
    }
}

// ------------------------------------------------------------------------------------------------ host side
struct ScanSizes {
    long long ncyl, nsino, nrecon, npix;
    int el_tiles, sn_tiles, rc_tiles, flt_tiles;
    BpfPlan bpp;  // subset back projection
    CbPlan fpp;   // subset (and initial) forward projection
    BpfPlan ibp;  // initial back projection over the region of reconstruction
    BpfPlan hbp;  // Hessian back projection over every pixel
    int hbp_slices;  // > 0: hbp is planned on one slice and broadcast to this many (unit-weight parallel beam)
    bool setup;   // the scan carries the set-up inputs
};

static int scan_sizes(const mbx_scan &sc, ScanSizes &z) {
    const mbx_geom &g = sc.geom;
    int rc = validate_geom(&g);
    if (rc != MBX_OK) return rc;
    if (!sc.flat_recon || !sc.error_sinogram || !sc.fm_hessian || !sc.partition) return MBX_ERR_INVALID_ARG;
    if (sc.num_subsets <= 0 || sc.subset_size <= 0) return MBX_ERR_INVALID_ARG;
    if (!(sc.qp.sigma_x > 0.0f) || !(sc.qp.T > 0.0f) || !(sc.qp.p > 0.0f)) return MBX_ERR_INVALID_ARG;
    z.bpp = plan_bp_fast(g, sc.subset_size, g.num_views);
    z.fpp = plan_fp_cb(g, 0, 0, 2, 128, 0, MBX_BATCHED_FP_CAP);
    if (!z.bpp.ok || !z.fpp.ok) return MBX_ERR_UNSUPPORTED;  // batched path needs the radius-1 kernels
    if ((long long)sc.subset_size * g.num_recon_slices >= (1LL << 31)) return MBX_ERR_UNSUPPORTED;
    if (sc.subset_size > (1 << 24)) return MBX_ERR_UNSUPPORTED;  // list positions share a word with the bin
    z.ncyl = (long long)sc.subset_size * g.num_recon_slices;
    z.nsino = (long long)g.num_views * g.num_det_rows * g.num_det_channels;
    z.npix = (long long)g.num_recon_rows * g.num_recon_cols;
    z.nrecon = z.npix * g.num_recon_slices;
    z.el_tiles = (int)((z.ncyl + BT_ELEM_TILE - 1) / BT_ELEM_TILE);
    z.sn_tiles = (int)((z.nsino + BT_SINO_TILE - 1) / BT_SINO_TILE);
    z.rc_tiles = (int)((z.nrecon + BT_SINO_TILE - 1) / BT_SINO_TILE);
    z.setup = sc.sinogram != nullptr || sc.full_indices != nullptr || sc.num_full_indices != 0;
    z.flt_tiles = 0;
    if (z.setup) {
        if (!sc.sinogram || !sc.full_indices || sc.num_full_indices <= 0 || sc.num_full_indices > z.npix)
            return MBX_ERR_INVALID_ARG;
        // the initial forward projection reads voxels by pixel index, which shares a word with the bin
        if (z.npix > (1 << 24) || z.nrecon >= (1LL << 31)) return MBX_ERR_UNSUPPORTED;
        z.hbp_slices = 0;
        if (bp_unit_broadcast(g, nullptr, sc.weights)) {  // unit-weight parallel Hessian: one slice, broadcast
            z.hbp = plan_bp_fast(one_slice_geometry(g), z.npix, g.num_views);
            if (z.hbp.ok && z.hbp.splits == 1) z.hbp_slices = g.num_recon_slices;
        }
        if (z.hbp_slices == 0) z.hbp = plan_bp_fast(g, z.npix, g.num_views);
        if (!z.hbp.ok) return MBX_ERR_UNSUPPORTED;
        if (g.kind != MBX_GEOM_TRANSLATION) {  // translation geometry starts from zeros (no direct recon)
            if (filter_smem_bytes(g.num_det_channels, g.kind != MBX_GEOM_PARALLEL) > 200 * 1024)
                return MBX_ERR_UNSUPPORTED;
            z.ibp = plan_bp_fast(g, sc.num_full_indices, g.num_views);
            if (!z.ibp.ok) return MBX_ERR_UNSUPPORTED;
            z.flt_tiles = (int)(((long long)g.num_views * g.num_det_rows + FILT_ROWS - 1) / FILT_ROWS);
        } else {
            z.ibp = z.hbp;  // unused
        }
    }
    return MBX_OK;
}

// Tiles of scan s in a projection work list, the list's per-scan dimension (gx or channel blocks) and the cost
// of one of its tiles (to order the list: most expensive tiles first).
static void list_dims(int which, const mbx_scan &sc, const ScanSizes &z, int &tiles, int &dim, double &cost,
                      bool planned = false) {
    const mbx_geom &g = sc.geom;
    auto bp_cost = [&](const BpfPlan &b) {
        return (double)g.num_views * std::min(g.num_recon_slices, b.ts * b.nsl) * 32.0 * b.npg;
    };
    auto fp_cost = [&](long long npix) {
        return (double)npix * (2.0 + (double)(z.fpp.nb + 2) * z.fpp.rpad / g.num_det_channels);
    };
    switch (which) {
        case PL_BP: tiles = z.bpp.gx * z.bpp.gy; dim = z.bpp.gx; cost = bp_cost(z.bpp); break;
        case PL_FP: tiles = g.num_views * z.fpp.cblocks; dim = z.fpp.cblocks; cost = fp_cost(sc.subset_size); break;
        case PL_INIT_BP:
            tiles = (z.setup && g.kind != MBX_GEOM_TRANSLATION) ? z.ibp.gx * z.ibp.gy : 0;
            dim = z.ibp.gx;
            cost = bp_cost(z.ibp);
            break;
        case PL_INIT_FP:
            tiles = (z.setup && g.kind != MBX_GEOM_TRANSLATION) ? g.num_views * z.fpp.cblocks : 0;
            dim = z.fpp.cblocks;
            cost = fp_cost(sc.num_full_indices);
            break;
        case PL_BUILD:
            tiles = planned ? sc.num_subsets * g.num_views * z.fpp.cblocks : 0;
            dim = z.fpp.cblocks;
            cost = fp_cost(sc.subset_size);
            break;
        default: tiles = z.setup ? z.hbp.gx * z.hbp.gy : 0; dim = z.hbp.gx; cost = bp_cost(z.hbp); break;
    }
}

// Storage of the planned forward projection of one (scan, subset) pixel list: records for about every pixel in
// every view plus the pixels shared by neighbouring channel blocks (a tile whose passes find no room is walked
// instead), pass slots for the most passes the records can need (every pass but a tile's last holds more than
// 256 records), and per-tile pass tables.
struct PlannedSizes {
    long long rec_cap;
    int pass_cap, tiles, nbins;
    size_t rec, rec2, sbin, pass_rec, pass_count, pass_bstart, tile_npass, tile_pass, total;
};

static PlannedSizes planned_sizes(const mbx_scan &sc, const ScanSizes &z) {
    PlannedSizes q;
    const mbx_geom &g = sc.geom;
    q.tiles = g.num_views * z.fpp.cblocks;
    q.nbins = z.fpp.nbins;
    q.rec_cap = (long long)std::ceil(1.06 * g.num_views * (double)sc.subset_size) + 16LL * q.tiles;
    q.pass_cap = (int)(q.rec_cap / 257 + q.tiles + 1);
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += align256(bytes); return o; };
    q.rec = take(sizeof(float4) * (size_t)q.rec_cap);
    q.rec2 = take(g.kind != MBX_GEOM_PARALLEL ? sizeof(float4) * (size_t)q.rec_cap : 0);
    q.sbin = take((size_t)q.rec_cap);
    q.pass_rec = take(sizeof(long long) * (size_t)q.pass_cap);
    q.pass_count = take(sizeof(int) * (size_t)q.pass_cap);
    q.pass_bstart = take(sizeof(int) * (size_t)q.pass_cap * (q.nbins + 1));
    q.tile_npass = take(sizeof(int) * (size_t)q.tiles);
    q.tile_pass = take(sizeof(int) * (size_t)q.tiles * CB_MAX_PASSES);
    q.total = off;
    return q;
}

struct Layout {
    size_t scans, fm, qp, bpargs, fpargs, ibp, ifp, hbp, filt, planned, pl_off, pl_dim, pl_order, offs, box_first,
        counters, sched, p_prior, p_fwd, p_l1, p_iter, p_init, alpha, alpha_init, arange, cursors, total;
    bool plan_fp;
    std::vector<size_t> plan_off;  // per scan: its subsets' planned storage, [K][PlannedSizes::total]
    int pl_total[PL_COUNT];
    int el_total, sn_total, rc_total, flt_total, box_total, ksum, max_npix;
    bool setup;
    std::vector<size_t> buf_off;   // per scan: bp, delta, dsino
    std::vector<size_t> box_off;   // per scan: chunk boxes of its subsets, [K][chunks]
    std::vector<size_t> fbox_off;  // per scan: chunk boxes of its region-of-reconstruction list
};

static int layout(const mbx_scan *scans, int n, int num_steps, Layout &L, std::vector<ScanSizes> &zs,
                  int flags = 0) {
    L.plan_fp = (flags & MBX_BATCHED_PLAN_FORWARD) != 0;
    zs.resize(n);
    for (int w = 0; w < PL_COUNT; ++w) L.pl_total[w] = 0;
    L.el_total = L.sn_total = L.rc_total = L.flt_total = L.box_total = L.ksum = L.max_npix = 0;
    int kind = -1, nsetup = 0;
    for (int s = 0; s < n; ++s) {
        int rc = scan_sizes(scans[s], zs[s]);
        if (rc != MBX_OK) return rc;
        if (kind >= 0 && scans[s].geom.kind != kind) return MBX_ERR_UNSUPPORTED;  // one geometry kind per batch
        if (scans[s].num_subsets != scans[0].num_subsets) return MBX_ERR_UNSUPPORTED;  // argument table is [scan][K]
        kind = scans[s].geom.kind;
        for (int w = 0; w < PL_COUNT; ++w) {
            int tiles, dim;
            double cost;
            list_dims(w, scans[s], zs[s], tiles, dim, cost, L.plan_fp);
            L.pl_total[w] += tiles;
        }
        L.el_total += zs[s].el_tiles;
        L.sn_total += zs[s].sn_tiles;
        L.rc_total += zs[s].rc_tiles;
        L.flt_total += zs[s].flt_tiles;
        L.ksum += scans[s].num_subsets;
        L.box_total += scans[s].num_subsets * (int)((scans[s].subset_size + CB_CHUNK - 1) / CB_CHUNK);
        L.max_npix = std::max<int>(L.max_npix, (int)zs[s].npix);
        nsetup += zs[s].setup ? 1 : 0;
    }
    if (nsetup != 0 && nsetup != n) return MBX_ERR_INVALID_ARG;  // set-up inputs for every scan or for none
    L.setup = nsetup == n;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += align256(bytes); return o; };
    L.scans = take(sizeof(VcdScan) * n);
    L.fm = take(sizeof(float) * n);
    L.qp = take(sizeof(QParams) * n);
    L.bpargs = take(sizeof(BpArgs) * L.ksum);
    L.fpargs = take(sizeof(FpArgs) * L.ksum);
    L.ibp = take(sizeof(BpArgs) * n);
    L.ifp = take(sizeof(FpArgs) * n);
    L.hbp = take(sizeof(BpArgs) * n);
    L.filt = take(sizeof(FiltScan) * n);
    L.planned = take(L.plan_fp ? sizeof(CbPlanned) * L.ksum : 0);
    L.pl_off = take(sizeof(int) * PL_COUNT * (n + 1));
    L.pl_dim = take(sizeof(int) * PL_COUNT * n);
    L.pl_order = take(sizeof(int) * PL_COUNT * n);
    L.offs = take(sizeof(int) * 4 * (n + 1));
    L.box_first = take(sizeof(int) * (L.ksum + 1));
    L.counters = take(sizeof(int) * PL_COUNT);
    L.sched = take(sizeof(int) * (size_t)num_steps * n);  // the host-built tables end here
    L.p_prior = take(sizeof(double) * 2 * (size_t)L.el_total);
    L.p_fwd = take(sizeof(double) * 2 * (size_t)L.sn_total);
    L.p_l1 = take(sizeof(double) * (size_t)L.el_total);
    L.p_iter = take(sizeof(double) * ((size_t)L.sn_total + L.rc_total));
    L.p_init = take(sizeof(double) * 2 * (size_t)L.sn_total);
    L.alpha = take(sizeof(float) * n);
    L.alpha_init = take(sizeof(float) * n);
    L.arange = take(L.setup ? sizeof(int32_t) * (size_t)L.max_npix : 0);
    L.cursors = take(L.plan_fp ? 16 * (size_t)L.ksum : 0);  // {unsigned long long records, int passes, pad}
    L.buf_off.resize(3 * (size_t)n);
    for (int s = 0; s < n; ++s) {
        L.buf_off[3 * s] = take(4 * (size_t)zs[s].ncyl);
        L.buf_off[3 * s + 1] = take(4 * (size_t)zs[s].ncyl);
        L.buf_off[3 * s + 2] = take(4 * (size_t)zs[s].nsino);
    }
    L.box_off.resize(n);
    L.fbox_off.assign(n, 0);
    for (int s = 0; s < n; ++s) {
        L.box_off[s] = take((size_t)scans[s].num_subsets * fp_chunk_box_bytes(scans[s].subset_size));
        if (L.setup) L.fbox_off[s] = take(fp_chunk_box_bytes(scans[s].num_full_indices));
    }
    L.plan_off.assign(n, 0);
    for (int s = 0; s < n && L.plan_fp; ++s)
        L.plan_off[s] = take((size_t)scans[s].num_subsets * planned_sizes(scans[s], zs[s]).total);
    L.total = off;
    return MBX_OK;
}

template <typename K>
static int occupancy_grid(K kern, int threads, size_t smem, int total) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem) != cudaSuccess || per_sm < 1) {
        cudaGetLastError();
        per_sm = 1;
    }
    const long long g = (long long)per_sm * num_sms();
    return (int)std::max(1LL, std::min<long long>(g, total));
}

// The projection stage kernels of a geometry kind.
static const void *bp_kernel_of(int kind) {
    return kind == MBX_GEOM_PARALLEL ? reinterpret_cast<const void *>(b_bp<MBX_GEOM_PARALLEL>)
           : kind == MBX_GEOM_CONE   ? reinterpret_cast<const void *>(b_bp<MBX_GEOM_CONE>)
                                     : reinterpret_cast<const void *>(b_bp<MBX_GEOM_TRANSLATION>);
}

// The forward stage kernels of each geometry kind (compiled in b_fp_parallel.cu, b_fp_cone.cu, b_fp_translation.cu).
const void *fp_stage_kernel_parallel(int minb, int mode);
const void *fp_stage_kernel_cone(int minb, int mode);
const void *fp_stage_kernel_translation(int minb, int mode);
void launch_fp_stage_parallel(int minb, int mode, int grid, size_t smem, cudaStream_t st, const ProjList &L, int n,
                              int step, int first, int total, int *err);
void launch_fp_stage_cone(int minb, int mode, int grid, size_t smem, cudaStream_t st, const ProjList &L, int n,
                          int step, int first, int total, int *err);
void launch_fp_stage_translation(int minb, int mode, int grid, size_t smem, cudaStream_t st, const ProjList &L, int n,
                                 int step, int first, int total, int *err);

const void *fp_stage_kernel(int kind, int minb, int mode) {
    return kind == MBX_GEOM_PARALLEL ? fp_stage_kernel_parallel(minb, mode)
           : kind == MBX_GEOM_CONE   ? fp_stage_kernel_cone(minb, mode)
                                     : fp_stage_kernel_translation(minb, mode);
}

void launch_fp_stage(int kind, int minb, int mode, int grid, size_t smem, cudaStream_t st, const ProjList &L, int n,
                     int step, int first, int total, int *err) {
    if (kind == MBX_GEOM_PARALLEL)
        launch_fp_stage_parallel(minb, mode, grid, smem, st, L, n, step, first, total, err);
    else if (kind == MBX_GEOM_CONE)
        launch_fp_stage_cone(minb, mode, grid, smem, st, L, n, step, first, total, err);
    else
        launch_fp_stage_translation(minb, mode, grid, smem, st, L, n, step, first, total, err);
}

// The forward stage kernel of a mode: CB_WALK (b_fp), CB_REPLAY (b_fp_replay) or CB_BUILD (b_fp_build).
static const void *fp_kernel_of(int kind, int minb, int mode = CB_WALK) { return fp_stage_kernel(kind, minb, mode); }

// Preferred shared-memory carveout of a kernel: what its resident CTAs of `threads` threads and smem bytes of
// dynamic shared memory need (a hint; the driver rounds it up to a supported split of the SM's unified storage).
static cudaError_t set_smem_carveout(const void *kern, int threads, size_t smem) {
    int dev = 0, max_sm = 0, reserved = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&max_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    if (e != cudaSuccess || max_sm <= 0 || per_sm <= 0) return e;
    const double need = (double)per_sm * (double)(smem + (size_t)reserved);
    const int pct = std::min(100, (int)std::ceil(100.0 * need / max_sm));
    return cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
}

static int bp_grid(int kind, size_t smem, int total) {
    return occupancy_grid(bp_kernel_of(kind), BPF_THREADS, smem, total);
}

static int fp_grid(int kind, int minb, size_t smem, int total, int mode = CB_WALK) {
    return occupancy_grid(fp_kernel_of(kind, minb, mode), CB_THREADS, smem, total);
}

// One launch of a back-projection work list over tiles [first, total) (resets the list's counter first).
static cudaError_t launch_bp_list(const BatchedPlanHost &P, int which, int step, int first, int total, int grid,
                                  size_t smem, cudaStream_t st) {
    ProjList L = proj_list(P.t, which, P.num_scans);
    L.stride = which == PL_BP ? P.ksum / P.num_scans : 1;
    cudaError_t e = cudaMemsetAsync(L.counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    int *err = device_error_ptr();
    if (P.kind == MBX_GEOM_PARALLEL)
        b_bp<MBX_GEOM_PARALLEL><<<grid, BPF_THREADS, smem, st>>>(L, P.num_scans, step, first, total, err);
    else if (P.kind == MBX_GEOM_CONE)
        b_bp<MBX_GEOM_CONE><<<grid, BPF_THREADS, smem, st>>>(L, P.num_scans, step, first, total, err);
    else
        b_bp<MBX_GEOM_TRANSLATION><<<grid, BPF_THREADS, smem, st>>>(L, P.num_scans, step, first, total, err);
    note_launch();
    return cudaGetLastError();
}

// One launch of a forward-projection work list (kernel variant for minb resident CTAs per SM): the walk
// (mode CB_WALK), the replay of planned passes (CB_REPLAY, subset list) or their build (CB_BUILD, PL_BUILD).
static cudaError_t launch_fp_list(const BatchedPlanHost &P, int which, int minb, int step, int first, int total,
                                  int grid, size_t smem, cudaStream_t st, int mode = CB_WALK) {
    ProjList L = proj_list(P.t, which, P.num_scans);
    const bool subsets = which == PL_FP || which == PL_BUILD;
    L.stride = subsets ? P.ksum / P.num_scans : 1;
    if (which == PL_BUILD) {
        L.fp = P.t.fpargs;
        L.schedule = nullptr;
    }
    if (mode != CB_WALK) L.planned = P.t.planned;
    cudaError_t e = cudaMemsetAsync(L.counter, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    int *err = device_error_ptr();
    launch_fp_stage(P.kind, minb, mode, grid, smem, st, L, P.num_scans, step, first, total, err);
    note_launch();
    return cudaGetLastError();
}

// Key of a batch shape for the autotune cache (every scan's sizes, subsets and pixels per subset).
static std::vector<long long> batch_key(long long tag, const BatchedPlanHost &P, const mbx_scan *scans, bool weights) {
    std::vector<long long> key = {tag, P.kind, P.num_scans, P.fp_minb, -1};
    for (int s = 0; s < P.num_scans; ++s) {
        const mbx_geom &g = scans[s].geom;
        key.insert(key.end(), {g.num_views, g.num_det_rows, g.num_det_channels, g.num_recon_rows, g.num_recon_cols,
                               g.num_recon_slices, scans[s].num_subsets, scans[s].subset_size});
        if (weights) key.push_back(scans[s].weights ? 1 : 0);
    }
    return key;
}

// Autotuning of the forward-projection stage: the plans of every scan with the kernel variant compiled for 2
// resident CTAs per SM (the tables as built) against the same channel blocks with smaller passes and the variant
// compiled for 3.  Each is timed on step 0 (the stage only writes the scans' projection scratch, whose input is
// zeroed first); the faster one's argument table stays on the device, and the choice is remembered for the
// batch shape, so later plans of the same batch do not time again.
static int tune_batched_fp(BatchedPlanHost &P, const Layout &L, const std::vector<ScanSizes> &zs,
                           const mbx_scan *scans, const FpArgs *hf2, cudaStream_t st) {
    const int num_scans = P.num_scans;
    std::vector<FpArgs> f3(hf2, hf2 + L.ksum);
    size_t smem3 = 0, smem3r = 0;
    int ki = 0;
    for (int s = 0; s < num_scans; ++s) {
        const CbPlan c3 = plan_fp_cb(scans[s].geom, 0, 0, 3, zs[s].fpp.nb, 0, MBX_BATCHED_FP_CAP);
        if (!c3.ok || c3.nb != zs[s].fpp.nb || c3.cblocks != zs[s].fpp.cblocks) return MBX_OK;  // same work list only
        smem3 = std::max(smem3, c3.walk.smem);
        smem3r = std::max(smem3r, c3.replay.smem);
        for (int k = 0; k < scans[s].num_subsets; ++k, ++ki) f3[ki].plan = c3;
    }
    char *base = reinterpret_cast<char *>(P.t.scans) - L.scans;
    const std::vector<long long> key = batch_key(2, P, scans, false);
    auto use3 = [&]() -> int {
        cudaError_t e3 = cudaMemcpyAsync(base + L.fpargs, f3.data(), sizeof(FpArgs) * L.ksum, cudaMemcpyHostToDevice,
                                         st);
        if (e3 == cudaSuccess) e3 = cudaStreamSynchronize(st);
        if (e3 != cudaSuccess) return set_cuda_error(e3);
        P.fp_minb = 3;
        P.pl_smem[PL_FP] = smem3;
        P.fp_smem_replay = smem3r;
        P.pl_grid[PL_FP] = fp_grid(P.kind, 3, smem3, P.pl_total[PL_FP]);
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
    auto run = [&]() {
        return launch_fp_list(P, PL_FP, P.fp_minb, 0, 0, P.pl_total[PL_FP], P.pl_grid[PL_FP], P.pl_smem[PL_FP], st);
    };
    float t2 = 0.0f, t3 = 0.0f;
    e = time_on_stream(run, st, t2);
    if (e != cudaSuccess) return set_cuda_error(e);
    const BatchedPlanHost keep = P;
    int rc = use3();
    if (rc != MBX_OK) return rc;
    e = time_on_stream(run, st, t3);
    if (e != cudaSuccess) return set_cuda_error(e);
    autotune_store(key.data(), (int)key.size(), t2 <= t3 ? 2 : 3);
    if (t2 <= t3) {  // back to the tables as built
        P = keep;
        e = cudaMemcpyAsync(base + L.fpargs, hf2, sizeof(FpArgs) * L.ksum, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return set_cuda_error(e);
    }
    return MBX_OK;
}

// Per-scan lane layout of the forward-projection stage, after the kernel variant is chosen: each scan is timed
// alone on step 0 with its plan and with the best layout that has another number of sub-groups per warp (same
// channel blocks, so the same tiles), and keeps the faster.  Cached per batch shape.
static int tune_batched_fp_layouts(BatchedPlanHost &P, const Layout &L, const mbx_scan *scans, const int *o_fp,
                                   const int *order_fp, cudaStream_t st) {
    const int num_scans = P.num_scans;
    const int K = scans[0].num_subsets;  // every scan of a batch has the same number of subsets
    const int ksum = L.ksum;
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
        const CbPlan q = plan_fp_cb(scans[sc].geom, 0, 0, c0.minb, c0.nb, c0.ppw, MBX_BATCHED_FP_CAP);
        if (!q.ok || q.nb != c0.nb || q.cblocks != c0.cblocks || q.minb != c0.minb) continue;
        can[sc] = 1;
        for (int j = 0; j < K; ++j) alt[sc * K + j].plan = q;
        smem_alt = std::max(smem_alt, q.walk.smem);
    }
    std::vector<long long> key = batch_key(5, P, scans, false);
    auto use = [&](int sc, int c) {
        for (int j = 0; j < K; ++j) cur[sc * K + j] = c ? alt[sc * K + j] : orig[sc * K + j];
    };
    auto upload = [&]() -> cudaError_t {
        cudaError_t e2 = cudaMemcpyAsync(base + L.fpargs, cur.data(), sizeof(FpArgs) * ksum, cudaMemcpyHostToDevice, st);
        return e2 == cudaSuccess ? cudaStreamSynchronize(st) : e2;
    };
    auto apply_smem = [&]() {
        size_t sm = 0;
        size_t smr = 0;
        for (int k = 0; k < ksum; ++k) {
            sm = std::max(sm, cur[k].plan.walk.smem);
            smr = std::max(smr, cur[k].plan.replay.smem);
        }
        P.pl_smem[PL_FP] = sm;
        P.fp_smem_replay = smr;
        P.pl_grid[PL_FP] = fp_grid(P.kind, P.fp_minb, sm, P.pl_total[PL_FP]);
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
    P.pl_smem[PL_FP] = std::max(P.pl_smem[PL_FP], smem_alt);  // tuning launches fit either plan
    for (int k = 0; k < num_scans; ++k) {
        const int sc = order_fp[k];
        if (!can[sc]) continue;
        const int first = o_fp[k], last = o_fp[k + 1];
        const int grid = std::min(P.pl_grid[PL_FP], last - first);
        auto run = [&]() {
            return launch_fp_list(P, PL_FP, P.fp_minb, 0, first, last, grid, P.pl_smem[PL_FP], st);
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
static int tune_batched_bp(BatchedPlanHost &P, const Layout &L, const mbx_scan *scans, const BpArgs *hb1,
                           const int *o_bp, const int *order_bp, cudaStream_t st) {
    const int num_scans = P.num_scans;
    const int K = scans[0].num_subsets;  // every scan of a batch has the same number of subsets
    const int ksum = L.ksum;
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
    std::vector<long long> key = batch_key(4, P, scans, true);
    key[3] = -1;
    auto upload = [&]() -> cudaError_t {
        cudaError_t e = cudaMemcpyAsync(base + L.bpargs, cur.data(), sizeof(BpArgs) * ksum, cudaMemcpyHostToDevice, st);
        return e == cudaSuccess ? cudaStreamSynchronize(st) : e;
    };
    auto apply_smem = [&]() {
        size_t sm = 0;
        for (int k = 0; k < ksum; ++k) sm = std::max(sm, cur[k].plan.smem);
        P.pl_smem[PL_BP] = sm;
        P.pl_grid[PL_BP] = bp_grid(P.kind, sm, P.pl_total[PL_BP]);
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
            key[4] = s;
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
    P.pl_smem[PL_BP] = std::max(P.pl_smem[PL_BP], smem_alt);  // tuning launches fit either plan
    for (int k = 0; k < num_scans; ++k) {
        const int s = order_bp[k];
        if (!can[s]) continue;
        const int first = o_bp[k], last = o_bp[k + 1];
        const int grid = std::min(P.pl_grid[PL_BP], last - first);
        auto run = [&]() { return launch_bp_list(P, PL_BP, 0, first, last, grid, P.pl_smem[PL_BP], st); };
        float t[2] = {0.0f, 0.0f};
        for (int c = 0; c < 2; ++c) {
            use(s, c);
            cudaError_t e = upload();
            if (e == cudaSuccess) e = time_on_stream(run, st, t[c]);
            if (e != cudaSuccess) return set_cuda_error(e);
        }
        choice[s] = t[1] < t[0] ? 1 : 0;
        use(s, choice[s]);
        key[4] = s;
        autotune_store(key.data(), (int)key.size(), choice[s]);
    }
    cudaError_t e = upload();
    if (e != cudaSuccess) return set_cuda_error(e);
    apply_smem();
    return MBX_OK;
}

// Per-call parameter tables: fm constants and qGGMRF parameters.
static void fill_params(const mbx_scan *scans, int n, float *fm, QParams *qp) {
    for (int s = 0; s < n; ++s) {
        fm[s] = scans[s].fm_constant;
        qp[s] = make_qparams(scans[s].qp);
    }
}

static int check_schedule(const mbx_scan *scans, int n, const int32_t *schedule, int num_steps) {
    for (int st = 0; st < num_steps; ++st)
        for (int s = 0; s < n; ++s) {
            const int v = schedule[(size_t)st * n + s];
            if (v < 0 || v >= scans[s].num_subsets) return MBX_ERR_INVALID_ARG;
        }
    return MBX_OK;
}

}  // namespace mbx

using namespace mbx;

extern "C" size_t mbx_vcd_batched_workspace_bytes2(const mbx_scan *scans, int32_t num_scans, int32_t num_steps,
                                                   int32_t flags) {
    if (!scans || num_scans <= 0 || num_steps <= 0 || (flags & ~MBX_BATCHED_PLAN_FORWARD)) return 0;
    Layout L;
    std::vector<ScanSizes> zs;
    if (layout(scans, num_scans, num_steps, L, zs, flags) != MBX_OK) return 0;
    return L.total;
}

extern "C" size_t mbx_vcd_batched_workspace_bytes(const mbx_scan *scans, int32_t num_scans, int32_t num_steps) {
    return mbx_vcd_batched_workspace_bytes2(scans, num_scans, num_steps, 0);
}

static const BatchedPlanHost *plan_of(const mbx_batched_plan *p) {
    if (!p) return nullptr;
    const BatchedPlanHost *P = reinterpret_cast<const BatchedPlanHost *>(p);
    return P->magic == BT_MAGIC ? P : nullptr;
}

extern "C" int mbx_vcd_batched_prepare(const mbx_scan *scans, int32_t num_scans, const int32_t *schedule,
                                       int32_t num_steps, int32_t num_iterations, double *step_stats,
                                       double *iter_stats, void *workspace, size_t workspace_bytes,
                                       mbx_batched_plan *plan_out, void *stream) {
    return mbx_vcd_batched_prepare2(scans, num_scans, schedule, num_steps, num_iterations, step_stats, iter_stats,
                                    workspace, workspace_bytes, 0, plan_out, stream);
}

extern "C" int mbx_vcd_batched_prepare2(const mbx_scan *scans, int32_t num_scans, const int32_t *schedule,
                                        int32_t num_steps, int32_t num_iterations, double *step_stats,
                                        double *iter_stats, void *workspace, size_t workspace_bytes, int32_t flags,
                                        mbx_batched_plan *plan_out, void *stream) {
    if (!scans || num_scans <= 0 || !schedule || num_steps <= 0 || num_iterations < 0 || !plan_out || !step_stats ||
        (num_iterations > 0 && !iter_stats) || (flags & ~MBX_BATCHED_PLAN_FORWARD))
        return MBX_ERR_INVALID_ARG;
    Layout L;
    std::vector<ScanSizes> zs;
    int rc = layout(scans, num_scans, num_steps, L, zs, flags);
    if (rc != MBX_OK) return rc;
    if (!workspace || workspace_bytes < L.total) return MBX_ERR_WORKSPACE;
    rc = check_schedule(scans, num_scans, schedule, num_steps);
    if (rc != MBX_OK) return rc;
    const int n = num_scans, n1 = num_scans + 1;
    char *base = static_cast<char *>(workspace);
    std::vector<char> host(L.sched + sizeof(int) * (size_t)num_steps * n, 0);
    VcdScan *hs = reinterpret_cast<VcdScan *>(host.data() + L.scans);
    BpArgs *hb = reinterpret_cast<BpArgs *>(host.data() + L.bpargs);
    FpArgs *hf = reinterpret_cast<FpArgs *>(host.data() + L.fpargs);
    BpArgs *hib = reinterpret_cast<BpArgs *>(host.data() + L.ibp);
    FpArgs *hif = reinterpret_cast<FpArgs *>(host.data() + L.ifp);
    BpArgs *hhb = reinterpret_cast<BpArgs *>(host.data() + L.hbp);
    FiltScan *hfl = reinterpret_cast<FiltScan *>(host.data() + L.filt);
    CbPlanned *hpn = reinterpret_cast<CbPlanned *>(host.data() + L.planned);
    int *hpl_off = reinterpret_cast<int *>(host.data() + L.pl_off);
    int *hpl_dim = reinterpret_cast<int *>(host.data() + L.pl_dim);
    int *hpl_order = reinterpret_cast<int *>(host.data() + L.pl_order);
    int *hoff = reinterpret_cast<int *>(host.data() + L.offs);
    int *hbox_first = reinterpret_cast<int *>(host.data() + L.box_first);
    int *o_el = hoff, *o_sn = hoff + n1, *o_rc = hoff + 2 * n1, *o_flt = hoff + 3 * n1;
    fill_params(scans, n, reinterpret_cast<float *>(host.data() + L.fm), reinterpret_cast<QParams *>(host.data() + L.qp));
    o_el[0] = o_sn[0] = o_rc[0] = o_flt[0] = 0;
    hbox_first[0] = 0;
    auto bp_args = [](const mbx_geom &g, const float *sino, const float *wts, const int32_t *pix, long long npix,
                      int cp, float *out, int by_index, const BpfPlan &plan) {
        BpArgs a;
        std::memset(&a, 0, sizeof(a));
        a.g = g;
        a.sino = sino;
        a.wts = wts;
        a.pix = pix;
        a.num_pixels = npix;
        a.order = nullptr;
        a.views = nullptr;
        a.num_views_sel = g.num_views;
        a.views_per_split = g.num_views;
        a.coeff_power = cp;
        a.scale = 1.0f;
        a.out = out;
        a.split_stride = 0;
        a.out_by_index = by_index;
        a.plan = plan;
        return a;
    };
    int ki = 0;
    for (int s = 0; s < n; ++s) {
        const mbx_scan &sc = scans[s];
        const ScanSizes &z = zs[s];
        const mbx_geom &g = sc.geom;
        VcdScan &v = hs[s];
        v.recon = sc.flat_recon;
        v.err = sc.error_sinogram;
        v.wts = sc.weights;
        v.hess = const_cast<float *>(sc.fm_hessian);
        v.partition = sc.partition;
        v.bp = reinterpret_cast<float *>(base + L.buf_off[3 * s]);
        v.delta = reinterpret_cast<float *>(base + L.buf_off[3 * s + 1]);
        v.dsino = reinterpret_cast<float *>(base + L.buf_off[3 * s + 2]);
        v.y = sc.sinogram;
        v.nsino = z.nsino;
        v.nrecon = z.nrecon;
        v.K = sc.num_subsets;
        v.M = sc.subset_size;
        v.nr = g.num_recon_rows;
        v.nc = g.num_recon_cols;
        v.ns = g.num_recon_slices;
        for (int k = 0; k < sc.num_subsets; ++k, ++ki) {
            const int32_t *pix = sc.partition + (size_t)k * sc.subset_size;
            hb[ki] = bp_args(g, sc.error_sinogram, sc.weights, pix, sc.subset_size, 1, v.bp, 0, z.bpp);
            if (sc.partition_order) hb[ki].order = sc.partition_order + (size_t)k * sc.subset_size;
            FpArgs &f = hf[ki];
            std::memset(&f, 0, sizeof(f));
            f.g = g;
            f.vox = v.delta;
            f.pix = pix;
            f.num_pixels = sc.subset_size;
            f.views = nullptr;
            f.num_views_sel = g.num_views;
            f.out = v.dsino;
            f.vox_by_index = 0;
            f.plan = z.fpp;
            f.chunk_box = reinterpret_cast<const int4 *>(base + L.box_off[s] + (size_t)k * fp_chunk_box_bytes(sc.subset_size));
            hbox_first[ki + 1] = hbox_first[ki] + (int)((sc.subset_size + CB_CHUNK - 1) / CB_CHUNK);
            if (L.plan_fp) {  // this subset's planned storage
                const PlannedSizes q = planned_sizes(sc, z);
                char *pb = base + L.plan_off[s] + (size_t)k * q.total;
                CbPlanned &pn = hpn[ki];
                pn.rec = reinterpret_cast<float4 *>(pb + q.rec);
                pn.rec2 = g.kind != MBX_GEOM_PARALLEL ? reinterpret_cast<float4 *>(pb + q.rec2) : nullptr;
                pn.sbin = reinterpret_cast<uint8_t *>(pb + q.sbin);
                pn.rec_cursor = reinterpret_cast<unsigned long long *>(base + L.cursors + 16 * (size_t)ki);
                pn.pass_cursor = reinterpret_cast<int *>(base + L.cursors + 16 * (size_t)ki + 8);
                pn.pass_rec = reinterpret_cast<long long *>(pb + q.pass_rec);
                pn.pass_count = reinterpret_cast<int *>(pb + q.pass_count);
                pn.pass_bstart = reinterpret_cast<int *>(pb + q.pass_bstart);
                pn.tile_npass = reinterpret_cast<int *>(pb + q.tile_npass);
                pn.tile_pass = reinterpret_cast<int *>(pb + q.tile_pass);
                pn.rec_cap = q.rec_cap;
                pn.pass_cap = q.pass_cap;
            }
        }
        if (L.setup) {
            // x0: back projection of the filtered sinogram (held in the error sinogram) into the recon, by index
            hib[s] = bp_args(g, sc.error_sinogram, nullptr, sc.full_indices, sc.num_full_indices, 1, sc.flat_recon, 1,
                             z.ibp);
            FpArgs &f = hif[s];
            std::memset(&f, 0, sizeof(f));
            f.g = g;
            f.vox = sc.flat_recon;
            f.pix = sc.full_indices;
            f.num_pixels = sc.num_full_indices;
            f.num_views_sel = g.num_views;
            f.out = v.dsino;
            f.vox_by_index = 1;
            f.plan = z.fpp;
            f.chunk_box = reinterpret_cast<const int4 *>(base + L.fbox_off[s]);
            // Hessian: the weights (or ones: no sinogram) with squared coefficients over every pixel
            hhb[s] = bp_args(z.hbp_slices > 0 ? one_slice_geometry(g) : g, sc.weights, nullptr,
                             reinterpret_cast<const int32_t *>(base + L.arange), z.npix, 2,
                             const_cast<float *>(sc.fm_hessian), 0, z.hbp);
            hhb[s].out_slices = z.hbp_slices;
            FiltScan &fl = hfl[s];
            fl.in = sc.sinogram;
            fl.out = sc.error_sinogram;
            fl.rows = (long long)g.num_views * g.num_det_rows;
            fl.R = g.num_det_rows;
            fl.C = g.num_det_channels;
            direct_filter_scales(g, fl.filter_scale, fl.out_scale, fl.fdk);
            fl.D = g.source_detector_dist;
            fl.ddc = g.delta_det_channel;
            fl.ddr = g.delta_det_row;
            fl.dco = g.det_channel_offset;
            fl.dro = g.det_row_offset;
        }
        o_el[s + 1] = o_el[s] + z.el_tiles;
        o_sn[s + 1] = o_sn[s] + z.sn_tiles;
        o_rc[s + 1] = o_rc[s] + z.rc_tiles;
        o_flt[s + 1] = o_flt[s] + z.flt_tiles;
    }
    // projection work lists: scans in decreasing order of per-tile cost, so that the dynamically scheduled tail of
    // a launch is made of the cheapest tiles
    size_t pl_smem[PL_COUNT] = {0, 0, 0, 0, 0, 0};
    for (int w = 0; w < PL_COUNT; ++w) {
        std::vector<int> ord(n), tiles(n), dim(n);
        std::vector<double> cost(n);
        for (int s = 0; s < n; ++s) {
            list_dims(w, scans[s], zs[s], tiles[s], dim[s], cost[s], L.plan_fp);
            ord[s] = s;
            const ScanSizes &z = zs[s];
            const size_t sm = w == PL_BP ? z.bpp.smem : (w == PL_FP || w == PL_INIT_FP || w == PL_BUILD) ? z.fpp.walk.smem
                              : w == PL_INIT_BP ? (z.setup ? z.ibp.smem : 0) : (z.setup ? z.hbp.smem : 0);
            pl_smem[w] = std::max(pl_smem[w], sm);
        }
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return cost[a] > cost[b]; });
        int *off = hpl_off + w * n1;
        off[0] = 0;
        for (int k = 0; k < n; ++k) {
            hpl_order[w * n + k] = ord[k];
            off[k + 1] = off[k] + tiles[ord[k]];
        }
        for (int s = 0; s < n; ++s) hpl_dim[w * n + s] = dim[s];
    }
    std::memcpy(host.data() + L.sched, schedule, sizeof(int) * (size_t)num_steps * n);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(base, host.data(), host.size(), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && L.setup) {
        std::vector<int32_t> ar((size_t)L.max_npix);
        for (int i = 0; i < L.max_npix; ++i) ar[i] = i;
        e = cudaMemcpyAsync(base + L.arange, ar.data(), sizeof(int32_t) * ar.size(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // ar is released at scope end
    }
    if (e != cudaSuccess) return set_cuda_error(e);

    BatchedPlanHost P;
    std::memset(&P, 0, sizeof(P));
    P.t.scans = reinterpret_cast<VcdScan *>(base + L.scans);
    P.t.fm = reinterpret_cast<float *>(base + L.fm);
    P.t.qp = reinterpret_cast<QParams *>(base + L.qp);
    P.t.bpargs = reinterpret_cast<BpArgs *>(base + L.bpargs);
    P.t.fpargs = reinterpret_cast<FpArgs *>(base + L.fpargs);
    P.t.init_bp = reinterpret_cast<BpArgs *>(base + L.ibp);
    P.t.init_fp = reinterpret_cast<FpArgs *>(base + L.ifp);
    P.t.hess_bp = reinterpret_cast<BpArgs *>(base + L.hbp);
    P.t.filt = reinterpret_cast<FiltScan *>(base + L.filt);
    P.t.planned = L.plan_fp ? reinterpret_cast<CbPlanned *>(base + L.planned) : nullptr;
    P.planned_fp = L.plan_fp ? 1 : 0;
    P.plan_cursors = L.plan_fp ? base + L.cursors : nullptr;
    P.plan_cursor_bytes = L.plan_fp ? 16 * (size_t)L.ksum : 0;
    P.t.pl_off = reinterpret_cast<int *>(base + L.pl_off);
    P.t.pl_dim = reinterpret_cast<int *>(base + L.pl_dim);
    P.t.pl_order = reinterpret_cast<int *>(base + L.pl_order);
    int *doff = reinterpret_cast<int *>(base + L.offs);
    P.t.el_off = doff;
    P.t.sn_off = doff + n1;
    P.t.rc_off = doff + 2 * n1;
    P.t.flt_off = doff + 3 * n1;
    P.t.box_first = reinterpret_cast<int *>(base + L.box_first);
    P.t.counters = reinterpret_cast<int *>(base + L.counters);
    P.t.schedule = reinterpret_cast<int *>(base + L.sched);
    P.t.p_prior = reinterpret_cast<double *>(base + L.p_prior);
    P.t.p_fwd = reinterpret_cast<double *>(base + L.p_fwd);
    P.t.p_l1 = reinterpret_cast<double *>(base + L.p_l1);
    P.t.p_iter = reinterpret_cast<double *>(base + L.p_iter);
    P.t.p_init = reinterpret_cast<double *>(base + L.p_init);
    P.t.alpha = reinterpret_cast<float *>(base + L.alpha);
    P.t.alpha_init = reinterpret_cast<float *>(base + L.alpha_init);
    P.t.step_stats = step_stats;
    P.t.iter_stats = iter_stats;
    P.num_scans = n;
    P.kind = scans[0].geom.kind;
    P.num_steps = num_steps;
    P.num_iterations = num_iterations;
    P.ksum = L.ksum;
    P.has_setup = L.setup ? 1 : 0;
    for (int w = 0; w < PL_COUNT; ++w) {
        P.pl_total[w] = L.pl_total[w];
        P.pl_smem[w] = pl_smem[w];
    }
    P.fp_smem_replay = 0;
    for (int s = 0; s < n; ++s) P.fp_smem_replay = std::max(P.fp_smem_replay, zs[s].fpp.replay.smem);
    P.el_total = L.el_total;
    P.sn_total = L.sn_total;
    P.rc_total = L.rc_total;
    P.flt_total = L.flt_total;
    P.box_total = L.box_total;
    P.fp_minb = 2;
    size_t flt_smem = 0;
    for (int s = 0; s < n; ++s)
        if (zs[s].setup)
            flt_smem = std::max(flt_smem, filter_smem_bytes(scans[s].geom.num_det_channels,
                                                            scans[s].geom.kind != MBX_GEOM_PARALLEL));
    P.flt_smem = flt_smem;
    // kernel attributes and resident-CTA grids
    const void *kbp = bp_kernel_of(P.kind), *kfp2 = fp_kernel_of(P.kind, 2), *kfp3 = fp_kernel_of(P.kind, 3);
    e = set_max_dynamic_smem(kbp, 100 * 1024);
    if (e == cudaSuccess) e = set_max_dynamic_smem(kfp2, 200 * 1024);
    if (e == cudaSuccess) e = set_max_dynamic_smem(kfp3, 200 * 1024);
    for (int mb = 2; mb <= 3 && e == cudaSuccess && L.plan_fp; ++mb) {
        e = set_max_dynamic_smem(fp_kernel_of(P.kind, mb, CB_REPLAY), 200 * 1024);
        if (e == cudaSuccess) e = set_max_dynamic_smem(fp_kernel_of(P.kind, mb, CB_BUILD), 200 * 1024);
    }
    if (e == cudaSuccess) e = set_max_dynamic_smem(reinterpret_cast<const void *>(b_filter), 200 * 1024);
    if (e != cudaSuccess) return set_cuda_error(e);
    P.pl_grid[PL_BP] = bp_grid(P.kind, P.pl_smem[PL_BP], P.pl_total[PL_BP]);
    P.pl_grid[PL_FP] = fp_grid(P.kind, 2, P.pl_smem[PL_FP], P.pl_total[PL_FP]);
    P.pl_grid[PL_INIT_BP] = bp_grid(P.kind, P.pl_smem[PL_INIT_BP], std::max(1, P.pl_total[PL_INIT_BP]));
    P.pl_grid[PL_INIT_FP] = fp_grid(P.kind, 2, P.pl_smem[PL_INIT_FP], std::max(1, P.pl_total[PL_INIT_FP]));
    P.pl_grid[PL_HESS] = bp_grid(P.kind, P.pl_smem[PL_HESS], std::max(1, P.pl_total[PL_HESS]));
    {   // load every stage kernel now (lazy module loading must not happen inside a stream capture)
        cudaFuncAttributes fa;
        const void *ks[] = {reinterpret_cast<const void *>(b_delta), reinterpret_cast<const void *>(b_linquad),
                            reinterpret_cast<const void *>(b_alpha), reinterpret_cast<const void *>(b_apply),
                            reinterpret_cast<const void *>(b_error), reinterpret_cast<const void *>(b_l1),
                            reinterpret_cast<const void *>(b_iter_partials),
                            reinterpret_cast<const void *>(b_iter_final),
                            reinterpret_cast<const void *>(b_zero_recon), reinterpret_cast<const void *>(b_filter),
                            reinterpret_cast<const void *>(b_init_partials),
                            reinterpret_cast<const void *>(b_init_alpha),
                            reinterpret_cast<const void *>(b_init_apply),
                            reinterpret_cast<const void *>(b_copy_sino),
                            reinterpret_cast<const void *>(b_chunk_bounds)};
        for (const void *k : ks) cudaFuncGetAttributes(&fa, k);
        device_error_ptr();
    }
    P.el_grid = occupancy_grid(b_delta, BT_THREADS, 0, L.el_total);
    P.sn_grid = occupancy_grid(b_linquad, BT_THREADS, 0, L.sn_total);
    P.rc_grid = occupancy_grid(b_iter_partials, BT_THREADS, 0, L.sn_total + L.rc_total);
    P.flt_grid = occupancy_grid(b_filter, FILT_THREADS, std::max<size_t>(flt_smem, 1), std::max(1, L.flt_total));
    P.box_grid = occupancy_grid(b_chunk_bounds, CB_CHUNK, 0, std::max(1, L.box_total));
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error(e);
    // chunk bounding boxes of every subset, and of every region-of-reconstruction list
    b_chunk_bounds<<<P.box_grid, CB_CHUNK, 0, st>>>(P.t, P.ksum, P.box_total);
    note_launch();
    for (int s = 0; s < n && L.setup; ++s) {
        const unsigned nch = (unsigned)((scans[s].num_full_indices + CB_CHUNK - 1) / CB_CHUNK);
        fp_chunk_bounds_kernel<<<nch, CB_CHUNK, 0, st>>>(scans[s].full_indices, scans[s].num_full_indices,
                                                         scans[s].geom.num_recon_rows, scans[s].geom.num_recon_cols,
                                                         reinterpret_cast<int4 *>(base + L.fbox_off[s]));
        note_launch();
    }
    // no planned tile is replayed before a build stores it
    for (int s2 = 0, k2 = 0; s2 < n && L.plan_fp; ++s2)
        for (int k = 0; k < scans[s2].num_subsets && e == cudaSuccess; ++k, ++k2) {
            const PlannedSizes q = planned_sizes(scans[s2], zs[s2]);
            e = cudaMemsetAsync(base + L.plan_off[s2] + (size_t)k * q.total + q.tile_npass, 0xFF,
                                sizeof(int) * (size_t)q.tiles, st);
        }
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (autotune_enabled()) {  // (also in forced mode: the tune functions then apply the forced choice)
        const int *o_bp = hpl_off + PL_BP * n1, *o_fp = hpl_off + PL_FP * n1;
        int rc2 = tune_batched_fp(P, L, zs, scans, hf, st);
        if (rc2 == MBX_OK) rc2 = tune_batched_fp_layouts(P, L, scans, o_fp, hpl_order + PL_FP * n, st);
        if (rc2 == MBX_OK) rc2 = tune_batched_bp(P, L, scans, hb, o_bp, hpl_order + PL_BP * n, st);
        if (rc2 != MBX_OK) return rc2;
    }
    if (P.planned_fp) {  // the replay and build kernels of the forward variant the tuner kept
        P.pl_grid_replay = fp_grid(P.kind, P.fp_minb, P.fp_smem_replay, P.pl_total[PL_FP], CB_REPLAY);
        // the shared-memory carveout the resident replay CTAs need, no more: the rest of the SM's unified
        // L1 / shared storage caches the row loads of the walk
        e = set_smem_carveout(fp_kernel_of(P.kind, P.fp_minb, CB_REPLAY), CB_THREADS, P.fp_smem_replay);
        if (e != cudaSuccess) return set_cuda_error(e);
        P.pl_grid_build = fp_grid(P.kind, P.fp_minb, P.pl_smem[PL_FP], std::max(1, P.pl_total[PL_BUILD]), CB_BUILD);
    }
    P.magic = BT_MAGIC;
    std::memset(plan_out, 0, sizeof(*plan_out));
    std::memcpy(plan_out, &P, sizeof(P));
    return MBX_OK;
}

static int launch_stage(const BatchedPlanHost *P, int step, int stage, cudaStream_t st) {
    const BatchedTables &T = P->t;
    const int n = P->num_scans;
    const int warp_blocks = (n + 7) / 8;
    int *err = device_error_ptr();
    cudaError_t e = cudaSuccess;
    switch (stage) {
        case 0:
            e = launch_bp_list(*P, PL_BP, step, 0, P->pl_total[PL_BP], P->pl_grid[PL_BP], P->pl_smem[PL_BP], st);
            return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
        case 1: b_delta<<<P->el_grid, BT_THREADS, 0, st>>>(T, n, step, P->el_total, err); break;
        case 2:
            e = launch_fp_list(*P, PL_FP, P->fp_minb, step, 0, P->pl_total[PL_FP],
                               P->planned_fp ? P->pl_grid_replay : P->pl_grid[PL_FP],
                               P->planned_fp ? P->fp_smem_replay : P->pl_smem[PL_FP], st,
                               P->planned_fp ? CB_REPLAY : CB_WALK);
            return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
        case 3: b_linquad<<<P->sn_grid, BT_THREADS, 0, st>>>(T, n, P->sn_total); break;
        case 4: b_alpha<<<warp_blocks, 256, 0, st>>>(T, n, step); break;
        case 5: b_apply<<<P->el_grid, BT_THREADS, 0, st>>>(T, n, step, P->el_total); break;
        case 6: b_error<<<P->sn_grid, BT_THREADS, 0, st>>>(T, n, P->sn_total); break;
        case 7: b_l1<<<warp_blocks, 256, 0, st>>>(T, n, step); break;
        default: return MBX_ERR_INVALID_ARG;
    }
    note_launch();
    e = cudaGetLastError();
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

extern "C" int mbx_vcd_batched_setup(const mbx_batched_plan *plan, void *stream) {
    const BatchedPlanHost *P = plan_of(plan);
    if (!P) return MBX_ERR_INVALID_ARG;
    if (!P->has_setup) return MBX_ERR_UNSUPPORTED;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const BatchedTables &T = P->t;
    const int n = P->num_scans;
    b_zero_recon<<<P->rc_grid, BT_THREADS, 0, st>>>(T, n, P->rc_total);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (P->kind == MBX_GEOM_TRANSLATION) {  // zero initial recon: e = y
        b_copy_sino<<<P->sn_grid, BT_THREADS, 0, st>>>(T, n, P->sn_total);
        note_launch();
        e = cudaGetLastError();
    } else {
        b_filter<<<P->flt_grid, FILT_THREADS, P->flt_smem, st>>>(T, n, P->flt_total);
        note_launch();
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = launch_bp_list(*P, PL_INIT_BP, 0, 0, P->pl_total[PL_INIT_BP], P->pl_grid[PL_INIT_BP],
                               P->pl_smem[PL_INIT_BP], st);
        if (e == cudaSuccess)
            e = launch_fp_list(*P, PL_INIT_FP, 2, 0, 0, P->pl_total[PL_INIT_FP], P->pl_grid[PL_INIT_FP],
                               P->pl_smem[PL_INIT_FP], st);
        if (e != cudaSuccess) return set_cuda_error(e);
        b_init_partials<<<P->sn_grid, BT_THREADS, 0, st>>>(T, n, P->sn_total);
        note_launch();
        b_init_alpha<<<(n + 7) / 8, 256, 0, st>>>(T, n);
        note_launch();
        b_init_apply<<<P->rc_grid, BT_THREADS, 0, st>>>(T, n, P->sn_total, P->rc_total);
        note_launch();
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = launch_bp_list(*P, PL_HESS, 0, 0, P->pl_total[PL_HESS], P->pl_grid[PL_HESS], P->pl_smem[PL_HESS], st);
    return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
}

extern "C" int mbx_vcd_batched_update(const mbx_batched_plan *plan, const mbx_scan *scans, int32_t num_scans,
                                      const int32_t *schedule, void *stream) {
    const BatchedPlanHost *P = plan_of(plan);
    if (!P || !scans || !schedule || num_scans != P->num_scans) return MBX_ERR_INVALID_ARG;
    int ksum = 0;
    for (int s = 0; s < num_scans; ++s) {
        if (!(scans[s].qp.sigma_x > 0.0f) || !(scans[s].qp.T > 0.0f) || !(scans[s].qp.p > 0.0f))
            return MBX_ERR_INVALID_ARG;
        ksum += scans[s].num_subsets;
    }
    if (ksum != P->ksum) return MBX_ERR_INVALID_ARG;
    int rc = check_schedule(scans, num_scans, schedule, P->num_steps);
    if (rc != MBX_OK) return rc;
    std::vector<float> fm(num_scans);
    std::vector<QParams> qp(num_scans);
    fill_params(scans, num_scans, fm.data(), qp.data());
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // from pageable host memory: each copy is staged before the call returns, so the vectors may go
    cudaError_t e = cudaMemcpyAsync(P->t.fm, fm.data(), sizeof(float) * num_scans, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->t.qp, qp.data(), sizeof(QParams) * num_scans, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(P->t.schedule, schedule, sizeof(int32_t) * (size_t)P->num_steps * num_scans,
                            cudaMemcpyHostToDevice, st);
    return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
}

extern "C" int mbx_vcd_batched_refresh(const mbx_batched_plan *plan, void *stream) {
    const BatchedPlanHost *P = plan_of(plan);
    if (!P) return MBX_ERR_INVALID_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    b_chunk_bounds<<<P->box_grid, CB_CHUNK, 0, st>>>(P->t, P->ksum, P->box_total);
    note_launch();
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess && P->planned_fp) {  // store the sorted passes of every subset's tiles
        e = cudaMemsetAsync(P->plan_cursors, 0, P->plan_cursor_bytes, st);
        if (e == cudaSuccess)
            e = launch_fp_list(*P, PL_BUILD, P->fp_minb, 0, 0, P->pl_total[PL_BUILD], P->pl_grid_build,
                               P->pl_smem[PL_FP], st, CB_BUILD);
    }
    return e == cudaSuccess ? MBX_OK : set_cuda_error(e);
}
