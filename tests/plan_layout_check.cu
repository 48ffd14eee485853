// Host-only check of the channel-block forward projector's shared-memory plans (fp_cb.cuh): for a sweep of
// geometries it builds every plan the library and the batched path can choose (variants for 2 and 3 resident CTAs,
// the alternative channel-block width and lane layout, passes of at most 2048 and 1024 records) and verifies
//  - the walk layout fits the 200 KB the kernels are allowed and holds its passes, sort buffers and cone tables in
//    order;
//  - the replay layout holds the tile, the records of a walk-sized pass and the bin starts;
//  - the smaller walk used by the replay kernel for tiles a build could not store fits the replay's shared memory;
// and for the back projector's plans (bp_fast.cuh, staged and per-thread footprints, any pixel count and view
// selection) that the CTA shape, slice tiles, view chunks and splits cover the work, that shared memory stays
// within the 100 KB its launches allow, and that a cone slice tile's rows fit the row cache;
// printing "ok <plans checked>" or the first failure.  Runs on the CPU (no device call).
#include <cmath>
#include <cstdio>

#include "../mbirjax_b200/csrc/bp_fast.cuh"
#include "../mbirjax_b200/csrc/fp_cb.cuh"

namespace mbx {
int num_sms() { return 148; }  // the device query of the library, for a B200
}  // namespace mbx

using namespace mbx;

// Back-projection plan invariants; returns a failure text or nullptr.
static const char *bp_plan_error(const mbx_geom &g, const BpfPlan &pl, long long n, int nv) {
    const int S = g.num_recon_slices;
    if (pl.nsl * pl.npg != 8 || (1 << pl.lg_pcta) != 32 * pl.npg) return "CTA shape";
    if (pl.ts < 1 || pl.ts > BPF_ST || (long long)pl.tiles * pl.ts < S || (long long)(pl.tiles - 1) * pl.ts >= S)
        return "slice tiles";
    if (pl.gy != (pl.tiles + pl.nsl - 1) / pl.nsl) return "grid y";
    if ((long long)pl.gx * 32 * pl.npg < n) return "grid x";
    if (!pl.inline_fp && (pl.chunk % (32 * pl.npg) || pl.vc != pl.chunk / (32 * pl.npg) || pl.vc < 1)) return "chunk";
    if (pl.splits < 1 || pl.splits > 64 || (long long)pl.splits * pl.views_per_split < nv ||
        (long long)(pl.splits - 1) * pl.views_per_split >= nv)
        return "view splits";
    if ((pl.splits > 1) != (pl.workspace > 0) || (pl.splits > 1 && pl.workspace < (size_t)pl.splits * n * S * 4))
        return "workspace";
    if (pl.smem > 100 * 1024) return "shared memory";
    if (g.kind != MBX_GEOM_PARALLEL && pl.ok) {
        const double half_r = 0.5 * (g.num_recon_rows - 1), half_c = 0.5 * (g.num_recon_cols - 1);
        const double rho = g.delta_voxel * std::sqrt(half_r * half_r + half_c * half_c);
        const double inv = 1.0 / g.magnification - rho / g.source_detector_dist;
        const double mag = g.kind == MBX_GEOM_TRANSLATION ? g.max_magnification : 1.0 / inv;
        if (pl.ts * mag * g.delta_voxel / g.delta_det_row + 4 > BPF_CACHE_ROWS) return "row cache";
    }
    return nullptr;
}

static int fail(const char *what, int kind, int R, int C) {
    std::printf("FAIL %s kind=%d R=%d C=%d\n", what, kind, R, C);
    return 1;
}

static bool layout_ok(const CbPlan &pl, const CbLayout &lo, int kind, int R, bool replay) {
    const size_t tile = (size_t)pl.ppw * pl.rpad * pl.pitch;
    if ((size_t)lo.o_rec < tile || lo.o_rec % 4) return false;            // float4 records after the tile copies
    if (lo.o_rec2 < lo.o_rec + 4 * (lo.cap + CB_PAD)) return false;
    if (lo.o_sbin < lo.o_rec2 + (kind != MBX_GEOM_PARALLEL ? 4 * lo.cap : 0)) return false;
    const int end_sbin = lo.o_sbin + lo.cap + CB_PAD;
    if (replay) {
        if (lo.o_bstart < end_sbin || lo.o_cone < lo.o_bstart + pl.nbins + 1) return false;
    } else {
        if (lo.o_ubin < end_sbin || lo.o_bstart < lo.o_ubin + lo.cap || lo.o_run < lo.o_bstart + pl.nbins + 1 ||
            lo.o_wcnt < lo.o_run + pl.nbins || lo.o_wstart < lo.o_wcnt + CB_WARPS * pl.nbins ||
            lo.o_cone < lo.o_wstart + CB_WARPS * pl.nbins)
            return false;
    }
    const size_t cone_end = (size_t)lo.o_cone + (kind != MBX_GEOM_PARALLEL ? 3 * (size_t)R : 0);
    if ((size_t)lo.o_win < cone_end) return false;
    const size_t win = kind != MBX_GEOM_PARALLEL
                           ? (size_t)CB_WARPS * cb_cone_records(pl.rpl) * pl.ppw * cb_cone_window(pl.ppw, pl.rpl)
                           : 0;
    return 4 * ((size_t)lo.o_win + win) <= lo.smem && lo.fill == lo.cap - CB_THREADS && lo.cap >= CB_THREADS;
}

int main() {
    long checked = 0;
    const int kinds[3] = {MBX_GEOM_PARALLEL, MBX_GEOM_CONE, MBX_GEOM_TRANSLATION};
    const int chans[7] = {32, 96, 131, 200, 317, 512, 1024};
    for (int kind : kinds)
        for (int R = 1; R <= 96; ++R)
            for (int C : chans) {
                mbx_geom g = {};
                g.kind = kind;
                g.num_views = 64;
                g.num_det_rows = R;
                g.num_det_channels = C;
                g.num_recon_rows = g.num_recon_cols = C;
                g.num_recon_slices = R;
                g.psf_radius = 1;
                g.bp_psf_radius = 1;
                g.entries_per_cylinder_batch = 128;
                g.delta_det_channel = g.delta_det_row = g.delta_voxel = 1.0f;
                g.source_detector_dist = kind == MBX_GEOM_PARALLEL ? INFINITY : 4.0f * C;
                g.magnification = kind == MBX_GEOM_PARALLEL ? 1.0f : 2.0f;
                g.delta_recon_row = 1.0f;
                g.max_magnification = kind == MBX_GEOM_TRANSLATION ? 2.0f : 0.0f;
                for (int minb = 2; minb <= 3; ++minb)
                    for (int max_cap : {2048, 1024})
                        for (int variant = 0; variant < 3; ++variant) {
                            const CbPlan base = plan_fp_cb(g, 0, 0, minb, 128, 0, max_cap);
                            if (!base.ok) continue;
                            const CbPlan pl = variant == 0   ? base
                                              : variant == 1 ? plan_fp_cb(g, 0, 0, minb, base.nb / 2 >= 32 ? base.nb / 2 : 32, 0, max_cap)
                                                             : plan_fp_cb(g, 0, 0, minb, 128, base.ppw, max_cap);
                            if (!pl.ok) continue;
                            ++checked;
                            if (pl.walk.smem > 200 * 1024) return fail("walk over 200 KB", kind, R, C);
                            if (pl.walk.cap > max_cap) return fail("pass over max_cap", kind, R, C);
                            if (!layout_ok(pl, pl.walk, kind, R, false)) return fail("walk layout", kind, R, C);
                            if (pl.replay.cap != pl.walk.cap) return fail("replay pass size", kind, R, C);
                            if (!layout_ok(pl, pl.replay, kind, R, true)) return fail("replay layout", kind, R, C);
                            if (pl.replay.smem > pl.walk.smem) return fail("replay larger than walk", kind, R, C);
                            if (pl.small.cap > pl.walk.cap) return fail("small pass size", kind, R, C);
                            if (!layout_ok(pl, pl.small, kind, R, false)) return fail("small layout", kind, R, C);
                            if (pl.small.smem > pl.replay.smem) return fail("small walk over replay smem", kind, R, C);
                            if (pl.rpad < R || pl.rpad != pl.row_passes * pl.rl * pl.rpl) return fail("rows", kind, R, C);
                        }
            }
    for (int kind : kinds)
        for (int S = 1; S <= 200; S += (S < 40 ? 1 : 7))
            for (int C : chans) {
                mbx_geom g = {};
                g.kind = kind;
                g.num_views = 180;
                g.num_det_rows = S;
                g.num_det_channels = C;
                g.num_recon_rows = g.num_recon_cols = C;
                g.num_recon_slices = S;
                g.psf_radius = g.bp_psf_radius = 1;
                g.entries_per_cylinder_batch = 128;
                g.delta_det_channel = g.delta_det_row = g.delta_voxel = 1.0f;
                g.source_detector_dist = kind == MBX_GEOM_PARALLEL ? INFINITY : 4.0f * C;
                g.magnification = kind == MBX_GEOM_PARALLEL ? 1.0f : 2.0f;
                g.delta_recon_row = 1.0f;
                g.max_magnification = kind == MBX_GEOM_TRANSLATION ? 2.0f : 0.0f;
                for (long long n : {1LL, 31LL, 1000LL, 20000LL, (long long)C * C})
                    for (int nv : {1, 16, 180})
                        for (int inl = 0; inl <= 1; ++inl) {
                            const BpfPlan pl = plan_bp_fast(g, n, nv, inl);
                            if (!pl.ok) continue;
                            ++checked;
                            const char *e = bp_plan_error(g, pl, n, nv);
                            if (e) return fail(e, kind, S, C);
                        }
            }
    std::printf("ok %ld\n", checked);
    return checked > 0 ? 0 : 1;
}
