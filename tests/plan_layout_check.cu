// Host-only check of the channel-block forward projector's shared-memory plans (fp_cb.cuh): for a sweep of
// geometries it builds every plan the library and the batched path can choose (variants for 2 and 3 resident CTAs,
// the alternative channel-block width and lane layout, passes of at most 2048 and 1024 records) and verifies
//  - the walk layout fits the 200 KB the kernels are allowed and holds its passes, sort buffers and cone tables in
//    order;
//  - the replay layout holds the tile, the records of a walk-sized pass and the bin starts;
//  - the smaller walk used by the replay kernel for tiles a build could not store fits the replay's shared memory;
// printing "ok <plans checked>" or the first failure.  Runs on the CPU (no device call).
#include <cmath>
#include <cstdio>

#include "../mbirjax_b200/csrc/fp_cb.cuh"

using namespace mbx;

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
    std::printf("ok %ld\n", checked);
    return checked > 0 ? 0 : 1;
}
