// Translation-geometry instantiations of the batched forward-projection stage kernels (compiled separately for build
// parallelism).
#include "b_fp_stage.cuh"

namespace mbx {

const void *fp_stage_kernel_translation(int minb, int mode) { return fp_stage_kernel_kind<MBX_GEOM_TRANSLATION>(minb, mode); }

void launch_fp_stage_translation(int minb, int mode, int grid, size_t smem, cudaStream_t st, const ProjList &L, int n,
                        int step, int first, int total, int *err) {
    launch_fp_stage_kind<MBX_GEOM_TRANSLATION>(minb, mode, grid, smem, st, L, n, step, first, total, err);
}

}  // namespace mbx
