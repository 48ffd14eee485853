// Translation-geometry instantiations of the back-projection kernel (compiled separately for build parallelism).
#include "back_project.cuh"

namespace mbx {

cudaError_t launch_bp_translation(const mbx_geom &g, const BpPlan &pl, const float *sino, const float *w,
                                  const int32_t *pix, long long n, const int32_t *views, int nv, int cp, float scale,
                                  float *dst, long long ss, cudaStream_t st) {
    return launch_bp_kind<MBX_GEOM_TRANSLATION>(g, pl, sino, w, pix, n, views, nv, cp, scale, dst, ss, st);
}

}  // namespace mbx
