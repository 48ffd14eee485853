// Sparse back projection that allocates nothing: its scratch lives in a static device array.
//
// Some callers of this library cannot allocate GPU memory at call time.  JAX, for example, hands about 98%
// of the device to its own allocator at start-up (the mbirjax reference sets
// XLA_PYTHON_CLIENT_MEM_FRACTION=0.98), so a projector called from inside such a program finds no room for
// cudaMalloc.  Real-time pipelines that reserve all memory up front have the same constraint.  This entry
// point takes the same inputs and outputs as mbx_sparse_back_project but no workspace.  When the back
// projector splits the views over CTAs it keeps the partial sums in g_bp_scratch, a file-scope device array of
// MBX_NOALLOC_SCRATCH_BYTES that every GPU which uses this entry point holds until the process exits.
//
// Its device address is looked up once per device (cudaGetSymbolAddress with that device current) on the
// first call on that device; make that first call before any stream capture.  Every call on a device shares
// the one array: calls whose GPU work overlaps (two streams, or two host threads) race on it and must be
// serialised by the caller.  The array keeps the last call's contents; nothing needs clearing, because each call
// writes every scratch element it later reads.
#include <mutex>

#include "mbx_common.cuh"
#include "mbx_host.hpp"

// The scratch array (file scope, one per device that loads this module).
static __device__ __align__(256) float g_bp_scratch[MBX_NOALLOC_SCRATCH_BYTES / sizeof(float)];

namespace {

std::mutex g_scratch_mutex;
void *g_scratch_ptr[64] = {nullptr};

// Device address of g_bp_scratch on the current device (set up on the first call per device).
int scratch_for_current_device(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return mbx::set_cuda_error(e);
    if (dev < 0 || dev >= 64) return MBX_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_bp_scratch);
        if (e != cudaSuccess) return mbx::set_cuda_error(e);
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return MBX_OK;
}

}  // namespace

extern "C" int mbx_sparse_back_project_noalloc(const mbx_geom *g, const float *sinogram, const float *weights,
                                               const int32_t *pixel_indices, int64_t num_pixels,
                                               const int32_t *view_indices, int32_t num_views_sel,
                                               int32_t coeff_power, float scale, float *out, void *stream) {
    int rc = mbx::validate_geom(g);
    if (rc != MBX_OK) return rc;
    if (num_pixels < 0 || num_views_sel <= 0) return MBX_ERR_INVALID_ARG;
    if (num_pixels > 0 && (!pixel_indices || !out)) return MBX_ERR_INVALID_ARG;
    if (coeff_power != 1 && coeff_power != 2) return MBX_ERR_UNSUPPORTED;
    if (!view_indices && num_views_sel > g->num_views) return MBX_ERR_INVALID_ARG;
    if (num_pixels == 0) return MBX_OK;
    if (!sinogram) {  // as mbx_sparse_back_project: the weights, or 1 everywhere
        sinogram = weights;
        weights = nullptr;
    }
    const size_t need = mbx::bp_workspace_bytes(*g, num_pixels, num_views_sel);
    if (need > MBX_NOALLOC_SCRATCH_BYTES) return MBX_ERR_WORKSPACE;  // more scratch than the static array holds
    void *scratch = nullptr;
    if (need > 0) {
        rc = scratch_for_current_device(&scratch);
        if (rc != MBX_OK) return rc;
    }
    return mbx::back_project(*g, sinogram, weights, pixel_indices, num_pixels, view_indices, num_views_sel,
                             coeff_power, scale, out, scratch, need, static_cast<cudaStream_t>(stream));
}
