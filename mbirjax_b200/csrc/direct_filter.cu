// FBP / FDK sinogram filtering (sm_100a).
//
// Replaces ParallelBeamModel.fbp_filter (parallel_beam.py:303-348) and ConeBeamModel.fdk_filter
// (cone_beam.py:779-846) with the ramp filter of generate_direct_recon_filter (tomography_utils.py:4-35):
//   h[d] = 1/2 sinc(d) - 1/4 sinc(d/2)^2, d in [-(C-1), C-1]  ->  h[0] = 1/4, h[odd d] = -1/(pi d)^2, h[even] = 0
// and the 'valid' part of fftconvolve(row, h): out[i] = sum_j row[j] h[i - j].
// The convolution is evaluated directly (only the C/2 odd taps and the centre tap are nonzero), which on a
// B200 costs less than the back projection that follows it by orders of magnitude.  One CTA filters
// FILT_ROWS detector rows: it stages them transposed in shared memory ([channel][row], so one float4 pair
// feeds FILT_ROWS accumulators), stages the scaled filter taps, and each thread produces channel outputs.
// FDK: the pre-weight D / sqrt(D^2 + u^2 + v^2) (cone_beam.py:806-818, detector_mn_to_uv :709-738) is applied
// while staging; both geometries apply the final pi / num_views.  Taps, pre-weight and sums are float64 (the
// float32 sums of a direct convolution are off by a few 1e-6 of the row's scale, which the VCD iterations that
// start from this recon can amplify).
#include "direct_filter.cuh"
#include "mbx_host.hpp"

namespace mbx {

__global__ void __launch_bounds__(FILT_THREADS)
direct_filter_kernel(const float *__restrict__ sino, float *__restrict__ out, long long num_rows_total, int R, int C,
                     double filter_scale, double out_scale, int fdk, double D, double delta_det_channel,
                     double delta_det_row, double det_channel_offset, double det_row_offset) {
    extern __shared__ __align__(16) float sm[];
    direct_filter_rows(sino, out, (long long)blockIdx.x * FILT_ROWS, num_rows_total, R, C, filter_scale, out_scale,
                       fdk, D, delta_det_channel, delta_det_row, det_channel_offset, det_row_offset, sm);
}

}  // namespace mbx

extern "C" int mbx_direct_filter(const mbx_geom *g, const float *sinogram, float *out, void *stream) {
    int rc = mbx::validate_geom(g);
    if (rc != MBX_OK) return rc;
    if (!sinogram || !out || sinogram == out) return MBX_ERR_INVALID_ARG;
    // translation geometry has no direct reconstruction (the base TomographyModel's zeros,
    // tomography_model.py:934-964)
    if (g->kind == MBX_GEOM_TRANSLATION) return MBX_ERR_UNSUPPORTED;
    const int C = g->num_det_channels, R = g->num_det_rows;
    const size_t smem = mbx::filter_smem_bytes(C, g->kind != MBX_GEOM_PARALLEL);
    if (smem > 200 * 1024) return MBX_ERR_UNSUPPORTED;
    {
        cudaError_t e = mbx::set_max_dynamic_smem(reinterpret_cast<const void *>(mbx::direct_filter_kernel),
                                                  200 * 1024);
        if (e != cudaSuccess) return mbx::set_cuda_error(e);
    }
    const long long rows_total = (long long)g->num_views * R;
    double filter_scale, out_scale;
    int fdk;
    mbx::direct_filter_scales(*g, filter_scale, out_scale, fdk);
    const unsigned blocks = (unsigned)((rows_total + mbx::FILT_ROWS - 1) / mbx::FILT_ROWS);
    mbx::direct_filter_kernel<<<blocks, mbx::FILT_THREADS, smem, static_cast<cudaStream_t>(stream)>>>(
        sinogram, out, rows_total, R, C, filter_scale, out_scale, fdk, g->source_detector_dist, g->delta_det_channel,
        g->delta_det_row, g->det_channel_offset, g->det_row_offset);
    mbx::note_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MBX_OK : mbx::set_cuda_error(e);
}
