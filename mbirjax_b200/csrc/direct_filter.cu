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
// while staging; both geometries apply the final pi / num_views.
#include <cmath>

#include "mbx_common.cuh"
#include "mbx_host.hpp"

namespace mbx {

constexpr int FILT_ROWS = 8;
constexpr int FILT_THREADS = 256;

__global__ void __launch_bounds__(FILT_THREADS)
direct_filter_kernel(const float *__restrict__ sino, float *__restrict__ out, long long num_rows_total, int R, int C,
                     float filter_scale, float out_scale, int fdk, float D, float delta_det_channel,
                     float delta_det_row, float det_channel_offset, float det_row_offset) {
    extern __shared__ __align__(16) float sm[];
    float *rows_t = sm;                         // [C][FILT_ROWS]
    float *filt = sm + (size_t)C * FILT_ROWS;   // [2C-1]
    const long long row0 = (long long)blockIdx.x * FILT_ROWS;
    const int nrows = (int)min((long long)FILT_ROWS, num_rows_total - row0);

    const double kInvPi2 = 0.10132118364233778;  // 1 / pi^2
    for (int t = threadIdx.x; t < 2 * C - 1; t += blockDim.x) {
        const int d = t - (C - 1);
        float h;
        if (d == 0)
            h = 0.25f;
        else if (d & 1)
            h = (float)(-kInvPi2 / ((double)d * (double)d));
        else
            h = 0.0f;
        filt[t] = filter_scale * h;
    }
    const float det_center_row = 0.5f * (float)(R - 1);
    const float det_center_channel = 0.5f * (float)(C - 1);
    for (int t = threadIdx.x; t < C * FILT_ROWS; t += blockDim.x) {
        const int rr = t / C;
        const int j = t - rr * C;
        float v = 0.0f;
        if (rr < nrows) {
            const long long grow = row0 + rr;
            v = sino[grow * C + j];
            if (fdk && isfinite(D)) {
                const int m = (int)(grow % R);
                const float vv = ((float)m - det_center_row) * delta_det_row - det_row_offset;
                const float uu = ((float)j - det_center_channel) * delta_det_channel - det_channel_offset;
                v *= D / sqrtf(D * D + uu * uu + vv * vv);
            }
        }
        rows_t[j * FILT_ROWS + rr] = v;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < C; i += blockDim.x) {
        float acc[FILT_ROWS];
        {
            const float h0 = filt[C - 1];
            const float4 a = *reinterpret_cast<const float4 *>(rows_t + i * FILT_ROWS);
            const float4 b = *reinterpret_cast<const float4 *>(rows_t + i * FILT_ROWS + 4);
            acc[0] = h0 * a.x; acc[1] = h0 * a.y; acc[2] = h0 * a.z; acc[3] = h0 * a.w;
            acc[4] = h0 * b.x; acc[5] = h0 * b.y; acc[6] = h0 * b.z; acc[7] = h0 * b.w;
        }
        // odd differences i - j only
        for (int j = (i + 1) & 1; j < C; j += 2) {
            const float h = filt[i - j + C - 1];
            const float4 a = *reinterpret_cast<const float4 *>(rows_t + j * FILT_ROWS);
            const float4 b = *reinterpret_cast<const float4 *>(rows_t + j * FILT_ROWS + 4);
            acc[0] = fmaf(h, a.x, acc[0]); acc[1] = fmaf(h, a.y, acc[1]);
            acc[2] = fmaf(h, a.z, acc[2]); acc[3] = fmaf(h, a.w, acc[3]);
            acc[4] = fmaf(h, b.x, acc[4]); acc[5] = fmaf(h, b.y, acc[5]);
            acc[6] = fmaf(h, b.z, acc[6]); acc[7] = fmaf(h, b.w, acc[7]);
        }
#pragma unroll
        for (int rr = 0; rr < FILT_ROWS; ++rr)
            if (rr < nrows) out[(row0 + rr) * C + i] = out_scale * acc[rr];
    }
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
    const size_t smem = ((size_t)C * mbx::FILT_ROWS + 2 * (size_t)C - 1) * sizeof(float);
    if (smem > 200 * 1024) return MBX_ERR_UNSUPPORTED;
    {
        cudaError_t e = mbx::set_max_dynamic_smem(reinterpret_cast<const void *>(mbx::direct_filter_kernel),
                                                  200 * 1024);
        if (e != cudaSuccess) return mbx::set_cuda_error(e);
    }
    const long long rows_total = (long long)g->num_views * R;
    const double pi = 3.14159265358979323846;
    float filter_scale, out_scale = (float)(pi / g->num_views);
    int fdk = 0;
    if (g->kind == MBX_GEOM_PARALLEL) {
        filter_scale = (float)(1.0 / ((double)g->delta_voxel * g->delta_voxel));
    } else {
        filter_scale = (float)((double)g->delta_det_row /
                               ((double)g->delta_voxel * g->delta_voxel * g->delta_voxel * g->magnification));
        fdk = 1;
    }
    const unsigned blocks = (unsigned)((rows_total + mbx::FILT_ROWS - 1) / mbx::FILT_ROWS);
    mbx::direct_filter_kernel<<<blocks, mbx::FILT_THREADS, smem, static_cast<cudaStream_t>(stream)>>>(
        sinogram, out, rows_total, R, C, filter_scale, out_scale, fdk, g->source_detector_dist, g->delta_det_channel,
        g->delta_det_row, g->det_channel_offset, g->det_row_offset);
    mbx::note_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? MBX_OK : mbx::set_cuda_error(e);
}
