// Ramp filtering of detector rows for FBP / FDK (sm_100a): the device function shared by the plain entry point
// (direct_filter.cu) and the batched VCD set-up (vcd_batched.cu).  See direct_filter.cu for the arithmetic.
#pragma once

#include <cmath>

#include "mbx_common.cuh"

namespace mbx {

constexpr int FILT_ROWS = 8;
constexpr int FILT_THREADS = 256;

// Scales of the ramp filter for a geometry: the filter times 1/delta_voxel^2 (FBP, parallel_beam.py:325-327) or
// delta_det_row / (delta_voxel^3 magnification) after the FDK pre-weight (cone_beam.py:825-827), and pi / views.
inline void direct_filter_scales(const mbx_geom &g, double &filter_scale, double &out_scale, int &fdk) {
    const double pi = 3.14159265358979323846;
    out_scale = pi / g.num_views;
    if (g.kind == MBX_GEOM_PARALLEL) {
        filter_scale = 1.0 / ((double)g.delta_voxel * g.delta_voxel);
        fdk = 0;
    } else {
        filter_scale = (double)g.delta_det_row /
                       ((double)g.delta_voxel * g.delta_voxel * g.delta_voxel * g.magnification);
        fdk = 1;
    }
}

// Shared memory of one filter tile for rows of C channels: the rows and, for FDK, the low parts of the
// pre-weighted rows ([C][FILT_ROWS] floats each), then the 2C-1 taps in float64.
inline size_t filter_smem_bytes(int C, int fdk) {
    return (fdk ? 2 : 1) * (size_t)C * FILT_ROWS * sizeof(float) + (2 * (size_t)C - 1) * sizeof(double);
}

// Filters rows row0 .. row0 + FILT_ROWS - 1 (fewer at the end) of a (num_rows_total, C) stack of detector rows
// (R rows per view) with the whole block; sm holds filter_smem_bytes(C).
// The taps, the FDK pre-weight, the sums and the scales are float64 and each output is rounded once, as the
// reference's filter is specified (a float64 evaluation of the convolution differs from any float32 one by
// rounding only).  An FDK pre-weighted sample is held as a float pair (hi + lo), which carries it to about 48
// bits, so one float4 pair of shared memory still feeds FILT_ROWS accumulators.
__device__ __forceinline__ void direct_filter_rows(const float *__restrict__ sino, float *__restrict__ out,
                                                   long long row0, long long num_rows_total, int R, int C,
                                                   double filter_scale, double out_scale, int fdk, double D,
                                                   double delta_det_channel, double delta_det_row,
                                                   double det_channel_offset, double det_row_offset, float *sm) {
    float *rows_t = sm;                                    // [C][FILT_ROWS]
    float *rows_lo = sm + (size_t)C * FILT_ROWS;           // FDK: [C][FILT_ROWS]
    double *filt = reinterpret_cast<double *>(sm + (fdk ? 2 : 1) * (size_t)C * FILT_ROWS);  // [2C-1]
    const int nrows = (int)min((long long)FILT_ROWS, num_rows_total - row0);

    const double kInvPi2 = 0.10132118364233778;  // 1 / pi^2
    for (int t = threadIdx.x; t < 2 * C - 1; t += blockDim.x) {
        const int d = t - (C - 1);
        double h;
        if (d == 0)
            h = 0.25;
        else if (d & 1)
            h = -kInvPi2 / ((double)d * (double)d);
        else
            h = 0.0;
        filt[t] = filter_scale * h;
    }
    const bool weighted = fdk && isfinite(D);
    const double det_center_row = 0.5 * (double)(R - 1);
    const double det_center_channel = 0.5 * (double)(C - 1);
    for (int t = threadIdx.x; t < C * FILT_ROWS; t += blockDim.x) {
        const int rr = t / C;
        const int j = t - rr * C;
        float hi = 0.0f, lo = 0.0f;
        if (rr < nrows) {
            const long long grow = row0 + rr;
            hi = sino[grow * C + j];
            if (weighted) {
                const int m = (int)(grow % R);
                const double vv = ((double)m - det_center_row) * delta_det_row - det_row_offset;
                const double uu = ((double)j - det_center_channel) * delta_det_channel - det_channel_offset;
                const double v = (double)hi * (D / sqrt(D * D + uu * uu + vv * vv));
                hi = (float)v;
                lo = (float)(v - (double)hi);
            }
        }
        rows_t[j * FILT_ROWS + rr] = hi;
        if (fdk) rows_lo[j * FILT_ROWS + rr] = lo;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < C; i += blockDim.x) {
        double acc[FILT_ROWS];
        {
            const double h0 = filt[C - 1];
            const float4 a = *reinterpret_cast<const float4 *>(rows_t + i * FILT_ROWS);
            const float4 b = *reinterpret_cast<const float4 *>(rows_t + i * FILT_ROWS + 4);
            acc[0] = h0 * a.x; acc[1] = h0 * a.y; acc[2] = h0 * a.z; acc[3] = h0 * a.w;
            acc[4] = h0 * b.x; acc[5] = h0 * b.y; acc[6] = h0 * b.z; acc[7] = h0 * b.w;
        }
        // odd differences i - j only (the even taps are zero)
        for (int j = (i + 1) & 1; j < C; j += 2) {
            const double h = filt[i - j + C - 1];
            const float4 a = *reinterpret_cast<const float4 *>(rows_t + j * FILT_ROWS);
            const float4 b = *reinterpret_cast<const float4 *>(rows_t + j * FILT_ROWS + 4);
            acc[0] = fma(h, (double)a.x, acc[0]); acc[1] = fma(h, (double)a.y, acc[1]);
            acc[2] = fma(h, (double)a.z, acc[2]); acc[3] = fma(h, (double)a.w, acc[3]);
            acc[4] = fma(h, (double)b.x, acc[4]); acc[5] = fma(h, (double)b.y, acc[5]);
            acc[6] = fma(h, (double)b.z, acc[6]); acc[7] = fma(h, (double)b.w, acc[7]);
        }
        if (weighted) {  // the low parts of the pre-weighted samples
            {
                const double h0 = filt[C - 1];
                const float4 a = *reinterpret_cast<const float4 *>(rows_lo + i * FILT_ROWS);
                const float4 b = *reinterpret_cast<const float4 *>(rows_lo + i * FILT_ROWS + 4);
                acc[0] = fma(h0, (double)a.x, acc[0]); acc[1] = fma(h0, (double)a.y, acc[1]);
                acc[2] = fma(h0, (double)a.z, acc[2]); acc[3] = fma(h0, (double)a.w, acc[3]);
                acc[4] = fma(h0, (double)b.x, acc[4]); acc[5] = fma(h0, (double)b.y, acc[5]);
                acc[6] = fma(h0, (double)b.z, acc[6]); acc[7] = fma(h0, (double)b.w, acc[7]);
            }
            for (int j = (i + 1) & 1; j < C; j += 2) {
                const double h = filt[i - j + C - 1];
                const float4 a = *reinterpret_cast<const float4 *>(rows_lo + j * FILT_ROWS);
                const float4 b = *reinterpret_cast<const float4 *>(rows_lo + j * FILT_ROWS + 4);
                acc[0] = fma(h, (double)a.x, acc[0]); acc[1] = fma(h, (double)a.y, acc[1]);
                acc[2] = fma(h, (double)a.z, acc[2]); acc[3] = fma(h, (double)a.w, acc[3]);
                acc[4] = fma(h, (double)b.x, acc[4]); acc[5] = fma(h, (double)b.y, acc[5]);
                acc[6] = fma(h, (double)b.z, acc[6]); acc[7] = fma(h, (double)b.w, acc[7]);
            }
        }
#pragma unroll
        for (int rr = 0; rr < FILT_ROWS; ++rr)
            if (rr < nrows) out[(row0 + rr) * C + i] = (float)(out_scale * acc[rr]);
    }
    __syncthreads();  // the block may stage its next tile into sm
}

}  // namespace mbx
