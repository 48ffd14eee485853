// Shared device helpers for the mbirjax_b200 kernels (sm_100a).
//
// The per-pixel geometry below restates, in float32 as the reference evaluates it, the footprint
// quantities of mbirjax v0.6.7:
//   parallel: compute_proj_data / recon_ij_to_x          parallel_beam.py:223-284
//   cone:     compute_horizontal_data / recon_ijk_to_xyz  cone_beam.py:593-666
//             vertical fan (FP, detector-row-centric)     cone_beam.py:286-377
//             vertical fan (BP, voxel-centric)            cone_beam.py:480-591
//   translation: compute_horizontal_data / recon_ijk_to_xyz  translation_model.py:595-656
//             vertical fans as the cone's, with the slice axis shifted by -tz per view
//             (translation_model.py:286-378 FP, :482-593 BP)
// One deliberate difference: 1/cos(phi) of the vertical cone angle is evaluated as sqrt(1 + (v/D)^2)
// (the same quantity as 1/cos(atan2(v, D))) because it is needed per voxel tap in the inner loops.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/mbirjax_b200.h"

#define MBX_ERRFLAG_PIXEL 1
#define MBX_ERRFLAG_VIEW 2
#define MBX_ERRFLAG_CACHE 4

namespace mbx {

constexpr int kNumSMsDefault = 148;

// Kernels receive the address of the device error word (defined in common.cu) as `err`.
__device__ __forceinline__ void flag_error(int *err, int bit) {
    if (err) atomicOr(err, bit);
}

// Quotient of i by d > 0, and the remainder in r: in 32-bit arithmetic when i fits in 31 bits (every element
// index of a cylinder list the library admits), a fraction of the instructions of a 64-bit division.
__device__ __forceinline__ long long div_rem(long long i, int d, int &r) {
    if (i >= 0 && i <= 0x7fffffffLL) {
        const unsigned q = (unsigned)i / (unsigned)d;
        r = (int)((unsigned)i - q * (unsigned)d);
        return (long long)q;
    }
    const long long q = i / d;
    r = (int)(i - q * d);
    return q;
}

// Recon (row, col) of a flat pixel index, as offsets from the recon centre in ALU (y_tilde, x_tilde).
__device__ __forceinline__ void pixel_tilde(const mbx_geom &g, int idx, float &x_tilde, float &y_tilde) {
    const int row = idx / g.num_recon_cols;
    const int col = idx - row * g.num_recon_cols;
    y_tilde = g.delta_voxel * ((float)row - 0.5f * (float)(g.num_recon_rows - 1));
    x_tilde = g.delta_voxel * ((float)col - 0.5f * (float)(g.num_recon_cols - 1));
}

// Same, with the row / column split of the flat index done by a float reciprocal (inv_cols = 1/num_recon_cols)
// and an exact integer correction instead of an integer division; row_pitch > 0 replaces delta_voxel as the row
// spacing (translation geometry's delta_recon_row).
__device__ __forceinline__ void pixel_tilde_fast(const mbx_geom &g, int idx, float inv_cols, float &x_tilde,
                                                 float &y_tilde, float row_pitch = 0.0f) {
    int row = __float2int_rz(__int2float_rz(idx) * inv_cols);
    int col = idx - row * g.num_recon_cols;
    if (col < 0) {
        --row;
        col += g.num_recon_cols;
    } else if (col >= g.num_recon_cols) {
        ++row;
        col -= g.num_recon_cols;
    }
    y_tilde = (row_pitch > 0.0f ? row_pitch : g.delta_voxel) * ((float)row - 0.5f * (float)(g.num_recon_rows - 1));
    x_tilde = g.delta_voxel * ((float)col - 0.5f * (float)(g.num_recon_cols - 1));
}

// Horizontal (channel) footprint of one pixel in one view: fractional channel n_p, centre channel,
// projected width W (in channels) and cos(alpha).
struct ChannelFootprint {
    float n_p;
    int n_c;
    float w;
    float cos_alpha;
    float mag;  // pixel magnification (cone); 1 for parallel beam
};

__device__ __forceinline__ ChannelFootprint parallel_footprint(const mbx_geom &g, float cs, float sn,
                                                              float x_tilde, float y_tilde) {
    ChannelFootprint f;
    const float x = cs * x_tilde - sn * y_tilde;
    const float det_center_channel = 0.5f * (float)(g.num_det_channels - 1);
    f.n_p = (x + g.det_channel_offset) / g.delta_det_channel + det_center_channel;
    f.n_c = (int)rintf(f.n_p);
    f.cos_alpha = fmaxf(fabsf(cs), fabsf(sn));
    f.w = (g.delta_voxel / g.delta_det_channel) * f.cos_alpha;
    f.mag = 1.0f;
    return f;
}

__device__ __forceinline__ float cone_pixel_mag(const mbx_geom &g, float y) {
    return 1.0f / (1.0f / g.magnification - y / g.source_detector_dist);
}

__device__ __forceinline__ ChannelFootprint cone_footprint(const mbx_geom &g, float angle, float cs, float sn,
                                                          float x_tilde, float y_tilde) {
    ChannelFootprint f;
    const float x_p = cs * x_tilde - sn * y_tilde;
    const float y_p = sn * x_tilde + cs * y_tilde;
    f.mag = cone_pixel_mag(g, y_p);
    const float u_p = f.mag * x_p;
    const float det_center_channel = 0.5f * (float)(g.num_det_channels - 1);
    f.n_p = (u_p + g.det_channel_offset) / g.delta_det_channel + det_center_channel;
    f.n_c = (int)rintf(f.n_p);
    const float theta_p = atan2f(u_p, g.source_detector_dist);
    const float d = angle - theta_p;
    f.cos_alpha = fmaxf(fabsf(cosf(d)), fabsf(sinf(d)));
    f.w = f.mag * (g.delta_voxel / g.delta_det_channel) * (f.cos_alpha / cosf(theta_p));
    return f;
}

// Translation geometry (translation_model.py:595-656): no rotation; the pixel sits at
// x = delta_voxel (col - (Nc-1)/2) - tx, y = delta_recon_row (row - (Nr-1)/2) - ty for the view's translation
// (tx, ty); W = mag delta_voxel / delta_det_channel and cos_alpha = cos(theta_p), theta_p = atan2(u_p, D).
__device__ __forceinline__ ChannelFootprint translation_footprint(const mbx_geom &g, int idx, float tx, float ty) {
    ChannelFootprint f;
    const int row = idx / g.num_recon_cols;
    const int col = idx - row * g.num_recon_cols;
    const float x_p = g.delta_voxel * ((float)col - 0.5f * (float)(g.num_recon_cols - 1)) - tx;
    const float y_p = g.delta_recon_row * ((float)row - 0.5f * (float)(g.num_recon_rows - 1)) - ty;
    f.mag = cone_pixel_mag(g, y_p);
    const float u_p = f.mag * x_p;
    const float det_center_channel = 0.5f * (float)(g.num_det_channels - 1);
    f.n_p = (u_p + g.det_channel_offset) / g.delta_det_channel + det_center_channel;
    f.n_c = (int)rintf(f.n_p);
    f.cos_alpha = cosf(atan2f(u_p, g.source_detector_dist));
    f.w = f.mag * (g.delta_voxel / g.delta_det_channel);
    return f;
}

// Translation channel coefficient L / cos(theta_p) (translation_model.py:275-281, :443-449): unlike the
// rotating geometries there is no delta_voxel factor.
__device__ __forceinline__ float translation_channel_coeff(const mbx_geom &g, const ChannelFootprint &f, int k) {
    const int n = f.n_c + k;
    if (n < 0 || n >= g.num_det_channels) return 0.0f;
    const float l_max = fminf(1.0f, f.w);
    const float l = fminf(fmaxf((f.w + 1.0f) * 0.5f - fabsf(f.n_p - (float)n), 0.0f), l_max);
    return l / f.cos_alpha;
}

// Channel coefficient A_chan_n for channel offset k from the centre (parallel_beam.py:170-175,
// cone_beam.py:276-281); 0 outside the detector.
__device__ __forceinline__ float channel_coeff(const mbx_geom &g, const ChannelFootprint &f, int k) {
    const int n = f.n_c + k;
    if (n < 0 || n >= g.num_det_channels) return 0.0f;
    const float l_max = fminf(1.0f, f.w);
    const float l = fminf(fmaxf((f.w + 1.0f) * 0.5f - fabsf(f.n_p - (float)n), 0.0f), l_max);
    return g.delta_voxel * l / f.cos_alpha;
}

// 1/cos(phi) for the vertical cone angle of a point at detector height v.
__device__ __forceinline__ float sec_phi(float v, float source_detector_dist) {
    const float t = v / source_detector_dist;
    return sqrtf(fmaf(t, t, 1.0f));
}

// Fractional slice index hit by the centre of detector row m (cone_beam.py:351-355) for slice-axis offset zoff
// (recon_slice_offset for the cone; -tz for a translation view, translation_model.py:353-356).
__device__ __forceinline__ float fan_row_to_slice(const mbx_geom &g, float mag, int m, float zoff) {
    const float det_center_row = 0.5f * (float)(g.num_det_rows - 1);
    const float v_m = ((float)m - det_center_row) * g.delta_det_row - g.det_row_offset;
    const float z_m = v_m / mag;
    return (z_m - zoff) / g.delta_voxel + 0.5f * (float)(g.num_recon_slices - 1);
}

__device__ __forceinline__ float cone_row_to_slice(const mbx_geom &g, float mag, int m) {
    return fan_row_to_slice(g, mag, m, g.recon_slice_offset);
}

// Vertical forward fan for detector row m of one pixel (cone_beam.py:347-372, translation_model.py:348-372):
// sum over the 2*rbp+1 slices around the slice hit by the row centre, slice k at height
// delta_voxel (k - (S-1)/2) + zoff.
template <int MAXRBP>
__device__ __forceinline__ float fan_fp_vertical(const mbx_geom &g, const float *__restrict__ cyl, float mag, int m,
                                                 float zoff, int rbp) {
    const int num_slices = g.num_recon_slices;
    const float w_r = (mag * g.delta_voxel) / g.delta_det_row;
    const float l_max = fminf(1.0f, w_r);
    int rows_per_batch = g.entries_per_cylinder_batch;
    if (rows_per_batch > g.num_det_rows) rows_per_batch = g.num_det_rows;
    const int batch_start = (m / rows_per_batch) * rows_per_batch;
    const float k_m = fan_row_to_slice(g, mag, m, zoff);
    const float k_m0 = fan_row_to_slice(g, mag, batch_start, zoff);
    const int k_c = (int)rintf(k_m);
    const float m_p = w_r * ((float)k_c - k_m0) + (float)batch_start;
    const float half_w = (w_r + 1.0f) * 0.5f;
    const float center_slice = 0.5f * (float)(num_slices - 1);
    float acc = 0.0f;
#pragma unroll
    for (int ko = -MAXRBP; ko <= MAXRBP; ++ko) {
        if (ko < -rbp || ko > rbp) continue;
        const int k = k_c + ko;
        if (k < 0 || k >= num_slices) continue;
        const float a = fminf(fmaxf(half_w - fabsf(m_p + w_r * (float)ko - (float)m), 0.0f), l_max);
        const float z = g.delta_voxel * ((float)k - center_slice) + zoff;
        acc += a * (__ldg(cyl + k) * sec_phi(mag * z, g.source_detector_dist));
    }
    return acc;
}

template <int MAXRBP>
__device__ __forceinline__ float cone_fp_vertical(const mbx_geom &g, const float *__restrict__ cyl, float mag,
                                                  int m) {
    return fan_fp_vertical<MAXRBP>(g, cyl, mag, m, g.recon_slice_offset, g.bp_psf_radius);
}

__host__ __device__ __forceinline__ int ceil_div(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace mbx
