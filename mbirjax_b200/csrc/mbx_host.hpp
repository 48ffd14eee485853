// Internal host-side helpers shared by the mbirjax_b200 translation units (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/mbirjax_b200.h"

namespace mbx {

// Number of SMs of the current device (cached per device; 148 when no device can be queried).
int num_sms();

// Counts kernel launches submitted by this library (host-side, all devices); read by mbx_launch_count().
void note_launch();

// Records a CUDA error for mbx_last_cuda_error() and returns MBX_ERR_CUDA.
int set_cuda_error(cudaError_t e);

// A 1-D grid of `threads`-wide blocks covering n elements, capped at a few waves of the device.
unsigned grid_for(long long n, int threads);

int validate_geom(const mbx_geom *g);

// Device address of the error word of the current device (cached per device; NULL if unavailable).
int *device_error_ptr();

size_t fp_workspace_bytes(const mbx_geom &g, long long num_pixels, int num_views_sel);
size_t bp_workspace_bytes(const mbx_geom &g, long long num_pixels, int num_views_sel);

int forward_project(const mbx_geom &g, const float *vox, const int32_t *pix, long long num_pixels,
                    const int32_t *views, int num_views_sel, float *out, void *ws, size_t ws_bytes,
                    cudaStream_t st);

int back_project(const mbx_geom &g, const float *sino, const float *w, const int32_t *pix, long long num_pixels,
                 const int32_t *views, int num_views_sel, int coeff_power, float scale, float *out, void *ws,
                 size_t ws_bytes, cudaStream_t st);

// Bytes rounded up to a 256-byte boundary (workspace carving).
inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Compile-time psf-radius bucket a kernel is instantiated for (1, 2 or MBX_MAX_PSF_RADIUS).
inline int psf_bucket(int r) { return r <= 1 ? 1 : (r <= 2 ? 2 : MBX_MAX_PSF_RADIUS); }

// out[i] = scale * sum_s ws[s * stride + i] over s = 0..splits-1 in order (deterministic split reduction).
void launch_split_sum(const float *ws, long long stride, int splits, float scale, float *out, long long n,
                      cudaStream_t st);

}  // namespace mbx
