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

// cudaFuncSetAttribute(func, MaxDynamicSharedMemorySize, bytes) once per (kernel, device), under a mutex, so that
// host threads launching the same kernel on one or several devices neither race on the record of what is set
// nor skip a device.
cudaError_t set_max_dynamic_smem(const void *func, int bytes);

size_t fp_workspace_bytes(const mbx_geom &g, long long num_pixels, int num_views_sel);
size_t bp_workspace_bytes(const mbx_geom &g, long long num_pixels, int num_views_sel);

int forward_project(const mbx_geom &g, const float *vox, const int32_t *pix, long long num_pixels,
                    const int32_t *views, int num_views_sel, float *out, void *ws, size_t ws_bytes,
                    cudaStream_t st);

int back_project(const mbx_geom &g, const float *sino, const float *w, const int32_t *pix, long long num_pixels,
                 const int32_t *views, int num_views_sel, int coeff_power, float scale, float *out, void *ws,
                 size_t ws_bytes, cudaStream_t st);

// Autotuning.  The first call of a projector for a given call shape (geometry sizes, views, pixel count rounded
// up to a power of two) times its candidate plans on the caller's stream and remembers the fastest; later calls
// of that shape launch it directly.  Calls made while their stream is being captured into a CUDA graph use the
// default plan and do not tune.  The cache is host memory only; mbx_set_autotune(0) selects the default plans.
bool autotune_enabled();
int autotune_forced();  // mbx_set_autotune(k >= 2): candidate k-1 is used everywhere without timing; else -1
int autotune_lookup(const long long *key, int n);  // -1 if the shape has not been tuned
void autotune_store(const long long *key, int n, int choice);
bool stream_is_capturing(cudaStream_t st);
// Milliseconds of the launches `launch` enqueues on st (one untimed call first, then the best of two).
template <class F>
cudaError_t time_on_stream(F launch, cudaStream_t st, float &ms) {
    cudaError_t e = launch();
    if (e != cudaSuccess) return e;
    cudaEvent_t a, b;
    if ((e = cudaEventCreate(&a)) != cudaSuccess) return e;
    if ((e = cudaEventCreate(&b)) != cudaSuccess) {
        cudaEventDestroy(a);
        return e;
    }
    ms = 3.0e38f;
    for (int r = 0; r < 2 && e == cudaSuccess; ++r) {
        e = cudaEventRecord(a, st);
        if (e == cudaSuccess) e = launch();
        if (e == cudaSuccess) e = cudaEventRecord(b, st);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        float t = 0.0f;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
        if (e == cudaSuccess && t < ms) ms = t;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return e;
}

// A call whose default plan alone takes longer than this is not tuned: timing its other candidates would cost
// more than a handful of calls could win back.
constexpr float MBX_TUNE_BUDGET_MS = 100.0f;

// Milliseconds of one run of `launch` on st (synchronises st).
template <class F>
cudaError_t time_once(F launch, cudaStream_t st, float &ms) {
    cudaEvent_t a, b;
    cudaError_t e = cudaEventCreate(&a);
    if (e != cudaSuccess) return e;
    if ((e = cudaEventCreate(&b)) != cudaSuccess) {
        cudaEventDestroy(a);
        return e;
    }
    e = cudaEventRecord(a, st);
    if (e == cudaSuccess) e = launch();
    if (e == cudaSuccess) e = cudaEventRecord(b, st);
    if (e == cudaSuccess) e = cudaEventSynchronize(b);
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return e;
}

// Best-of-three milliseconds of each of n candidates on st: every candidate runs once untimed first, then the
// timed runs go round-robin, so clock ramp-up and cache state do not favour one candidate.
template <class F>
cudaError_t time_candidates(int n, F launch, cudaStream_t st, float *ms) {
    cudaError_t e = cudaSuccess;
    for (int c = 0; c < n && e == cudaSuccess; ++c) e = launch(c);
    if (e != cudaSuccess) return e;
    cudaEvent_t a, b;
    if ((e = cudaEventCreate(&a)) != cudaSuccess) return e;
    if ((e = cudaEventCreate(&b)) != cudaSuccess) {
        cudaEventDestroy(a);
        return e;
    }
    for (int c = 0; c < n; ++c) ms[c] = 3.0e38f;
    for (int r = 0; r < 3 && e == cudaSuccess; ++r)
        for (int c = 0; c < n && e == cudaSuccess; ++c) {
            e = cudaEventRecord(a, st);
            if (e == cudaSuccess) e = launch(c);
            if (e == cudaSuccess) e = cudaEventRecord(b, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(b);
            float t = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
            if (e == cudaSuccess && t < ms[c]) ms[c] = t;
        }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return e;
}

// Bytes rounded up to a 256-byte boundary (workspace carving).
inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Compile-time psf-radius bucket a kernel is instantiated for (1, 2 or MBX_MAX_PSF_RADIUS).
inline int psf_bucket(int r) { return r <= 1 ? 1 : (r <= 2 ? 2 : MBX_MAX_PSF_RADIUS); }

// out[i] = scale * sum_s ws[s * stride + i] over s = 0..splits-1 in order (deterministic split reduction).
void launch_split_sum(const float *ws, long long stride, int splits, float scale, float *out, long long n,
                      cudaStream_t st);

}  // namespace mbx
