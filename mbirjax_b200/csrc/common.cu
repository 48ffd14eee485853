// Library identification, error reporting and device queries for the mbirjax_b200 C ABI.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <set>
#include <utility>
#include <vector>

#include "mbx_common.cuh"
#include "mbx_host.hpp"

// Device error word: bit flags set by kernels that met an out-of-range pixel or view index.
__device__ int g_mbx_device_error = 0;

namespace mbx {

int *device_error_ptr() {
    static std::atomic<int *> cache[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return nullptr;
    }
    int *c = cache[dev].load(std::memory_order_acquire);
    if (!c) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_mbx_device_error) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        c = static_cast<int *>(p);
        cache[dev].store(c, std::memory_order_release);  // every thread that races here stores the same address
    }
    return c;
}

static std::mutex g_attr_mutex;
static std::set<std::pair<const void *, int>> g_attr_done;

cudaError_t set_max_dynamic_smem(const void *func, int bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(g_attr_mutex);
    const auto key = std::make_pair(func, dev);
    if (g_attr_done.count(key)) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) g_attr_done.insert(key);
    return e;
}

static std::atomic<int> g_autotune{1};
static std::mutex g_tune_mutex;
static std::map<std::vector<long long>, int> g_tune_cache;

bool autotune_enabled() { return g_autotune.load(std::memory_order_relaxed) != 0; }

int autotune_forced() {
    const int m = g_autotune.load(std::memory_order_relaxed);
    return m >= 2 ? m - 1 : -1;
}

int autotune_lookup(const long long *key, int n) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::vector<long long> k(key, key + n);
    k.push_back(dev);
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(k);
    return it == g_tune_cache.end() ? -1 : it->second;
}

void autotune_store(const long long *key, int n, int choice) {
    int dev = 0;
    cudaGetDevice(&dev);
    std::vector<long long> k(key, key + n);
    k.push_back(dev);
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[k] = choice;
}

bool stream_is_capturing(cudaStream_t st) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
        cudaGetLastError();
        return true;  // unknown: do not synchronise on it
    }
    return cs != cudaStreamCaptureStatusNone;
}

static std::atomic<unsigned long long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

static thread_local int t_last_cuda_error = 0;

int set_cuda_error(cudaError_t e) {
    t_last_cuda_error = (int)e;
    return MBX_ERR_CUDA;
}

int num_sms() {
    static std::atomic<int> cache[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return kNumSMsDefault;
    }
    int n = cache[dev].load(std::memory_order_relaxed);
    if (n == 0) {
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
            cudaGetLastError();
            n = kNumSMsDefault;
        }
        cache[dev].store(n, std::memory_order_relaxed);
    }
    return n;
}

int validate_geom(const mbx_geom *g) {
    if (!g) return MBX_ERR_INVALID_ARG;
    if (g->kind != MBX_GEOM_PARALLEL && g->kind != MBX_GEOM_CONE && g->kind != MBX_GEOM_TRANSLATION)
        return MBX_ERR_INVALID_ARG;
    if (g->num_views <= 0 || g->num_det_rows <= 0 || g->num_det_channels <= 0) return MBX_ERR_INVALID_ARG;
    if (g->num_recon_rows <= 0 || g->num_recon_cols <= 0 || g->num_recon_slices <= 0) return MBX_ERR_INVALID_ARG;
    if ((long long)g->num_recon_rows * g->num_recon_cols > 2147483647LL) return MBX_ERR_UNSUPPORTED;
    if (g->psf_radius < 0 || g->psf_radius > MBX_MAX_PSF_RADIUS) return MBX_ERR_UNSUPPORTED;
    if (g->kind == MBX_GEOM_CONE && (g->bp_psf_radius < 0 || g->bp_psf_radius > MBX_MAX_PSF_RADIUS))
        return MBX_ERR_UNSUPPORTED;
    if (g->kind == MBX_GEOM_CONE && g->entries_per_cylinder_batch <= 0) return MBX_ERR_INVALID_ARG;
    if (g->kind == MBX_GEOM_PARALLEL && g->num_recon_slices != g->num_det_rows) return MBX_ERR_INVALID_ARG;
    if (!(g->delta_voxel > 0.0f) || !(g->delta_det_channel > 0.0f) || !(g->delta_det_row > 0.0f))
        return MBX_ERR_INVALID_ARG;
    if (g->kind == MBX_GEOM_CONE && (!(g->magnification > 0.0f) || !(g->source_detector_dist > 0.0f)))
        return MBX_ERR_INVALID_ARG;
    if (g->kind == MBX_GEOM_TRANSLATION) {
        // a finite source distance: with the source at infinity every translated view carries the same
        // information (translation_model.py:69-81)
        if (!g->translations || !(g->delta_recon_row > 0.0f) || !(g->magnification > 0.0f) ||
            !(g->source_detector_dist > 0.0f) || !std::isfinite(g->source_detector_dist) ||
            g->entries_per_cylinder_batch <= 0)
            return MBX_ERR_INVALID_ARG;
        return MBX_OK;
    }
    if (!g->angles) return MBX_ERR_INVALID_ARG;
    return MBX_OK;
}

unsigned grid_for(long long n, int threads) {
    long long blocks = (n + threads - 1) / threads;
    const long long cap = 16LL * num_sms();
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    return (unsigned)blocks;
}

}  // namespace mbx

extern "C" const char *mbx_version(void) { return "mbirjax_b200 0.1.0 (sm_100a)"; }

extern "C" const char *mbx_error_string(int code) {
    switch (code) {
        case MBX_OK: return "ok";
        case MBX_ERR_INVALID_ARG: return "invalid argument";
        case MBX_ERR_UNSUPPORTED: return "unsupported configuration";
        case MBX_ERR_CUDA: return "CUDA error (see mbx_last_cuda_error)";
        case MBX_ERR_WORKSPACE: return "workspace missing or too small";
        default: return "unknown error";
    }
}

extern "C" int mbx_last_cuda_error(void) { return mbx::t_last_cuda_error; }

extern "C" uint64_t mbx_launch_count(void) { return mbx::g_launches.load(std::memory_order_relaxed); }

extern "C" int mbx_set_autotune(int mode) {
    if (mode < 0) return MBX_ERR_INVALID_ARG;
    return mbx::g_autotune.exchange(mode);
}

extern "C" int mbx_get_device_error(int *flags_out) {
    if (!flags_out) return MBX_ERR_INVALID_ARG;
    int value = 0;
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaMemcpyFromSymbol(&value, g_mbx_device_error, sizeof(int));
    const int zero = 0;
    if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_mbx_device_error, &zero, sizeof(int));
    if (e != cudaSuccess) return mbx::set_cuda_error(e);
    *flags_out = value;
    return MBX_OK;
}
