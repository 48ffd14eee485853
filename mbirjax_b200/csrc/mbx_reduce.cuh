// Deterministic float64 block reductions: a fixed warp-shuffle tree inside each block, one partial per block,
// and a single-block fixed-order final sum.  Given the same grid, results are bit-identical run to run.
#pragma once

#include <cuda_runtime.h>

namespace mbx {

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Reduces NV values over the block (blockDim.x a multiple of 32, at most 1024) and stores them to
// partials[blockIdx.x * NV + i] from thread 0.
template <int NV>
__device__ __forceinline__ void block_reduce_store_n(const double (&v)[NV], double *partials) {
    __shared__ double sh[32][NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
        const double s = warp_sum(v[i]);
        if (lane == 0) sh[warp][i] = s;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int i = 0; i < NV; ++i) {
            double s = lane < nwarps ? sh[lane][i] : 0.0;
            s = warp_sum(s);
            if (lane == 0) partials[blockIdx.x * NV + i] = s;
        }
    }
}

__device__ __forceinline__ void block_reduce_store(double v, double *partials) {
    const double a[1] = {v};
    block_reduce_store_n<1>(a, partials);
}

// out[i] = sum_b partials[b * nv + i] for i < nv, b = 0..nblocks-1 in a fixed order (defined in vcd.cu).
void launch_sum_partials(const double *partials, int nblocks, int nv, double *out, cudaStream_t st);

}  // namespace mbx
