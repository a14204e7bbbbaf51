// Device helpers for fixed-order block reductions.
#pragma once
#include <cuda_runtime.h>

namespace mgg {

// Sum of v over the block in a fixed order: xor-shuffle tree inside each warp,
// then warp 0 adds the warp totals in warp order.  Valid in thread 0.
// blockDim.x must be a multiple of 32 and at most 1024.
__device__ __forceinline__ double block_sum_fixed(double v) {
    __shared__ double warp_tot[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) warp_tot[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int i = 0; i < nw; ++i) s += warp_tot[i];
    }
    return s;
}

}  // namespace mgg
