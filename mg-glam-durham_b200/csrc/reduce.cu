// Deterministic reductions and the exclusive scan used by the CIC bucketing.
//
// Every FP64 sum in the step (MG residual norms, kinetic energy) is reduced in a
// fixed order: a fixed shuffle tree inside each warp, a fixed order across the
// warps of a block, one partial per block, then one block that walks the
// partials in index order.  The result is bit-identical run to run for a given
// grid size, unlike the reference's OpenMP REDUCTION whose order follows the
// thread count (scripts/compare_residuals.py checks exactly that drift).
#include "mgg_internal.cuh"
#include "reduce.cuh"

namespace mgg {

namespace {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 2 * kScanThreads;

// Block-local exclusive scan of 2048 uint32 (Blelloch in shared memory).
__global__ void k_scan_block(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                             uint32_t* __restrict__ block_sums, int64_t n) {
    __shared__ uint32_t s[kScanItems];
    const int t = threadIdx.x;
    const int64_t base = (int64_t)blockIdx.x * kScanItems;
    const int64_t g0 = base + 2 * t, g1 = g0 + 1;
    s[2 * t] = g0 < n ? in[g0] : 0u;
    s[2 * t + 1] = g1 < n ? in[g1] : 0u;
    int offset = 1;
    for (int d = kScanItems >> 1; d > 0; d >>= 1) {
        __syncthreads();
        if (t < d) {
            int ai = offset * (2 * t + 1) - 1, bi = offset * (2 * t + 2) - 1;
            s[bi] += s[ai];
        }
        offset <<= 1;
    }
    __syncthreads();
    if (t == 0) {
        if (block_sums) block_sums[blockIdx.x] = s[kScanItems - 1];
        s[kScanItems - 1] = 0;
    }
    for (int d = 1; d < kScanItems; d <<= 1) {
        offset >>= 1;
        __syncthreads();
        if (t < d) {
            int ai = offset * (2 * t + 1) - 1, bi = offset * (2 * t + 2) - 1;
            uint32_t tmp = s[ai];
            s[ai] = s[bi];
            s[bi] += tmp;
        }
    }
    __syncthreads();
    if (g0 < n) out[g0] = s[2 * t];
    if (g1 < n) out[g1] = s[2 * t + 1];
}

__global__ void k_scan_add(uint32_t* __restrict__ out, const uint32_t* __restrict__ block_off, int64_t n) {
    const int64_t base = (int64_t)blockIdx.x * kScanItems;
    const uint32_t add = block_off[blockIdx.x];
    for (int e = threadIdx.x; e < kScanItems; e += blockDim.x) {
        int64_t g = base + e;
        if (g < n) out[g] += add;
    }
}

__global__ void k_sum_partials(const double* __restrict__ part, int n, double* __restrict__ out) {
    double v = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
    v = block_sum_fixed(v);
    if (threadIdx.x == 0) out[0] = v;
}

}  // namespace

void scan_exclusive(Ctx& c, const uint32_t* in, uint32_t* out, int64_t n) {
    ProfScope ps(c, K_SCAN, 8.0 * (double)n);
    const int nb = div_up(n, kScanItems);
    if (nb == 1) {
        k_scan_block<<<1, kScanThreads, 0, c.stream>>>(in, out, nullptr, n);
        MGG_CHECK_LAUNCH();
        return;
    }
    if (nb > kScanItems * kScanItems) throw Error{MGG_ERR_ARG, "scan: too many elements"};
    uint32_t* sums = c.scan_tmp;
    uint32_t* sums_scan = c.scan_tmp + kScanItems * 2;
    k_scan_block<<<nb, kScanThreads, 0, c.stream>>>(in, out, sums, n);
    MGG_CHECK_LAUNCH();
    const int nb2 = div_up(nb, kScanItems);
    if (nb2 == 1) {
        k_scan_block<<<1, kScanThreads, 0, c.stream>>>(sums, sums_scan, nullptr, nb);
        MGG_CHECK_LAUNCH();
    } else {
        throw Error{MGG_ERR_ARG, "scan: more than 2048 blocks"};
    }
    k_scan_add<<<nb, 256, 0, c.stream>>>(out, sums_scan, n);
    MGG_CHECK_LAUNCH();
}

void ensure_partials(Ctx& c, int n) {
    if (n <= c.red_capacity) return;
    if (c.red_partial) MGG_CUDA(cudaFree(c.red_partial));
    c.red_partial = nullptr;
    int cap = n < 4096 ? 4096 : n;
    MGG_CUDA(cudaMalloc(&c.red_partial, sizeof(double) * cap));
    c.red_capacity = cap;
}

void reduce_sum_blocks_async(Ctx& c, int nblocks, double* out) {
    ProfScope ps(c, K_MG_REDUCE, 8.0 * nblocks);
    k_sum_partials<<<1, 1024, 0, c.stream>>>(c.red_partial, nblocks, out);
    MGG_CHECK_LAUNCH();
}

double reduce_sum_blocks(Ctx& c, int nblocks) {
    reduce_sum_blocks_async(c, nblocks, c.red_out);
    MGG_CUDA(cudaMemcpyAsync(c.h_red, c.red_out, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaStreamSynchronize(c.stream));
    return c.h_red[0];
}

}  // namespace mgg
