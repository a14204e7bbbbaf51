// Kernel (a): deterministic cloud-in-cell density, the replacement of DENSIT
// (PMP2mod_density.f90:17-301).
//
// The reference scatters eight FP64 weights per particle into the FP32 grid FI
// with `!$OMP ATOMIC` (PMP2mod_density.f90:263-279), so its summation order --
// and its last bits -- change with the thread count.  Here:
//
//   1. k_cic_count   : integer cell key of every particle; the row part of the
//                      key (J + N*K) is histogrammed with integer atomics
//                      (one per row and warp).
//   2. scan          : exclusive prefix of the N^2 row counts = row offsets.
//   3. k_cic_scatter : every particle's position is written to its row bucket
//                      (a counting sort on the row key).
//   4. k_cic_deposit : one CTA per 2 x 2 block of output rows.  It walks the source
//                      rows that can reach its rows in a fixed order, forms the
//                      reference's FP64 weights, and accumulates them in shared
//                      memory as 32.32 fixed-point integers.  Integer addition
//                      is associative, so each cell's sum -- and therefore FI --
//                      is bit-identical for any particle order, launch shape or
//                      run; the single rounding to FP32 happens at the end.
//
// Weights follow the reference exactly: D = X - INT(X) in FP64,
// w = T3*T1*(T2*WPAR) etc. (PMP2mod_density.f90:249-279), WPAR = NGRID^3/Np in
// Real*4 (line 41), FI starts at -1 (lines 47-55).
#include "mgg_internal.cuh"

#include <mutex>

namespace mgg {

namespace {

constexpr double kFix = 4294967296.0;          // 2^32
constexpr double kUnfix = 1.0 / 4294967296.0;

__device__ __forceinline__ int cell_of(float v, int N, int32_t* flags) {
    int I = (int)v;   // 1-based, positions live in [1, N+1)
    if (!(I >= 1 && I <= N)) {
        atomicOr(flags, 1);
        I = I < 1 ? 1 : N;
    }
    return I;
}

__global__ void k_cic_count(const float* __restrict__ x, const float* __restrict__ y,
                            const float* __restrict__ z, int64_t np, int N,
                            uint32_t* __restrict__ rowcnt, uint32_t* __restrict__ slot,
                            int32_t* __restrict__ flags) {
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * blockDim.x) {
        (void)cell_of(__ldg(x + p), N, flags);
        const int J = cell_of(__ldg(y + p), N, flags);
        const int K = cell_of(__ldg(z + p), N, flags);
        const uint32_t r = (uint32_t)(J - 1) + (uint32_t)N * (uint32_t)(K - 1);
        // lanes with the same row (neighbouring particles usually share one) take
        // one atomic per row: the leader adds the group size, each lane its rank
        const unsigned act = __activemask();
        const unsigned grp = __match_any_sync(act, r);
        const int leader = __ffs(grp) - 1, lane = threadIdx.x & 31;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(rowcnt + r, (uint32_t)__popc(grp));
        base = __shfl_sync(act, base, leader);
        slot[p] = base + (uint32_t)__popc(grp & ((1u << lane) - 1u));
    }
}

__global__ void k_cic_scatter(const float* __restrict__ x, const float* __restrict__ y,
                              const float* __restrict__ z, int64_t np, int N,
                              const uint32_t* __restrict__ rowstart, const uint32_t* __restrict__ slot,
                              float4* __restrict__ rec) {
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np;
         p += (int64_t)gridDim.x * blockDim.x) {
        const float X = __ldg(x + p), Y = __ldg(y + p), Z = __ldg(z + p);
        int J = (int)Y, K = (int)Z;
        J = J < 1 ? 1 : (J > N ? N : J);
        K = K < 1 ? 1 : (K > N ? N : K);
        const uint32_t r = (uint32_t)(J - 1) + (uint32_t)N * (uint32_t)(K - 1);
        rec[rowstart[r] + slot[p]] = make_float4(X, Y, Z, 0.f);
    }
}

// One CTA per TY x TZ block of output rows (all N cells of each row), N = 2^lgN.
// Shared memory: TY*TZ*N 64-bit accumulators (32 KB for 2 x 2 rows at N = 1024,
// so several CTAs share an SM and hide each other's latency).
constexpr int kDepTY = 2, kDepTZ = 2, kDepThreads = 256;

template <int TY, int TZ>
__global__ void __launch_bounds__(kDepThreads) k_cic_deposit(const float4* __restrict__ rec,
                                                             const uint32_t* __restrict__ rowstart, int N, int lgN,
                                                             float wpar, float* __restrict__ fi) {
    extern __shared__ unsigned long long acc[];
    const int j0 = blockIdx.x * TY, k0 = blockIdx.y * TZ;
    const int nacc = (TY * TZ) << lgN;
    for (int e = threadIdx.x; e < nacc; e += kDepThreads) acc[e] = 0ull;
    __syncthreads();
    const double W = (double)wpar;
#pragma unroll 1
    for (int sr = 0; sr < (TY + 1) * (TZ + 1); ++sr) {
        int sj = j0 - 1 + sr % (TY + 1);
        int sk = k0 - 1 + sr / (TY + 1);
        sj = sj < 0 ? sj + N : sj;
        sk = sk < 0 ? sk + N : sk;
        const uint32_t row = (uint32_t)sj + ((uint32_t)sk << lgN);
        const uint32_t beg = __ldg(rowstart + row), end = __ldg(rowstart + row + 1);
        // target rows of this source row that fall inside the block
        const int jj0 = sj - j0, jj1 = (sj + 1 == N ? 0 : sj + 1) - j0;
        const int kk0 = sk - k0, kk1 = (sk + 1 == N ? 0 : sk + 1) - k0;
        const bool vj0 = jj0 >= 0 && jj0 < TY, vj1 = jj1 >= 0 && jj1 < TY;
        const bool vk0 = kk0 >= 0 && kk0 < TZ, vk1 = kk1 >= 0 && kk1 < TZ;
        if (!((vj0 || vj1) && (vk0 || vk1))) continue;
        for (uint32_t q = beg + threadIdx.x; q < end; q += kDepThreads) {
            const float4 r = __ldg(rec + q);
            const double X = r.x, Y = r.y, Z = r.z;
            int I = (int)r.x;
            I = I < 1 ? 1 : (I > N ? N : I);
            const int Jc = (int)r.y, Kc = (int)r.z;
            const double D1 = X - (double)(float)I, D2 = Y - (double)(float)Jc, D3 = Z - (double)(float)Kc;
            const double T1 = 1.0 - D1, T2 = 1.0 - D2, T3 = 1.0 - D3;
            const double T2W = T2 * W, D2W = D2 * W;
            const int i0 = I - 1, i1 = (I == N) ? 0 : I;
            if (vk0) {
                if (vj0) {
                    unsigned long long* a = acc + ((kk0 * TY + jj0) << lgN);
                    atomicAdd(a + i0, __double2ull_rn(T3 * T1 * T2W * kFix));
                    atomicAdd(a + i1, __double2ull_rn(T3 * D1 * T2W * kFix));
                }
                if (vj1) {
                    unsigned long long* a = acc + ((kk0 * TY + jj1) << lgN);
                    atomicAdd(a + i0, __double2ull_rn(T3 * T1 * D2W * kFix));
                    atomicAdd(a + i1, __double2ull_rn(T3 * D1 * D2W * kFix));
                }
            }
            if (vk1) {
                if (vj0) {
                    unsigned long long* a = acc + ((kk1 * TY + jj0) << lgN);
                    atomicAdd(a + i0, __double2ull_rn(D3 * T1 * T2W * kFix));
                    atomicAdd(a + i1, __double2ull_rn(D3 * D1 * T2W * kFix));
                }
                if (vj1) {
                    unsigned long long* a = acc + ((kk1 * TY + jj1) << lgN);
                    atomicAdd(a + i0, __double2ull_rn(D3 * T1 * D2W * kFix));
                    atomicAdd(a + i1, __double2ull_rn(D3 * D1 * D2W * kFix));
                }
            }
        }
    }
    __syncthreads();
    const int64_t NN = (int64_t)N;
    for (int e = threadIdx.x; e < nacc; e += kDepThreads) {
        const int i = e & (N - 1), rowl = e >> lgN;
        const int jj = rowl % TY, kk = rowl / TY;
        const double v = (double)acc[e] * kUnfix - 1.0;
        fi[(int64_t)i + NN * ((int64_t)(j0 + jj) + NN * (int64_t)(k0 + kk))] = (float)v;
    }
}

int ilog2i(int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

// deposit launch for an N^3 grid (N a power of two, 16 <= N <= 1024)
void launch_deposit(const float4* rec, const uint32_t* rowstart, int N, float wpar, float* fi, cudaStream_t s) {
    const size_t smem = (size_t)kDepTY * kDepTZ * N * 8;   // <= 32 KB
    k_cic_deposit<kDepTY, kDepTZ><<<dim3(N / kDepTY, N / kDepTZ), kDepThreads, smem, s>>>(rec, rowstart, N, ilog2i(N),
                                                                                         wpar, fi);
}

}  // namespace

void cic_alloc(Ctx& c) {
    const int64_t rows = (int64_t)c.N * c.N;
    MGG_CUDA(cudaMalloc(&c.cic_rowcnt, sizeof(uint32_t) * (rows + 1)));
    MGG_CUDA(cudaMalloc(&c.cic_rowstart, sizeof(uint32_t) * (rows + 1)));
    MGG_CUDA(cudaMalloc(&c.cic_slot, sizeof(uint32_t) * c.np));
    MGG_CUDA(cudaMalloc(&c.cic_rec, sizeof(float4) * c.np));
}

void cic_grid(Ctx& c, const float* x, const float* y, const float* z, int N, float* out) {
    const int64_t rows = (int64_t)N * N;
    c.cic_last_n = N;
    const int threads = 256;
    const int blocks = (int)std::min<int64_t>(div_up(c.np, threads), 148 * 16);
    MGG_CUDA(cudaMemsetAsync(c.cic_rowcnt, 0, sizeof(uint32_t) * (rows + 1), c.stream));
    {
        ProfScope ps(c, K_CIC_COUNT, 16.0 * c.np);
        k_cic_count<<<blocks, threads, 0, c.stream>>>(x, y, z, c.np, N, c.cic_rowcnt, c.cic_slot, c.d_flags);
        MGG_CHECK_LAUNCH();
    }
    scan_exclusive(c, c.cic_rowcnt, c.cic_rowstart, rows + 1);
    {
        ProfScope ps(c, K_CIC_SCATTER, 32.0 * c.np);
        k_cic_scatter<<<blocks, threads, 0, c.stream>>>(x, y, z, c.np, N, c.cic_rowstart, c.cic_slot, c.cic_rec);
        MGG_CHECK_LAUNCH();
    }
    {
        ProfScope ps(c, K_CIC_DEPOSIT, 12.0 * c.np + 4.0 * (double)N * N * N);
        launch_deposit(c.cic_rec, c.cic_rowstart, N, (float)((double)N * N * N / (double)(float)c.np), out, c.stream);
        MGG_CHECK_LAUNCH();
    }
}

namespace {

// Per-cell counts recounted from the row buckets: block r walks bucket r and
// counts each record into cell (INT(X), r), so a record placed in the wrong
// bucket would land in the wrong cell.
__global__ void k_cic_cellcount(const float4* __restrict__ rec, const uint32_t* __restrict__ rowstart, int N,
                                uint32_t* __restrict__ cellcnt) {
    const uint32_t row = blockIdx.x + (uint32_t)N * blockIdx.y;
    const uint32_t beg = rowstart[row], end = rowstart[row + 1];
    for (uint32_t q = beg + threadIdx.x; q < end; q += blockDim.x) {
        int I = (int)rec[q].x;
        I = I < 1 ? 1 : (I > N ? N : I);
        atomicAdd(cellcnt + (size_t)row * N + (I - 1), 1u);
    }
}

}  // namespace

void cic_keys(Ctx& c, uint32_t* rowcnt, uint32_t* rowstart, uint32_t* cellcnt) {
    const int N = c.N;
    if (c.cic_last_n != N) throw Error{MGG_ERR_STATE, "cic_keys: no density on the NGRID mesh since the last analysis call"};
    const int64_t rows = (int64_t)N * N;
    if (rowcnt) MGG_CUDA(cudaMemcpyAsync(rowcnt, c.cic_rowcnt, sizeof(uint32_t) * rows, cudaMemcpyDeviceToHost, c.stream));
    if (rowstart)
        MGG_CUDA(cudaMemcpyAsync(rowstart, c.cic_rowstart, sizeof(uint32_t) * (rows + 1), cudaMemcpyDeviceToHost, c.stream));
    if (cellcnt) {
        uint32_t* d = nullptr;
        const size_t b = sizeof(uint32_t) * (size_t)c.ncell;
        if (cudaMalloc(&d, b) != cudaSuccess) {
            cudaGetLastError();
            throw Error{MGG_ERR_NOMEM, "cic_keys: no device memory for the cell counts"};
        }
        try {
            MGG_CUDA(cudaMemsetAsync(d, 0, b, c.stream));
            k_cic_cellcount<<<dim3(N, N), 128, 0, c.stream>>>(c.cic_rec, c.cic_rowstart, N, d);
            MGG_CHECK_LAUNCH();
            MGG_CUDA(cudaMemcpyAsync(cellcnt, d, b, cudaMemcpyDeviceToHost, c.stream));
            MGG_CUDA(cudaStreamSynchronize(c.stream));
        } catch (...) {
            cudaStreamSynchronize(c.stream);
            cudaFree(d);
            throw;
        }
        MGG_CUDA(cudaFree(d));
    }
    MGG_CUDA(cudaStreamSynchronize(c.stream));
}

void cic_density(Ctx& c) {
    if (!c.have_particles) throw Error{MGG_ERR_STATE, "density: no particles uploaded"};
    BucketScope bs(c, MGG_T_DENSITY);
    cic_grid(c, c.x, c.y, c.z, c.N, c.fi);
}

// ---------------------------------------------------------------------------
// Density without allocation.  Some callers cannot call cudaMalloc: a host
// that owns all device memory through its own pool or arena (and forbids
// other allocations in its process), or code that runs where an allocation
// could synchronise the device at the wrong moment.  This variant of the CIC
// pipeline above takes the caller's device arrays and keeps its bucketing
// scratch (row counts, row offsets, per-particle slots and records, the range
// flag) in one file-scope device array of fixed size, kNoAllocBytes (about
// 40.5 MiB), which every GPU that loads this library holds until the process
// exits.  Limits: NGRID a power of two in [16, 256] and at most 2^21
// particles.  The first call on each device looks up the array's device
// address (cudaGetSymbolAddress) with that device current and keeps it for
// the life of the process, so a cudaDeviceReset between calls is not
// supported.  The stream must belong to the current device.  Every call waits
// for its own range flag on the host, so no call can be made while its stream
// is being captured into a CUDA graph (such a call is refused before it
// queues any work).  All calls share the one array and it keeps the last
// call's contents: the row counts and the flag are cleared on every call, and
// calls that overlap on the GPU (other threads or streams) race.
// ---------------------------------------------------------------------------
namespace {

constexpr int kNoAllocMaxNgrid = 256;
constexpr int64_t kNoAllocMaxParticles = int64_t(1) << 21;
constexpr size_t kNoAllocRows = (size_t)kNoAllocMaxNgrid * kNoAllocMaxNgrid + 1;
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kNaOffRowcnt = 0;
constexpr size_t kNaOffRowstart = kNaOffRowcnt + align256(sizeof(uint32_t) * kNoAllocRows);
constexpr size_t kNaOffSlot = kNaOffRowstart + align256(sizeof(uint32_t) * kNoAllocRows);
constexpr size_t kNaOffRec = kNaOffSlot + align256(sizeof(uint32_t) * kNoAllocMaxParticles);
constexpr size_t kNaOffFlags = kNaOffRec + align256(sizeof(float4) * kNoAllocMaxParticles);
constexpr size_t kNoAllocBytes = kNaOffFlags + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
unsigned char* g_noalloc_ptr[kMaxDevices] = {};

// Exclusive scan of n <= 65537 row counts by one CTA: chunks of 1024 with a
// running carry (warp shuffles, then the warp totals).
__global__ void __launch_bounds__(1024) k_scan_rows_1cta(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                         int64_t n) {
    __shared__ uint32_t wsum[32];
    __shared__ uint32_t carry;
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    if (t == 0) carry = 0u;
    for (int64_t base = 0; base < n; base += 1024) {
        __syncthreads();
        const int64_t g = base + t;
        const uint32_t v = g < n ? in[g] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) wsum[w] = x;
        __syncthreads();
        if (w == 0) {
            uint32_t s = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            wsum[lane] = s;   // inclusive warp-total prefix
        }
        __syncthreads();
        const uint32_t c0 = carry;
        const uint32_t incl = x + (w > 0 ? wsum[w - 1] : 0u);
        if (g < n) out[g] = c0 + incl - v;
        __syncthreads();
        if (t == 1023) carry = c0 + incl;
    }
}

}  // namespace

void density_noalloc(const float* x, const float* y, const float* z, int64_t np, int ngrid, float* fi,
                     cudaStream_t stream) {
    if (!x || !y || !z || !fi) throw Error{MGG_ERR_ARG, "density_noalloc: null pointer"};
    if (ngrid < 16 || ngrid > kNoAllocMaxNgrid || (ngrid & (ngrid - 1)) != 0)
        throw Error{MGG_ERR_ARG, "density_noalloc: NGRID must be a power of two in [16, 256]"};
    if (np < 1 || np > kNoAllocMaxParticles)
        throw Error{MGG_ERR_ARG, "density_noalloc: particle count must be in [1, 2097152]"};
    int dev = 0;
    MGG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) throw Error{MGG_ERR_ARG, "density_noalloc: device index out of range"};
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    MGG_CUDA(cudaStreamIsCapturing(stream, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        throw Error{MGG_ERR_STATE, "density_noalloc: the stream is being captured (the call waits for its result)"};
    int sdev = dev;
    MGG_CUDA(cudaStreamGetDevice(stream, &sdev));
    if (sdev != dev) throw Error{MGG_ERR_ARG, "density_noalloc: the stream belongs to another device"};
    unsigned char* base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {   // once per device, with that device current
            void* p = nullptr;
            MGG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
            g_noalloc_ptr[dev] = static_cast<unsigned char*>(p);
        }
        base = g_noalloc_ptr[dev];
    }
    uint32_t* rowcnt = reinterpret_cast<uint32_t*>(base + kNaOffRowcnt);
    uint32_t* rowstart = reinterpret_cast<uint32_t*>(base + kNaOffRowstart);
    uint32_t* slot = reinterpret_cast<uint32_t*>(base + kNaOffSlot);
    float4* rec = reinterpret_cast<float4*>(base + kNaOffRec);
    int32_t* flags = reinterpret_cast<int32_t*>(base + kNaOffFlags);
    const int N = ngrid;
    const int64_t rows = (int64_t)N * N;
    const int threads = 256;
    const int blocks = (int)std::min<int64_t>(div_up(np, threads), 148 * 16);
    MGG_CUDA(cudaMemsetAsync(rowcnt, 0, sizeof(uint32_t) * (rows + 1), stream));
    MGG_CUDA(cudaMemsetAsync(flags, 0, sizeof(int32_t), stream));
    k_cic_count<<<blocks, threads, 0, stream>>>(x, y, z, np, N, rowcnt, slot, flags);
    MGG_CHECK_LAUNCH();
    k_scan_rows_1cta<<<1, 1024, 0, stream>>>(rowcnt, rowstart, rows + 1);
    MGG_CHECK_LAUNCH();
    k_cic_scatter<<<blocks, threads, 0, stream>>>(x, y, z, np, N, rowstart, slot, rec);
    MGG_CHECK_LAUNCH();
    launch_deposit(rec, rowstart, N, (float)((double)N * N * N / (double)(float)np), fi, stream);
    MGG_CHECK_LAUNCH();
    int32_t h = 0;
    MGG_CUDA(cudaMemcpyAsync(&h, flags, sizeof(int32_t), cudaMemcpyDeviceToHost, stream));
    MGG_CUDA(cudaStreamSynchronize(stream));
    if (h) throw Error{MGG_ERR_NUMERIC, "density_noalloc: particle position outside [1, NGRID+1) (clamped)"};
}

}  // namespace mgg
