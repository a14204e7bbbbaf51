// Kernel (b): a hand-written Stockham 3-D real FFT, the replacement of the
// FFTPACK5 halfcomplex transforms (PMP2mod_fft5.f90) used by POTENTfft5
// (PMP2main.f90:705-867) and POWERfft5 (PMP2mod_power.f90:209-463).
//
// The reference transforms FI with separable real halfcomplex FFTs and divides
// every coefficient by the eigenvalue of the 7-point Laplacian,
//   A1 = GREENf(i) + GREENf(j) + GREENf(k) - 6,  GREENf = 2 cos(2 pi m / N),
// keeping the DC coefficient (A1 := 1, PMP2main.f90:815).  Because the kernel
// depends only on |m| along each axis, the same operator is diagonal in the
// complex Fourier basis, so a real-to-complex 3-D transform with the same A1
// reproduces it up to rounding.  Pipeline (each pass one kernel, FP32 data,
// FP32 twiddles tabulated from FP64):
//   x  : real rows -> half spectrum (N/2 complex FFT + split),      R2C
//   y  : complex lines along y,                                       forward
//   z  : forward along z, * trfi / A1 * 2 / N^3, inverse along z      (fused)
//   y  : inverse
//   x  : half spectrum -> real rows (merge + N/2 complex FFT),        C2R
// Butterflies: radix-4 Stockham autosort stages (one radix-2 stage first when
// log2 L is odd) on a shared-memory tile of lines; every thread keeps its
// butterflies of a stage in registers between the read and write barriers.
#include "mgg_internal.cuh"
#include "fft.cuh"
#include "reduce.cuh"

namespace mgg {

namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// multiply by SIGN * i
template <int SIGN>
__device__ __forceinline__ float2 mul_si(float2 a) {
    return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

constexpr int kMaxR = 8;

// In-place Stockham FFT of `nlines` lines of length L (power of two) held in
// shared memory; element e of line q lives at s[q*ls + e*es].
// SIGN = -1 forward, +1 inverse (unnormalised).  tw = exp(-2 pi i t / n) with
// n = L * twmul.  Must be called by all threads of the block.
template <int SIGN>
__device__ void stockham(float2* s, int L, int nlines, int ls, int es, bool lanes_over_lines,
                         const float2* __restrict__ tw, int twmul) {
    const int nt = blockDim.x, tid = threadIdx.x;
    int lg = 0;
    while ((1 << lg) < L) ++lg;
    int Ns = 1;
    if (lg & 1) {
        const int Lr = L >> 1;
        const int nb = nlines * Lr;
        float2 o0[kMaxR], o1[kMaxR];
#pragma unroll
        for (int r = 0; r < kMaxR; ++r) {
            const int b = tid + r * nt;
            if (b < nb) {
                const int q = lanes_over_lines ? b % nlines : b / Lr;
                const int j = lanes_over_lines ? b / nlines : b % Lr;
                const float2 v0 = s[q * ls + j * es], v1 = s[q * ls + (j + Lr) * es];
                o0[r] = cadd(v0, v1);
                o1[r] = csub(v0, v1);
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kMaxR; ++r) {
            const int b = tid + r * nt;
            if (b < nb) {
                const int q = lanes_over_lines ? b % nlines : b / Lr;
                const int j = lanes_over_lines ? b / nlines : b % Lr;
                s[q * ls + (2 * j) * es] = o0[r];
                s[q * ls + (2 * j + 1) * es] = o1[r];
            }
        }
        __syncthreads();
        Ns = 2;
    }
    const int Lr = L >> 2;
    const int nb = nlines * Lr;
    for (; Ns < L; Ns <<= 2) {
        float2 o[kMaxR / 2][4];
        const int tstep = (L / (4 * Ns)) * twmul;
#pragma unroll
        for (int r = 0; r < kMaxR / 2; ++r) {
            const int b = tid + r * nt;
            if (b < nb) {
                const int q = lanes_over_lines ? b % nlines : b / Lr;
                const int j = lanes_over_lines ? b / nlines : b % Lr;
                const int k = j & (Ns - 1);
                float2 v0 = s[q * ls + j * es];
                float2 v1 = s[q * ls + (j + Lr) * es];
                float2 v2 = s[q * ls + (j + 2 * Lr) * es];
                float2 v3 = s[q * ls + (j + 3 * Lr) * es];
                if (Ns > 1) {
                    float2 w1 = __ldg(tw + k * tstep), w2 = __ldg(tw + 2 * k * tstep), w3 = __ldg(tw + 3 * k * tstep);
                    if (SIGN > 0) { w1 = cconj(w1); w2 = cconj(w2); w3 = cconj(w3); }
                    v1 = cmul(v1, w1);
                    v2 = cmul(v2, w2);
                    v3 = cmul(v3, w3);
                }
                const float2 a = cadd(v0, v2), bb = csub(v0, v2), cc = cadd(v1, v3);
                const float2 d = mul_si<SIGN>(csub(v1, v3));
                o[r][0] = cadd(a, cc);
                o[r][2] = csub(a, cc);
                o[r][1] = cadd(bb, d);
                o[r][3] = csub(bb, d);
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < kMaxR / 2; ++r) {
            const int b = tid + r * nt;
            if (b < nb) {
                const int q = lanes_over_lines ? b % nlines : b / Lr;
                const int j = lanes_over_lines ? b / nlines : b % Lr;
                const int k = j & (Ns - 1);
                const int base = (j / Ns) * 4 * Ns + k;
                s[q * ls + (base) * es] = o[r][0];
                s[q * ls + (base + Ns) * es] = o[r][1];
                s[q * ls + (base + 2 * Ns) * es] = o[r][2];
                s[q * ls + (base + 3 * Ns) * es] = o[r][3];
            }
        }
        __syncthreads();
    }
}

// --------------------------------------------------------------- x pass ----
// Rows of n reals = L = n/2 complex; TB rows per block.
__global__ void k_fft_x_r2c(const float* __restrict__ in, float2* __restrict__ out, int n, int nxp,
                            int64_t nrows, int TB, const float2* __restrict__ tw) {
    extern __shared__ float2 sm[];
    const int L = n >> 1;
    const int ls = L + 1;
    const int64_t row0 = (int64_t)blockIdx.x * TB;
    const float2* in2 = reinterpret_cast<const float2*>(in);
    for (int e = threadIdx.x; e < TB * L; e += blockDim.x) {
        const int q = e / L, m = e % L;
        const int64_t row = row0 + q;
        sm[q * ls + m] = row < nrows ? __ldg(in2 + row * L + m) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    stockham<-1>(sm, L, TB, ls, 1, false, tw, 2);
    // split: X[k] = (Z[k] + conj Z[L-k])/2 - i/2 W^k (Z[k] - conj Z[L-k]),  k = 0..L
    for (int e = threadIdx.x; e < TB * (L + 1); e += blockDim.x) {
        const int q = e / (L + 1), k = e % (L + 1);
        const int64_t row = row0 + q;
        if (row >= nrows) continue;
        const float2 zk = sm[q * ls + (k == L ? 0 : k)];
        const float2 zc = cconj(sm[q * ls + (k == 0 ? 0 : L - k)]);
        const float2 fe = cscale(cadd(zk, zc), 0.5f);
        const float2 fo = mul_si<-1>(cscale(csub(zk, zc), 0.5f));
        const float2 w = __ldg(tw + k);
        out[row * nxp + k] = cadd(fe, cmul(w, fo));
    }
}

// Half spectrum rows -> real rows.  Output = (n/2) * x (unnormalised inverse / 2).
__global__ void k_fft_x_c2r(const float2* __restrict__ in, float* __restrict__ out, int n, int nxp,
                            int64_t nrows, int TB, const float2* __restrict__ tw) {
    extern __shared__ float2 sm[];
    const int L = n >> 1;
    const int ls = L + 1;
    const int64_t row0 = (int64_t)blockIdx.x * TB;
    for (int e = threadIdx.x; e < TB * (L + 1); e += blockDim.x) {
        const int q = e / (L + 1), m = e % (L + 1);
        const int64_t row = row0 + q;
        sm[q * ls + m] = row < nrows ? __ldg(in + row * nxp + m) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    // merge pairs (k, L-k) in place: Z[k] = Fe + i Fo,
    //   Fe = (X[k] + conj X[L-k]) / 2,  Fo = (X[k] - conj X[L-k]) conj(W^k) / 2
    for (int e = threadIdx.x; e < TB * (L / 2 + 1); e += blockDim.x) {
        const int q = e / (L / 2 + 1), k = e % (L / 2 + 1);
        const float2 xk = sm[q * ls + k], xl = sm[q * ls + (L - k)];
        const float2 fe = cscale(cadd(xk, cconj(xl)), 0.5f);
        const float2 fo = cscale(cmul(csub(xk, cconj(xl)), cconj(__ldg(tw + k))), 0.5f);
        const float2 z = cadd(fe, mul_si<1>(fo));
        // partner index L-k (equal to k when k = L/2, unused when k = 0)
        const int k2 = L - k;
        const float2 fe2 = cscale(cadd(xl, cconj(xk)), 0.5f);
        const float2 fo2 = cscale(cmul(csub(xl, cconj(xk)), cconj(__ldg(tw + k2))), 0.5f);
        const float2 z2 = cadd(fe2, mul_si<1>(fo2));
        sm[q * ls + k] = z;
        if (k2 < L && k2 != k) sm[q * ls + k2] = z2;
    }
    __syncthreads();
    stockham<1>(sm, L, TB, ls, 1, false, tw, 2);
    float2* out2 = reinterpret_cast<float2*>(out);
    for (int e = threadIdx.x; e < TB * L; e += blockDim.x) {
        const int q = e / L, m = e % L;
        const int64_t row = row0 + q;
        if (row < nrows) out2[row * L + m] = sm[q * ls + m];
    }
}

// ---------------------------------------------------------- y / z lines ----
// Tile: TX consecutive kx columns x n elements of one line set.
//   element (x, e) of tile o at buf[o*ostride + e*estride + x0 + x]
template <int MODE>
__global__ void k_fft_lines(float2* __restrict__ buf, int n, int nxp, int TX, int64_t estride,
                            int64_t ostride, int axis, const float2* __restrict__ tw, LineExtra ex) {
    extern __shared__ float2 sm[];
    const int x0 = blockIdx.x * TX;
    const int o = blockIdx.y;
    const int nxh = n / 2 + 1;
    const int nvalid = min(TX, nxh - x0);
    const float2* src = (MODE == LM_DISP) ? ex.src : buf;
    const int64_t base = (int64_t)o * ostride + x0;
    for (int e = threadIdx.x; e < TX * n; e += blockDim.x) {
        const int x = e % TX, el = e / TX;
        sm[el * TX + x] = x < nvalid ? __ldg(src + base + (int64_t)el * estride + x) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    if (MODE == LM_INV) {
        stockham<1>(sm, n, TX, 1, TX, true, tw, 1);
    } else if (MODE == LM_DISP) {
        // spectrum -> displacement component: psi_c(k) = i k_c / k^2 * T(k) * delta(k)
        for (int e = threadIdx.x; e < TX * n; e += blockDim.x) {
            const int x = e % TX, kz = e / TX;
            const int kx = x0 + x, ky = o;
            const int mx = kx, my = ky <= n / 2 ? ky : ky - n, mz = kz <= n / 2 ? kz : kz - n;
            const int m2 = mx * mx + my * my + mz * mz;
            float2 v = sm[e];
            float f = 0.f;
            if (m2 > 0 && x < nvalid) {
                int mc = ex.comp == 0 ? mx : (ex.comp == 1 ? my : mz);
                // Nyquist planes carry no odd (sine) part
                if ((ex.comp == 0 && kx == n / 2) || (ex.comp == 1 && ky == n / 2) || (ex.comp == 2 && kz == n / 2)) mc = 0;
                f = __ldg(ex.tk + m2) * (float)mc / (float)m2;
            }
            sm[e] = mul_si<1>(cscale(v, f));
        }
        __syncthreads();
        stockham<1>(sm, n, TX, 1, TX, true, tw, 1);
    } else {
        stockham<-1>(sm, n, TX, 1, TX, true, tw, 1);
        if (MODE == LM_GREEN) {
            // axis == 2: o = ky, element = kz
            for (int e = threadIdx.x; e < TX * n; e += blockDim.x) {
                const int x = e % TX, kz = e / TX;
                const int kx = min(x0 + x, n / 2);
                double A1 = (__ldg(ex.green + o) - 6.0 + __ldg(ex.green + kx)) + __ldg(ex.green + kz);
                if (fabs(A1) < 1.0e-7) A1 = 1.0;
                sm[e] = cscale(sm[e], (float)(ex.green_scale / A1));
            }
            __syncthreads();
            stockham<1>(sm, n, TX, 1, TX, true, tw, 1);
        } else if (MODE == LM_POWER) {
            unsigned long long* hl = reinterpret_cast<unsigned long long*>(sm + TX * n);
            unsigned long long* hg = hl + (n + 1);
            for (int e = threadIdx.x; e < 2 * (n + 1); e += blockDim.x) hl[e] = 0ull;
            __syncthreads();
            for (int e = threadIdx.x; e < TX * n; e += blockDim.x) {
                const int x = e % TX, kz = e / TX;
                if (x >= nvalid) continue;
                const int kx = x0 + x, ky = o;
                const int my = ky <= n / 2 ? ky : n - ky, mz = kz <= n / 2 ? kz : n - kz;
                const int m2 = kx * kx + my * my + mz * mz;
                if (m2 == 0) continue;
                const float RK = sqrtf((float)m2);
                int MP = (int)(RK + 0.5f);
                MP = MP < 1 ? 1 : MP;
                const int ML = __ldg(ex.logbin + m2);
                const float2 v = sm[e];
                const double w = (kx == 0 || kx == n / 2) ? 1.0 : 2.0;
                const double amp = w * ((double)v.x * v.x + (double)v.y * v.y) * ex.amp_scale;
                const unsigned long long fx = __double2ull_rn(amp);
                atomicAdd(hl + MP, fx);
                atomicAdd(hg + ML, fx);
            }
            __syncthreads();
            for (int e = threadIdx.x; e < 2 * (n + 1); e += blockDim.x)
                if (hl[e]) atomicAdd(ex.hist + e, hl[e]);
            return;
        }
    }
    float2* dst = buf;
    for (int e = threadIdx.x; e < TX * n; e += blockDim.x) {
        const int x = e % TX, el = e / TX;
        if (x < nvalid) dst[base + (int64_t)el * estride + x] = sm[el * TX + x];
    }
}

int x_rows_per_block(int n) {
    // keep TB * n/2 / 4 butterflies <= 4 * 256 threads
    int TB = 8;
    while (TB > 1 && TB * (n / 2) > 8192) TB >>= 1;
    return TB;
}

int line_tile(int n) { return 8; }

int line_threads(int n, int TX) {
    int t = TX * n / 4;
    if (t > 512) t = 512;
    if (t < 32) t = 32;
    return t;
}

}  // namespace

void fft_set_attributes() {
    const int big = 200 * 1024;
    MGG_CUDA(cudaFuncSetAttribute(k_fft_x_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_x_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_FWD>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_INV>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_GREEN>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_POWER>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_DISP>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
}

void fft_x_r2c(const FftPlan& p, const float* in, float2* out, cudaStream_t s) {
    const int n = p.n;
    const int64_t nrows = (int64_t)n * n;
    const int TB = x_rows_per_block(n);
    const int threads = min(512, max(32, TB * (n / 2) / 4));
    const size_t smem = (size_t)TB * (n / 2 + 1) * sizeof(float2);
    k_fft_x_r2c<<<div_up(nrows, TB), threads, smem, s>>>(in, out, n, p.nxp, nrows, TB, p.tw);
    MGG_CHECK_LAUNCH();
}

void fft_x_c2r(const FftPlan& p, const float2* in, float* out, cudaStream_t s) {
    const int n = p.n;
    const int64_t nrows = (int64_t)n * n;
    const int TB = x_rows_per_block(n);
    const int threads = min(512, max(32, TB * (n / 2) / 4));
    const size_t smem = (size_t)TB * (n / 2 + 1) * sizeof(float2);
    k_fft_x_c2r<<<div_up(nrows, TB), threads, smem, s>>>(in, out, n, p.nxp, nrows, TB, p.tw);
    MGG_CHECK_LAUNCH();
}

void fft_lines(const FftPlan& p, float2* buf, int axis, int mode, const LineExtra& ex, cudaStream_t s) {
    const int n = p.n;
    const int TX = line_tile(n);
    const int nxh = n / 2 + 1;
    dim3 grid(div_up(nxh, TX), n);
    int64_t estride, ostride;
    if (axis == 1) { estride = p.nxp; ostride = (int64_t)n * p.nxp; }       // o = z
    else { estride = (int64_t)n * p.nxp; ostride = p.nxp; }                  // o = y
    const int threads = line_threads(n, TX);
    size_t smem = (size_t)TX * n * sizeof(float2);
    switch (mode) {
    case LM_FWD: k_fft_lines<LM_FWD><<<grid, threads, smem, s>>>(buf, n, p.nxp, TX, estride, ostride, axis, p.tw, ex); break;
    case LM_INV: k_fft_lines<LM_INV><<<grid, threads, smem, s>>>(buf, n, p.nxp, TX, estride, ostride, axis, p.tw, ex); break;
    case LM_GREEN: k_fft_lines<LM_GREEN><<<grid, threads, smem, s>>>(buf, n, p.nxp, TX, estride, ostride, axis, p.tw, ex); break;
    case LM_POWER:
        smem += 2 * (size_t)(n + 1) * sizeof(unsigned long long);
        k_fft_lines<LM_POWER><<<grid, threads, smem, s>>>(buf, n, p.nxp, TX, estride, ostride, axis, p.tw, ex);
        break;
    case LM_DISP: k_fft_lines<LM_DISP><<<grid, threads, smem, s>>>(buf, n, p.nxp, TX, estride, ostride, axis, p.tw, ex); break;
    default: throw Error{MGG_ERR_ARG, "fft_lines: bad mode"};
    }
    MGG_CHECK_LAUNCH();
}

// ------------------------------------------------------------- context ----
void fft_alloc(Ctx& c) {
    const int N = c.N;
    c.nxp = ((N / 2 + 1) + 15) / 16 * 16;
    MGG_CUDA(cudaMalloc(&c.cbuf, sizeof(float2) * (size_t)c.nxp * N * N));
    std::vector<float2> tw(N);
    for (int k = 0; k < N; ++k) {
        const double a = -2.0 * M_PI * (double)k / (double)N;
        tw[k] = make_float2((float)cos(a), (float)sin(a));
    }
    MGG_CUDA(cudaMalloc(&c.tw_n, sizeof(float2) * N));
    MGG_CUDA(cudaMemcpy(c.tw_n, tw.data(), sizeof(float2) * N, cudaMemcpyHostToDevice));
    // GREENf of PMP2main.f90:736-742 mapped to the complex index k (m = min(k, N-k)),
    // with the reference's 2*pi constant P16 = 6.28318530718
    const double P16 = 6.28318530718;
    std::vector<double> g(N);
    for (int k = 0; k < N; ++k) {
        const int m = k <= N / 2 ? k : N - k;
        if (m == 0) g[k] = 2.0;
        else if (m == N / 2) g[k] = -2.0;
        else g[k] = 2.0 * cos(P16 * m / N);
    }
    MGG_CUDA(cudaMalloc(&c.green, sizeof(double) * N));
    MGG_CUDA(cudaMemcpy(c.green, g.data(), sizeof(double) * N, cudaMemcpyHostToDevice));
    // log-bin table per integer |k|^2 with the reference's Real*4 arithmetic
    // (MPlog = max(1, min(NPOWER, INT(Log10(RK)/dLog + 1000.) - 1000)), PMP2mod_power.f90:396)
    const int m2max = 3 * (N / 2) * (N / 2);
    std::vector<uint8_t> lb(m2max + 1, 0);
    for (int m2 = 1; m2 <= m2max; ++m2) {
        const float RK = sqrtf((float)m2);
        int ml = (int)(log10f(RK) / 0.02f + 1000.0f) - 1000;
        ml = ml < 1 ? 1 : (ml > N ? N : ml);
        if (ml > 255) ml = 255;
        lb[m2] = (uint8_t)ml;
    }
    MGG_CUDA(cudaMalloc(&c.pk_logbin, m2max + 1));
    MGG_CUDA(cudaMemcpy(c.pk_logbin, lb.data(), m2max + 1, cudaMemcpyHostToDevice));
    MGG_CUDA(cudaMalloc(&c.pk_hist, sizeof(unsigned long long) * 2 * (N + 1)));
    fft_set_attributes();
}

void poisson_solve(Ctx& c) {
    BucketScope bs(c, MGG_T_FORCE);
    const int N = c.N;
    FftPlan p;
    p.n = N;
    p.nxp = c.nxp;
    p.tw = c.tw_n;
    const double cells = (double)c.ncell;
    const double cplx = 8.0 * (double)N * N * (N / 2 + 1);
    // trfi (PMP2main.f90:728-732), Real*4
    float trfi;
    if (c.cfg.omb < 0.005f) trfi = 1.5f * (c.cfg.om - c.cfg.omb) / c.aexpn;
    else trfi = 1.5f * c.cfg.om / c.aexpn;
    LineExtra ex;
    ex.green = c.green;
    ex.green_scale = (double)trfi * 2.0 / (cells);
    {
        ProfScope ps(c, K_FFT_X_R2C, 4.0 * cells + cplx);
        fft_x_r2c(p, c.fi, c.cbuf, c.stream);
    }
    {
        ProfScope ps(c, K_FFT_Y, 2.0 * cplx);
        fft_lines(p, c.cbuf, 1, LM_FWD, ex, c.stream);
    }
    {
        ProfScope ps(c, K_FFT_Z_GREEN, 2.0 * cplx);
        fft_lines(p, c.cbuf, 2, LM_GREEN, ex, c.stream);
    }
    {
        ProfScope ps(c, K_FFT_Y, 2.0 * cplx);
        fft_lines(p, c.cbuf, 1, LM_INV, ex, c.stream);
    }
    {
        ProfScope ps(c, K_FFT_X_C2R, 4.0 * cells + cplx);
        fft_x_c2r(p, c.cbuf, c.fi, c.stream);
    }
}

namespace {
__global__ void k_sumsq(const float* __restrict__ f, int64_t n, double* __restrict__ part) {
    double v = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const double a = f[q];
        v += a * a;
    }
    v = block_sum_fixed(v);
    if (threadIdx.x == 0) part[blockIdx.x] = v;
}
}  // namespace

// Mode counts per integer |k|^2 over the full N^3 spectrum (each axis index
// m in [0, N/2] stands for 1 (m = 0, N/2) or 2 halfcomplex entries), the
// reference's iVolume/dk sums (PMP2mod_power.f90:406-409), computed once.
static void mode_counts(int N, std::vector<double>& cnt) {
    const int h = N / 2;
    const int m2max = 3 * h * h;
    cnt.assign(m2max + 1, 0.0);
    for (int a = 0; a <= h; ++a) {
        const double ca = (a == 0 || a == h) ? 1.0 : 2.0;
        for (int b = 0; b <= h; ++b) {
            const double cb = (b == 0 || b == h) ? 1.0 : 2.0;
            const int ab = a * a + b * b;
            for (int d = 0; d <= h; ++d) {
                const double cd = (d == 0 || d == h) ? 1.0 : 2.0;
                cnt[ab + d * d] += ca * cb * cd;
            }
        }
    }
}

void power_spectrum(Ctx& c, int nbins, double* k_out, double* n_out, double* p_out, double* kl_out,
                    double* nl_out, double* pl_out) {
    BucketScope bs(c, MGG_T_POWER);
    const int N = c.N;
    const double cells = (double)c.ncell;
    // Parseval bound for the fixed-point scale: sum_k |delta_k|^2 = sum delta^2 / N^3
    const int blocks = 148 * 8;
    ensure_partials(c, blocks);
    {
        ProfScope ps(c, K_GRID_OP, 4.0 * cells);
        k_sumsq<<<blocks, 256, 0, c.stream>>>(c.fi, c.ncell, c.red_partial);
        MGG_CHECK_LAUNCH();
    }
    const double s2 = reduce_sum_blocks(c, blocks);
    const double total = s2 / cells;   // >= any bin sum
    double scale = 1.0;
    if (total > 0.0) {
        int e;
        frexp(total, &e);                    // total < 2^e
        scale = ldexp(1.0, 61 - e);          // sums stay below 2^61
    }
    FftPlan p;
    p.n = N;
    p.nxp = c.nxp;
    p.tw = c.tw_n;
    LineExtra ex;
    ex.logbin = c.pk_logbin;
    ex.hist = c.pk_hist;
    ex.amp_scale = scale / (cells * cells);
    MGG_CUDA(cudaMemsetAsync(c.pk_hist, 0, sizeof(unsigned long long) * 2 * (N + 1), c.stream));
    const double cplx = 8.0 * (double)N * N * (N / 2 + 1);
    {
        ProfScope ps(c, K_FFT_X_R2C, 4.0 * cells + cplx);
        fft_x_r2c(p, c.fi, c.cbuf, c.stream);
    }
    {
        ProfScope ps(c, K_FFT_Y, 2.0 * cplx);
        fft_lines(p, c.cbuf, 1, LM_FWD, ex, c.stream);
    }
    {
        ProfScope ps(c, K_FFT_Z_POWER, cplx);
        fft_lines(p, c.cbuf, 2, LM_POWER, ex, c.stream);
    }
    std::vector<unsigned long long> h(2 * (N + 1));
    MGG_CUDA(cudaMemcpyAsync(h.data(), c.pk_hist, sizeof(unsigned long long) * 2 * (N + 1),
                             cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaStreamSynchronize(c.stream));
    // mode counts and <k> per bin (exact, data independent)
    static thread_local int cached_n = -1;
    static thread_local std::vector<double> cnt;
    if (cached_n != N) {
        mode_counts(N, cnt);
        cached_n = N;
    }
    std::vector<double> iV(N + 1, 0.0), dk(N + 1, 0.0), iVl(N + 1, 0.0), dkl(N + 1, 0.0);
    std::vector<uint8_t> lb(cnt.size());
    MGG_CUDA(cudaMemcpy(lb.data(), c.pk_logbin, cnt.size(), cudaMemcpyDeviceToHost));
    for (size_t m2 = 1; m2 < cnt.size(); ++m2) {
        if (cnt[m2] == 0.0) continue;
        const float RK = sqrtf((float)m2);
        int MP = (int)(RK + 0.5f);
        MP = MP < 1 ? 1 : MP;
        iV[MP] += cnt[m2];
        dk[MP] += cnt[m2] * (double)RK;
        iVl[lb[m2]] += cnt[m2];
        dkl[lb[m2]] += cnt[m2] * (double)RK;
    }
    const float Pi = 3.141592653f;
    const float Scale = 2.0f * Pi / c.cfg.box;
    const float b3 = c.cfg.box * c.cfg.box * c.cfg.box;
    const double unfix = 1.0 / scale;
    for (int I = 1; I <= nbins && I <= N / 2; ++I) {
        double kv = 0, nv = 0, pv = 0, klv = 0, nlv = 0, plv = 0;
        if (iV[I] > 0) {
            kv = (float)(dk[I] / iV[I] * (double)Scale);
            nv = (float)iV[I];
            pv = (float)((double)b3 * ((double)h[I] * unfix) / iV[I]);
        }
        if (iVl[I] > 0) {
            klv = (float)(dkl[I] / iVl[I] * (double)Scale);
            nlv = (float)iVl[I];
            plv = (float)((double)b3 * ((double)h[(N + 1) + I] * unfix) / iVl[I]);
        }
        if (k_out) k_out[I - 1] = kv;
        if (n_out) n_out[I - 1] = nv;
        if (p_out) p_out[I - 1] = pv;
        if (kl_out) kl_out[I - 1] = klv;
        if (nl_out) nl_out[I - 1] = nlv;
        if (pl_out) pl_out[I - 1] = plv;
    }
}

}  // namespace mgg
