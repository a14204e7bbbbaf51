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
// reproduces it up to rounding.  Pipeline (each pass one kernel, FP32 data
// between passes; the lines of a pass are computed in FP64 on the plain path,
// as FFTPACK5's real(kind=8), and in FP32 in the precision form, with twiddles
// tabulated in FP64):
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
#include <cuda.h>   // CUtensorMap (encoded on the host through the runtime's driver entry point)
#include <cstdlib>
#include <initializer_list>
#include <map>
#include <mutex>
#include <tuple>
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
// the same in FP64 (the plain path's line arithmetic, as FFTPACK5's real(kind=8))
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
template <int SIGN>
__device__ __forceinline__ double2 mul_si(double2 a) {
    return SIGN < 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}
// scalar type of a complex type; FP32 storage <-> the arithmetic type
template <class C> struct Scal;
template <> struct Scal<float2> { typedef float T; };
template <> struct Scal<double2> { typedef double T; };
template <class C> __device__ __forceinline__ C from_f2(float2 v);
template <> __device__ __forceinline__ float2 from_f2<float2>(float2 v) { return v; }
template <> __device__ __forceinline__ double2 from_f2<double2>(float2 v) { return make_double2(v.x, v.y); }
__device__ __forceinline__ float2 to_f2(float2 v) { return v; }
__device__ __forceinline__ float2 to_f2(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <class C> __device__ __forceinline__ C czero();
template <> __device__ __forceinline__ float2 czero<float2>() { return make_float2(0.f, 0.f); }
template <> __device__ __forceinline__ double2 czero<double2>() { return make_double2(0.0, 0.0); }

constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v >> 1); }

// W16^p = exp(-2 pi i p / 16) for p = 0..15, as (cos, sin) pairs
__device__ __forceinline__ float w16c(int p) {
    constexpr float c[16] = {1.0f, 0.92387953251f, 0.70710678119f, 0.38268343237f, 0.0f, -0.38268343237f,
                             -0.70710678119f, -0.92387953251f, -1.0f, -0.92387953251f, -0.70710678119f,
                             -0.38268343237f, 0.0f, 0.38268343237f, 0.70710678119f, 0.92387953251f};
    return c[p & 15];
}
__device__ __forceinline__ float w16s(int p) { return w16c(p + 12); }   // sin(2 pi p/16) = cos(2 pi (p-4)/16)
__device__ __forceinline__ double w16c_d(int p) {
    constexpr double c[16] = {1.0, 0.92387953251128674, 0.70710678118654752, 0.38268343236508977, 0.0,
                              -0.38268343236508977, -0.70710678118654752, -0.92387953251128674, -1.0,
                              -0.92387953251128674, -0.70710678118654752, -0.38268343236508977, 0.0,
                              0.38268343236508977, 0.70710678118654752, 0.92387953251128674};
    return c[p & 15];
}
// v * exp(SIGN 2 pi i p / 16), p a compile-time constant after unrolling
template <int SIGN>
__device__ __forceinline__ float2 rot16(float2 v, int p) {
    if ((p & 15) == 0) return v;
    if ((p & 15) == 4) return mul_si<SIGN>(v);
    if ((p & 15) == 8) return make_float2(-v.x, -v.y);
    if ((p & 15) == 12) return mul_si<-SIGN>(v);
    const float c = w16c(p), sn = (float)SIGN * w16s(p);
    return make_float2(v.x * c - v.y * sn, v.x * sn + v.y * c);
}
template <int SIGN>
__device__ __forceinline__ double2 rot16(double2 v, int p) {
    if ((p & 15) == 0) return v;
    if ((p & 15) == 4) return mul_si<SIGN>(v);
    if ((p & 15) == 8) return make_double2(-v.x, -v.y);
    if ((p & 15) == 12) return mul_si<-SIGN>(v);
    const double c = w16c_d(p), sn = (double)SIGN * w16c_d(p + 12);
    return make_double2(v.x * c - v.y * sn, v.x * sn + v.y * c);
}

// In-register DFTs of size R = 2, 4, 8, 16, natural order in and out:
// X[m] = sum_r v[r] exp(SIGN 2 pi i r m / R)
template <int SIGN, class C>
__device__ __forceinline__ void dft4(C& v0, C& v1, C& v2, C& v3) {
    const C a = cadd(v0, v2), bb = csub(v0, v2), cc = cadd(v1, v3);
    const C d = mul_si<SIGN>(csub(v1, v3));
    v0 = cadd(a, cc);
    v2 = csub(a, cc);
    v1 = cadd(bb, d);
    v3 = csub(bb, d);
}
template <int SIGN, int R, class C>
__device__ __forceinline__ void dft(C* v) {
    if (R == 2) {
        const C a = v[0], b = v[1];
        v[0] = cadd(a, b);
        v[1] = csub(a, b);
    } else if (R == 4) {
        dft4<SIGN>(v[0], v[1], v[2], v[3]);
    } else if (R == 8) {   // r = r1 + 2 r2, m = m1 + 4 m2
        C y[2][4];
#pragma unroll
        for (int r1 = 0; r1 < 2; ++r1) {
            y[r1][0] = v[r1]; y[r1][1] = v[r1 + 2]; y[r1][2] = v[r1 + 4]; y[r1][3] = v[r1 + 6];
            dft4<SIGN>(y[r1][0], y[r1][1], y[r1][2], y[r1][3]);
#pragma unroll
            for (int m1 = 0; m1 < 4; ++m1) y[r1][m1] = rot16<SIGN>(y[r1][m1], 2 * r1 * m1);
        }
#pragma unroll
        for (int m1 = 0; m1 < 4; ++m1) {
            v[m1] = cadd(y[0][m1], y[1][m1]);
            v[m1 + 4] = csub(y[0][m1], y[1][m1]);
        }
    } else {               // R == 16: r = r1 + 4 r2, m = m1 + 4 m2
        C y[4][4];
#pragma unroll
        for (int r1 = 0; r1 < 4; ++r1) {
            y[r1][0] = v[r1]; y[r1][1] = v[r1 + 4]; y[r1][2] = v[r1 + 8]; y[r1][3] = v[r1 + 12];
            dft4<SIGN>(y[r1][0], y[r1][1], y[r1][2], y[r1][3]);
#pragma unroll
            for (int m1 = 0; m1 < 4; ++m1) y[r1][m1] = rot16<SIGN>(y[r1][m1], r1 * m1);
        }
#pragma unroll
        for (int m1 = 0; m1 < 4; ++m1) {
            dft4<SIGN>(y[0][m1], y[1][m1], y[2][m1], y[3][m1]);
            v[m1] = y[0][m1]; v[m1 + 4] = y[1][m1]; v[m1 + 8] = y[2][m1]; v[m1 + 12] = y[3][m1];
        }
    }
}

// One radix-2^LGR Stockham stage (sub-transform size Ns = 2^LGNS -> R Ns) of NL
// lines of length L in shared memory; element e of line q lives at
// s[q*LS + e*ES].  tw[t] = exp(-2 pi i t / (L * TWM)).  Each thread keeps its
// butterflies in registers between the read and the write barrier.
template <int SIGN, int LGR, int L, int NL, int LS, int ES, bool LOL, int NT, int TWM, int LGNS, class C>
__device__ __forceinline__ void stockham_stage(C* s, const C* __restrict__ tw) {
    constexpr int R = 1 << LGR, LG = ilog2c(L), LGNL = ilog2c(NL);
    constexpr int LR = L / R, LGLR = LG - LGR, NB = NL * LR, RB = (NB + NT - 1) / NT;
    constexpr int NS = 1 << LGNS;
    constexpr int TSTEP = (L / (R * NS)) * TWM;
    const int tid = threadIdx.x;
    C v[RB][R];
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
        const int b = tid + rb * NT;
        if (NB % NT == 0 || b < NB) {
            const int q = LOL ? (b & (NL - 1)) : (b >> LGLR);
            const int j = LOL ? (b >> LGNL) : (b & (LR - 1));
            const int k = j & (NS - 1);
#pragma unroll
            for (int r = 0; r < R; ++r) v[rb][r] = s[q * LS + (j + r * LR) * ES];
            if (LGNS > 0) {
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    C w = __ldg(tw + r * k * TSTEP);
                    if (SIGN > 0) w = cconj(w);
                    v[rb][r] = cmul(v[rb][r], w);
                }
            }
            dft<SIGN, R>(v[rb]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) {
        const int b = tid + rb * NT;
        if (NB % NT == 0 || b < NB) {
            const int q = LOL ? (b & (NL - 1)) : (b >> LGLR);
            const int j = LOL ? (b >> LGNL) : (b & (LR - 1));
            const int k = j & (NS - 1);
            const int base = ((j >> LGNS) << (LGNS + LGR)) + k;
#pragma unroll
            for (int r = 0; r < R; ++r) s[q * LS + (base + r * NS) * ES] = v[rb][r];
        }
    }
    __syncthreads();
}

// In-place Stockham FFT of NL lines of length L (powers of two) in shared
// memory; element e of line q lives at s[q*LS + e*ES].  SIGN = -1 forward,
// +1 inverse (unnormalised).  tw[t] = exp(-2 pi i t / (L * TWM)).  NT threads;
// with LOL, consecutive butterflies run over lines first (lines are the fast
// index in shared memory), otherwise along a line.  Stages are radix 16 (one
// smaller radix first when log2 L is not a multiple of 4), so a 1024-point
// line takes three shared-memory passes; all sizes are compile-time.
template <int SIGN, int L, int NL, int LS, int ES, bool LOL, int NT, int TWM, int LGNS = 0, class C>
__device__ __forceinline__ void stockham_t(C* s, const C* __restrict__ tw) {
    constexpr int LG = ilog2c(L);
    if constexpr (LGNS < LG) {
        constexpr int LGR = LGNS == 0 ? (LG % 4 == 0 ? 4 : LG % 4) : 4;
        stockham_stage<SIGN, LGR, L, NL, LS, ES, LOL, NT, TWM, LGNS, C>(s, tw);
        stockham_t<SIGN, L, NL, LS, ES, LOL, NT, TWM, LGNS + LGR, C>(s, tw);
    }
}

// Radix-4 variant (used by the x pass, whose rows sit along shared memory and
// leave radix-16 stages short of butterflies).  In-place Stockham FFT of NL lines
// of length L (powers of two) in shared memory; element e of line q lives at s[q*LS + e*ES].  SIGN = -1 forward,
// +1 inverse (unnormalised).  tw[t] = exp(-2 pi i t / (L * TWM)).  NT threads;
// with LOL, consecutive butterflies run over lines first (lines are the fast
// index in shared memory), otherwise along a line.  All sizes are
// compile-time, so index arithmetic is shifts and masks and every stage is
// unrolled; each thread keeps its butterflies of a stage in registers between
// the read and the write barrier.
template <int SIGN, int L, int NL, int LS, int ES, bool LOL, int NT, int TWM, class C>
__device__ __forceinline__ void stockham_r4(C* s, const C* __restrict__ tw) {
    constexpr int LG = ilog2c(L), LGNL = ilog2c(NL);
    const int tid = threadIdx.x;
    if (LG & 1) {   // one radix-2 stage first
        constexpr int LR = L / 2, LGLR = LG - 1, NB = NL * LR, R = (NB + NT - 1) / NT;
        C o0[R], o1[R];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int b = tid + r * NT;
            if (NB % NT == 0 || b < NB) {
                const int q = LOL ? (b & (NL - 1)) : (b >> LGLR);
                const int j = LOL ? (b >> LGNL) : (b & (LR - 1));
                const C v0 = s[q * LS + j * ES], v1 = s[q * LS + (j + LR) * ES];
                o0[r] = cadd(v0, v1);
                o1[r] = csub(v0, v1);
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int b = tid + r * NT;
            if (NB % NT == 0 || b < NB) {
                const int q = LOL ? (b & (NL - 1)) : (b >> LGLR);
                const int j = LOL ? (b >> LGNL) : (b & (LR - 1));
                s[q * LS + (2 * j) * ES] = o0[r];
                s[q * LS + (2 * j + 1) * ES] = o1[r];
            }
        }
        __syncthreads();
    }
    constexpr int LR = L / 4, LGLR = LG - 2, NB = NL * LR, R = (NB + NT - 1) / NT;
#pragma unroll
    for (int lgns = (LG & 1); lgns < LG; lgns += 2) {
        const int Ns = 1 << lgns;
        const int tstep = (L / (4 * Ns)) * TWM;
        C o[R][4];
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int b = tid + r * NT;
            if (NB % NT == 0 || b < NB) {
                const int q = LOL ? (b & (NL - 1)) : (b >> LGLR);
                const int j = LOL ? (b >> LGNL) : (b & (LR - 1));
                const int k = j & (Ns - 1);
                C v0 = s[q * LS + j * ES];
                C v1 = s[q * LS + (j + LR) * ES];
                C v2 = s[q * LS + (j + 2 * LR) * ES];
                C v3 = s[q * LS + (j + 3 * LR) * ES];
                if (lgns > 0) {
                    C w1 = __ldg(tw + k * tstep), w2 = __ldg(tw + 2 * k * tstep), w3 = __ldg(tw + 3 * k * tstep);
                    if (SIGN > 0) { w1 = cconj(w1); w2 = cconj(w2); w3 = cconj(w3); }
                    v1 = cmul(v1, w1);
                    v2 = cmul(v2, w2);
                    v3 = cmul(v3, w3);
                }
                const C a = cadd(v0, v2), bb = csub(v0, v2), cc = cadd(v1, v3);
                const C d = mul_si<SIGN>(csub(v1, v3));
                o[r][0] = cadd(a, cc);
                o[r][2] = csub(a, cc);
                o[r][1] = cadd(bb, d);
                o[r][3] = csub(bb, d);
            }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int b = tid + r * NT;
            if (NB % NT == 0 || b < NB) {
                const int q = LOL ? (b & (NL - 1)) : (b >> LGLR);
                const int j = LOL ? (b >> LGNL) : (b & (LR - 1));
                const int k = j & (Ns - 1);
                const int base = ((j >> lgns) << (lgns + 2)) + k;
                s[q * LS + (base) * ES] = o[r][0];
                s[q * LS + (base + Ns) * ES] = o[r][1];
                s[q * LS + (base + 2 * Ns) * ES] = o[r][2];
                s[q * LS + (base + 3 * Ns) * ES] = o[r][3];
            }
        }
        __syncthreads();
    }
}

// Launch shapes per grid size N (powers of two, 16..1024)
template <int N>
struct XShape {   // x pass: TB rows of L = N/2 complex per block
    static constexpr int L = N / 2;
    static constexpr int TB = (4096 / L) < N * N ? (4096 / L) : N * N;
    static constexpr int NT = (TB * L / 4) < 512 ? (TB * L / 4 < 32 ? 32 : TB * L / 4) : 512;
    static constexpr int LS = L + 1;
};
template <int N>
struct LShape {   // y / z lines: TX kx columns x N elements per block
    static constexpr int TX = 8;
    static constexpr int NT = (TX * N / 4) < 512 ? (TX * N / 4 < 32 ? 32 : TX * N / 4) : 512;
};

// --------------------------------------------------------------- x pass ----
// Rows of N reals = L = N/2 complex; TB rows per block.
template <int N, class C>
__global__ void __launch_bounds__(XShape<N>::NT, sizeof(C) == 8 ? 4 : 1) k_fft_x_r2c(const float* __restrict__ in, float2* __restrict__ out,
                                                             int nxp, const C* __restrict__ tw) {
    using X = XShape<N>;
    using T = typename Scal<C>::T;
    constexpr int L = X::L, TB = X::TB, NT = X::NT, LS = X::LS, LGL = ilog2c(L);
    constexpr int64_t NROWS = (int64_t)N * N;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    C* sm = reinterpret_cast<C*>(sm_raw);
    const int64_t row0 = (int64_t)blockIdx.x * TB;
    const float2* in2 = reinterpret_cast<const float2*>(in);
#pragma unroll 4
    for (int e = threadIdx.x; e < TB * L; e += NT) {
        const int q = e >> LGL, m = e & (L - 1);
        const int64_t row = row0 + q;
        sm[q * LS + m] = (TB <= NROWS || row < NROWS) ? from_f2<C>(__ldg(in2 + row * L + m)) : czero<C>();
    }
    __syncthreads();
    stockham_r4<-1, L, TB, LS, 1, false, NT, 2>(sm, tw);
    // split: X[k] = (Z[k] + conj Z[L-k])/2 - i/2 W^k (Z[k] - conj Z[L-k]),  k = 0..L
#pragma unroll 4
    for (int e = threadIdx.x; e < TB * (L + 1); e += NT) {
        const int q = e / (L + 1), k = e - q * (L + 1);
        const int64_t row = row0 + q;
        if (row >= NROWS) continue;
        const C zk = sm[q * LS + (k == L ? 0 : k)];
        const C zc = cconj(sm[q * LS + (k == 0 ? 0 : L - k)]);
        const C fe = cscale(cadd(zk, zc), (T)0.5);
        const C fo = mul_si<-1>(cscale(csub(zk, zc), (T)0.5));
        const C w = __ldg(tw + k);
        out[row * nxp + k] = to_f2(cadd(fe, cmul(w, fo)));
    }
}

// Half spectrum rows -> real rows.  Output = (N/2) * x (unnormalised inverse / 2).
template <int N, class C>
__global__ void __launch_bounds__(XShape<N>::NT, sizeof(C) == 8 ? 4 : 1) k_fft_x_c2r(const float2* __restrict__ in, float* __restrict__ out,
                                                             int nxp, const C* __restrict__ tw) {
    using X = XShape<N>;
    using T = typename Scal<C>::T;
    constexpr int L = X::L, TB = X::TB, NT = X::NT, LS = X::LS, LGL = ilog2c(L);
    constexpr int64_t NROWS = (int64_t)N * N;
    extern __shared__ __align__(16) unsigned char sm_raw[];
    C* sm = reinterpret_cast<C*>(sm_raw);
    const int64_t row0 = (int64_t)blockIdx.x * TB;
#pragma unroll 4
    for (int e = threadIdx.x; e < TB * (L + 1); e += NT) {
        const int q = e / (L + 1), m = e - q * (L + 1);
        const int64_t row = row0 + q;
        sm[q * LS + m] = row < NROWS ? from_f2<C>(__ldg(in + row * nxp + m)) : czero<C>();
    }
    __syncthreads();
    // merge pairs (k, L-k) in place: Z[k] = Fe + i Fo,
    //   Fe = (X[k] + conj X[L-k]) / 2,  Fo = (X[k] - conj X[L-k]) conj(W^k) / 2
    for (int e = threadIdx.x; e < TB * (L / 2 + 1); e += NT) {
        const int q = e / (L / 2 + 1), k = e - q * (L / 2 + 1);
        const C xk = sm[q * LS + k], xl = sm[q * LS + (L - k)];
        const C fe = cscale(cadd(xk, cconj(xl)), (T)0.5);
        const C fo = cscale(cmul(csub(xk, cconj(xl)), cconj(__ldg(tw + k))), (T)0.5);
        const C z = cadd(fe, mul_si<1>(fo));
        // partner index L-k (equal to k when k = L/2, unused when k = 0)
        const int k2 = L - k;
        const C fe2 = cscale(cadd(xl, cconj(xk)), (T)0.5);
        const C fo2 = cscale(cmul(csub(xl, cconj(xk)), cconj(__ldg(tw + k2))), (T)0.5);
        const C z2 = cadd(fe2, mul_si<1>(fo2));
        sm[q * LS + k] = z;
        if (k2 < L && k2 != k) sm[q * LS + k2] = z2;
    }
    __syncthreads();
    stockham_r4<1, L, TB, LS, 1, false, NT, 2>(sm, tw);
    float2* out2 = reinterpret_cast<float2*>(out);
#pragma unroll 4
    for (int e = threadIdx.x; e < TB * L; e += NT) {
        const int q = e >> LGL, m = e & (L - 1);
        const int64_t row = row0 + q;
        if (TB <= NROWS || row < NROWS) out2[row * L + m] = to_f2(sm[q * LS + m]);
    }
}

// ---------------------------------------------------------- y / z lines ----
// Tile: TX consecutive kx columns x N elements of one line set.
//   element (x, e) of tile o at buf[o*ostride + e*estride + x0 + x]
// C: the arithmetic type of the lines (float2, or double2 for the plain path's
// FP64 line arithmetic); the spectrum is stored as float2 either way.
//
// The transform of one tile in shared memory (every mode but the loads and
// stores): LM_POWER adds the tile's modes into the block's histograms hl
// (zeroed by the caller) and leaves the tile as it is.
// Adds v to h[bin] for every lane of the warp (all 32 lanes call it together):
// the lanes of each distinct bin are summed by shuffles and one lane adds the
// sum with one shared-memory atomic.  The histograms are integers (fixed point),
// so the totals do not depend on the order of the additions.
__device__ __forceinline__ void warp_bin_add(unsigned long long* h, int bin, unsigned long long v) {
    const unsigned lane = threadIdx.x & 31u;
    unsigned rem = __ballot_sync(0xffffffffu, v != 0ull);
    while (rem) {
        const int lead = __ffs(rem) - 1;
        const int b = __shfl_sync(0xffffffffu, bin, lead);
        const bool mine = ((rem >> lane) & 1u) && bin == b;
        unsigned long long t = mine ? v : 0ull;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
        if ((int)lane == lead) atomicAdd(h + b, t);
        rem &= ~__ballot_sync(0xffffffffu, mine);
    }
}

template <int MODE, int N, class C, int TX = LShape<N>::TX, int NT = LShape<N>::NT>
__device__ __forceinline__ void lines_compute(C* sm, int x0, int o, int nvalid, const C* __restrict__ tw,
                                              const LineExtra& ex, unsigned long long* hl) {
    using T = typename Scal<C>::T;
    constexpr int LGTX = ilog2c(TX);
    if (MODE == LM_INV) {
        stockham_t<1, N, TX, 1, TX, true, NT, 1>(sm, tw);
    } else if (MODE == LM_DISP) {
        // spectrum -> displacement component: psi_c(k) = i k_c / k^2 * T(k) * delta(k)
        for (int e = threadIdx.x; e < TX * N; e += NT) {
            const int x = e & (TX - 1), kz = e >> LGTX;
            const int kx = x0 + x, ky = o;
            const int mx = kx, my = ky <= N / 2 ? ky : ky - N, mz = kz <= N / 2 ? kz : kz - N;
            const int m2 = mx * mx + my * my + mz * mz;
            C v = sm[e];
            T f = (T)0;
            if (m2 > 0 && x < nvalid) {
                int mc = ex.comp == 0 ? mx : (ex.comp == 1 ? my : mz);
                // Nyquist planes carry no odd (sine) part
                if ((ex.comp == 0 && kx == N / 2) || (ex.comp == 1 && ky == N / 2) || (ex.comp == 2 && kz == N / 2)) mc = 0;
                f = (T)(__ldg(ex.tk + m2) * (float)mc / (float)m2);
            }
            sm[e] = mul_si<1>(cscale(v, f));
        }
        __syncthreads();
        stockham_t<1, N, TX, 1, TX, true, NT, 1>(sm, tw);
    } else {
        stockham_t<-1, N, TX, 1, TX, true, NT, 1>(sm, tw);
        if (MODE == LM_GREEN) {
            // axis == 2: o = ky, element = kz
            const double go = __ldg(ex.green + o) - 6.0;
            for (int e = threadIdx.x; e < TX * N; e += NT) {
                const int x = e & (TX - 1), kz = e >> LGTX;
                const int kx = min(x0 + x, N / 2);
                double A1 = (go + __ldg(ex.green + kx)) + __ldg(ex.green + kz);
                if (fabs(A1) < 1.0e-7) A1 = 1.0;
                // green_scale / A1: SFU reciprocal seed refined by two Newton steps in FP64
                // (|A1| lies in [1e-7, 12], so the seed is a normal float)
                double r = (double)(1.0f / (float)A1);
                r = fma(r, fma(-A1, r, 1.0), r);
                r = fma(r, fma(-A1, r, 1.0), r);
                sm[e] = cscale(sm[e], (T)(ex.green_scale * r));
            }
            __syncthreads();
            stockham_t<1, N, TX, 1, TX, true, NT, 1>(sm, tw);
        } else if (MODE == LM_POWER) {
            // linear bins, log bins, quadrupole-weighted linear bins (two's-complement sums).
            // The loop's trip count is the same for every thread (TX N is a multiple of NT),
            // so whole warps bin together: one shared-memory atomic per distinct bin of a warp.
            unsigned long long* hg = hl + (N + 1);
            unsigned long long* hq = hl + 2 * (N + 1);
            static_assert((TX * N) % NT == 0 && NT % 32 == 0, "whole warps in every binning round");
            for (int e = threadIdx.x; e < TX * N; e += NT) {
                const int x = e & (TX - 1), kz = e >> LGTX;
                const int kx = x0 + x, ky = o;
                const int my = ky <= N / 2 ? ky : N - ky, mz = kz <= N / 2 ? kz : N - kz;
                const int m2 = kx * kx + my * my + mz * mz;
                int MP = 0, ML = 0;
                unsigned long long fx = 0ull, fq = 0ull;
                if (x < nvalid && m2 != 0) {
                    const float RK = sqrtf((float)m2);
                    MP = (int)(RK + 0.5f);
                    MP = MP < 1 ? 1 : MP;
                    ML = __ldg(ex.logbin + m2);
                    const C v = sm[e];
                    const double w = (kx == 0 || kx == N / 2) ? 1.0 : 2.0;
                    const double amp = w * ((double)v.x * v.x + (double)v.y * v.y) * ex.amp_scale;
                    fx = __double2ull_rn(amp);
                    if (ex.quad) {
                        // P2(mu) about z in Real*4 as the reference (cosmu2 = MI/RK**2, P2 = 1.5 cosmu2 - 0.5,
                        // PMP2mod_power.f90:386-388, its MI being the z index after its x<->z transposition)
                        const float cosmu2 = __fdiv_rn((float)(mz * mz), __fmul_rn(RK, RK));
                        const float p2 = __fsub_rn(__fmul_rn(1.5f, cosmu2), 0.5f);
                        fq = (unsigned long long)__double2ll_rn(amp * (double)p2);
                    }
                }
                warp_bin_add(hl, MP, fx);
                warp_bin_add(hg, ML, fx);
                if (ex.quad) warp_bin_add(hq, MP, fq);
            }
        }
    }
}

template <int MODE, int N, class C>
__global__ void __launch_bounds__(LShape<N>::NT, sizeof(C) == 8 ? 2 : 1) k_fft_lines(float2* __restrict__ buf,
                                                                                    int64_t estride, int64_t ostride,
                                                                                    const C* __restrict__ tw,
                                                                                    LineExtra ex) {
    constexpr int TX = LShape<N>::TX, NT = LShape<N>::NT, LGTX = ilog2c(TX);
    extern __shared__ __align__(16) unsigned char sm_raw[];
    C* sm = reinterpret_cast<C*>(sm_raw);
    const int x0 = blockIdx.x * TX;
    const int o = blockIdx.y;
    constexpr int nxh = N / 2 + 1;
    const int nvalid = min(TX, nxh - x0);
    const float2* src = (MODE == LM_DISP) ? ex.src : buf;
    const int64_t base = (int64_t)o * ostride + x0;
#pragma unroll 4
    for (int e = threadIdx.x; e < TX * N; e += NT) {
        const int x = e & (TX - 1), el = e >> LGTX;
        sm[e] = x < nvalid ? from_f2<C>(__ldg(src + base + (int64_t)el * estride + x)) : czero<C>();
    }
    __syncthreads();
    unsigned long long* hl = reinterpret_cast<unsigned long long*>(sm + TX * N);   // after the tile
    const int nh = ex.quad ? 3 * (N + 1) : 2 * (N + 1);
    if (MODE == LM_POWER) {
        for (int e = threadIdx.x; e < nh; e += NT) hl[e] = 0ull;
        __syncthreads();
    }
    lines_compute<MODE, N, C>(sm, x0, o, nvalid, tw, ex, hl);
    if constexpr (MODE == LM_POWER) {
        __syncthreads();
        for (int e = threadIdx.x; e < nh; e += NT)
            if (hl[e]) atomicAdd(ex.hist + e, hl[e]);
    } else {
#pragma unroll 4
        for (int e = threadIdx.x; e < TX * N; e += NT) {
            const int x = e & (TX - 1), el = e >> LGTX;
            if (x < nvalid) buf[base + (int64_t)el * estride + x] = to_f2(sm[e]);
        }
    }
}

// ------------------------------------------- y / z lines, TMA-staged pencils ----
// The precision form's y and z passes (FP32 lines) at NGRID >= 256 in a
// persistent form: each block walks a strided list of pencils (TX kx columns x
// N elements of one line set) with two pencil buffers in shared memory.  One
// thread stages the next pencil with tensor copies (cp.async.bulk.tensor.3d,
// boxes of 16 floats x 256 elements, completion counted on an mbarrier) while
// the block transforms the current one, so the strided global reads overlap
// the butterflies instead of preceding them.  The tensor map covers only this
// context's own spectrum (no multicast).  The arithmetic and the stores are
// those of k_fft_lines.  A wait that does not end within its bound sets bit 2
// of the context's flag word and ends the block (reported by the next call
// that reads the flags).
constexpr int kTmaBoxE = 256;   // box extent along the line (the tensor-copy limit)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

// Pencil widths of the staged passes, picked per size, pass and device by
// timing (fft_tune): TX kx columns of 8 bytes, so 64 or 32 bytes per row of a
// box (a multiple of 16 bytes either way).  The thread count gives every
// radix-16 butterfly of a stage its own thread (at least 128, at most 512).
template <int N, int TX>
struct TShape {
    static constexpr int NT = TX == LShape<N>::TX ? LShape<N>::NT
                                                  : (TX * N / 16 < 128 ? 128 : (TX * N / 16 > 512 ? 512 : TX * N / 16));
};
constexpr int kTileTX[2] = {8, 4};   // candidate pencil widths (index 0: the default)

template <int N, int TX>
constexpr size_t tma_lines_smem(bool power) {
    return 2 * (size_t)TX * N * sizeof(float2) + 16 + (power ? 3 * (size_t)(N + 1) * 8 : 0);
}

template <int MODE, int N, int TX>
__global__ void __launch_bounds__(TShape<N, TX>::NT, N >= 1024 && TX == 8 ? 1 : 2) k_fft_lines_tma(
    const __grid_constant__ CUtensorMap tmap, float2* __restrict__ buf, int axis, int64_t estride, int64_t ostride,
    const float2* __restrict__ tw, LineExtra ex, int32_t* __restrict__ flags) {
    constexpr int NT = TShape<N, TX>::NT, LGTX = ilog2c(TX);
    constexpr int nxh = N / 2 + 1, NXG = (nxh + TX - 1) / TX;
    constexpr int BE = N < kTmaBoxE ? N : kTmaBoxE, NCH = N / BE;
    constexpr uint32_t PBYTES = TX * N * (uint32_t)sizeof(float2);
    static_assert(TX * 2 * sizeof(float) % 16 == 0, "the box's inner extent must be a multiple of 16 bytes");
    extern __shared__ __align__(128) unsigned char sm_tma[];
    float2* pb0 = reinterpret_cast<float2*>(sm_tma);
    float2* pb1 = pb0 + TX * N;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm_tma + 2 * PBYTES);
    unsigned long long* hl = reinterpret_cast<unsigned long long*>(sm_tma + 2 * PBYTES + 16);
    const int tid = threadIdx.x;
    const int npencils = NXG * N;
    const int nh = ex.quad ? 3 * (N + 1) : 2 * (N + 1);
    auto issue = [&](int p, int b) {   // one thread: stage pencil p into buffer b
        const int xg = p % NXG, o = p / NXG;
        float2* dst = b ? pb1 : pb0;
        mbar_expect_tx(bar + b, PBYTES);
#pragma unroll
        for (int c = 0; c < NCH; ++c) {
            // x coordinate in floats: 2 TX xg, a multiple of 16 floats (64 bytes)
            if (axis == 1) tma_load_3d(dst + c * BE * TX, &tmap, bar + b, 2 * TX * xg, c * BE, o);
            else tma_load_3d(dst + c * BE * TX, &tmap, bar + b, 2 * TX * xg, o, c * BE);
        }
    };
    if (smem_u32(pb0) & 127) {   // tensor copies need 128-byte aligned destinations
        if (tid == 0) atomicOr(flags, 4);
        return;
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(bar + 1, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (MODE == LM_POWER)
        for (int e = tid; e < nh; e += NT) hl[e] = 0ull;
    __syncthreads();
    int p = blockIdx.x;
    if (tid == 0 && p < npencils) issue(p, 0);
    for (int i = 0; p < npencils; ++i, p += gridDim.x) {
        const int b = i & 1;
        float2* sm = b ? pb1 : pb0;
        const int pn = p + gridDim.x;
        if (tid == 0 && pn < npencils) {
            // the other buffer's reads (the previous pencil) ended at the last barrier
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            issue(pn, b ^ 1);
        }
        // wait for this pencil, for at most two seconds of the GPU's global timer
        bool ok = mbar_try_wait(bar + b, (uint32_t)((i >> 1) & 1));
        if (!ok) {
            const uint64_t t0 = global_ns();
            while (!(ok = mbar_try_wait(bar + b, (uint32_t)((i >> 1) & 1))) && global_ns() - t0 < 2000000000ull) {
            }
        }
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicOr(flags, 4);
            return;
        }
        const int xg = p % NXG, o = p / NXG, x0 = xg * TX;
        const int nvalid = min(TX, nxh - x0);
        lines_compute<MODE, N, float2, TX, NT>(sm, x0, o, nvalid, tw, ex, hl);
        if (MODE != LM_POWER) {
            const int64_t base = (int64_t)o * ostride + x0;
#pragma unroll 4
            for (int e = tid; e < TX * N; e += NT) {
                const int x = e & (TX - 1), el = e >> LGTX;
                if (x < nvalid) buf[base + (int64_t)el * estride + x] = sm[e];
            }
        }
        __syncthreads();
    }
    if (MODE == LM_POWER) {
        __syncthreads();
        for (int e = tid; e < nh; e += NT)
            if (hl[e]) atomicAdd(ex.hist + e, hl[e]);
    }
}

#define MGG_FFT_SIZES(F) F(16) F(32) F(64) F(128) F(256) F(512) F(1024)

template <int N>
void set_attrs_n() {
    const int big = 200 * 1024;
    if constexpr (N >= 256) {
#define MGG_TMA_ATTR(M, T) \
        MGG_CUDA(cudaFuncSetAttribute(k_fft_lines_tma<M, N, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, big))
        MGG_TMA_ATTR(LM_FWD, 8); MGG_TMA_ATTR(LM_INV, 8); MGG_TMA_ATTR(LM_GREEN, 8); MGG_TMA_ATTR(LM_POWER, 8);
        MGG_TMA_ATTR(LM_FWD, 4); MGG_TMA_ATTR(LM_INV, 4); MGG_TMA_ATTR(LM_GREEN, 4); MGG_TMA_ATTR(LM_POWER, 4);
#undef MGG_TMA_ATTR
    }
    MGG_CUDA(cudaFuncSetAttribute(k_fft_x_r2c<N, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_x_c2r<N, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_FWD, N, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_INV, N, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_GREEN, N, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_POWER, N, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_DISP, N, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_x_r2c<N, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_x_c2r<N, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_FWD, N, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_INV, N, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_GREEN, N, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
    MGG_CUDA(cudaFuncSetAttribute(k_fft_lines<LM_POWER, N, double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
}

template <int N>
void x_r2c_n(const FftPlan& p, const float* in, float2* out, cudaStream_t s) {
    using X = XShape<N>;
    if (p.tw64) {
        const size_t smem = (size_t)X::TB * X::LS * sizeof(double2);
        k_fft_x_r2c<N, double2><<<div_up((int64_t)N * N, X::TB), X::NT, smem, s>>>(in, out, p.nxp, p.tw64);
    } else {
        const size_t smem = (size_t)X::TB * X::LS * sizeof(float2);
        k_fft_x_r2c<N, float2><<<div_up((int64_t)N * N, X::TB), X::NT, smem, s>>>(in, out, p.nxp, p.tw);
    }
    MGG_CHECK_LAUNCH();
}

template <int N>
void x_c2r_n(const FftPlan& p, const float2* in, float* out, cudaStream_t s) {
    using X = XShape<N>;
    if (p.tw64) {
        const size_t smem = (size_t)X::TB * X::LS * sizeof(double2);
        k_fft_x_c2r<N, double2><<<div_up((int64_t)N * N, X::TB), X::NT, smem, s>>>(in, out, p.nxp, p.tw64);
    } else {
        const size_t smem = (size_t)X::TB * X::LS * sizeof(float2);
        k_fft_x_c2r<N, float2><<<div_up((int64_t)N * N, X::TB), X::NT, smem, s>>>(in, out, p.nxp, p.tw);
    }
    MGG_CHECK_LAUNCH();
}

// the persistent TMA-staged pass: as many blocks as fit on the device at once
template <int MODE, int N, int TX>
void lines_tma_launch(const FftPlan& p, float2* buf, int axis, int64_t estride, int64_t ostride, const LineExtra& ex,
                      cudaStream_t s) {
    constexpr int NT = TShape<N, TX>::NT;
    const size_t smem = tma_lines_smem<N, TX>(MODE == LM_POWER);
    static const int resident = [&] {   // blocks resident on the whole device
        int dev = 0, sms = 0, per_sm = 0;
        MGG_CUDA(cudaGetDevice(&dev));
        MGG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        MGG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fft_lines_tma<MODE, N, TX>, NT, smem));
        if (per_sm < 1) throw Error{MGG_ERR_CUDA, "fft: the staged line pass does not fit on an SM"};
        return per_sm * sms;
    }();
    constexpr int nxh = N / 2 + 1, NXG = (nxh + TX - 1) / TX;
    const int grid = (int)std::min<int64_t>((int64_t)NXG * N, (int64_t)resident);
    const int ti = TX == kTileTX[0] ? 0 : 1;
    const CUtensorMap* map = reinterpret_cast<const CUtensorMap*>(p.tmap[ti][axis - 1]);
    k_fft_lines_tma<MODE, N, TX><<<grid, NT, smem, s>>>(*map, buf, axis, estride, ostride, p.tw, ex, p.flags);
    MGG_CHECK_LAUNCH();
}

template <int MODE, int N>
void lines_tma_tx(const FftPlan& p, float2* buf, int axis, int64_t estride, int64_t ostride, const LineExtra& ex,
                  cudaStream_t s) {
    if (p.tile_tx[MODE] == kTileTX[1]) lines_tma_launch<MODE, N, kTileTX[1]>(p, buf, axis, estride, ostride, ex, s);
    else lines_tma_launch<MODE, N, kTileTX[0]>(p, buf, axis, estride, ostride, ex, s);
}

template <int N>
void lines_n(const FftPlan& p, float2* buf, int axis, int mode, const LineExtra& ex, cudaStream_t s) {
    constexpr int TX = LShape<N>::TX, NT = LShape<N>::NT;
    constexpr int nxh = N / 2 + 1;
    dim3 grid(div_up(nxh, TX), N);
    int64_t estride, ostride;
    if (axis == 1) { estride = p.nxp; ostride = (int64_t)N * p.nxp; }       // o = z
    else { estride = (int64_t)N * p.nxp; ostride = p.nxp; }                  // o = y
    if constexpr (N >= 256) {
        if (p.tmap[0][0] && !p.tw64 && mode != LM_DISP) {   // TMA-staged pencils (the context's own spectrum)
            switch (mode) {
            case LM_FWD: lines_tma_tx<LM_FWD, N>(p, buf, axis, estride, ostride, ex, s); return;
            case LM_INV: lines_tma_tx<LM_INV, N>(p, buf, axis, estride, ostride, ex, s); return;
            case LM_GREEN: lines_tma_tx<LM_GREEN, N>(p, buf, axis, estride, ostride, ex, s); return;
            case LM_POWER: lines_tma_tx<LM_POWER, N>(p, buf, axis, estride, ostride, ex, s); return;
            default: break;
            }
        }
    }
    if (p.tw64) {   // FP64 line arithmetic
        size_t smem = (size_t)TX * N * sizeof(double2);
        const double2* tw = p.tw64;
        switch (mode) {
        case LM_FWD: k_fft_lines<LM_FWD, N, double2><<<grid, NT, smem, s>>>(buf, estride, ostride, tw, ex); break;
        case LM_INV: k_fft_lines<LM_INV, N, double2><<<grid, NT, smem, s>>>(buf, estride, ostride, tw, ex); break;
        case LM_GREEN: k_fft_lines<LM_GREEN, N, double2><<<grid, NT, smem, s>>>(buf, estride, ostride, tw, ex); break;
        case LM_POWER:
            smem += 3 * (size_t)(N + 1) * sizeof(unsigned long long);
            k_fft_lines<LM_POWER, N, double2><<<grid, NT, smem, s>>>(buf, estride, ostride, tw, ex);
            break;
        default: throw Error{MGG_ERR_ARG, "fft_lines: no FP64 form of this mode"};
        }
        MGG_CHECK_LAUNCH();
        return;
    }
    size_t smem = (size_t)TX * N * sizeof(float2);
    switch (mode) {
    case LM_FWD: k_fft_lines<LM_FWD, N, float2><<<grid, NT, smem, s>>>(buf, estride, ostride, p.tw, ex); break;
    case LM_INV: k_fft_lines<LM_INV, N, float2><<<grid, NT, smem, s>>>(buf, estride, ostride, p.tw, ex); break;
    case LM_GREEN: k_fft_lines<LM_GREEN, N, float2><<<grid, NT, smem, s>>>(buf, estride, ostride, p.tw, ex); break;
    case LM_POWER:
        smem += 3 * (size_t)(N + 1) * sizeof(unsigned long long);
        k_fft_lines<LM_POWER, N, float2><<<grid, NT, smem, s>>>(buf, estride, ostride, p.tw, ex);
        break;
    case LM_DISP: k_fft_lines<LM_DISP, N, float2><<<grid, NT, smem, s>>>(buf, estride, ostride, p.tw, ex); break;
    default: throw Error{MGG_ERR_ARG, "fft_lines: bad mode"};
    }
    MGG_CHECK_LAUNCH();
}

}  // namespace

void fft_set_attributes() {
#define MGG_F(N) set_attrs_n<N>();
    MGG_FFT_SIZES(MGG_F)
#undef MGG_F
}

#define MGG_FFT_SWITCH(n, CALL)                                              \
    switch (n) {                                                             \
    case 16: CALL(16); break;                                                \
    case 32: CALL(32); break;                                                \
    case 64: CALL(64); break;                                                \
    case 128: CALL(128); break;                                              \
    case 256: CALL(256); break;                                              \
    case 512: CALL(512); break;                                              \
    case 1024: CALL(1024); break;                                            \
    default: throw Error{MGG_ERR_ARG, "fft: NGRID must be a power of two in [16, 1024]"}; \
    }

void fft_x_r2c(const FftPlan& p, const float* in, float2* out, cudaStream_t s) {
#define MGG_C(N) x_r2c_n<N>(p, in, out, s)
    MGG_FFT_SWITCH(p.n, MGG_C)
#undef MGG_C
}

void fft_x_c2r(const FftPlan& p, const float2* in, float* out, cudaStream_t s) {
#define MGG_C(N) x_c2r_n<N>(p, in, out, s)
    MGG_FFT_SWITCH(p.n, MGG_C)
#undef MGG_C
}

void fft_lines(const FftPlan& p, float2* buf, int axis, int mode, const LineExtra& ex, cudaStream_t s) {
#define MGG_C(N) lines_n<N>(p, buf, axis, mode, ex, s)
    MGG_FFT_SWITCH(p.n, MGG_C)
#undef MGG_C
}

// ------------------------------------------------------------- context ----
int fft_pitch(int N) { return ((N / 2 + 1) + 15) / 16 * 16; }

float2* make_twiddles(int N) {
    std::vector<float2> tw(N);
    for (int k = 0; k < N; ++k) {
        const double a = -2.0 * M_PI * (double)k / (double)N;
        tw[k] = make_float2((float)cos(a), (float)sin(a));
    }
    float2* d = nullptr;
    MGG_CUDA(cudaMalloc(&d, sizeof(float2) * N));
    MGG_CUDA(cudaMemcpy(d, tw.data(), sizeof(float2) * N, cudaMemcpyHostToDevice));
    return d;
}

double2* make_twiddles64(int N) {
    std::vector<double2> tw(N);
    for (int k = 0; k < N; ++k) {
        const double a = -2.0 * M_PI * (double)k / (double)N;
        tw[k] = make_double2(cos(a), sin(a));
    }
    double2* d = nullptr;
    MGG_CUDA(cudaMalloc(&d, sizeof(double2) * N));
    MGG_CUDA(cudaMemcpy(d, tw.data(), sizeof(double2) * N, cudaMemcpyHostToDevice));
    return d;
}

// log-bin table per integer |k|^2 with the reference's Real*4 arithmetic
// (MPlog = max(1, min(NPOWER, INT(Log10(RK)/dLog + 1000.) - 1000)), PMP2mod_power.f90:396)
uint8_t* make_logbins(int N) {
    const int m2max = 3 * (N / 2) * (N / 2);
    std::vector<uint8_t> lb(m2max + 1, 0);
    for (int m2 = 1; m2 <= m2max; ++m2) {
        const float RK = sqrtf((float)m2);
        int ml = (int)(log10f(RK) / 0.02f + 1000.0f) - 1000;
        ml = ml < 1 ? 1 : (ml > N ? N : ml);
        if (ml > 255) ml = 255;
        lb[m2] = (uint8_t)ml;
    }
    uint8_t* d = nullptr;
    MGG_CUDA(cudaMalloc(&d, m2max + 1));
    MGG_CUDA(cudaMemcpy(d, lb.data(), m2max + 1, cudaMemcpyHostToDevice));
    return d;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library); null when the driver does not provide it
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
    static const EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (EncodeTiledFn) nullptr;
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

// Tensor map of the half spectrum [kz][ky][kx] (float2, row pitch nxp) as FP32
// {2 nxp, N, N}, with boxes of one pencil chunk: 2 tx floats (tx kx columns,
// 8 tx bytes) x 256 elements along y (axis 1) or z (axis 2).
static bool make_line_map(void* out, float2* cbuf, int N, int nxp, int axis, int tx) {
    const EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)2 * nxp, (cuuint64_t)N, (cuuint64_t)N};
    const cuuint64_t strides[2] = {(cuuint64_t)2 * nxp * sizeof(float), (cuuint64_t)2 * nxp * N * sizeof(float)};
    const cuuint32_t be = (cuuint32_t)(N < kTmaBoxE ? N : kTmaBoxE);
    const cuuint32_t box[3] = {(cuuint32_t)(2 * tx), axis == 1 ? be : 1u, axis == 1 ? 1u : be};
    const cuuint32_t estr[3] = {1u, 1u, 1u};
    return enc(reinterpret_cast<CUtensorMap*>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, cbuf, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

void fft_alloc(Ctx& c) {
    const int N = c.N;
    c.nxp = fft_pitch(N);
    MGG_CUDA(cudaMalloc(&c.cbuf, sizeof(float2) * (size_t)c.nxp * N * N));
    static_assert(sizeof(CUtensorMap) == sizeof(c.tmap[0][0]), "tensor map storage");
    // MGG_FFT_DIRECT=1 in the environment keeps the direct pencil loads (tests compare the two)
    c.tmaps = N >= 256 && !std::getenv("MGG_FFT_DIRECT");
    for (int t = 0; t < 2 && c.tmaps; ++t)
        for (int a = 0; a < 2 && c.tmaps; ++a) c.tmaps = make_line_map(c.tmap[t][a], c.cbuf, N, c.nxp, a + 1, kTileTX[t]);
    c.tw_n = make_twiddles(N);
    c.tw64_n = make_twiddles64(N);
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
    c.pk_logbin = make_logbins(N);
    MGG_CUDA(cudaMalloc(&c.pk_hist, sizeof(unsigned long long) * 3 * (N + 1)));
    fft_set_attributes();
}

namespace {

// the staged pencils' tensor maps and flag word of a context
void staged_plan(Ctx& c, FftPlan& p) {
    for (int t = 0; t < 2; ++t)
        for (int a = 0; a < 2; ++a) p.tmap[t][a] = c.tmap[t][a];
    p.flags = c.d_flags;
}

LineExtra ex_tune_green(Ctx& c) {
    LineExtra ex;
    ex.green = c.green;
    ex.green_scale = 1.0;
    return ex;
}

std::mutex g_fft_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_fft_tile;   // (device, N, mode, axis) -> pencil width

// Pencil widths of the staged passes: picked per device, size, pass and axis by
// timing both widths the first time the pass runs outside a CUDA-graph
// capture, on the spectrum buffer before the transform fills it (its contents
// do not change the timing), and cached for the process.  The narrower width
// replaces the default only when at least 3 % faster.  The width changes no
// result: every line gets the same butterflies.  MGG_FFT_TX=4 or 8 in the
// environment forces one (tests compare the two).
void fft_tune(Ctx& c, FftPlan& p, const LineExtra& ex, std::initializer_list<std::pair<int, int>> passes) {
    static const int forced = [] {
        const char* e = std::getenv("MGG_FFT_TX");
        return e ? std::atoi(e) : 0;
    }();
    const int N = p.n;
    for (const auto& pa : passes) {
        const int mode = pa.first, axis = pa.second;
        if (forced == kTileTX[0] || forced == kTileTX[1]) {
            p.tile_tx[mode] = forced;
            continue;
        }
        const auto key = std::make_tuple(c.dev, N, mode, axis);
        std::lock_guard<std::mutex> lk(g_fft_tune_mu);
        auto it = g_fft_tile.find(key);
        if (it != g_fft_tile.end()) {
            p.tile_tx[mode] = it->second;
            continue;
        }
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        MGG_CUDA(cudaStreamIsCapturing(c.stream, &cs));
        if (cs != cudaStreamCaptureStatusNone) {
            p.tile_tx[mode] = kTileTX[0];
            continue;
        }
        cudaEvent_t ea, eb;
        MGG_CUDA(cudaEventCreate(&ea));
        MGG_CUDA(cudaEventCreate(&eb));
        float best_ms = 0.f;
        int best = kTileTX[0];
        for (int t = 0; t < 2; ++t) {
            p.tile_tx[mode] = kTileTX[t];
            fft_lines(p, c.cbuf, axis, mode, ex, c.stream);   // warm-up
            MGG_CUDA(cudaEventRecord(ea, c.stream));
            fft_lines(p, c.cbuf, axis, mode, ex, c.stream);
            fft_lines(p, c.cbuf, axis, mode, ex, c.stream);
            MGG_CUDA(cudaEventRecord(eb, c.stream));
            MGG_CUDA(cudaEventSynchronize(eb));
            float ms = 0.f;
            MGG_CUDA(cudaEventElapsedTime(&ms, ea, eb));
            if (t == 0 || ms < 0.97f * best_ms) {
                best_ms = ms;
                best = kTileTX[t];
            }
        }
        cudaEventDestroy(ea);
        cudaEventDestroy(eb);
        g_fft_tile[key] = best;
        p.tile_tx[mode] = best;
    }
}

}  // namespace

void poisson_solve(Ctx& c) {
    BucketScope bs(c, MGG_T_FORCE);
    const int N = c.N;
    FftPlan p;
    p.n = N;
    p.nxp = c.nxp;
    p.tw = c.tw_n;
    if (c.cfg.precision == MGG_PREC_PLAIN) p.tw64 = c.tw64_n;   // FP64 lines, as FFTPACK5
    else if (c.tmaps) staged_plan(c, p);                         // FP32 lines, TMA-staged pencils
    const double cells = (double)c.ncell;
    const double cplx = 8.0 * (double)N * N * (N / 2 + 1);
    if (p.tmap[0][0]) fft_tune(c, p, ex_tune_green(c), {{LM_FWD, 1}, {LM_GREEN, 2}, {LM_INV, 1}});
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

void power_bins(Ctx& c, const float* grid, int N, const float2* tw, const double2* tw64, const uint8_t* logbin,
                bool quad, PkBins& out) {
    const double cells = (double)N * N * N;
    // Parseval bound for the fixed-point scale: sum_k |delta_k|^2 = sum delta^2 / N^3
    const int blocks = 148 * 8;
    ensure_partials(c, blocks);
    {
        ProfScope ps(c, K_GRID_OP, 4.0 * cells);
        k_sumsq<<<blocks, 256, 0, c.stream>>>(grid, (int64_t)cells, c.red_partial);
        MGG_CHECK_LAUNCH();
    }
    const double s2 = reduce_sum_blocks(c, blocks);
    const double total = s2 / cells;   // >= any bin sum (and any |quadrupole bin sum|)
    double scale = 1.0;
    if (total > 0.0) {
        int e;
        frexp(total, &e);                    // total < 2^e
        scale = ldexp(1.0, 61 - e);          // sums stay below 2^61
    }
    FftPlan p;
    p.n = N;
    p.nxp = fft_pitch(N);
    p.tw = tw;
    p.tw64 = tw64;
    if (!tw64 && N == c.N && c.tmaps) staged_plan(c, p);   // the context's own mesh: TMA-staged pencils
    LineExtra ex;
    ex.logbin = logbin;
    ex.hist = c.pk_hist;
    ex.amp_scale = scale / (cells * cells);
    ex.quad = quad ? 1 : 0;
    const int nh = 3 * (N + 1);
    if (p.tmap[0][0]) fft_tune(c, p, ex, {{LM_FWD, 1}, {LM_POWER, 2}});   // before the histograms are cleared
    MGG_CUDA(cudaMemsetAsync(c.pk_hist, 0, sizeof(unsigned long long) * nh, c.stream));
    const double cplx = 8.0 * (double)N * N * (N / 2 + 1);
    {
        ProfScope ps(c, K_FFT_X_R2C, 4.0 * cells + cplx);
        fft_x_r2c(p, grid, c.cbuf, c.stream);
    }
    {
        ProfScope ps(c, K_FFT_Y, 2.0 * cplx);
        fft_lines(p, c.cbuf, 1, LM_FWD, ex, c.stream);
    }
    {
        ProfScope ps(c, K_FFT_Z_POWER, cplx);
        fft_lines(p, c.cbuf, 2, LM_POWER, ex, c.stream);
    }
    std::vector<unsigned long long> h(nh);
    MGG_CUDA(cudaMemcpyAsync(h.data(), c.pk_hist, sizeof(unsigned long long) * nh, cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaStreamSynchronize(c.stream));
    // mode counts and <k> per bin (exact, data independent)
    static thread_local std::map<int, std::vector<double>> counts;
    std::vector<double>& cnt = counts[N];
    if (cnt.empty()) mode_counts(N, cnt);
    std::vector<double> iV(N + 1, 0.0), dk(N + 1, 0.0), iVl(N + 1, 0.0), dkl(N + 1, 0.0);
    std::vector<uint8_t> lb(cnt.size());
    MGG_CUDA(cudaMemcpy(lb.data(), logbin, cnt.size(), cudaMemcpyDeviceToHost));
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
    const int nb = N / 2;
    for (auto* v : {&out.k, &out.n, &out.p, &out.kl, &out.nl, &out.pl, &out.q}) v->assign(nb + 1, 0.0);
    for (int I = 1; I <= nb; ++I) {
        if (iV[I] > 0) {
            out.k[I] = (float)(dk[I] / iV[I] * (double)Scale);
            out.n[I] = (float)iV[I];
            out.p[I] = (float)((double)b3 * ((double)h[I] * unfix) / iV[I]);
            // iPol = 1: DPOWER = 2.5 DPOWER ((2L+1)/2, PMP2mod_power.f90:420)
            if (quad) out.q[I] = (float)((double)b3 * (2.5 * ((double)(int64_t)h[2 * (N + 1) + I] * unfix)) / iV[I]);
        }
        if (iVl[I] > 0) {
            out.kl[I] = (float)(dkl[I] / iVl[I] * (double)Scale);
            out.nl[I] = (float)iVl[I];
            out.pl[I] = (float)((double)b3 * ((double)h[(N + 1) + I] * unfix) / iVl[I]);
        }
    }
}

void power_spectrum(Ctx& c, int nbins, double* k_out, double* n_out, double* p_out, double* kl_out,
                    double* nl_out, double* pl_out) {
    BucketScope bs(c, MGG_T_POWER);
    PkBins b;
    power_bins(c, c.fi, c.N, c.tw_n, c.cfg.precision == MGG_PREC_PLAIN ? c.tw64_n : nullptr, c.pk_logbin, false, b);
    for (int I = 1; I <= nbins && I <= c.N / 2; ++I) {
        if (k_out) k_out[I - 1] = b.k[I];
        if (n_out) n_out[I - 1] = b.n[I];
        if (p_out) p_out[I - 1] = b.p[I];
        if (kl_out) kl_out[I - 1] = b.kl[I];
        if (nl_out) nl_out[I - 1] = b.nl[I];
        if (pl_out) pl_out[I - 1] = b.pl[I];
    }
}

}  // namespace mgg
