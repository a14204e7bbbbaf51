// ORACLE -- TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement, in C++17 + OpenMP, of the reference MG-GLAM particle-mesh
// step (chzruan/MG-GLAM-Durham, Fortran 90).  Only the tests, the smoke check
// and the CPU-baseline leg of the benchmark load it, and only as the checker or
// the timed CPU baseline.  The product library never links or calls it.
//
// Parity status: UNPINNED by reference fixtures.  The reference ships no
// golden vectors, no unit tests and no fixtures, and it cannot be built in this
// container (Fortran only, no Fortran compiler).  This restatement is pinned
// instead by analytic known-answer tests (single-mode Poisson solve against the
// 7-point eigenvalue, FFT round trips against the halfcomplex definition, mass
// conservation of CIC, the reference's own MG convergence criterion, the f(R)
// background solution) in tests/test_oracle_*.py.
//
// Precision follows the reference: grids are stored in the storage type S
// (float = the reference's Real*4 FI/FI2/FI3, double = the FP64 oracle); every
// expression is evaluated in the kind the Fortran source gives it, including the
// Real*4 products and sums of grid values inside the multigrid stencils and the
// Real*4 cosmological scalars (AEXPN, ASTEP, Om, OmL are Real*4 in Module Tools).
// Red-black sweeps run in the serial lexicographic order of one OpenMP thread.

#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#include <complex>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/mgglam.h"

namespace {

typedef std::complex<double> cd;

// ---------------------------------------------------------------------------
// 1-D real transforms with FFTPACK5's halfcomplex convention
// (PMP2mod_fft5.f90:8-326, rfftf1 scaling 1937-1972):
//   forward  r(1)    = (1/n)  sum x_j
//            r(2m)   = (2/n)  sum x_j cos(2 pi m j / n)
//            r(2m+1) = (2/n)  sum x_j sin(2 pi m j / n)      m = 1..n/2-1
//            r(n)    = (1/n)  sum (-1)^j x_j                 (n even)
//   backward is the exact inverse (Fourier synthesis).
// Computed here with an iterative radix-2 complex FFT in double; FFTPACK's own
// radix-4/2 factorisation differs only in the last bits of the FP64 result.
// ---------------------------------------------------------------------------
struct CFFT {
    int n = 0;
    std::vector<cd> w;      // exp(-2 pi i k / n)
    std::vector<int> rev;
    void init(int n_) {
        if (n == n_) return;
        n = n_;
        w.resize(n / 2 > 0 ? n / 2 : 1);
        for (int k = 0; k < n / 2; ++k) {
            double a = -2.0 * M_PI * (double)k / (double)n;
            w[k] = cd(std::cos(a), std::sin(a));
        }
        rev.resize(n);
        int lg = 0;
        while ((1 << lg) < n) ++lg;
        for (int i = 0; i < n; ++i) {
            int r = 0;
            for (int b = 0; b < lg; ++b) if (i & (1 << b)) r |= 1 << (lg - 1 - b);
            rev[i] = r;
        }
    }
    // in-place forward DFT (sign -1); inverse = conj trick
    void forward(cd* a) const {
        for (int i = 0; i < n; ++i) if (i < rev[i]) std::swap(a[i], a[rev[i]]);
        for (int len = 2; len <= n; len <<= 1) {
            int step = n / len;
            for (int i = 0; i < n; i += len)
                for (int j = 0; j < len / 2; ++j) {
                    cd u = a[i + j], v = a[i + j + len / 2] * w[j * step];
                    a[i + j] = u + v;
                    a[i + j + len / 2] = u - v;
                }
        }
    }
};

thread_local CFFT t_fft;
thread_local std::vector<cd> t_buf;

// rfft1f: r[0..n-1] (0-based storage of the 1-based halfcomplex vector)
void rfft1f(double* r, int n) {
    t_fft.init(n);
    t_buf.resize(n);
    for (int j = 0; j < n; ++j) t_buf[j] = cd(r[j], 0.0);
    t_fft.forward(t_buf.data());
    // scale constants are computed in single precision by rfftf1 (1937-1938)
    const double sn = (double)(1.0f / (float)n);
    const double tsn = (double)(2.0f / (float)n);
    r[0] = sn * t_buf[0].real();
    for (int m = 1; m < n / 2; ++m) {
        r[2 * m - 1] = tsn * t_buf[m].real();   // r(2m)
        r[2 * m] = -tsn * t_buf[m].imag();      // r(2m+1)
    }
    r[n - 1] = sn * t_buf[n / 2].real();
}

// rfft1b: exact inverse of rfft1f
void rfft1b(double* r, int n) {
    t_fft.init(n);
    t_buf.resize(n);
    // x_j = r1 + sum_m [r(2m) cos + r(2m+1) sin] + r(n) (-1)^j
    //     = Re sum_k G_k e^{+2 pi i k j/n}  with G_0 = r1, G_m = r(2m) - i r(2m+1), G_{n/2} = r(n)
    // computed as conj(DFT(conj(G))) on the full Hermitian spectrum / appropriate weights.
    t_buf[0] = cd(r[0], 0.0);
    for (int m = 1; m < n / 2; ++m) {
        cd g(0.5 * r[2 * m - 1], -0.5 * r[2 * m]);
        t_buf[m] = g;
        t_buf[n - m] = std::conj(g);
    }
    t_buf[n / 2] = cd(r[n - 1], 0.0);
    for (int k = 0; k < n; ++k) t_buf[k] = std::conj(t_buf[k]);
    t_fft.forward(t_buf.data());
    for (int j = 0; j < n; ++j) r[j] = t_buf[j].real();   // real part of conj == real part
}

inline int64_t gidx(int i, int j, int k, int n) {   // 0-based
    return (int64_t)i + (int64_t)n * ((int64_t)j + (int64_t)n * (int64_t)k);
}

inline int wrapu(int m, int n) { return m >= n ? m - n : m; }
inline int wrapl(int m, int n) { return m < 0 ? m + n : m; }

// Fortran DSIGN(a, b)
inline double dsign(double a, double b) { return b >= 0.0 ? std::fabs(a) : -std::fabs(a); }

// Fortran real*4 integer power x**3 evaluated in single precision
inline float fpow2(float x) { return x * x; }
inline float fpow3(float x) { return x * x * x; }

// ---------------------------------------------------------------------------
// DENSIT (PMP2mod_density.f90:17-301): FI := -1, then CIC.  Serial particle
// order: the reference's OMP ATOMIC scatter reduces to this order at T=1.
// ---------------------------------------------------------------------------
template <class S>
void density(const float* xp, const float* yp, const float* zp, int64_t np, int ng, S* fi,
             int threads) {
    const int64_t ncell = (int64_t)ng * ng * ng;
    const double YN = (double)ng;
    const float Wpar = (float)(YN * YN * YN / (double)(float)np);   // Real*4 WPAR (41)
    for (int64_t c = 0; c < ncell; ++c) fi[c] = (S)-1.0f;          // (47-55)
    auto add = [&](int64_t c, double w) {
        if (threads > 1) {
#pragma omp atomic
            fi[c] += (S)w;          // reference-style unordered scatter (timing mode)
        } else {
            fi[c] = (S)((double)fi[c] + w);
        }
    };
#pragma omp parallel for num_threads(threads > 1 ? threads : 1) schedule(static) if (threads > 1)
    for (int64_t p = 0; p < np; ++p) {
        double X = xp[p], Y = yp[p], Z = zp[p];
        int I = (int)X, J = (int)Y, K = (int)Z;               // 1-based cell
        double D1 = X - (double)(float)I, D2 = Y - (double)(float)J, D3 = Z - (double)(float)K;
        double T1 = 1.0 - D1, T2 = 1.0 - D2, T3 = 1.0 - D3;
        double T2W = T2 * (double)Wpar, D2W = D2 * (double)Wpar;
        int I1 = I + 1; if (I1 > ng) I1 = 1;
        int J1 = J + 1; if (J1 > ng) J1 = 1;
        int K1 = K + 1; if (K1 > ng) K1 = 1;
        // 0-based
        int i0 = I - 1, j0 = J - 1, k0 = K - 1, i1 = I1 - 1, j1 = J1 - 1, k1 = K1 - 1;
        add(gidx(i0, j0, k0, ng), T3 * T1 * T2W);
        add(gidx(i1, j0, k0, ng), T3 * D1 * T2W);
        add(gidx(i0, j1, k0, ng), T3 * T1 * D2W);
        add(gidx(i1, j1, k0, ng), T3 * D1 * D2W);
        add(gidx(i0, j0, k1, ng), D3 * T1 * T2W);
        add(gidx(i1, j0, k1, ng), D3 * D1 * T2W);
        add(gidx(i0, j1, k1, ng), D3 * T1 * D2W);
        add(gidx(i1, j1, k1, ng), D3 * D1 * D2W);
    }
}

// ---------------------------------------------------------------------------
// POTENTfft5 (PMP2main.f90:705-867).  The two x<->z transpositions are pure
// data movement, so the z lines are transformed in place instead.
// ---------------------------------------------------------------------------
template <class S>
void potential(S* fi, int ng, float aexpn, float om, float omb, int threads) {
    const int N = ng;
    float trfi;
    if (omb < 0.005f) trfi = 1.5f * (om - omb) / aexpn;   // (728-732)
    else trfi = 1.5f * om / aexpn;
    const double P16 = 6.28318530718;                       // (711)
    std::vector<double> G(N);
    G[0] = 2.0;
    G[N - 1] = -2.0;
    for (int i = 1; i <= N / 2 - 1; ++i) {                  // (736-742)
        double XX = 2.0 * std::cos(P16 * i / N);
        G[2 * i - 1] = XX;   // GREENf(2i)
        G[2 * i] = XX;       // GREENf(2i+1)
    }
    // x and y forward per z plane (749-772)
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int k = 0; k < N; ++k) {
        std::vector<double> r(N);
        for (int j = 0; j < N; ++j) {
            for (int i = 0; i < N; ++i) r[i] = (double)fi[gidx(i, j, k, N)];
            rfft1f(r.data(), N);
            for (int i = 0; i < N; ++i) fi[gidx(i, j, k, N)] = (S)r[i];
        }
        for (int i = 0; i < N; ++i) {
            for (int j = 0; j < N; ++j) r[j] = (double)fi[gidx(i, j, k, N)];
            rfft1f(r.data(), N);
            for (int j = 0; j < N; ++j) fi[gidx(i, j, k, N)] = (S)r[j];
        }
    }
    // z forward (789-801)
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int j = 0; j < N; ++j) {
        std::vector<double> r(N);
        for (int i = 0; i < N; ++i) {
            for (int k = 0; k < N; ++k) r[k] = (double)fi[gidx(i, j, k, N)];
            rfft1f(r.data(), N);
            for (int k = 0; k < N; ++k) fi[gidx(i, j, k, N)] = (S)r[k];
        }
    }
    // Green's function multiply + z backward (803-823)
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int j = 0; j < N; ++j) {
        std::vector<double> r(N);
        double A3 = G[j] - 6.0;
        for (int i = 0; i < N; ++i) {
            double A2 = G[i] + A3;
            for (int k = 0; k < N; ++k) {
                double A1 = A2 + G[k];
                if (std::fabs(A1) < 1.0e-7) A1 = 1.0;
                // FI*trfi is a Real*4 product, the division is in Real*8
                S prod = (S)((S)fi[gidx(i, j, k, N)] * (S)trfi);
                r[k] = (double)prod / A1;
            }
            rfft1b(r.data(), N);
            for (int k = 0; k < N; ++k) fi[gidx(i, j, k, N)] = (S)r[k];
        }
    }
    // x and y backward per z plane (841-862)
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int k = 0; k < N; ++k) {
        std::vector<double> r(N);
        for (int j = 0; j < N; ++j) {
            for (int i = 0; i < N; ++i) r[i] = (double)fi[gidx(i, j, k, N)];
            rfft1b(r.data(), N);
            for (int i = 0; i < N; ++i) fi[gidx(i, j, k, N)] = (S)r[i];
        }
        for (int i = 0; i < N; ++i) {
            for (int j = 0; j < N; ++j) r[j] = (double)fi[gidx(i, j, k, N)];
            rfft1b(r.data(), N);
            for (int j = 0; j < N; ++j) fi[gidx(i, j, k, N)] = (S)r[j];
        }
    }
}

// Background-table interpolation at a (PMP2main.f90:351-358 pattern):
// first row with a_row >= a, then linear interpolation of column col.
double bg_interp(const double* tab, int rows, double a, double aval, int col) {
    int ist = 0;
    while (ist < rows - 1 && tab[ist * 6 + 0] < a) ++ist;
    if (ist == 0) ist = 1;
    const double* r0 = tab + (ist - 1) * 6;
    const double* r1 = tab + ist * 6;
    return r0[col] + (r1[col] - r0[col]) / (r1[0] - r0[0]) * (aval - r0[0]);
}

// ---------------------------------------------------------------------------
// POTENT_FOR_MG (PMP2main.f90:869-1015)
// ---------------------------------------------------------------------------
template <class S>
void potential_mg(S* fi, const S* fi2, const mgg_config* c, float aexpn, int threads) {
    const int N = c->ngrid;
    const int64_t ncell = (int64_t)N * N * N;
    double fct1 = 0.0;
    int kind = 0;   // 0: fct1*FI2, 1: fct1*FI2^2, 2: fct1*FI2^3 ; sign folded in fct1
    switch (c->mg_model) {
    case 1: {
        double ctilde = 2.99792458e3 * (double)N / (double)c->box;
        double R_bg = 3.0 * ((double)(c->om / fpow3(aexpn)) + 4.0 * (double)c->oml);
        double R0_bg = 3.0 * ((double)c->om + 4.0 * (double)c->oml);
        double fR_bg = c->fr0 * std::pow(R0_bg / R_bg, c->fr_n + 1);
        fct1 = -(ctilde * ctilde * 0.5 * fR_bg);
        kind = c->fr_n;
        break;
    }
    case 2: fct1 = 0.5; kind = 0; break;
    case 3: {
        double ctilde = 2.99792458e3 * (double)N / (double)c->box;
        fct1 = 3.0 * c->sym_xi * c->sym_xi * (double)c->om * c->sym_beta * c->sym_beta * ctilde * ctilde /
               (c->sym_astar * c->sym_astar * c->sym_astar);
        kind = 1;
        break;
    }
    case 4: {
        double ctilde = 2.99792458e3 * (double)N / (double)c->box;
        fct1 = c->kmf_beta * ctilde;
        kind = 0;
        break;
    }
    case 5: fct1 = (c->csf_coupling == 1) ? c->csf_beta : 0.0; kind = 0; break;
    default: return;
    }
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int64_t q = 0; q < ncell; ++q) {
        S u = fi2[q];
        double sf;
        if (kind == 0) sf = fct1 * (double)u;
        else if (kind == 1) sf = fct1 * (double)(S)(u * u);      // FI2**2 in Real*4
        else sf = fct1 * (double)(S)(u * u * u);                  // FI2**3 in Real*4
        fi[q] = (S)((double)fi[q] + sf);
    }
}

// ---------------------------------------------------------------------------
// MOVE(FactV) (PMP2main.f90:304-685), models 1-3 (models 4/5 need the table).
// ---------------------------------------------------------------------------
template <class S>
double move(const S* fi, const S* fi2, float* xp, float* yp, float* zp, float* vxp, float* vyp,
            float* vzp, int64_t np, const mgg_config* c, float AEXPN, float ASTEP, float FactV,
            const double* bgtab, int bgrows, int threads) {
    const int N = c->ngrid;
    const float Om = c->om, OmL = c->oml;
    double PCONST = (double)(-std::sqrt(AEXPN / (Om + OmL * fpow3(AEXPN))) * ASTEP * 0.5f / FactV);
    float Ahalf = AEXPN + ASTEP / 2.0f;
    double XCONST = (double)(ASTEP / std::sqrt(Ahalf * (Om + OmL * fpow3(Ahalf))) / Ahalf);
    double bs_fct = 1.0;
    if (c->mg_model == 4) {
        const float r = 9.116748693e-5f;
        PCONST = (double)(-std::sqrt(AEXPN / (Om + r / AEXPN + (OmL - r) * fpow3(AEXPN))) * ASTEP * 0.5f / FactV);
        XCONST = (double)(ASTEP / std::sqrt(Ahalf * (Om + r / Ahalf + (OmL - r) * fpow3(Ahalf))) / Ahalf);
    }
    if (c->mg_flag == 1 && (c->mg_model == 4 || c->mg_model == 5) && bgtab) {
        double pc = bg_interp(bgtab, bgrows, AEXPN, AEXPN, 4);
        PCONST = 1.0 / pc;
        PCONST = -PCONST * ASTEP * 0.5 / FactV;
        double xc = bg_interp(bgtab, bgrows, Ahalf, Ahalf, 4);
        xc = (double)(Ahalf * Ahalf) * xc;
        XCONST = 1.0 / xc * ASTEP;
        // bs_fct interpolates column 2 with the Ahalf bracket but the AEXPN abscissa (380-383)
        bs_fct = bg_interp(bgtab, bgrows, Ahalf, AEXPN, 1);
        if (c->mg_model == 4) bs_fct = std::exp(c->kmf_beta * bs_fct);
        if (c->mg_model == 5 && c->csf_coupling == 1) bs_fct = std::exp(c->csf_beta * bs_fct);
    }
    double fric_fac = 0.0;
    bool sym_fric = false, bg_fric = false;
    if (c->mg_flag == 1) {
        if (c->mg_model == 3 && AEXPN > c->sym_astar) {
            double sa = c->sym_astar / (double)AEXPN;
            fric_fac = (double)(-9.0f * Om) * c->sym_beta * c->sym_beta * c->sym_xi * c->sym_xi *
                       std::sqrt(1.0 - sa * sa * sa);
            sym_fric = true;
        }
        if ((c->mg_model == 4 || c->mg_model == 5) && bgtab) {
            double pb = (c->mg_model == 4) ? c->kmf_beta : c->csf_beta;
            double f = bg_interp(bgtab, bgrows, AEXPN, AEXPN, 2);
            f = f / (double)AEXPN;
            fric_fac = -f * pb;
            bg_fric = true;
        }
    }
    const double XN = (double)((float)N + 1.0f - 1.0e-8f);
    const double YN = (double)(float)N;
    const float WPAR = (float)(YN * YN * YN / (double)(float)np);
    const double ast = (double)ASTEP, fv = (double)FactV;
    double SVEL = 0.0;
    int nth = threads > 0 ? threads : 1;
    std::vector<double> part(nth, 0.0);
#pragma omp parallel num_threads(nth)
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double sv = 0.0;
#pragma omp for schedule(static)
        for (int64_t IN = 0; IN < np; ++IN) {
            double X = xp[IN], Y = yp[IN], Z = zp[IN];
            double VVX = vxp[IN], VVY = vyp[IN], VVZ = vzp[IN];
            int I = (int)X, J = (int)Y, K = (int)Z;
            double D1 = X - (double)(float)I, D2 = Y - (double)(float)J, D3 = Z - (double)(float)K;
            double T1 = 1.0 - D1, T2 = 1.0 - D2, T3 = 1.0 - D3;
            double T2T1 = T2 * T1, T2D1 = T2 * D1, D2T1 = D2 * T1, D2D1 = D2 * D1;
            int I1 = I + 1; if (I1 > N) I1 = 1;
            int J1 = J + 1; if (J1 > N) J1 = 1;
            int K1 = K + 1; if (K1 > N) K1 = 1;
            int K2 = K + 2; if (K2 > N) K2 -= N;
            int K3 = K - 1; if (K3 < 1) K3 = N;
            int I2 = I + 2; if (I2 > N) I2 -= N;
            int J2 = J + 2; if (J2 > N) J2 -= N;
            int I0 = I - 1; if (I0 < 1) I0 = N;
            int J0 = J - 1; if (J0 < 1) J0 = N;
            auto F = [&](int a, int b, int cc) -> float { return (float)fi[gidx(a - 1, b - 1, cc - 1, N)]; };
            float F111 = F(I, J, K), F211 = F(I1, J, K), F121 = F(I, J1, K), F221 = F(I1, J1, K);
            float F112 = F(I, J, K1), F212 = F(I1, J, K1), F122 = F(I, J1, K1), F222 = F(I1, J1, K1);
            float F113 = F(I, J, K2), F213 = F(I1, J, K2), F123 = F(I, J1, K2), F223 = F(I1, J1, K2);
            float F110 = F(I, J, K3), F210 = F(I1, J, K3), F120 = F(I, J1, K3), F220 = F(I1, J1, K3);
            float F311 = F(I2, J, K), F321 = F(I2, J1, K), F131 = F(I, J2, K), F231 = F(I1, J2, K);
            float F312 = F(I2, J, K1), F322 = F(I2, J1, K1), F132 = F(I, J2, K1), F232 = F(I1, J2, K1);
            float F011 = F(I0, J, K), F021 = F(I0, J1, K), F101 = F(I, J0, K), F201 = F(I1, J0, K);
            float F012 = F(I0, J, K1), F022 = F(I0, J1, K1), F102 = F(I, J0, K1), F202 = F(I1, J0, K1);
            // Real*4 differences stored in Real*8 (566-594)
            double GX111 = F211 - F011, GX211 = F311 - F111, GX121 = F221 - F021, GX221 = F321 - F121;
            double GX112 = F212 - F012, GX212 = F312 - F112, GX122 = F222 - F022, GX222 = F322 - F122;
            double GY111 = F121 - F101, GY211 = F221 - F201, GY121 = F131 - F111, GY221 = F231 - F211;
            double GY112 = F122 - F102, GY212 = F222 - F202, GY122 = F132 - F112, GY222 = F232 - F212;
            double GZ111 = F112 - F110, GZ211 = F212 - F210, GZ121 = F122 - F120, GZ221 = F222 - F220;
            double GZ112 = F113 - F111, GZ212 = F213 - F211, GZ122 = F123 - F121, GZ222 = F223 - F221;
            double GX = PCONST * (T3 * (T2T1 * GX111 + T2D1 * GX211 + D2T1 * GX121 + D2D1 * GX221) +
                                  D3 * (T2T1 * GX112 + T2D1 * GX212 + D2T1 * GX122 + D2D1 * GX222));
            double GY = PCONST * (T3 * (T2T1 * GY111 + T2D1 * GY211 + D2T1 * GY121 + D2D1 * GY221) +
                                  D3 * (T2T1 * GY112 + T2D1 * GY212 + D2T1 * GY122 + D2D1 * GY222));
            double GZ = PCONST * (T3 * (T2T1 * GZ111 + T2D1 * GZ211 + D2T1 * GZ121 + D2D1 * GZ221) +
                                  D3 * (T2T1 * GZ112 + T2D1 * GZ212 + D2T1 * GZ122 + D2D1 * GZ222));
            if (c->mg_flag == 1) {
                if (sym_fric) {
                    double f2 = (double)fi2[gidx(I - 1, J - 1, K - 1, N)];
                    VVX = VVX + fric_fac * f2 * VVX * ast / fv;
                    VVY = VVY + fric_fac * f2 * VVY * ast / fv;
                    VVZ = VVZ + fric_fac * f2 * VVZ * ast / fv;
                }
                if (bg_fric) {
                    VVX = VVX + fric_fac * VVX * ast / fv;
                    VVY = VVY + fric_fac * VVY * ast / fv;
                    VVZ = VVZ + fric_fac * VVZ * ast / fv;
                    VVX = VVX + (bs_fct - 1.0) * GX;
                    VVY = VVY + (bs_fct - 1.0) * GY;
                    VVZ = VVZ + (bs_fct - 1.0) * GZ;
                }
            }
            VVX = VVX + GX;
            VVY = VVY + GY;
            VVZ = VVZ + GZ;
            X = X + VVX * XCONST;
            Y = Y + VVY * XCONST;
            Z = Z + VVZ * XCONST;
            if (X < 1.0) X = X + YN;
            if (X >= XN) X = X - YN;
            if (Y < 1.0) Y = Y + YN;
            if (Y >= XN) Y = Y - YN;
            if (Z < 1.0) Z = Z + YN;
            if (Z >= XN) Z = Z - YN;
            sv = sv + (VVX * VVX + VVY * VVY + VVZ * VVZ) * (double)WPAR;
            float xf = (float)X, yf = (float)Y, zf = (float)Z;
            if ((int)xf == N + 1) xf = xf - 1.e-3f;
            if ((int)yf == N + 1) yf = yf - 1.e-3f;
            if ((int)zf == N + 1) zf = zf - 1.e-3f;
            xp[IN] = xf; yp[IN] = yf; zp[IN] = zf;
            vxp[IN] = (float)VVX; vyp[IN] = (float)VVY; vzp[IN] = (float)VVZ;
        }
        part[tid] = sv;
    }
    for (int t = 0; t < nth; ++t) SVEL += part[t];
    float ah = AEXPN + ASTEP / 2.0f;
    float ENKIN = (float)(SVEL / 2.0 / (double)(ah * ah));
    return (double)ENKIN;
}

// ---------------------------------------------------------------------------
// Multigrid: per-level arena in place of the packed FI3 array (the sections of
// FI3 listed in PMP2MGsolver_fR.f90:76-83 become separate arrays):
//   RR  = section 1 (0,0,koffset)  restricted residual
//   D   = section 2 (n,0,koffset)  restricted density
//   RU  = section 3 (0,n,koffset)  restricted fine solution (frozen)
//   U   = section 4 (n,n,koffset)  working coarse solution
//   TAU = section 5 (0,n,koffset2) FAS right-hand side
//   RES = section 6 (n,0,koffset2) coarse residual
// Level 0 uses D = FI and U = FI2.
// ---------------------------------------------------------------------------
template <class S>
struct MG {
    const mgg_config* c;
    int N, levelmax, levelmin;
    float AEXPN;
    int threads;
    S* fi;    // level-0 density contrast
    S* fi2;   // level-0 field
    std::vector<std::vector<S>> RR, D, RU, U, TAU, RES;
    double phibar = 0.0;   // csf background field at AEXPN (correct_solution)
    const double* bgtab = nullptr;
    int bgrows = 0;

    int n_of(int l) const { return N >> l; }
    S* Ul(int l) { return l == 0 ? fi2 : U[l].data(); }
    S* Dl(int l) { return l == 0 ? fi : D[l].data(); }

    void setup() {
        levelmax = 0;
        while ((1 << levelmax) < N) ++levelmax;
        int ngridmax = N;
        while (ngridmax % 2 == 0) ngridmax /= 2;
        levelmin = 0;
        while ((1 << levelmin) < ngridmax) ++levelmin;
        levelmin += 1;
        RR.assign(levelmax + 1, {}); D.assign(levelmax + 1, {}); RU.assign(levelmax + 1, {});
        U.assign(levelmax + 1, {}); TAU.assign(levelmax + 1, {}); RES.assign(levelmax + 1, {});
        for (int l = 1; l <= levelmax; ++l) {
            int64_t n3 = (int64_t)n_of(l) * n_of(l) * n_of(l);
            RR[l].assign(n3, 0); D[l].assign(n3, 0); RU[l].assign(n3, 0);
            U[l].assign(n3, 0); TAU[l].assign(n3, 0); RES[l].assign(n3, 0);
        }
    }

    double ctilde() const { return 2.99792458e3 * (double)N / (double)c->box; }

    // ---------------- f(R) (PMP2MGsolver_fR.f90) ----------------
    struct FRc {
        double R_bg, R0_bg, fR_bg, s_fR_bg, a_fR_bg;
    };
    FRc frc() const {
        FRc r;
        r.R_bg = 3.0 * ((double)(c->om / fpow3(AEXPN)) + 4.0 * (double)c->oml);
        r.R0_bg = 3.0 * ((double)c->om + 4.0 * (double)c->oml);
        r.fR_bg = c->fr0 * std::pow(r.R0_bg / r.R_bg, c->fr_n + 1);
        r.s_fR_bg = dsign(1.0, r.fR_bg);
        r.a_fR_bg = std::fabs(r.fR_bg);
        return r;
    }
    // Real*4 power u**(n+1) as the Fortran product chain
    static S upow(S u, int n) {
        if (n == 0) return u;
        if (n == 1) return (S)(u * u);
        return (S)(u * u * u);
    }

    void relax_fR(int l, bool red) {   // (20-301)
        const int n = n_of(l);
        const int frn = c->fr_n;
        FRc r = frc();
        const double ctl = ctilde();
        const double dx = (double)(1 << l), dx2 = dx * dx;
        const double fct2 = dx2 / (ctl * ctl * dsign(1.0, r.fR_bg)) / 6.0;
        const double fct1 = -((double)(c->om / AEXPN) * fct2);
        const double Q2 = r.R_bg * (double)fpow2(AEXPN) * fct2 / 3.0;
        const double Q = Q2 * std::pow(std::fabs(r.fR_bg), 1.0 / ((double)frn + 1.0));
        const double ZERO = 1.0e-20, ONEOVERTHREE = 1.0 / 3.0, TWOOVERTHREE = 2.0 / 3.0;
        const double TWOPIOVERTHREE = 2.0 / 3.0 * std::acos(-1.0);
        const double Q2onethird = std::pow(-Q, ONEOVERTHREE);
        const double Q4 = 4.0 * Q, Delta11 = 27.0 * Q, Delta20 = 12.0 * Q;
        S* u = Ul(l);
        const S* d = Dl(l);
        const S* tau = l > 0 ? TAU[l].data() : nullptr;
        const int parity_off = red ? 0 : 1;
#pragma omp parallel for num_threads(threads) schedule(static) collapse(2)
        for (int M3 = 1; M3 <= n; ++M3)
            for (int M2 = 1; M2 <= n; ++M2) {
                int M1start = 1 + (M2 + M3 + parity_off) % 2;
                for (int M1 = M1start; M1 <= n; M1 += 2) {
                    int i = M1 - 1, j = M2 - 1, k = M3 - 1;
                    int iu = wrapu(i + 1, n), il = wrapl(i - 1, n), ju = wrapu(j + 1, n),
                        jl = wrapl(j - 1, n), ku = wrapu(k + 1, n), kl = wrapl(k - 1, n);
                    // Real*4 sum of Real*4 powers of the six neighbours
                    S s = upow(u[gidx(iu, j, k, n)], frn);
                    s = (S)(s + upow(u[gidx(il, j, k, n)], frn));
                    s = (S)(s + upow(u[gidx(i, ju, k, n)], frn));
                    s = (S)(s + upow(u[gidx(i, jl, k, n)], frn));
                    s = (S)(s + upow(u[gidx(i, j, ku, n)], frn));
                    s = (S)(s + upow(u[gidx(i, j, kl, n)], frn));
                    const int64_t q = gidx(i, j, k, n);
                    double P = fct1 * (double)d[q] - Q2;
                    if (l > 0) P = P + fct2 * (double)tau[q];
                    P = P - (double)s / 6.0;
                    double val;
                    if (frn == 0) {
                        val = 0.5 * (-P + std::sqrt(P * P - Q4));
                    } else if (frn == 1) {
                        double Delta10 = -3.0 * P;
                        double CC = Delta11 * Delta11 - 4.0 * Delta10 * Delta10 * Delta10;
                        if (CC >= 0.0) {
                            double tmp1 = 0.5 * (std::sqrt(CC) + Delta11);
                            double tmp2 = tmp1 - Delta11;
                            if (std::fabs(P) < ZERO) val = Q2onethird;
                            else
                                val = -(dsign(std::pow(std::fabs(tmp1), ONEOVERTHREE), tmp1) -
                                        dsign(std::pow(std::fabs(tmp2), ONEOVERTHREE), tmp2)) *
                                      ONEOVERTHREE;
                        } else {
                            double sqrt_Delta0 = std::sqrt(Delta10);
                            double S_ = std::acos(0.5 * Delta11 / (sqrt_Delta0 * sqrt_Delta0 * sqrt_Delta0));
                            val = -TWOOVERTHREE * sqrt_Delta0 * std::cos(S_ * ONEOVERTHREE + TWOPIOVERTHREE);
                        }
                    } else {
                        double Delta21 = 27.0 * P * P;
                        double tmp1 = 0.5 * (std::sqrt(Delta21 * Delta21 - 4.0 * Delta20 * Delta20 * Delta20) + Delta21);
                        double cr = dsign(std::pow(std::fabs(tmp1), ONEOVERTHREE), tmp1);
                        double S_ = std::sqrt(cr + Delta20 / cr) / std::sqrt(12.0);
                        if (P > ZERO) val = -S_ + 0.5 * std::sqrt(-4.0 * S_ * S_ + P / S_);
                        else if (P < -ZERO) val = S_ + 0.5 * std::sqrt(-4.0 * S_ * S_ - P / S_);
                        else val = std::sqrt(std::sqrt(-Q));
                    }
                    u[q] = (S)val;
                }
            }
    }

    // (308-561); level 0 returns the RMS, level > 0 writes RES[l]
    double resid_fR(int l) {
        const int n = n_of(l);
        const int frn = c->fr_n;
        FRc r = frc();
        const double ctl = ctilde(), ctl2 = ctl * ctl;
        const double dx = (double)(1 << l), dx2 = dx * dx;
        const double a_fR_rt = std::pow(r.a_fR_bg, 1.0 / (double)(frn + 1));
        const double fct1 = (double)(c->om / AEXPN);
        const double fct2 = -r.R_bg * (double)fpow2(AEXPN) / 3.0;
        const double fct3 = ctl2 * r.s_fR_bg / dx2;
        const S* u = Ul(l);
        const S* d = Dl(l);
        S* res = l > 0 ? RES[l].data() : nullptr;
        const S* tau = l > 0 ? TAU[l].data() : nullptr;
        int nth = threads > 0 ? threads : 1;
        std::vector<double> part(nth, 0.0);
#pragma omp parallel num_threads(nth)
        {
            int tid = 0;
#ifdef _OPENMP
            tid = omp_get_thread_num();
#endif
            double acc = 0.0;
#pragma omp for schedule(static) collapse(2)
            for (int k = 0; k < n; ++k)
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i) {
                        int iu = wrapu(i + 1, n), il = wrapl(i - 1, n), ju = wrapu(j + 1, n),
                            jl = wrapl(j - 1, n), ku = wrapu(k + 1, n), kl = wrapl(k - 1, n);
                        const int64_t q = gidx(i, j, k, n);
                        S s = upow(u[gidx(iu, j, k, n)], frn);
                        s = (S)(s + upow(u[gidx(il, j, k, n)], frn));
                        s = (S)(s + upow(u[gidx(i, ju, k, n)], frn));
                        s = (S)(s + upow(u[gidx(i, jl, k, n)], frn));
                        s = (S)(s + upow(u[gidx(i, j, ku, n)], frn));
                        s = (S)(s + upow(u[gidx(i, j, kl, n)], frn));
                        double OP = (double)s - (double)upow(u[q], frn) * 6.0;
                        OP = OP * fct3;
                        OP = OP + fct1 * (double)d[q];
                        OP = OP + fct2 * (a_fR_rt / (double)u[q] - 1.0);
                        if (l > 0) {
                            OP = OP - (double)tau[q];
                            res[q] = (S)OP;
                        } else {
                            acc += OP * OP;
                        }
                    }
            part[tid] = acc;
        }
        double RES = 0.0;
        for (int t = 0; t < nth; ++t) RES += part[t];
        return std::sqrt(RES / std::pow((double)n, 3));
    }

    // (569-782)
    void restrict_resid_fR(int l) {
        const int n = n_of(l);
        const int frn = c->fr_n;
        FRc r = frc();
        const double ctl = ctilde(), ctl2 = ctl * ctl;
        const double fct1 = (double)(c->om / AEXPN);
        const double fct2 = -r.R_bg * (double)fpow2(AEXPN) / 3.0;
        const double fct3 = ctl2 * r.s_fR_bg / 1.0;
        const double fct4 = fct2 * std::pow(r.a_fR_bg, 1.0 / (1.0 + (double)frn));
        S* rr = RR[l].data();
        if (l == 1) {
            const int Nf = N;
#pragma omp parallel for num_threads(threads) schedule(static) collapse(2)
            for (int k = 0; k < n; ++k)
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i) {
                        // 0-based fine indices of the children: 2i, 2i+1
                        const int a0 = 2 * i, a1 = 2 * i + 1, b0 = 2 * j, b1 = 2 * j + 1, c0 = 2 * k, c1 = 2 * k + 1;
                        const int ch[8][3] = {{a0, b0, c0}, {a1, b0, c0}, {a0, b1, c0}, {a1, b1, c0},
                                              {a0, b0, c1}, {a1, b0, c1}, {a0, b1, c1}, {a1, b1, c1}};
                        double Q = -8.0 * fct2;
                        for (int m = 0; m < 8; ++m) {
                            int64_t q = gidx(ch[m][0], ch[m][1], ch[m][2], Nf);
                            Q = Q + fct1 * (double)fi[q] + fct4 / (double)fi2[q];
                        }
                        const int Mu = wrapu(a1 + 1, Nf), Ml = wrapl(a0 - 1, Nf);
                        const int Ju = wrapu(b1 + 1, Nf), Jl = wrapl(b0 - 1, Nf);
                        const int Ku = wrapu(c1 + 1, Nf), Kl = wrapl(c0 - 1, Nf);
                        S s8 = upow(fi2[gidx(a0, b0, c0, Nf)], frn);
                        for (int m = 1; m < 8; ++m)
                            s8 = (S)(s8 + upow(fi2[gidx(ch[m][0], ch[m][1], ch[m][2], Nf)], frn));
                        double P = -3.0 * (double)s8;
                        auto U = [&](int x, int y, int z) { return (double)upow(fi2[gidx(x, y, z, Nf)], frn); };
                        P = P + U(Ml, b0, c0) + U(Ml, b1, c0) + U(Ml, b0, c1) + U(Ml, b1, c1);
                        P = P + U(Mu, b0, c0) + U(Mu, b1, c0) + U(Mu, b0, c1) + U(Mu, b1, c1);
                        P = P + U(a0, Jl, c0) + U(a1, Jl, c0) + U(a0, Jl, c1) + U(a1, Jl, c1);
                        P = P + U(a0, Ju, c0) + U(a1, Ju, c0) + U(a0, Ju, c1) + U(a1, Ju, c1);
                        P = P + U(a0, b0, Kl) + U(a1, b0, Kl) + U(a0, b1, Kl) + U(a1, b1, Kl);
                        P = P + U(a0, b0, Ku) + U(a1, b0, Ku) + U(a0, b1, Ku) + U(a1, b1, Ku);
                        rr[gidx(i, j, k, n)] = (S)((P * fct3 + Q) / 8.0);
                    }
        } else {
            avg8(RES[l - 1].data(), rr, n);
        }
    }

    // 8-child average into one coarse array (restrict_density / scalar_field order)
    void avg8(const S* f, S* out, int n, S* out2 = nullptr) {
        const int nf = 2 * n;
#pragma omp parallel for num_threads(threads) schedule(static) collapse(2)
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    double P = (double)f[gidx(2 * i, 2 * j, 2 * k, nf)];
                    P = P + (double)f[gidx(2 * i + 1, 2 * j, 2 * k, nf)];
                    P = P + (double)f[gidx(2 * i, 2 * j + 1, 2 * k, nf)];
                    P = P + (double)f[gidx(2 * i + 1, 2 * j + 1, 2 * k, nf)];
                    P = P + (double)f[gidx(2 * i, 2 * j, 2 * k + 1, nf)];
                    P = P + (double)f[gidx(2 * i + 1, 2 * j, 2 * k + 1, nf)];
                    P = P + (double)f[gidx(2 * i, 2 * j + 1, 2 * k + 1, nf)];
                    P = P + (double)f[gidx(2 * i + 1, 2 * j + 1, 2 * k + 1, nf)];
                    out[gidx(i, j, k, n)] = (S)(P / 8.0);
                    if (out2) out2[gidx(i, j, k, n)] = (S)(P / 8.0);
                }
    }
    void restrict_scalar_field(int l) { avg8(Ul(l - 1), RU[l].data(), n_of(l), U[l].data()); }   // (1262-1349)
    void restrict_density(int l) { avg8(Dl(l - 1), D[l].data(), n_of(l)); }                        // (1168-1251)

    // (789-927)
    void rhs_fR(int l) {
        const int n = n_of(l);
        const int frn = c->fr_n;
        FRc r = frc();
        const double ctl = ctilde();
        const double dx = (double)(1 << l), dx2 = dx * dx;
        const double a_fR_rt = std::pow(r.a_fR_bg, 1.0 / (double)(frn + 1));
        const double fct1 = (double)(c->om / AEXPN);
        const double fct2 = -r.R_bg * (double)fpow2(AEXPN) / 3.0;
        const double fct3 = ctl * ctl * r.s_fR_bg / dx2;
        const S* ru = RU[l].data();
        const S* d = D[l].data();
        const S* rr = RR[l].data();
        S* tau = TAU[l].data();
#pragma omp parallel for num_threads(threads) schedule(static) collapse(2)
        for (int k = 0; k < n; ++k)
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    int iu = wrapu(i + 1, n), il = wrapl(i - 1, n), ju = wrapu(j + 1, n),
                        jl = wrapl(j - 1, n), ku = wrapu(k + 1, n), kl = wrapl(k - 1, n);
                    const int64_t q = gidx(i, j, k, n);
                    S s = upow(ru[gidx(iu, j, k, n)], frn);
                    s = (S)(s + upow(ru[gidx(il, j, k, n)], frn));
                    s = (S)(s + upow(ru[gidx(i, ju, k, n)], frn));
                    s = (S)(s + upow(ru[gidx(i, jl, k, n)], frn));
                    s = (S)(s + upow(ru[gidx(i, j, ku, n)], frn));
                    s = (S)(s + upow(ru[gidx(i, j, kl, n)], frn));
                    double OP = (double)s - (double)upow(ru[q], frn) * 6.0;
                    OP = OP * fct3;
                    OP = OP + fct1 * (double)d[q];
                    OP = OP + fct2 * (a_fR_rt / (double)ru[q] - 1.0);
                    OP = OP - (double)rr[q];
                    tau[q] = (S)OP;
                }
    }

    // correct_solution (PMP2extradof.f90:1361-1578)
    void correct(int l) {
        const int n = n_of(l), nf = 2 * n;
        const double a = 1.0 / 64.0, b = 3.0 * a, cw = 9.0 * a, d = 27.0 * a;
        const double bbb[8] = {a, b, b, cw, b, cw, cw, d};
        static const int ccc[8][8] = {{1, 2, 4, 5, 10, 11, 13, 14},   {3, 2, 6, 5, 12, 11, 15, 14},
                                      {7, 8, 4, 5, 16, 17, 13, 14},   {9, 8, 6, 5, 18, 17, 15, 14},
                                      {19, 20, 22, 23, 10, 11, 13, 14}, {21, 20, 24, 23, 12, 11, 15, 14},
                                      {25, 26, 22, 23, 16, 17, 13, 14}, {27, 26, 24, 23, 18, 17, 15, 14}};
        const S* uc = U[l].data();
        const S* ru = RU[l].data();
        S* uf = Ul(l - 1);
        const int model = c->mg_model;
        const double ctl2 = ctilde() * ctilde();
#pragma omp parallel for num_threads(threads) schedule(static) collapse(2)
        for (int M3 = 1; M3 <= n; ++M3)
            for (int M2 = 1; M2 <= n; ++M2)
                for (int M1 = 1; M1 <= n; ++M1) {
                    int pid1[27], pid2[27], pid3[27];
                    for (int pind = 1; pind <= 27; ++pind) {
                        int i3 = (pind - 1) / 9, i2 = (pind - 1 - i3 * 9) / 3, i1 = pind - 1 - i3 * 9 - i2 * 3;
                        int p1 = M1 + i1 - 1; if (p1 < 1) p1 = n; if (p1 > n) p1 = 1;
                        int p2 = M2 + i2 - 1; if (p2 < 1) p2 = n; if (p2 > n) p2 = 1;
                        int p3 = M3 + i3 - 1; if (p3 < 1) p3 = n; if (p3 > n) p3 = 1;
                        pid1[pind - 1] = p1; pid2[pind - 1] = p2; pid3[pind - 1] = p3;
                    }
                    for (int sind = 1; sind <= 8; ++sind) {
                        int i3 = (sind - 1) / 4, i2 = (sind - 1 - i3 * 4) / 2, i1 = sind - 1 - i3 * 4 - i2 * 2;
                        double P = 0.0;
                        for (int ind = 0; ind < 8; ++ind) {
                            int pp = ccc[sind - 1][ind] - 1;
                            int64_t q = gidx(pid1[pp] - 1, pid2[pp] - 1, pid3[pp] - 1, n);
                            P = P + bbb[ind] * (double)uc[q];
                            P = P - bbb[ind] * (double)ru[q];
                        }
                        int64_t qf = gidx(2 * M1 + i1 - 2, 2 * M2 + i2 - 2, 2 * M3 + i3 - 2, nf);
                        double tmpt = (double)uf[qf] + P;
                        if (model == 1 || model == 3) {
                            if (tmpt > 0.0) uf[qf] = (S)tmpt;
                        } else if (model == 5) {
                            if (phibar + tmpt / ctl2 > 0.0) uf[qf] = (S)tmpt;
                        } else {
                            uf[qf] = (S)tmpt;
                        }
                    }
                }
    }

    // model dispatch (only f(R) in this file; other models added alongside)
    void relax(int l, bool red);
    double resid(int l);
    void restrict_resid(int l);
    void rhs(int l);

    void smooth(int l, int nsmth) {
        for (int s = 0; s < nsmth; ++s) {
            relax(l, true);
            relax(l, false);
        }
    }
    void coarse_prepare(int l) {   // the block between pre-smoothing and the recursion
        restrict_resid(l + 1);
        restrict_scalar_field(l + 1);
        restrict_density(l + 1);
        rhs(l + 1);
    }
    // V_cycle (PMP2extradof.f90:352-555).  The level-0 calculate_residual call
    // inside the cycle (427) only feeds the level-1 restriction, which for every
    // model recomputes the fine residual from FI and FI2 (restrict_residual_*,
    // ilevel==1 branch), so its value is not needed here.
    void vcycle(int l) {
        const int Nsmth = 2;
        if (levelmax - l <= levelmin) {
            smooth(l, Nsmth);
            return;
        }
        smooth(l, Nsmth);
        if (l > 0) resid(l);
        coarse_prepare(l);
        vcycle(l + 1);
        correct(l + 1);
        smooth(l, Nsmth);
    }
    // F_cycle (PMP2extradof.f90:563-865): pre-smooth, coarse F-cycle, correct,
    // post-smooth, then the same level again as a V-cycle
    void fcycle(int l) {
        const int Nsmth = 2;
        if (levelmax - l <= levelmin) {
            smooth(l, Nsmth);
            return;
        }
        smooth(l, Nsmth);
        if (l > 0) resid(l);
        coarse_prepare(l);
        fcycle(l + 1);
        correct(l + 1);
        smooth(l, Nsmth);
        if (l > 0) resid(l);
        coarse_prepare(l);
        vcycle(l + 1);
        correct(l + 1);
        smooth(l, Nsmth);
    }
    // W_cycle (PMP2extradof.f90:867-1165): two coarse-grid corrections per level
    void wcycle(int l) {
        const int Nsmth = 2;
        if (levelmax - l <= levelmin) {
            smooth(l, Nsmth);
            return;
        }
        smooth(l, Nsmth);
        if (l > 0) resid(l);
        coarse_prepare(l);
        wcycle(l + 1);
        correct(l + 1);
        smooth(l, Nsmth);
        if (l > 0) resid(l);
        coarse_prepare(l);
        wcycle(l + 1);
        correct(l + 1);
        smooth(l, Nsmth);
    }
};

// Sweep order of the nDGP and k-mouflage relaxations, whose stencils read
// same-colour diagonal neighbours: 0 = the serial in-place order of one OpenMP
// thread (the reference at T = 1); 1 = snapshot order, every cell of a colour
// reading the field as it was before that colour's sweep (an order-independent
// schedule, the one a parallel sweep without in-place reads gives).  The other
// models' 7-point stencils read only the other colour, so both orders agree.
int g_snapshot_order = 0;

// -------- model dispatch (models other than f(R) live in oracle_models.inc) ----
#include "oracle_models.inc"

template <class S>
void MG<S>::relax(int l, bool red) {
    switch (c->mg_model) {
    case 1: relax_fR(l, red); break;
    case 2: relax_DGP(this, l, red); break;
    case 3: relax_sym(this, l, red); break;
    case 4: relax_kmf(this, l, red); break;
    case 5: relax_csf(this, l, red); break;
    default: break;
    }
}
template <class S>
double MG<S>::resid(int l) {
    switch (c->mg_model) {
    case 1: return resid_fR(l);
    case 2: return resid_DGP(this, l);
    case 3: return resid_sym(this, l);
    case 4: return resid_kmf(this, l);
    case 5: return resid_csf(this, l);
    default: return 0.0;
    }
}
template <class S>
void MG<S>::restrict_resid(int l) {
    switch (c->mg_model) {
    case 1: restrict_resid_fR(l); break;
    case 2: restrict_resid_DGP(this, l); break;
    case 3: restrict_resid_sym(this, l); break;
    case 4: restrict_resid_kmf(this, l); break;
    case 5: restrict_resid_csf(this, l); break;
    default: break;
    }
}
template <class S>
void MG<S>::rhs(int l) {
    switch (c->mg_model) {
    case 1: rhs_fR(l); break;
    case 2: rhs_DGP(this, l); break;
    case 3: rhs_sym(this, l); break;
    case 4: rhs_kmf(this, l); break;
    case 5: rhs_csf(this, l); break;
    default: break;
    }
}

// scalar_field (PMP2extradof.f90:12-178) with initialise_extradof (181-344)
template <class S>
int scalar_field(S* fi, S* fi2, const mgg_config* c, float AEXPN, int i_step, mgg_mg_report* rep,
                 int threads, const double* bg = nullptr, int bgrows = 0) {
    MG<S> mg;
    mg.bgtab = bg;
    mg.bgrows = bgrows;
    if (bg && c->mg_model == 5) mg.phibar = bg_interp(bg, bgrows, AEXPN, AEXPN, 1);
    mg.c = c;
    mg.N = c->ngrid;
    mg.AEXPN = AEXPN;
    mg.threads = threads;
    mg.fi = fi;
    mg.fi2 = fi2;
    mg.setup();
    const int64_t ncell = (int64_t)mg.N * mg.N * mg.N;
    if (rep) std::memset(rep, 0, sizeof(*rep));
    auto fr_ubg = [&](double expo) {
        double R_bg = 3.0 * ((double)(c->om / fpow3(AEXPN)) + 4.0 * (double)c->oml);
        double R0_bg = 3.0 * ((double)c->om + 4.0 * (double)c->oml);
        double fR_bg = c->fr0 * std::pow(R0_bg / R_bg, c->fr_n + 1);
        return std::pow(std::fabs(fR_bg), expo);
    };
    if (i_step == 1) {
        // initialise_extradof
        double ubg = 0.0;
        if (c->mg_model == 1) ubg = fr_ubg(1.0 / (1.0 + (double)c->fr_n));
        else if (c->mg_model == 3) {
            if (AEXPN > c->sym_astar) {
                double sa = c->sym_astar / (double)AEXPN;
                ubg = std::sqrt(1.0 - sa * sa * sa);
            }
        }
        for (int64_t q = 0; q < ncell; ++q) fi2[q] = (S)ubg;
    }
    if (c->mg_model == 3 && AEXPN < c->sym_astar) return 0;   // (37-41)
    double res_old_1 = 1.0e5, res_old_2 = 1.0e10;
    int iter_count = 1;
    for (;;) {
        if (i_step > 1 && iter_count == 1) {
            if (c->mg_model == 1) {
                double ubg = fr_ubg(1.0 / (1.0 + (double)c->fr_n));
                for (int64_t q = 0; q < ncell; ++q) fi2[q] = (S)((double)fi2[q] * ubg);
            }
            if (c->mg_model == 3) {
                double sa = c->sym_astar / (double)AEXPN;
                double ubg = std::sqrt(1.0 - sa * sa * sa);
                for (int64_t q = 0; q < ncell; ++q) fi2[q] = (S)ubg;
            }
        }
        if (c->vcycle == 1) mg.vcycle(0);
        if (c->fcycle == 1) mg.fcycle(0);
        if (c->wcycle == 1) mg.wcycle(0);
        double res = mg.resid(0);
        if (rep && iter_count <= 64) rep->residual[iter_count - 1] = res;
        bool can_exit = false;
        int reason = 0;
        if (res <= c->res_conv) { can_exit = true; reason = 1; }
        if (iter_count > 2) {
            if (std::fabs(res / res_old_1 - 1.0) <= 5.0e-3) { can_exit = true; if (!reason) reason = 2; }
            if (std::fabs(res / res_old_1 - 1.0) <= 1.0e-2 && std::fabs(res_old_1 / res_old_2 - 1.0) <= 1.0e-2) {
                can_exit = true;
                if (!reason) reason = 2;
            }
        }
        if (iter_count >= c->iter_count_max) { can_exit = true; if (!reason) reason = 3; }
        if (can_exit) {
            if (c->mg_model == 1) {
                double ubg = fr_ubg(-1.0 / (1.0 + (double)c->fr_n));
                for (int64_t q = 0; q < ncell; ++q) fi2[q] = (S)((double)fi2[q] * ubg);
            }
            if (rep) { rep->cycles = iter_count; rep->exit_reason = reason; }
            break;
        }
        iter_count++;
        res_old_2 = res_old_1;
        res_old_1 = res;
    }
    return 0;
}

// ---------------------------------------------------------------------------
// DENSITrsd(iSwitch, NGRID_old) (PMP2mod_density.f90:407-557) with sigv = 0, so
// the added dispersion vv is zero: FI := -1 on the ng mesh, then CIC of the
// particles at X = (XPAR-1)*Xscale+1, Xscale = ng/ng_old, all in Real*4; for
// iSwitch = 1, 2, 3 the axes rotate so that the displaced one is the third
// (line of sight) and it moves by (V*Xscale+vv)*factor, factor =
// sqrt(AEXPN/(Om+AEXPN**3*OmL))/AEXPN.  The periodic wrap and the CIC weights
// are Real*8 (X, D1, T1 are Real*8 there); WPAR = ng^3/Np in Real*4.
// ---------------------------------------------------------------------------
template <class S>
void density_rsd(const float* xp, const float* yp, const float* zp, const float* vxp, const float* vyp,
                 const float* vzp, int64_t np, int ng_old, int ng, int iswitch, float aexpn, float om, float oml,
                 S* fi) {
    const int64_t ncell = (int64_t)ng * ng * ng;
    const float Xscale = (float)ng / (float)ng_old;
    const float factor = std::sqrt(aexpn / (om + aexpn * aexpn * aexpn * oml)) / aexpn;
    const float W = ((float)ng * (float)ng * (float)ng) / (float)np;
    const float vv = 0.0f;
    for (int64_t c = 0; c < ncell; ++c) fi[c] = (S)-1.0f;
    for (int64_t p = 0; p < np; ++p) {
        const float px = (xp[p] - 1.0f) * Xscale + 1.0f;
        const float py = (yp[p] - 1.0f) * Xscale + 1.0f;
        const float pz = (zp[p] - 1.0f) * Xscale + 1.0f;
        float Xf = px, Yf = py, Zf = pz;
        if (iswitch == 1) { Zf = px + (vxp[p] * Xscale + vv) * factor; Yf = py; Xf = pz; }
        else if (iswitch == 2) { Xf = px; Zf = py + (vyp[p] * Xscale + vv) * factor; Yf = pz; }
        else if (iswitch == 3) { Zf = pz + (vzp[p] * Xscale + vv) * factor; }
        double X = Xf, Y = Yf, Z = Zf;
        const double top = (double)((float)ng + 1.0f);
        if (X >= top) X -= ng;
        if (Y >= top) Y -= ng;
        if (Z >= top) Z -= ng;
        if (X < 1.0) X += ng;
        if (Y < 1.0) Y += ng;
        if (Z < 1.0) Z += ng;
        const int I = (int)X, J = (int)Y, K = (int)Z;
        const double D1 = X - (double)(float)I, D2 = Y - (double)(float)J, D3 = Z - (double)(float)K;
        const double T1 = 1.0 - D1, T2 = 1.0 - D2, T3 = 1.0 - D3;
        const double T2W = T2 * (double)W, D2W = D2 * (double)W;
        int I1 = I + 1; if (I1 > ng) I1 = 1;
        int J1 = J + 1; if (J1 > ng) J1 = 1;
        int K1 = K + 1; if (K1 > ng) K1 = 1;
        const int i0 = I - 1, j0 = J - 1, k0 = K - 1, i1 = I1 - 1, j1 = J1 - 1, k1 = K1 - 1;
        auto add = [&](int64_t c, double w) { fi[c] = (S)((double)fi[c] + w); };
        add(gidx(i0, j0, k0, ng), T3 * T1 * T2W);
        add(gidx(i1, j0, k0, ng), T3 * D1 * T2W);
        add(gidx(i0, j1, k0, ng), T3 * T1 * D2W);
        add(gidx(i1, j1, k0, ng), T3 * D1 * D2W);
        add(gidx(i0, j0, k1, ng), D3 * T1 * T2W);
        add(gidx(i1, j0, k1, ng), D3 * D1 * T2W);
        add(gidx(i0, j1, k1, ng), D3 * T1 * D2W);
        add(gidx(i1, j1, k1, ng), D3 * D1 * D2W);
    }
}

// ---------------------------------------------------------------------------
// DensDistr (PMP2mod_density.f90:1041-1126): bins of 0.001 dex in 1 + delta
// from iMin = -2001 to iMax = 2001 (cells outside go to the end bins), cell
// counts and density sums per bin, and the mean and RMS of 1 + delta.  The
// Real*4 LOG10 of the reference is taken as the correctly rounded FP32 log10;
// an empty cell (1 + delta = 0) goes to bin iMin.
// ---------------------------------------------------------------------------
template <class S>
void density_pdf(const S* fi, int ng, int64_t* ncells, double* den, double* rms, double* mean) {
    const int iMin = -2001, iMax = 2001;
    const double dlog = 0.001;
    for (int i = 0; i <= iMax - iMin; ++i) { ncells[i] = 0; den[i] = 0.0; }
    double SUM1 = 0.0, SUM2 = 0.0;
    const int64_t ncell = (int64_t)ng * ng * ng;
    for (int64_t q = 0; q < ncell; ++q) {
        const float v = (float)fi[q] + 1.0f;
        SUM1 += (double)v;
        SUM2 += (double)(v * v);
        int ind = iMin;
        if (v > 0.0f) {
            const double l = (double)(float)std::log10((double)v);
            const double f = std::floor(l / dlog);
            ind = f < iMin ? iMin : (f > iMax ? iMax : (int)f);
        }
        ncells[ind - iMin] += 1;
        den[ind - iMin] += (double)v;
    }
    const float Total = (float)ng * (float)ng * (float)ng;
    const double DENM = SUM1 / (double)Total;
    *mean = DENM;
    *rms = std::sqrt(SUM2 / (double)Total - DENM * DENM);
}

// ---------------------------------------------------------------------------
// POWERfft5(iPol,0) (PMP2mod_power.f90:209-463) with the GetPower(0) output
// conversion (437-456).  Transpositions skipped as in potential(), so the
// reference's first index after its x<->z transposition (the z axis, which
// the quadrupole's cos(mu) refers to) is the third index here.  iPol = 1
// weights every mode by P2(mu) = 1.5 cos^2(mu) - 0.5 in Real*4 and scales the
// sums by 2.5 (no log bins).
// ---------------------------------------------------------------------------
template <class S>
void power(S* fi, int ng, float box, int nbins, double* k_out, double* n_out, double* p_out,
           double* kl_out, double* nl_out, double* pl_out, int threads, int pol = 0) {
    const int N = ng;
    const float sq2 = std::sqrt(2.0f);
    // x lines, then the sqrt(2) of the DC and Nyquist x rows
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int k = 0; k < N; ++k) {
        std::vector<double> r(N);
        for (int j = 0; j < N; ++j) {
            for (int i = 0; i < N; ++i) r[i] = (double)fi[gidx(i, j, k, N)];
            rfft1f(r.data(), N);
            for (int i = 0; i < N; ++i) fi[gidx(i, j, k, N)] = (S)r[i];
        }
    }
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j) {
            fi[gidx(0, j, k, N)] = (S)(fi[gidx(0, j, k, N)] * sq2);
            fi[gidx(N - 1, j, k, N)] = (S)(fi[gidx(N - 1, j, k, N)] * sq2);
        }
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int k = 0; k < N; ++k) {
        std::vector<double> r(N);
        for (int i = 0; i < N; ++i) {
            for (int j = 0; j < N; ++j) r[j] = (double)fi[gidx(i, j, k, N)];
            rfft1f(r.data(), N);
            for (int j = 0; j < N; ++j) fi[gidx(i, j, k, N)] = (S)r[j];
        }
    }
    for (int k = 0; k < N; ++k)
        for (int i = 0; i < N; ++i) {
            fi[gidx(i, 0, k, N)] = (S)(fi[gidx(i, 0, k, N)] * sq2);
            fi[gidx(i, N - 1, k, N)] = (S)(fi[gidx(i, N - 1, k, N)] * sq2);
        }
#pragma omp parallel for num_threads(threads) schedule(static)
    for (int j = 0; j < N; ++j) {
        std::vector<double> r(N);
        for (int i = 0; i < N; ++i) {
            for (int k = 0; k < N; ++k) r[k] = (double)fi[gidx(i, j, k, N)];
            rfft1f(r.data(), N);
            for (int k = 0; k < N; ++k) fi[gidx(i, j, k, N)] = (S)r[k];
        }
    }
    for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i) {
            fi[gidx(i, j, 0, N)] = (S)(fi[gidx(i, j, 0, N)] * sq2);
            fi[gidx(i, j, N - 1, N)] = (S)(fi[gidx(i, j, N - 1, N)] * sq2);
        }
    const int64_t ncell = (int64_t)N * N * N;
    for (int64_t q = 0; q < ncell; ++q) fi[q] = (S)(fi[q] * fi[q] / (S)8.0f);
    fi[0] = 0;
    const int NPOWER = N;
    const float dLog = 0.02f;
    std::vector<double> DP(NPOWER + 1, 0.0), iV(NPOWER + 1, 0.0), dk(NPOWER + 1, 0.0);
    std::vector<double> DPl(NPOWER + 1, 0.0), iVl(NPOWER + 1, 0.0), dkl(NPOWER + 1, 0.0);
    for (int K = 1; K <= N; ++K) {
        int MK = (K / 2) * (K / 2);
        for (int J = 1; J <= N; ++J) {
            int MJ = (J / 2) * (J / 2);
            for (int I = 1; I <= N; ++I) {
                int MI = (I / 2) * (I / 2);
                float AMP = (float)fi[gidx(I - 1, J - 1, K - 1, N)];
                float RK = (float)(MI + MJ + MK);
                if (RK < 0.5f) continue;
                RK = std::sqrt(RK);
                int MP = std::max((int)(RK + 0.5f), 1);
                int MPlog = std::max(1, std::min(NPOWER, (int)(std::log10(RK) / dLog + 1000.0f) - 1000));
                if (pol) {
                    const float cosmu2 = (float)MK / (RK * RK);
                    const float P2 = 1.5f * cosmu2 - 0.5f;
                    DP[MP] += (double)(AMP * P2);
                } else {
                    DP[MP] += AMP;
                    DPl[MPlog] += AMP;
                }
                iV[MP] += 1.0;
                dk[MP] += RK;
                iVl[MPlog] += 1.0;
                dkl[MPlog] += RK;
            }
        }
    }
    if (pol)
        for (auto& v : DP) v = 2.5 * v;   // (2L+1)/2 for the quadrupole
    const float Pi = 3.141592653f;
    const float Scale = 2.0f * Pi / box;
    const float b3 = box * box * box;
    for (int I = 1; I <= nbins && I <= N / 2; ++I) {
        if (k_out) k_out[I - 1] = 0;
        if (n_out) n_out[I - 1] = 0;
        if (p_out) p_out[I - 1] = 0;
        if (kl_out) kl_out[I - 1] = 0;
        if (nl_out) nl_out[I - 1] = 0;
        if (pl_out) pl_out[I - 1] = 0;
        if (iV[I] > 0) {
            float wk = (float)(dk[I] / iV[I] * (double)Scale);
            double Pkk = (double)b3 * DP[I] / iV[I];
            if (k_out) k_out[I - 1] = wk;
            if (n_out) n_out[I - 1] = (float)iV[I];
            if (p_out) p_out[I - 1] = (float)Pkk;
        }
        if (iVl[I] > 0) {
            float wk = (float)(dkl[I] / iVl[I] * (double)Scale);
            double Pkk = (double)b3 * DPl[I] / iVl[I];
            if (kl_out) kl_out[I - 1] = wk;
            if (nl_out) nl_out[I - 1] = (float)iVl[I];
            if (pl_out) pl_out[I - 1] = (float)Pkk;
        }
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// C entry points (ctypes).  Suffix _f = Real*4 storage, _d = FP64 storage.
// ---------------------------------------------------------------------------
extern "C" {

void orc_rfft1f(double* r, int n) { rfft1f(r, n); }
void orc_rfft1b(double* r, int n) { rfft1b(r, n); }

void orc_density_f(const float* x, const float* y, const float* z, int64_t np, int ng, float* fi, int threads) {
    density<float>(x, y, z, np, ng, fi, threads);
}
void orc_density_d(const float* x, const float* y, const float* z, int64_t np, int ng, double* fi, int threads) {
    density<double>(x, y, z, np, ng, fi, threads);
}
void orc_potential_f(float* fi, int ng, float aexpn, float om, float omb, int threads) {
    potential<float>(fi, ng, aexpn, om, omb, threads);
}
void orc_potential_d(double* fi, int ng, float aexpn, float om, float omb, int threads) {
    potential<double>(fi, ng, aexpn, om, omb, threads);
}
void orc_potential_mg_f(float* fi, const float* fi2, const mgg_config* c, float aexpn, int threads) {
    potential_mg<float>(fi, fi2, c, aexpn, threads);
}
void orc_potential_mg_d(double* fi, const double* fi2, const mgg_config* c, float aexpn, int threads) {
    potential_mg<double>(fi, fi2, c, aexpn, threads);
}
double orc_move_f(const float* fi, const float* fi2, float* x, float* y, float* z, float* vx, float* vy,
                  float* vz, int64_t np, const mgg_config* c, float aexpn, float astep, float factv,
                  const double* bg, int bgrows, int threads) {
    return move<float>(fi, fi2, x, y, z, vx, vy, vz, np, c, aexpn, astep, factv, bg, bgrows, threads);
}
double orc_move_d(const double* fi, const double* fi2, float* x, float* y, float* z, float* vx, float* vy,
                  float* vz, int64_t np, const mgg_config* c, float aexpn, float astep, float factv,
                  const double* bg, int bgrows, int threads) {
    return move<double>(fi, fi2, x, y, z, vx, vy, vz, np, c, aexpn, astep, factv, bg, bgrows, threads);
}
int orc_scalar_field_f(float* fi, float* fi2, const mgg_config* c, float aexpn, int i_step, mgg_mg_report* rep,
                       int threads, const double* bg, int bgrows) {
    return scalar_field<float>(fi, fi2, c, aexpn, i_step, rep, threads, bg, bgrows);
}
int orc_scalar_field_d(double* fi, double* fi2, const mgg_config* c, float aexpn, int i_step,
                       mgg_mg_report* rep, int threads, const double* bg, int bgrows) {
    return scalar_field<double>(fi, fi2, c, aexpn, i_step, rep, threads, bg, bgrows);
}
void orc_power_f(float* fi, int ng, float box, int nbins, double* k, double* n, double* p, double* kl,
                 double* nl, double* pl, int threads) {
    power<float>(fi, ng, box, nbins, k, n, p, kl, nl, pl, threads);
}
void orc_power_pol_f(float* fi, int ng, float box, int nbins, double* k, double* n, double* p, int pol,
                     int threads) {
    power<float>(fi, ng, box, nbins, k, n, p, nullptr, nullptr, nullptr, threads, pol);
}
void orc_density_rsd_f(const float* x, const float* y, const float* z, const float* vx, const float* vy,
                       const float* vz, int64_t np, int ng_old, int ng, int iswitch, float aexpn, float om, float oml,
                       float* fi) {
    density_rsd<float>(x, y, z, vx, vy, vz, np, ng_old, ng, iswitch, aexpn, om, oml, fi);
}
void orc_density_pdf_f(const float* fi, int ng, int64_t* ncells, double* den, double* rms, double* mean) {
    density_pdf<float>(fi, ng, ncells, den, rms, mean);
}

// GetPower(1) (PMP2mod_power.f90:20-108) with sigv = 0: on the NGRID/2 mesh the
// real-space P(k) (iSwitch = 0) and, for the three lines of sight, the monopole
// and quadrupole of the redshift-space density; P0 and P2 are the Real*4
// averages over the three.  Outputs per bin I = 1..nbins (nbins <= NGRID/4).
void orc_power_rsd_f(const float* x, const float* y, const float* z, const float* vx, const float* vy,
                     const float* vz, int64_t np, int ng_old, float box, float aexpn, float om, float oml, int nbins,
                     double* k, double* n, double* preal, double* p0, double* p2, int threads) {
    const int ng = ng_old / 2;
    std::vector<float> fi((size_t)ng * ng * ng);
    std::vector<double> pk[7];
    for (auto& v : pk) v.assign(nbins, 0.0);
    for (int sw = 0; sw <= 3; ++sw) {
        density_rsd<float>(x, y, z, vx, vy, vz, np, ng_old, ng, sw, aexpn, om, oml, fi.data());
        power<float>(fi.data(), ng, box, nbins, sw == 0 ? k : nullptr, sw == 0 ? n : nullptr, pk[2 * sw].data(),
                     nullptr, nullptr, nullptr, threads, 0);
        if (sw != 0) {
            density_rsd<float>(x, y, z, vx, vy, vz, np, ng_old, ng, sw, aexpn, om, oml, fi.data());
            power<float>(fi.data(), ng, box, nbins, nullptr, nullptr, pk[2 * sw - 1].data(), nullptr, nullptr,
                         nullptr, threads, 1);
        }
    }
    for (int i = 0; i < nbins; ++i) {
        preal[i] = pk[0][i];
        const float a2 = (float)pk[1][i] + (float)pk[3][i] + (float)pk[5][i];
        const float a0 = (float)pk[2][i] + (float)pk[4][i] + (float)pk[6][i];
        p2[i] = a2 / 3.0f;
        p0[i] = a0 / 3.0f;
    }
}

// The level-0 k-mouflage operator (kmf_op, PMP2MGsolver_kmf.f90:262-~505) at
// every cell into out (FP64): tests build manufactured solutions from it (the
// operator is affine in the density contrast).
void orc_kmf_operator_f(float* fi, float* fi2, const mgg_config* c, float aexpn, double* out, const double* bg,
                        int bgrows) {
    MG<float> mg;
    mg.bgtab = bg;
    mg.bgrows = bgrows;
    mg.c = c;
    mg.N = c->ngrid;
    mg.AEXPN = aexpn;
    mg.threads = 1;
    mg.fi = fi;
    mg.fi2 = fi2;
    mg.setup();
    const KMFc K = kmf_consts(&mg);
    const int n = mg.N;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) out[gidx(i, j, k, n)] = kmf_op(fi2, fi, i, j, k, n, 1.0, c->kmf_n, K);
}

// The density contrast for which the level-0 nDGP operator (resid_DGP,
// PMP2MGsolver_DGP.f90:240-388) vanishes at every cell of the field fi2:
// lap/dx^2 = 0.75 (sign(alpha) sqrt(alpha^2 + 8/3 Sigma) - alpha) gives
// Sigma = ((alpha + 4/3 lap)^2 - alpha^2) 3/8, and Sigma = fct1 delta + G(u).
// Returns the number of cells where the root does not exist (sign(alpha)
// (alpha + 4/3 lap) < 0); tests build manufactured solutions from it.
int64_t orc_dgp_root_density_f(float* fi2, const mgg_config* c, float aexpn, double* out) {
    const int n = c->ngrid;
    const DGPc K = dgp_consts(c, aexpn, true);
    const double sa = K.alpha >= 0.0 ? 1.0 : -1.0;
    int64_t bad = 0;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                const double lap = lap7(fi2, i, j, k, n);
                const double t = K.alpha + 4.0 / 3.0 * lap;
                if (sa * t < 0.0) ++bad;
                const double sigma = (t * t - K.alpha * K.alpha) * 3.0 / 8.0;
                out[gidx(i, j, k, n)] = (sigma - dgp_sigma(fi2, i, j, k, n, 1.0, 0.0)) / K.fct1;
            }
    return bad;
}

// Single MG building blocks for unit tests: op selects the routine,
// 0 relax red, 1 relax black, 2 level-0 residual RMS.
double orc_mg_op_f(float* fi, float* fi2, const mgg_config* c, float aexpn, int op, int threads) {
    MG<float> mg;
    mg.c = c;
    mg.N = c->ngrid;
    mg.AEXPN = aexpn;
    mg.threads = threads;
    mg.fi = fi;
    mg.fi2 = fi2;
    mg.setup();
    if (op == 0) mg.relax(0, true);
    else if (op == 1) mg.relax(0, false);
    else if (op == 2) return mg.resid(0);
    else if (op == 3) mg.vcycle(0);
    return 0.0;
}

void orc_set_sweep_order(int snapshot) { g_snapshot_order = snapshot ? 1 : 0; }

int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

}  // extern "C"
