// Kernel (d): FAS nonlinear multigrid for the scalar field, the replacement of
// scalar_field / V_cycle / F_cycle / W_cycle and the transfer operators
// (PMP2extradof.f90:12-578, 1168-1578) and of the model solvers
// PMP2MGsolver_fR.f90 (f(R), n = 0, 1, 2), PMP2MGsolver_DGP.f90 (nDGP) and
// PMP2MGsolver_sym.f90 (symmetron).
//
// Storage: FP32 grids, one array per FI3 section per level (mgg_internal.cuh
// Level); level 0 uses FI (density contrast) and FI2 (field).  Arithmetic
// follows the reference: Real*8 for everything except the Real*4 sums and
// products of grid values that the Fortran expressions form in single
// precision.
//
// Red-black smoothing with the 7-point stencil (f(R), symmetron) updates each
// colour from the other colour only, so the parallel sweep equals the
// reference's serial sweep.  The nDGP stencil also reads same-colour diagonal
// neighbours; the reference's result there depends on the OpenMP schedule.
// Here every nDGP colour pass reads a snapshot of the field taken before the
// pass, which is deterministic.
#include "mgg_internal.cuh"
#include "reduce.cuh"
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <vector>

namespace mgg {

namespace {

// ---------------------------------------------------------------- consts ----
struct LevelConsts {
    int n;
    double dx2, dx4;
    // reciprocals of level constants: divisions by them in the nDGP, k-mouflage
    // and csf stencils become multiplications (within 1 ulp of the division)
    double rdx2, rdx4, r4dx2;
    // f(R)
    int frn;
    double fr_fct1, fr_fct2, fr_Q2, fr_Q, fr_Q2third, fr_Q4, fr_D11, fr_D20;   // relaxation
    double fr_rt, fr_r1, fr_r2, fr_r3;                                          // residual / rhs
    double fr_r4;                                                               // level-1 restriction
    float f_fct1, f_fct2, f_mQ2, f_Q;   // precision form: fct1, fct2, -Q2, Q rounded to FP32
    float f_r1, f_r2, f_r3, f_rt;       // precision form: residual constants rounded to FP32
    // precision form, other models: FP32 copies of their sweep constants
    float f_dg_fct1, f_dg_alpha2, f_dg_absalpha, f_dg_sa, f_dg_c23, f_dg_c18, f_dg_rdLphi, f_rdx2;
    float f_sy_fct1, f_sy_f3, f_sy_f2, f_sy_fct4;
    float f_km_fct2, f_km_fct4, f_km_fct5, f_km_c3, f_km_dx2ctl, f_r4dx2, f_rdx4;
    float f_cs_fct1, f_cs_beta, f_cs_a1, f_cs_Aphibar, f_cs_Vphibar, f_cs_rphibar, f_rctl2;
    float f_sy_f2r, f_ctl;
    // DGP
    double dg_alpha, dg_fct1, dg_sa, dg_dLphi, dg_fct2, dg_fct3, dg_rdLphi, dg_c23, dg_c18;
    // symmetron
    double sy_fct1, sy_fct4, sy_f2, sy_f3, sy_f2r;
    // k-mouflage (PMP2MGsolver_kmf.f90:49-86)
    int km_n;
    double km_fct2, km_fct3, km_fct4, km_fct5, km_phidot2, ctl, km_dx2ctl;
    // coupled scalar field (PMP2MGsolver_csf.f90:40-62)
    double cs_fct1, cs_Aphibar, cs_Vphibar, cs_Vamp, cs_beta, cs_alpha;
    // prolongation clamp
    int model;
    double phibar, ctl2, rctl2;
};

// first row with a >= AEXPN, then linear interpolation (PMP2MGsolver_kmf.f90:62-77)
double bg_at(const Ctx& c, int col) {
    const std::vector<double>& t = c.h_bg;
    const double a = (double)c.aexpn;
    int ist = 0;
    while (ist < c.bgrows - 1 && t[ist * 6] < a) ++ist;
    if (ist == 0) ist = 1;
    const double* r0 = &t[(ist - 1) * 6];
    const double* r1 = &t[ist * 6];
    return r0[col] + (r1[col] - r0[col]) / (r1[0] - r0[0]) * (a - r0[0]);
}

inline float fcube(float a) { return a * a * a; }
inline float fsq(float a) { return a * a; }
inline double dsign(double a, double b) { return b >= 0.0 ? fabs(a) : -fabs(a); }

LevelConsts make_consts(const Ctx& c, int l) {
    const mgg_config& g = c.cfg;
    const float A = c.aexpn;
    LevelConsts k{};
    k.n = c.N >> l;
    const double dx = (double)(1 << l);
    k.dx2 = dx * dx;
    k.dx4 = k.dx2 * k.dx2;
    k.rdx2 = 1.0 / k.dx2;
    k.rdx4 = 1.0 / k.dx4;
    k.r4dx2 = 1.0 / (4.0 * k.dx2);
    k.model = g.mg_model;
    const double ctl = kCtildeC * (double)c.N / (double)g.box;
    k.ctl2 = ctl * ctl;
    k.rctl2 = 1.0 / k.ctl2;
    k.f_rdx2 = (float)k.rdx2;
    k.f_ctl = (float)ctl;
    if (g.mg_model == MGG_MODEL_FR) {
        k.frn = g.fr_n;
        const double R_bg = 3.0 * ((double)(g.om / fcube(A)) + 4.0 * (double)g.oml);
        const double R0_bg = 3.0 * ((double)g.om + 4.0 * (double)g.oml);
        const double fR_bg = g.fr0 * pow(R0_bg / R_bg, g.fr_n + 1);
        const double s = dsign(1.0, fR_bg), a_fR = fabs(fR_bg);
        // relaxation (PMP2MGsolver_fR.f90:59-73)
        k.fr_fct2 = k.dx2 / (ctl * ctl * s) / 6.0;
        k.fr_fct1 = -((double)(g.om / A) * k.fr_fct2);
        k.fr_Q2 = R_bg * (double)fsq(A) * k.fr_fct2 / 3.0;
        k.fr_Q = k.fr_Q2 * pow(a_fR, 1.0 / ((double)g.fr_n + 1.0));
        k.fr_Q2third = pow(-k.fr_Q, 1.0 / 3.0);
        k.fr_Q4 = 4.0 * k.fr_Q;
        k.fr_D11 = 27.0 * k.fr_Q;
        k.fr_D20 = 12.0 * k.fr_Q;
        // residual and rhs (338-348, 821-825)
        k.fr_rt = pow(a_fR, 1.0 / (double)(g.fr_n + 1));
        k.fr_r1 = (double)(g.om / A);
        k.fr_r2 = -R_bg * (double)fsq(A) / 3.0;
        k.fr_r3 = ctl * ctl * s / k.dx2;
        // level-1 restriction (591-605): fine spacing
        k.fr_r4 = k.fr_r2 * pow(a_fR, 1.0 / (1.0 + (double)g.fr_n));
        k.f_fct1 = (float)k.fr_fct1;
        k.f_fct2 = (float)k.fr_fct2;
        k.f_mQ2 = (float)(-k.fr_Q2);
        k.f_Q = (float)k.fr_Q;
        k.f_r1 = (float)k.fr_r1;
        k.f_r2 = (float)k.fr_r2;
        k.f_r3 = (float)k.fr_r3;
        k.f_rt = (float)k.fr_rt;
    } else if (g.mg_model == MGG_MODEL_DGP) {
        const double Orc = 1.0 / (4.0 * g.h0rc * g.h0rc);
        const double a3d = (double)fcube(A);
        double beta;
        if (g.n_branch) beta = 1.0 + (0.5 * (double)g.om / a3d + (double)g.oml) / sqrt(Orc * (double)(g.om / fcube(A) + g.oml));
        else beta = -(0.5 * (double)g.om / a3d + Orc) / sqrt(Orc * ((double)(g.om / fcube(A)) + Orc));
        const double Rc_sq = 1.0 / (4.0 * Orc);
        k.dg_alpha = 3.0 * beta * (double)fsq(A) / Rc_sq;
        k.dg_fct1 = k.dg_alpha * (double)g.om / beta / (double)A;
        k.dg_sa = dsign(1.0, k.dg_alpha);
        k.dg_dLphi = -6.0 / k.dx2;
        k.dg_rdLphi = 1.0 / k.dg_dLphi;
        k.dg_c23 = (2.0 / 3.0) / k.dx4;
        k.dg_c18 = 0.125 / k.dx4;
        k.f_dg_fct1 = (float)k.dg_fct1;
        k.f_dg_alpha2 = (float)(k.dg_alpha * k.dg_alpha);
        k.f_dg_absalpha = (float)fabs(k.dg_alpha);
        k.f_dg_sa = (float)k.dg_sa;
        k.f_dg_c23 = (float)k.dg_c23;
        k.f_dg_c18 = (float)k.dg_c18;
        k.f_dg_rdLphi = (float)k.dg_rdLphi;
        k.f_rdx2 = (float)k.rdx2;
        k.dg_fct2 = -0.75 * k.dg_alpha;
        k.dg_fct3 = dsign(0.75, k.dg_alpha);
    } else if (g.mg_model == MGG_MODEL_SYMMETRON) {
        const double sa = g.sym_astar / (double)A;
        k.sy_fct1 = sa * sa * sa;
        const double t = ctl * g.sym_xi / (double)A;
        k.sy_fct4 = 2.0 * t * t;
        k.sy_f2 = -k.sy_fct4 / k.dx2;
        k.sy_f3 = k.sy_fct4 / k.dx2 * 6.0;
        const double t2 = (double)A / (ctl * g.sym_xi);
        k.sy_f2r = 0.5 * t2 * t2;
        k.f_sy_fct1 = (float)k.sy_fct1;
        k.f_sy_f3 = (float)k.sy_f3;
        k.f_sy_f2 = (float)k.sy_f2;
        k.f_sy_fct4 = (float)k.sy_fct4;
        k.f_sy_f2r = (float)k.sy_f2r;
    } else if (g.mg_model == MGG_MODEL_KMOUFLAGE) {
        k.km_n = g.kmf_n;
        k.ctl = ctl;
        k.km_dx2ctl = k.dx2 / ctl;
        const double fct1 = 0.5 * pow(1.0 / ((double)A * g.kmf_lambda), 2);
        k.km_fct2 = 3.0 * g.kmf_beta * (double)g.om / (double)A;
        k.km_fct3 = g.kmf_n * g.kmf_k0 * pow(fct1, g.kmf_n - 1);
        k.km_fct4 = -k.km_fct3 * ((double)g.kmf_n - 1.0) * 2.0 * ctl;
        k.km_fct5 = k.km_fct3 * (2.0 * (double)g.kmf_n + 1.0) / 3.0;
        const double phibar = bg_at(c, 1), dphidN = bg_at(c, 2), HoH0 = bg_at(c, 4);
        k.km_fct2 = k.km_fct2 * exp(g.kmf_beta * phibar);
        const double phidot = dphidN * HoH0;
        k.km_phidot2 = phidot * phidot;
        k.f_km_fct2 = (float)k.km_fct2;
        k.f_km_fct4 = (float)k.km_fct4;
        k.f_km_fct5 = (float)k.km_fct5;
        k.f_km_c3 = (float)(k.km_n == 2 ? k.km_fct3 * k.km_phidot2 : k.km_fct3 * k.km_phidot2 * k.km_phidot2);
        k.f_km_dx2ctl = (float)k.km_dx2ctl;
        k.f_r4dx2 = (float)k.r4dx2;
        k.f_rdx4 = (float)k.rdx4;
    } else if (g.mg_model == MGG_MODEL_CSF) {
        k.cs_beta = g.csf_beta;
        k.cs_alpha = g.csf_alpha;
        k.cs_fct1 = 3.0 * (double)g.om / (double)A;
        k.phibar = bg_at(c, 1);
        k.cs_Aphibar = g.csf_beta * exp(g.csf_beta * k.phibar);
        k.cs_Vamp = -g.csf_alpha * g.csf_lambda * g.csf_lambda * (double)fsq(A);
        k.cs_Vphibar = k.cs_Vamp / pow(k.phibar, 1.0 + g.csf_alpha);
        k.f_cs_fct1 = (float)k.cs_fct1;
        k.f_cs_beta = (float)g.csf_beta;
        k.f_cs_a1 = (float)(1.0 + g.csf_alpha);
        k.f_cs_Aphibar = (float)k.cs_Aphibar;
        k.f_cs_Vphibar = (float)k.cs_Vphibar;
        k.f_cs_rphibar = (float)(1.0 / k.phibar);
        k.f_rctl2 = (float)k.rctl2;
        k.f_rdx2 = (float)k.rdx2;
    }
    return k;
}

// ------------------------------------------------------------- helpers -----
struct Nb {
    int64_t c, xu, xl, yu, yl, zu, zl;
};
__device__ __forceinline__ Nb nb6(int i, int j, int k, int n) {
    const int64_t nn = n;
    const int iu = i + 1 == n ? 0 : i + 1, il = i == 0 ? n - 1 : i - 1;
    const int ju = j + 1 == n ? 0 : j + 1, jl = j == 0 ? n - 1 : j - 1;
    const int ku = k + 1 == n ? 0 : k + 1, kl = k == 0 ? n - 1 : k - 1;
    Nb r;
    r.c = i + nn * (j + nn * k);
    r.xu = iu + nn * (j + nn * k);
    r.xl = il + nn * (j + nn * k);
    r.yu = i + nn * (ju + nn * k);
    r.yl = i + nn * (jl + nn * k);
    r.zu = i + nn * (j + nn * ku);
    r.zl = i + nn * (j + nn * kl);
    return r;
}

template <int FRN>
__device__ __forceinline__ float upow(float u) {
    if (FRN == 0) return u;
    if (FRN == 1) return u * u;
    return u * u * u;
}

// Real*4 sum of the six neighbour powers, in the reference's order
template <int FRN>
__device__ __forceinline__ float nbsum_pow(const float* __restrict__ u, const Nb& q) {
    float s = upow<FRN>(u[q.xu]);
    s = s + upow<FRN>(u[q.xl]);
    s = s + upow<FRN>(u[q.yu]);
    s = s + upow<FRN>(u[q.yl]);
    s = s + upow<FRN>(u[q.zu]);
    s = s + upow<FRN>(u[q.zl]);
    return s;
}

// cube root with the sign of x (the reference's DSIGN(DABS(x)**(1/3), x))
__device__ __forceinline__ double scbrt(double x) { return cbrt(x); }

// Roots of the depressed cubic u^3 + P u + Q = 0 as the reference selects them
// (PMP2MGsolver_fR.f90:165-179, PMP2MGsolver_sym.f90:110-129), with
// D0 = -3P, D1 = 27Q, CC = D1^2 - 4 D0^3:
//   CC >= 0 : Cardano, u = -(cbrt(t1) - cbrt(t2))/3, t1 = (sqrt(CC) + D1)/2, t2 = t1 - D1
//   CC <  0 : u = -(2/3) sqrt(D0) cos(acos(c)/3 + 2 pi/3), c = D1 / (2 D0^(3/2))
// Each root is evaluated as an FP32 seed of the same closed form and refined by
// two chord-Newton steps on the cubic in FP64.  Cardano's seed uses
// cbrt(t1) cbrt(t2) = -D0: with T = (D1 + sign(D1) sqrt(CC))/2 (no cancellation)
// and C = cbrt(T), u = -(C + D0/C)/3, so one cube root, taken as
// exp2(log2|T|/3) on the special-function unit, gives a seed with relative
// error ~1e-6.  The chord slope 3u0^2 + P is of order |P| or larger away from
// a double root, so each step multiplies the relative error by ~1e-6 and the
// result equals the closed form to FP64 rounding.  Whenever the seed is not
// finite, leaves [1e-15, 1e15], or sits near a double root, the FP64 closed
// form itself is evaluated.
__device__ __forceinline__ bool f32_ok(float v) {
    const float a = fabsf(v);
    return a < 1.0e30f && (a > 1.0e-30f || a == 0.0f);
}

// Special-function-unit approximations (PTX *.approx.ftz.f32, relative error
// ~2^-22; subnormal inputs and results flush to zero), used only for seeds
// that are refined in FP64 or checked and replaced
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ double chord_refine(double u, double P, double Q) {
    const float uf = (float)u;
    const float fp = 3.0f * uf * uf + (float)P;
    const double r = (double)rcp_approx(fp);   // chord slope: any close value converges
#pragma unroll
    for (int it = 0; it < 2; ++it) {
        const double f = fma(u * u + P, u, Q);
        u = fma(-f, r, u);
    }
    return u;
}

__device__ __noinline__ double cardano_fp64(double CC, double D1) {
    const double tmp1 = 0.5 * (sqrt(CC) + D1);
    const double tmp2 = tmp1 - D1;
    return -(scbrt(tmp1) - scbrt(tmp2)) * (1.0 / 3.0);
}

__device__ __noinline__ double trig_fp64(double D0, double D1) {
    const double sq = sqrt(D0);
    const double S = acos(0.5 * D1 / (sq * sq * sq));
    return -(2.0 / 3.0) * sq * cos(S * (1.0 / 3.0) + 2.0 / 3.0 * 3.141592653589793);
}

__device__ __forceinline__ double cardano_root(double P, double Q, double CC, double D0, double D1) {
    const float D0f = (float)D0, D1f = (float)D1, CCf = (float)CC;
    const float sf = CCf * rsqrt_approx(CCf);               // sqrt(CC) (CC > 0; CC = 0 gives NaN -> FP64)
    const float T = 0.5f * (D1f >= 0.0f ? D1f + sf : D1f - sf);
    const float C = copysignf(ex2_approx(lg2_approx(fabsf(T)) * (1.0f / 3.0f)), T);
    const float u0 = -(C + D0f * rcp_approx(C)) * (1.0f / 3.0f);
    const float au = fabsf(u0);
    const float fp = 3.0f * u0 * u0 + (float)P;
    if (!(au > 1.0e-15f && au < 1.0e15f && fabsf(fp) > 3.0e-3f * u0 * u0)) return cardano_fp64(CC, D1);
    return chord_refine((double)u0, P, Q);
}

__device__ __forceinline__ double trig_root(double P, double Q, double D0, double D1) {
    const float Pf = (float)P, Qf = (float)Q;
    const float sqf = sqrtf(-3.0f * Pf);
    const float cf = 0.5f * (27.0f * Qf) / (sqf * sqf * sqf);
    if (!(f32_ok(Pf) && f32_ok(Qf) && f32_ok(sqf * sqf * sqf) && cf > -1.0f && cf < 0.9f)) return trig_fp64(D0, D1);
    const float y = cosf(acosf(cf) * (1.0f / 3.0f) + 2.09439510239f);
    return chord_refine((double)(-(2.0f / 3.0f) * sqf * y), P, Q);
}

// ------------------------------------------------------------- f(R) -------
// c / u in FP64: an SFU reciprocal seed of u refined by two Newton steps
// (relative error 2^-22 -> 2^-44 -> FP64 rounding), exact division outside
// [1e-30, 1e30]
__device__ __forceinline__ double div_by(double c, float u) {
    const float au = fabsf(u);
    if (!(au > 1.0e-30f && au < 1.0e30f)) return c / (double)u;
    const double ud = (double)u;
    double r = (double)__fdividef(1.0f, u);
    r = fma(r, fma(-ud, r, 1.0), r);
    r = fma(r, fma(-ud, r, 1.0), r);
    return c * r;
}

template <int FRN>
__device__ __forceinline__ double fr_root(double P, const LevelConsts& k) {
    if (FRN == 0) return 0.5 * (-P + sqrt(P * P - k.fr_Q4));
    if (FRN == 1) {
        const double Delta10 = -3.0 * P;
        const double CC = k.fr_D11 * k.fr_D11 - 4.0 * Delta10 * Delta10 * Delta10;
        if (CC >= 0.0) {
            if (fabs(P) < 1.0e-20) return k.fr_Q2third;
            return cardano_root(P, k.fr_Q, CC, Delta10, k.fr_D11);
        }
        return trig_root(P, k.fr_Q, Delta10, k.fr_D11);
    }
    const double Delta21 = 27.0 * P * P;
    const double tmp1 = 0.5 * (sqrt(Delta21 * Delta21 - 4.0 * k.fr_D20 * k.fr_D20 * k.fr_D20) + Delta21);
    const double cr = scbrt(tmp1);
    const double S = sqrt(cr + k.fr_D20 / cr) / sqrt(12.0);
    if (P > 1.0e-20) return -S + 0.5 * sqrt(-4.0 * S * S + P / S);
    if (P < -1.0e-20) return S + 0.5 * sqrt(-4.0 * S * S - P / S);
    return sqrt(sqrt(-k.fr_Q));
}

__device__ __forceinline__ int lg2(int n) { return __ffs(n) - 1; }   // n is a power of two

// idx-th cell of one colour (0: (i+j+k) even, the reference's red M1+M2+M3 odd)
__device__ __forceinline__ void colour_cell(uint32_t idx, int n, int colour, int& i, int& j, int& k) {
    const int lg = lg2(n);
    const uint32_t ih = lg > 0 ? (idx & ((1u << (lg - 1)) - 1u)) : 0u;
    const uint32_t r = lg > 0 ? (idx >> (lg - 1)) : idx;
    j = (int)(r & (uint32_t)(n - 1));
    k = (int)(r >> lg);
    i = 2 * (int)ih + ((j + k + colour) & 1);
}

__device__ __forceinline__ void decode3(uint32_t idx, int n, int& i, int& j, int& k) {
    const int lg = lg2(n);
    const uint32_t m = (uint32_t)(n - 1);
    i = (int)(idx & m);
    j = (int)((idx >> lg) & m);
    k = (int)(idx >> (2 * lg));
}

template <int FRN, bool L0>
__device__ __forceinline__ void relax_fr_cells(float* __restrict__ u, const float* __restrict__ d,
                                               const float* __restrict__ tau, int n, int colour,
                                               const LevelConsts& kc, uint32_t first, uint32_t stride) {
    const uint32_t total = (uint32_t)n * n * (n >> 1);
    for (uint32_t idx = first; idx < total; idx += stride) {
        int i, j, k;
        colour_cell(idx, n, colour, i, j, k);
        const Nb q = nb6(i, j, k, n);
        const float s = nbsum_pow<FRN>(u, q);
        double P = kc.fr_fct1 * (double)d[q.c] - kc.fr_Q2;
        if (!L0) P = P + kc.fr_fct2 * (double)tau[q.c];
        P = P - (double)s * (1.0 / 6.0);
        u[q.c] = (float)fr_root<FRN>(P, kc);
    }
}

template <int FRN, bool L0>
__global__ void k_relax_fr(float* __restrict__ u, const float* __restrict__ d, const float* __restrict__ tau,
                           int n, int colour, LevelConsts kc) {
    relax_fr_cells<FRN, L0>(u, d, tau, n, colour, kc, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

template <int FRN>
__device__ __forceinline__ double fr_op(const float* __restrict__ u, const Nb& q, double dval, const LevelConsts& k) {
    const float s = nbsum_pow<FRN>(u, q);
    const float uc = u[q.c];
    double OP = (double)s - (double)upow<FRN>(uc) * 6.0;
    OP = OP * k.fr_r3;
    OP = OP + k.fr_r1 * dval;
    OP = OP + k.fr_r2 * (div_by(k.fr_rt, uc) - 1.0);
    return OP;
}

// ------------------------------------------------------- k-mouflage -------
// The 19-point neighbourhood (faces and the 12 edge diagonals) of one cell.
struct Nb19 {
    float c, xu, xl, yu, yl, zu, zl;
    float xyPP, xyMM, xyPM, xyMP, xzPP, xzMM, xzPM, xzMP, yzPP, yzMM, yzPM, yzMP;
};

__device__ __forceinline__ Nb19 nb19_global(const float* __restrict__ u, int i, int j, int k, int n) {
    const int64_t nn = n;
    const int iu = i + 1 == n ? 0 : i + 1, il = i == 0 ? n - 1 : i - 1;
    const int ju = j + 1 == n ? 0 : j + 1, jl = j == 0 ? n - 1 : j - 1;
    const int ku = k + 1 == n ? 0 : k + 1, kl = k == 0 ? n - 1 : k - 1;
    auto U = [&](int a, int b, int cc) { return u[a + nn * (b + nn * cc)]; };
    Nb19 r;
    r.c = U(i, j, k);
    r.xu = U(iu, j, k); r.xl = U(il, j, k); r.yu = U(i, ju, k); r.yl = U(i, jl, k); r.zu = U(i, j, ku); r.zl = U(i, j, kl);
    r.xyPP = U(iu, ju, k); r.xyMM = U(il, jl, k); r.xyPM = U(iu, jl, k); r.xyMP = U(il, ju, k);
    r.xzPP = U(iu, j, ku); r.xzMM = U(il, j, kl); r.xzPM = U(iu, j, kl); r.xzMP = U(il, j, ku);
    r.yzPP = U(i, ju, ku); r.yzMM = U(i, jl, kl); r.yzPM = U(i, ju, kl); r.yzMP = U(i, jl, ku);
    return r;
}

// Neighbour sum (Real*4) and the source (fct2 delta + Sigma2)/Sigma1 of
// PMP2MGsolver_kmf.f90:100-173 at one cell.
// r4dx2 = 1 / (4 dx^2), rdx4 = 1 / dx^4 of the spacing the stencil is taken at.
__device__ __forceinline__ double kmf_src(const Nb19& v, double dval, double r4dx2, double rdx4, const LevelConsts& k,
                                          float& qsum) {
    float q = v.xu;
    q = q + v.xl; q = q + v.yu; q = q + v.yl; q = q + v.zu; q = q + v.zl;
    qsum = q;
    const float dx_ = v.xu - v.xl, dy_ = v.yu - v.yl, dz_ = v.zu - v.zl;
    const float t1f = (dx_ * dx_ + dy_ * dy_) + dz_ * dz_;
    const double tmp1 = (double)t1f * r4dx2;
    double Sigma1, Sigma2;
    if (k.km_n == 2) { Sigma1 = k.km_fct5 * tmp1 + k.km_fct3 * k.km_phidot2; Sigma2 = 1.0; }
    else { Sigma1 = k.km_fct5 * tmp1 * tmp1 + k.km_fct3 * k.km_phidot2 * k.km_phidot2; Sigma2 = tmp1; }
    Sigma1 = Sigma1 + 1.0;
    Sigma2 = Sigma2 * k.km_fct4;
    const double X = v.xu, Xl = v.xl, Y = v.yu, Yl = v.yl, Z = v.zu, Zl = v.zl;
    constexpr double r12 = 1.0 / 12.0;
    double tmp2 = (double)(dx_ * dx_) * ((((2.0 * X + 2.0 * Xl) - Y) - Yl - Z) - Zl) * r12 +
                  (double)(dy_ * dy_) * ((((2.0 * Y + 2.0 * Yl) - X) - Xl - Z) - Zl) * r12 +
                  (double)(dz_ * dz_) * ((((2.0 * Z + 2.0 * Zl) - X) - Xl - Y) - Yl) * r12;
    const float axy = ((v.xyPP + v.xyMM) - v.xyPM) - v.xyMP;
    const float axz = ((v.xzPP + v.xzMM) - v.xzPM) - v.xzMP;
    const float ayz = ((v.yzPP + v.yzMM) - v.yzPM) - v.yzMP;
    tmp2 = tmp2 + (double)((axy * dx_) * dy_) / 8.0 + (double)((axz * dx_) * dz_) / 8.0 + (double)((ayz * dy_) * dz_) / 8.0;
    tmp2 = tmp2 * rdx4;
    Sigma2 = Sigma2 * tmp2;
    return (k.km_fct2 * dval + Sigma2) / Sigma1;
}

__device__ __forceinline__ double kmf_op(const Nb19& v, double dval, const LevelConsts& k) {
    float qs;
    const double src = kmf_src(v, dval, k.r4dx2, k.rdx4, k, qs);
    double OP = (double)qs - (double)v.c * 6.0;
    OP = OP * k.rdx2 * k.ctl;
    return OP - src;
}

template <bool L0>
// one colour sweep src (us) -> dst (u), other colour copied (as k_relax_dgp)
__device__ __forceinline__ void relax_kmf_cells(float* __restrict__ u, const float* __restrict__ us,
                                                const float* __restrict__ d, const float* __restrict__ tau, int n,
                                                int colour, const LevelConsts& kc, uint32_t first, uint32_t stride) {
    const uint32_t total = (uint32_t)n * n * (n >> 1);
    for (uint32_t idx = first; idx < total; idx += stride) {
        int i, j, k;
        colour_cell(idx, n, colour, i, j, k);
        const int64_t q = i + (int64_t)n * (j + (int64_t)n * k);
        const int64_t partner = q + ((i & 1) ? -1 : 1);
        u[partner] = us[partner];
        const Nb19 v = nb19_global(us, i, j, k, n);
        float qs;
        const double src = kmf_src(v, (double)d[q], kc.r4dx2, kc.rdx4, kc, qs);
        const double Q = L0 ? (double)qs : -(double)tau[q] * kc.km_dx2ctl + (double)qs;
        const double P = src * kc.km_dx2ctl;
        u[q] = (float)((Q - P) * (1.0 / 6.0));
    }
}

template <bool L0>
__global__ void k_relax_kmf(float* __restrict__ u, const float* __restrict__ us, const float* __restrict__ d,
                            const float* __restrict__ tau, int n, int colour, LevelConsts kc) {
    relax_kmf_cells<L0>(u, us, d, tau, n, colour, kc, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ------------------------------------------------ coupled scalar field -----
// A'(phi) and V'(phi) at phi = phibar + u / c~^2 (PMP2MGsolver_csf.f90:96-117)
__device__ __forceinline__ void csf_phi(double uval, const LevelConsts& k, double& phi, double& A_phi, double& V_phi) {
    phi = k.phibar + uval * k.rctl2;
    A_phi = k.cs_beta * exp(k.cs_beta * phi);
    V_phi = k.cs_Vamp / pow(phi, 1.0 + k.cs_alpha);
}

// Newton update of one cell (PMP2MGsolver_csf.f90:96-150)
template <bool L0>
__device__ __forceinline__ void relax_csf_cells(float* __restrict__ u, const float* __restrict__ d,
                                                const float* __restrict__ tau, int n, int colour,
                                                const LevelConsts& kc, uint32_t first, uint32_t stride) {
    const uint32_t total = (uint32_t)n * n * (n >> 1);
    for (uint32_t idx = first; idx < total; idx += stride) {
        int i, j, k;
        colour_cell(idx, n, colour, i, j, k);
        const Nb q = nb6(i, j, k, n);
        const float uc = u[q.c];
        double L;
        if (L0) {
            float s = u[q.xu];
            s = s + u[q.xl]; s = s + u[q.yu]; s = s + u[q.yl]; s = s + u[q.zu]; s = s + u[q.zl];
            L = (double)s - (double)uc * 6.0;
        } else {
            L = -(double)tau[q.c] * kc.dx2 + (double)u[q.xu];
            L = L + (double)u[q.xl]; L = L + (double)u[q.yu]; L = L + (double)u[q.yl];
            L = L + (double)u[q.zu]; L = L + (double)u[q.zl]; L = L - (double)uc * 6.0;
        }
        double phi, A_phi, V_phi;
        csf_phi((double)uc, kc, phi, A_phi, V_phi);
        const double rho = (double)d[q.c] + 1.0;
        const double A_pp = kc.cs_beta * A_phi * kc.rctl2;
        const double V_pp = -(1.0 + kc.cs_alpha) * V_phi * kc.rctl2 / phi;
        L = L * kc.rdx2;
        L = L - kc.cs_fct1 * (A_phi * rho - kc.cs_Aphibar);
        L = L - (V_phi - kc.cs_Vphibar);
        const double dL = -6.0 * kc.rdx2 - kc.cs_fct1 * rho * A_pp - V_pp;
        u[q.c] = (float)((double)uc - L / dL);
    }
}

template <bool L0>
__global__ void k_relax_csf(float* __restrict__ u, const float* __restrict__ d, const float* __restrict__ tau, int n,
                            int colour, LevelConsts kc) {
    relax_csf_cells<L0>(u, d, tau, n, colour, kc, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// Residual (tau subtracted first, level > 0) and coarse-grid operator
// (PMP2MGsolver_csf.f90:179-353, 574-686).  s is the Real*4 neighbour sum.
__device__ __forceinline__ double csf_op(float uc, float s, double dval, const LevelConsts& k) {
    const double OP = ((double)s - (double)uc * 6.0) * k.rdx2;
    double phi, A_phi, V_phi;
    csf_phi((double)uc, k, phi, A_phi, V_phi);
    double r = OP - k.cs_fct1 * (A_phi * (dval + 1.0) - k.cs_Aphibar);
    return r - (V_phi - k.cs_Vphibar);
}
__device__ __forceinline__ double csf_res(float uc, float s, double dval, double tval, const LevelConsts& k) {
    double OP = ((double)s - (double)uc * 6.0) * k.rdx2;
    OP = OP - tval;
    double phi, A_phi, V_phi;
    csf_phi((double)uc, k, phi, A_phi, V_phi);
    OP = OP - k.cs_fct1 * (A_phi * (dval + 1.0) - k.cs_Aphibar);
    return OP - (V_phi - k.cs_Vphibar);
}

// ------------------------------------------------------------- nDGP -------
__device__ __forceinline__ double dgp_sigma(const float* __restrict__ u, int i, int j, int k, int n,
                                            const LevelConsts& kc, double base) {
    const int64_t nn = n;
    const int iu = i + 1 == n ? 0 : i + 1, il = i == 0 ? n - 1 : i - 1;
    const int ju = j + 1 == n ? 0 : j + 1, jl = j == 0 ? n - 1 : j - 1;
    const int ku = k + 1 == n ? 0 : k + 1, kl = k == 0 ? n - 1 : k - 1;
    auto U = [&](int a, int b, int c) { return u[a + nn * (b + nn * c)]; };
    const double uc2 = 2.0 * (double)U(i, j, k);
    const double dxx = (double)(U(iu, j, k) + U(il, j, k)) - uc2;
    const double dyy = (double)(U(i, ju, k) + U(i, jl, k)) - uc2;
    const double dzz = (double)(U(i, j, ku) + U(i, j, kl)) - uc2;
    const float dxy = ((U(iu, ju, k) + U(il, jl, k)) - U(iu, jl, k)) - U(il, ju, k);
    const float dxz = ((U(iu, j, ku) + U(il, j, kl)) - U(iu, j, kl)) - U(il, j, ku);
    const float dyz = ((U(i, ju, ku) + U(i, jl, kl)) - U(i, ju, kl)) - U(i, jl, ku);
    const float diag = (dxy * dxy + dxz * dxz) + dyz * dyz;
    return base + (dxx * dxx + dyy * dyy + dzz * dzz) * kc.dg_c23 - (dxx * dyy + dxx * dzz + dyy * dzz) * kc.dg_c23 +
           (double)diag * kc.dg_c18;
}

__device__ __forceinline__ double lap7(const float* __restrict__ u, const Nb& q) {
    float s = u[q.xu];
    s = s + u[q.xl];
    s = s + u[q.yu];
    s = s + u[q.yl];
    s = s + u[q.zu];
    s = s + u[q.zl];
    return (double)s - (double)u[q.c] * 6.0;
}

__device__ __forceinline__ double dgp_op(const float* __restrict__ u, const Nb& q, int i, int j, int k, int n, double dval,
                                         const LevelConsts& kc) {
    const double Sigma = dgp_sigma(u, i, j, k, n, kc, kc.dg_fct1 * dval);
    double OP = lap7(u, q) * kc.rdx2;
    OP = OP - (kc.dg_sa * sqrt(kc.dg_alpha * kc.dg_alpha + 8.0 / 3.0 * Sigma) - kc.dg_alpha) * 0.75;
    return OP;
}

template <bool L0>
// One colour sweep from src into dst: cells of the colour are updated from src
// (same-colour diagonal neighbours included, as they were before the sweep),
// each thread also copies the other-colour cell of its x pair, so a red sweep
// U -> snap and a black sweep snap -> U leave the result in U without a
// separate snapshot copy.
__device__ __forceinline__ void relax_dgp_cells(float* __restrict__ u, const float* __restrict__ us,
                                                const float* __restrict__ d, const float* __restrict__ tau, int n,
                                                int colour, const LevelConsts& kc, uint32_t first, uint32_t stride) {
    const uint32_t total = (uint32_t)n * n * (n >> 1);
    for (uint32_t idx = first; idx < total; idx += stride) {
        int i, j, k;
        colour_cell(idx, n, colour, i, j, k);
        const Nb q = nb6(i, j, k, n);
        const int64_t partner = q.c + ((i & 1) ? -1 : 1);
        u[partner] = us[partner];
        double L = dgp_op(us, q, i, j, k, n, (double)d[q.c], kc);
        if (!L0) L = L - (double)tau[q.c];
        u[q.c] = (float)((double)us[q.c] - L * kc.dg_rdLphi);
    }
}

template <bool L0>
__global__ void k_relax_dgp(float* __restrict__ u, const float* __restrict__ us, const float* __restrict__ d,
                            const float* __restrict__ tau, int n, int colour, LevelConsts kc) {
    relax_dgp_cells<L0>(u, us, d, tau, n, colour, kc, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// -------------------------------------------------------- symmetron -------
__device__ __forceinline__ double sym_op(const float* __restrict__ u, const Nb& q, double dval, const LevelConsts& kc) {
    const float uc = u[q.c];
    double OP = lap7(u, q) / kc.dx2;
    OP = OP - kc.sy_f2r * (kc.sy_fct1 * (dval + 1.0) - 1.0) * (double)uc;
    OP = OP - kc.sy_f2r * (double)(uc * uc * uc);
    return OP;
}

template <bool L0>
__device__ __forceinline__ void relax_sym_cells(float* __restrict__ u, const float* __restrict__ d,
                                                const float* __restrict__ tau, int n, int colour,
                                                const LevelConsts& kc, uint32_t first, uint32_t stride) {
    const uint32_t total = (uint32_t)n * n * (n >> 1);
    for (uint32_t idx = first; idx < total; idx += stride) {
        int i, j, k;
        colour_cell(idx, n, colour, i, j, k);
        const Nb q = nb6(i, j, k, n);
        float s = u[q.xu];
        s = s + u[q.xl];
        s = s + u[q.yu];
        s = s + u[q.yl];
        s = s + u[q.zu];
        s = s + u[q.zl];
        const double P = kc.sy_fct1 * ((double)d[q.c] + 1.0) - 1.0 + kc.sy_f3;
        const double Q = L0 ? kc.sy_f2 * (double)s : kc.sy_fct4 * (double)tau[q.c] + kc.sy_f2 * (double)s;
        const double D0 = -3.0 * P, D1 = 27.0 * Q;
        const double CC = D1 * D1 - 4.0 * D0 * D0 * D0;
        double val;
        if (CC >= 0.0) {
            if (fabs(P) < 1.0e-20) val = -scbrt(Q);
            else val = cardano_root(P, Q, CC, D0, D1);
        } else {
            val = trig_root(P, Q, D0, D1);
        }
        u[q.c] = (float)val;
    }
}

template <bool L0>
__global__ void k_relax_sym(float* __restrict__ u, const float* __restrict__ d, const float* __restrict__ tau, int n,
                            int colour, LevelConsts kc) {
    relax_sym_cells<L0>(u, d, tau, n, colour, kc, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ------------------------------------------------ fused red-black sweep ----
// One smoothing iteration (red pass, then black pass) of a 7-point model in a
// single sweep.  A block owns an interior tile of FB_X x FB_Y cells in x-y and a
// chunk of planes in z, and marches up the chunk keeping five planes of the
// field (with a 2-cell halo) in a shared-memory ring.  Step m has two phases:
//   A: red cells of plane m (tile and its 1-cell ring) and black cells of
//      plane m-2 (tile), side by side;
//   B: write plane m-2; plane m+2 (prefetched into registers during A)
//      replaces plane m-3 in the ring.
// Red(m) reads only old black values (black(m-1) comes one step later) and
// black(m-2) only new red values of planes m-3 .. m-1, so every cell gets
// exactly the arithmetic of the two separate passes, with two barriers per
// plane.  The result goes to a second buffer (blocks read halos that other
// blocks own), so two calls per smoothing step return the field to its buffer.
// Each interior thread updates two cells of a colour per plane, 64 apart in x.
constexpr int FB_X = 128, FB_Y = 16, FB_PX = FB_X + 4, FB_PY = FB_Y + 4, FB_PLANE = FB_PX * FB_PY;
constexpr int FB_HALO_RED = 2 * (FB_X + 2) / 2 + FB_Y;   // red cells on the 1-cell ring per plane (146)
constexpr int FB_INNER = FB_X / 4 * FB_Y;                // two interior updates per thread (512 threads)
constexpr int FB_THREADS = FB_INNER + 160;               // + 5 warps for the ring
constexpr int FB_PREF = (FB_PLANE / 2 + FB_THREADS - 1) / FB_THREADS;   // float2 prefetches per thread
constexpr int FB_OUT4 = FB_X * FB_Y / 4;                 // float4 stores of one interior plane (512)
constexpr int FB_SMEM = 5 * FB_PLANE * (int)sizeof(float);   // 52800 B of dynamic shared memory

// Precision form (MGG_PREC_MIXED), f(R) n = 1 and symmetron: the largest root
// of u^3 + P u + Q = 0 by Newton's method in FP32, from the cell's current
// value.  That is the root the reference's closed form returns: Cardano's
// single real root when CC >= 0, and for CC < 0 the trigonometric form
// -(2/3) sqrt(-3P) cos(acos(c)/3 + 2 pi/3), which lies in
// [sqrt(-P/3), 2 sqrt(-P/3)], right of the local minimum.
// To the right of the local minimum (3u^2 + P > 0) the cubic is convex, so
// Newton converges to that root from any such start, quadratically with
// eps' <= 3.3 eps^2 while 3u^2 + P >= 0.9 u^2: a step below 1e-4 u leaves an
// error below FP32 rounding.  Returns NaN when the start is outside that region
// or five steps do not converge; the caller then takes the FP64 closed form.
__device__ __forceinline__ float cubic_root_newton32(float u, float P, float Q) {
    if (!(u > 0.0f && u < 1.0e15f && fmaf(2.1f * u, u, P) > 0.0f)) return __int_as_float(0x7fffffff);
#pragma unroll 1
    for (int it = 0; it < 5; ++it) {
        const float fp = fmaf(3.0f * u, u, P);
        const float f = fmaf(fmaf(u, u, P), u, Q);
        const float du = f * rcp_approx(fp);
        u = u - du;
        if (fabsf(du) <= 1.0e-4f * u) return u;
    }
    return __int_as_float(0x7fffffff);
}

// Precision form, f(R) n = 2: the positive root of u^4 + P u + Q = 0 (Q < 0),
// the root the reference's Ferrari closed form returns, by Newton's method in
// FP32 from the cell's current value.  The quartic is convex with one positive
// root; right of its minimum (4u^3 + P > 0) Newton converges from any start,
// with eps' <= 5 eps^2 while 4u^3 + P >= 1.2 u^3.  NaN when the start is
// unusable or five steps do not converge.
__device__ __forceinline__ float quartic_root_newton32(float u, float P, float Q) {
    if (!(u > 0.0f && u < 1.0e10f && fmaf(2.8f * u * u, u, P) > 0.0f)) return __int_as_float(0x7fffffff);
#pragma unroll 1
    for (int it = 0; it < 5; ++it) {
        const float u2 = u * u;
        const float fp = fmaf(4.0f * u2, u, P);
        const float f = fmaf(fmaf(u2, u, P), u, Q);
        const float du = f * rcp_approx(fp);
        u = u - du;
        if (fabsf(du) <= 1.0e-4f * u) return u;
    }
    return __int_as_float(0x7fffffff);
}

// One cell of the precision-form f(R) sweep: P in FP32 from the FP32
// neighbour sum, then the root in FP32 -- n = 0: the larger root of
// u^2 + P u + Q in the cancellation-free closed form; n = 1, 2: Newton from the
// cell's value -- with the FP64 closed form of the plain path when the Newton
// start is unusable.
template <int FRN, bool L0>
__device__ __forceinline__ float fr_update_mixed(float s, float uold, float dvf, float tvf, const LevelConsts& kc) {
    float P = fmaf(kc.f_fct1, dvf, kc.f_mQ2);
    if (!L0) P = fmaf(kc.f_fct2, tvf, P);
    P = fmaf(s, -1.0f / 6.0f, P);
    float u;
    if (FRN == 0) {
        const float r = sqrtf(fmaf(P, P, -4.0f * kc.f_Q));
        u = P <= 0.0f ? 0.5f * (r - P) : -2.0f * kc.f_Q / (P + r);
    } else if (FRN == 1) {
        u = cubic_root_newton32(uold, P, kc.f_Q);
    } else {
        u = quartic_root_newton32(uold, P, kc.f_Q);
    }
    if (u == u) return u;
    double Pd = kc.fr_fct1 * (double)dvf - kc.fr_Q2;
    if (!L0) Pd = Pd + kc.fr_fct2 * (double)tvf;
    Pd = Pd - (double)s * (1.0 / 6.0);
    return (float)fr_root<FRN>(Pd, kc);
}

// One cell of a 7-point red-black sweep from its six neighbours (the reference's
// order x+, x-, y+, y-, z+, z-), its own value c0 (the Newton start of the
// precision form), its density dvf and FAS right-hand side tvf.
template <int MODEL, int FRN, bool L0, bool MIX>
__device__ __forceinline__ float cell_update(float nxu, float nxl, float nyu, float nyl, float nzu, float nzl,
                                             float c0, float dvf, float tvf, const LevelConsts& kc) {
    const double dval = (double)dvf, tval = (double)tvf;
    if (MODEL == MGG_MODEL_FR) {
        float s = upow<FRN>(nxu);
        s = s + upow<FRN>(nxl);
        s = s + upow<FRN>(nyu);
        s = s + upow<FRN>(nyl);
        s = s + upow<FRN>(nzu);
        s = s + upow<FRN>(nzl);
        if (MIX) return fr_update_mixed<FRN, L0>(s, c0, dvf, tvf, kc);
        double P = kc.fr_fct1 * dval - kc.fr_Q2;
        if (!L0) P = P + kc.fr_fct2 * tval;
        P = P - (double)s * (1.0 / 6.0);
        return (float)fr_root<FRN>(P, kc);
    } else {
        float s = nxu;
        s = s + nxl;
        s = s + nyu;
        s = s + nyl;
        s = s + nzu;
        s = s + nzl;
        if (MIX) {   // precision form: FP32 P and Q, FP32 Newton root (the closed form's largest root)
            const float Pf = fmaf(kc.f_sy_fct1, dvf + 1.0f, -1.0f) + kc.f_sy_f3;
            const float Qf = L0 ? kc.f_sy_f2 * s : fmaf(kc.f_sy_fct4, tvf, kc.f_sy_f2 * s);
            const float u = cubic_root_newton32(c0, Pf, Qf);
            if (u == u) return u;
        }
        const double P = kc.sy_fct1 * (dval + 1.0) - 1.0 + kc.sy_f3;
        const double Q = L0 ? kc.sy_f2 * (double)s : kc.sy_fct4 * tval + kc.sy_f2 * (double)s;
        const double D0 = -3.0 * P, D1 = 27.0 * Q;
        const double CC = D1 * D1 - 4.0 * D0 * D0 * D0;
        if (CC >= 0.0) {
            if (fabs(P) < 1.0e-20) return (float)(-scbrt(Q));
            return (float)cardano_root(P, Q, CC, D0, D1);
        }
        return (float)trig_root(P, Q, D0, D1);
    }
}

template <int MODEL, int FRN, bool L0, bool MIX>
__device__ __forceinline__ float fused_update(const float* __restrict__ S0, const float* __restrict__ Sm,
                                              const float* __restrict__ Sp, int p, float dvf, float tvf,
                                              const LevelConsts& kc) {
    return cell_update<MODEL, FRN, L0, MIX>(S0[p + 1], S0[p - 1], S0[p + FB_PX], S0[p - FB_PX], Sp[p], Sm[p],
                                            MIX ? S0[p] : 0.0f, dvf, tvf, kc);
}

// f(R) with n = 1 fits 32 registers: three blocks (63 warps) per SM
// three blocks per SM (32 registers) for the f(R) n = 1 smoother; on the coarse
// levels (which also load tau) the precision form at two blocks (40 registers)
// measured 1-2 % faster
template <int MODEL, int FRN, bool L0, bool MIX>
constexpr int fb_min_blocks() { return (MODEL == MGG_MODEL_FR && FRN == 1 && (L0 || !MIX)) ? 3 : 2; }

template <int MODEL, int FRN, bool L0, bool MIX = false>
__global__ void __launch_bounds__(FB_THREADS, fb_min_blocks<MODEL, FRN, L0, MIX>()) k_smooth_fused(
    const float* __restrict__ uin, float* __restrict__ uout, const float* __restrict__ d, const float* __restrict__ tau,
    int n, int cz, LevelConsts kc) {
    extern __shared__ __align__(16) float S[];   // FB_SMEM bytes: five padded planes
    const int x0 = blockIdx.x * FB_X, y0 = blockIdx.y * FB_Y, kbeg = blockIdx.z * cz, kend = kbeg + cz;
    const int nm = n - 1;
    const int plane = n * n;   // offsets fit 32 bits: n^3 <= 2^30
    const int tid = threadIdx.x;
    // x-y offsets (periodic) of this thread's float2 pairs of a padded plane; pairs
    // start at even x, so they never straddle the periodic wrap
    int pxy[FB_PREF], sxy[FB_PREF];
#pragma unroll
    for (int i = 0; i < FB_PREF; ++i) {
        const int e = min(tid + i * FB_THREADS, FB_PLANE / 2 - 1);
        const int yy = e / (FB_PX / 2), xx = 2 * (e - yy * (FB_PX / 2));
        pxy[i] = ((x0 + xx - 2) & nm) + n * ((y0 + yy - 2) & nm);
        sxy[i] = yy * FB_PX + xx;
    }
    // planes kbeg-2 .. kbeg go to ring slots 2, 3, 4 (planes m-1, m, m+1 of the
    // first step m = kbeg - 1)
    for (int z = kbeg - 2; z <= kbeg; ++z) {
        const float* uz = uin + (z & nm) * plane;
        float* Sz = S + (z - kbeg + 4) * FB_PLANE;
#pragma unroll
        for (int i = 0; i < FB_PREF; ++i)
            if (tid + i * FB_THREADS < FB_PLANE / 2)
                *reinterpret_cast<float2*>(Sz + sxy[i]) = __ldg(reinterpret_cast<const float2*>(uz + pxy[i]));
    }
    const bool inner = tid < FB_INNER;
    const int w = tid >> 5, lane = tid & 31;
    // interior cells of this thread: x = 2 lane + parity (+ 64), y = w (no wrap inside the tile)
    const int ixy = x0 + 2 * lane + n * (y0 + w);
    const int ip = (w + 2) * FB_PX + 2 * lane + 2;
    const int h = tid - FB_INNER;   // ring cell index of warps 16..20
    // this thread's float4 of the interior plane for the write-out
    const int oy = tid >> 5, ox = 4 * (tid & 31);
    const int oxy = (x0 + ox) + n * (y0 + oy), osm = (oy + 2) * FB_PX + ox + 2;
    float2 pre[FB_PREF];
    // One step m with the ring slots (float offsets into S) of planes m-3, m-2,
    // m-1, m, m+1: (j + 0..4) mod 5 planes with j = m - kbeg + 1.  The
    // precision-form sweeps run five steps per loop iteration and pass the slots
    // as compile-time constants; the plain sweeps (whose FP64 closed-form root is
    // the main path, five copies of which slowed the whole run) keep one step per
    // iteration and rotate the slots in registers.
    auto step = [&](int m, auto oE, auto oA, auto oB, auto oC, auto oD) {
        const bool fetch = m + 2 <= kend + 1;
        if (fetch) {
            const float* uz = uin + ((m + 2) & nm) * plane;
#pragma unroll
            for (int i = 0; i < FB_PREF; ++i)
                if (tid + i * FB_THREADS < FB_PLANE / 2) pre[i] = __ldg(reinterpret_cast<const float2*>(uz + pxy[i]));
        }
        __syncthreads();
        // phase A
        const bool black = m >= kbeg + 2;   // black cells of plane m-2 (its last red neighbour came at m-1)
        if (inner) {
            if (m <= kend) {   // red cells of plane m: (x0 + x + y0 + y + m) even, x0 even
                const int par = (y0 + w + m) & 1;
                const int g = (m & nm) * plane + ixy + par, p = ip + par;
                const float dv0 = __ldg(d + g), dv1 = __ldg(d + g + 64);
                const float tv0 = L0 ? 0.f : __ldg(tau + g), tv1 = L0 ? 0.f : __ldg(tau + g + 64);
                S[oC + p] = fused_update<MODEL, FRN, L0, MIX>(S + oC, S + oB, S + oD, p, dv0, tv0, kc);
                S[oC + p + 64] = fused_update<MODEL, FRN, L0, MIX>(S + oC, S + oB, S + oD, p + 64, dv1, tv1, kc);
            }
            if (black) {       // black cells of plane m-2: (x + y + z) odd
                const int par = (y0 + w + m - 1) & 1;
                const int g = ((m - 2) & nm) * plane + ixy + par, p = ip + par;
                const float dv0 = __ldg(d + g), dv1 = __ldg(d + g + 64);
                const float tv0 = L0 ? 0.f : __ldg(tau + g), tv1 = L0 ? 0.f : __ldg(tau + g + 64);
                S[oA + p] = fused_update<MODEL, FRN, L0, MIX>(S + oA, S + oE, S + oB, p, dv0, tv0, kc);
                S[oA + p + 64] = fused_update<MODEL, FRN, L0, MIX>(S + oA, S + oE, S + oB, p + 64, dv1, tv1, kc);
            }
        } else if (h < FB_HALO_RED && m <= kend) {
            int x, y;
            if (h < FB_X + 2) {               // rows y = -1 and y = FB_Y
                const int r = h / ((FB_X + 2) / 2), col = h - r * ((FB_X + 2) / 2);
                y = r == 0 ? -1 : FB_Y;
                x = -1 + 2 * col + (((y0 + y + m) & 1) ^ 1);
            } else {                          // columns x = -1 / FB_X
                y = h - (FB_X + 2);
                x = ((y0 + y + m) & 1) ? -1 : FB_X;
            }
            const int p = (y + 2) * FB_PX + (x + 2);
            const int g = (m & nm) * plane + ((x0 + x) & nm) + n * ((y0 + y) & nm);
            const float dv = __ldg(d + g), tv = L0 ? 0.f : __ldg(tau + g);
            S[oC + p] = fused_update<MODEL, FRN, L0, MIX>(S + oC, S + oB, S + oD, p, dv, tv, kc);
        }
        __syncthreads();
        // phase B
        if (black && tid < FB_OUT4) {
            const float2 a = *reinterpret_cast<const float2*>(S + oA + osm);
            const float2 b = *reinterpret_cast<const float2*>(S + oA + osm + 2);
            *reinterpret_cast<float4*>(uout + ((m - 2) & nm) * plane + oxy) = make_float4(a.x, a.y, b.x, b.y);
        }
        if (fetch) {   // plane m+2 goes to the slot of plane m-3, last read by black(m-2)
#pragma unroll
            for (int i = 0; i < FB_PREF; ++i)
                if (tid + i * FB_THREADS < FB_PLANE / 2) *reinterpret_cast<float2*>(S + oE + sxy[i]) = pre[i];
        }
    };
    if constexpr (MIX) {
        using S0 = std::integral_constant<int, 0>;
        using S1 = std::integral_constant<int, FB_PLANE>;
        using S2 = std::integral_constant<int, 2 * FB_PLANE>;
        using S3 = std::integral_constant<int, 3 * FB_PLANE>;
        using S4 = std::integral_constant<int, 4 * FB_PLANE>;
        for (int m = kbeg - 1; m <= kend + 1; m += 5) {
            step(m, S0{}, S1{}, S2{}, S3{}, S4{});
            if (m + 1 > kend + 1) break;
            step(m + 1, S1{}, S2{}, S3{}, S4{}, S0{});
            if (m + 2 > kend + 1) break;
            step(m + 2, S2{}, S3{}, S4{}, S0{}, S1{});
            if (m + 3 > kend + 1) break;
            step(m + 3, S3{}, S4{}, S0{}, S1{}, S2{});
            if (m + 4 > kend + 1) break;
            step(m + 4, S4{}, S0{}, S1{}, S2{}, S3{});
        }
    } else {
        int oE = 0, oA = FB_PLANE, oB = 2 * FB_PLANE, oC = 3 * FB_PLANE, oD = 4 * FB_PLANE;
        for (int m = kbeg - 1; m <= kend + 1; ++m) {
            step(m, oE, oA, oB, oC, oD);
            const int t = oE;
            oE = oA;
            oA = oB;
            oB = oC;
            oC = oD;
            oD = t;
        }
    }
}

// ---------------------------------------------- marching operator pass ----
// The residual (level 0: squared-norm partials; level > 0: coarse residual)
// and the FAS right-hand side evaluate the model operator on every cell.  A
// block owns a 128 x 16 tile and marches up a chunk of planes with three planes
// (1-cell halo) in a shared-memory ring, so each field value comes from DRAM
// once; the arithmetic per cell is the same as k_resid / k_rhs.
constexpr int OP_X = 128, OP_Y = 16, OP_PX = OP_X + 4, OP_PY = OP_Y + 2, OP_PLANE = OP_PX * OP_PY;
constexpr int OP_CPT = 4, OP_T = OP_X / OP_CPT * OP_Y;   // four cells per thread, 32 apart in x
enum { OPM_NORM = 0, OPM_RES = 1, OPM_RHS = 2, OPM_SWEEP = 3 };

// the 19-point neighbourhood of smem cell p from three padded planes
__device__ __forceinline__ Nb19 nb19_smem(const float* __restrict__ Sm, const float* __restrict__ S0,
                                          const float* __restrict__ Sp, int p) {
    Nb19 r;
    r.c = S0[p];
    r.xu = S0[p + 1]; r.xl = S0[p - 1]; r.yu = S0[p + OP_PX]; r.yl = S0[p - OP_PX]; r.zu = Sp[p]; r.zl = Sm[p];
    r.xyPP = S0[p + 1 + OP_PX]; r.xyMM = S0[p - 1 - OP_PX]; r.xyPM = S0[p + 1 - OP_PX]; r.xyMP = S0[p - 1 + OP_PX];
    r.xzPP = Sp[p + 1]; r.xzMM = Sm[p - 1]; r.xzPM = Sm[p + 1]; r.xzMP = Sp[p - 1];
    r.yzPP = Sp[p + OP_PX]; r.yzMM = Sm[p - OP_PX]; r.yzPM = Sm[p + OP_PX]; r.yzMP = Sp[p - OP_PX];
    return r;
}

// Precision form, f(R) n = 1: the operator of calculate_residual_fR
// (PMP2MGsolver_fR.f90:338-348) in FP32.  s - 6 u^2 is formed with the rounding
// error of u^2 carried by an FMA, so the cancellation of the Laplacian costs no
// more than the FP32 neighbour sum itself; the norm keeps its FP64 accumulation.
__device__ __forceinline__ float fr1_op_f32(float s, float uc, float dval, const LevelConsts& k) {
    const float p = uc * uc;
    const float e = fmaf(uc, uc, -p);
    const float lap = fmaf(-6.0f, e, fmaf(-6.0f, p, s));
    const float ratio = k.f_rt * __frcp_rn(uc);
    return fmaf(lap, k.f_r3, fmaf(k.f_r1, dval, k.f_r2 * (ratio - 1.0f)));
}

template <int MODEL, int FRN>
__device__ __forceinline__ double op_smem(const float* __restrict__ Sm, const float* __restrict__ S0,
                                          const float* __restrict__ Sp, int p, double dval, const LevelConsts& k) {
    const float uc = S0[p];
    const float nxu = S0[p + 1], nxl = S0[p - 1], nyu = S0[p + OP_PX], nyl = S0[p - OP_PX], nzu = Sp[p], nzl = Sm[p];
    if (MODEL == MGG_MODEL_FR) {
        float s = upow<FRN>(nxu);
        s = s + upow<FRN>(nxl);
        s = s + upow<FRN>(nyu);
        s = s + upow<FRN>(nyl);
        s = s + upow<FRN>(nzu);
        s = s + upow<FRN>(nzl);
        double OP = (double)s - (double)upow<FRN>(uc) * 6.0;
        OP = OP * k.fr_r3;
        OP = OP + k.fr_r1 * dval;
        OP = OP + k.fr_r2 * (div_by(k.fr_rt, uc) - 1.0);
        return OP;
    }
    float s = nxu;
    s = s + nxl;
    s = s + nyu;
    s = s + nyl;
    s = s + nzu;
    s = s + nzl;
    const double lap = (double)s - (double)uc * 6.0;
    if (MODEL == MGG_MODEL_SYMMETRON) {
        double OP = lap / k.dx2;
        OP = OP - k.sy_f2r * (k.sy_fct1 * (dval + 1.0) - 1.0) * (double)uc;
        OP = OP - k.sy_f2r * (double)(uc * uc * uc);
        return OP;
    }
    if (MODEL == MGG_MODEL_KMOUFLAGE) return kmf_op(nb19_smem(Sm, S0, Sp, p), dval, k);
    if (MODEL == MGG_MODEL_CSF) return csf_op(uc, s, dval, k);
    // nDGP: Sigma of PMP2MGsolver_DGP.f90:305-317
    const double uc2 = 2.0 * (double)uc;
    const double dxx = (double)(nxu + nxl) - uc2, dyy = (double)(nyu + nyl) - uc2, dzz = (double)(nzu + nzl) - uc2;
    const float dxy = ((S0[p + 1 + OP_PX] + S0[p - 1 - OP_PX]) - S0[p + 1 - OP_PX]) - S0[p - 1 + OP_PX];
    const float dxz = ((Sp[p + 1] + Sm[p - 1]) - Sm[p + 1]) - Sp[p - 1];
    const float dyz = ((Sp[p + OP_PX] + Sm[p - OP_PX]) - Sm[p + OP_PX]) - Sp[p - OP_PX];
    const float diag = (dxy * dxy + dxz * dxz) + dyz * dyz;
    const double Sigma = k.dg_fct1 * dval + (dxx * dxx + dyy * dyy + dzz * dzz) * k.dg_c23 -
                         (dxx * dyy + dxx * dzz + dyy * dzz) * k.dg_c23 + (double)diag * k.dg_c18;
    double OP = lap * k.rdx2;
    OP = OP - (k.dg_sa * sqrt(k.dg_alpha * k.dg_alpha + 8.0 / 3.0 * Sigma) - k.dg_alpha) * 0.75;
    return OP;
}

// One cell of a colour sweep of the 19-point models (nDGP, k-mouflage) and the
// csf Newton update, from neighbours in shared memory: the arithmetic of
// k_relax_dgp / k_relax_kmf / k_relax_csf.  l0: PM grid (no tau).
// Precision form of the nDGP colour-sweep update in FP32.  The second
// differences are one FMA from the FP32 pair sums, as the plain path forms
// them from Real*4 sums; sign(alpha) sqrt(alpha^2 + y) - alpha is evaluated as
// sign(alpha) y / (sqrt(alpha^2 + y) + |alpha|), which has no cancellation.
__device__ __forceinline__ float dgp_L_f32(const float* __restrict__ Sm, const float* __restrict__ S0,
                                           const float* __restrict__ Sp, int p, float dval, const LevelConsts& k) {
    const float uc = S0[p];
    const float nxu = S0[p + 1], nxl = S0[p - 1], nyu = S0[p + OP_PX], nyl = S0[p - OP_PX], nzu = Sp[p], nzl = Sm[p];
    float s = nxu;
    s = s + nxl; s = s + nyu; s = s + nyl; s = s + nzu; s = s + nzl;
    const float lap = fmaf(-6.0f, uc, s);
    const float dxx = fmaf(-2.0f, uc, nxu + nxl), dyy = fmaf(-2.0f, uc, nyu + nyl), dzz = fmaf(-2.0f, uc, nzu + nzl);
    const float dxy = ((S0[p + 1 + OP_PX] + S0[p - 1 - OP_PX]) - S0[p + 1 - OP_PX]) - S0[p - 1 + OP_PX];
    const float dxz = ((Sp[p + 1] + Sm[p - 1]) - Sm[p + 1]) - Sp[p - 1];
    const float dyz = ((Sp[p + OP_PX] + Sm[p - OP_PX]) - Sm[p + OP_PX]) - Sp[p - OP_PX];
    const float diag = (dxy * dxy + dxz * dxz) + dyz * dyz;
    const float sq = (dxx * dxx + dyy * dyy) + dzz * dzz, cr = (dxx * dyy + dxx * dzz) + dyy * dzz;
    const float Sigma = fmaf(k.f_dg_fct1, dval, fmaf(diag, k.f_dg_c18, (sq - cr) * k.f_dg_c23));
    const float y = (8.0f / 3.0f) * Sigma;
    const float root = k.f_dg_sa * y / (sqrtf(k.f_dg_alpha2 + y) + k.f_dg_absalpha);
    return fmaf(lap, k.f_rdx2, -0.75f * root);
}
__device__ __forceinline__ float dgp_sweep_f32(const float* __restrict__ Sm, const float* __restrict__ S0,
                                               const float* __restrict__ Sp, int p, float dval, float tval, bool l0,
                                               const LevelConsts& k) {
    float L = dgp_L_f32(Sm, S0, Sp, p, dval, k);
    if (!l0) L = L - tval;
    return fmaf(-L, k.f_dg_rdLphi, S0[p]);
}

// Precision form of the k-mouflage source term (kmf_src) in FP32.  The three
// second-difference brackets are sums of differences of neighbouring values
// (2X+2Xl-Y-Yl-Z-Zl = (X-Y)+(X-Z)+(Xl-Yl)+(Xl-Zl)), exact for nearby values.
__device__ __forceinline__ float kmf_src_f32(const Nb19& v, float dval, const LevelConsts& k, float& qsum) {
    float q = v.xu;
    q = q + v.xl; q = q + v.yu; q = q + v.yl; q = q + v.zu; q = q + v.zl;
    qsum = q;
    const float dx_ = v.xu - v.xl, dy_ = v.yu - v.yl, dz_ = v.zu - v.zl;
    const float t1f = (dx_ * dx_ + dy_ * dy_) + dz_ * dz_;
    const float tmp1 = t1f * k.f_r4dx2;
    float Sigma1, Sigma2;
    if (k.km_n == 2) { Sigma1 = fmaf(k.f_km_fct5, tmp1, k.f_km_c3); Sigma2 = 1.0f; }
    else { Sigma1 = fmaf(k.f_km_fct5 * tmp1, tmp1, k.f_km_c3); Sigma2 = tmp1; }
    Sigma1 = Sigma1 + 1.0f;
    Sigma2 = Sigma2 * k.f_km_fct4;
    const float bx = ((v.xu - v.yu) + (v.xu - v.zu)) + ((v.xl - v.yl) + (v.xl - v.zl));
    const float by = ((v.yu - v.xu) + (v.yu - v.zu)) + ((v.yl - v.xl) + (v.yl - v.zl));
    const float bz = ((v.zu - v.xu) + (v.zu - v.yu)) + ((v.zl - v.xl) + (v.zl - v.yl));
    const float axy = ((v.xyPP + v.xyMM) - v.xyPM) - v.xyMP;
    const float axz = ((v.xzPP + v.xzMM) - v.xzPM) - v.xzMP;
    const float ayz = ((v.yzPP + v.yzMM) - v.yzPM) - v.yzMP;
    float tmp2 = ((dx_ * dx_) * bx + (dy_ * dy_) * by + (dz_ * dz_) * bz) * (1.0f / 12.0f);
    tmp2 = fmaf((axy * dx_) * dy_ + (axz * dx_) * dz_ + (ayz * dy_) * dz_, 0.125f, tmp2);
    tmp2 = tmp2 * k.f_rdx4;
    Sigma2 = Sigma2 * tmp2;
    return fmaf(k.f_km_fct2, dval, Sigma2) / Sigma1;
}

// Precision form of the csf Newton update in FP32.  With e = u/c~^2 (phi =
// phibar + e), the coupling and potential terms are written as deviations from
// the background, which is what they are of order of:
//   A'(phi) rho - A'(phibar) = A'(phibar) (expm1(beta e) rho + delta),
//   V'(phi) - V'(phibar)     = V'(phibar) expm1(-(1+alpha) log1p(e/phibar)),
// identities of the reference's expressions that FP32 evaluates without the
// cancellation of the direct form.
// the csf nonlinear terms in deviation form: returns fct1 (A'(phi) rho - A'(phibar)) + (V'(phi) - V'(phibar))
__device__ __forceinline__ float csf_terms_f32(float uc, float dval, const LevelConsts& k) {
    const float e = uc * k.f_rctl2;
    const float em = expm1f(k.f_cs_beta * e);
    const float vm = expm1f(-k.f_cs_a1 * log1pf(e * k.f_cs_rphibar));
    return fmaf(k.f_cs_fct1 * k.f_cs_Aphibar, fmaf(em, dval + 1.0f, dval), k.f_cs_Vphibar * vm);
}

__device__ __forceinline__ float csf_sweep_f32(const float* __restrict__ Sm, const float* __restrict__ S0,
                                               const float* __restrict__ Sp, int p, float dval, float tval, bool l0,
                                               const LevelConsts& k) {
    const float uc = S0[p];
    float s = S0[p + 1];
    s = s + S0[p - 1]; s = s + S0[p + OP_PX]; s = s + S0[p - OP_PX]; s = s + Sp[p]; s = s + Sm[p];
    float L = fmaf(-6.0f, uc, s) * k.f_rdx2;
    if (!l0) L = L - tval;
    const float e = uc * k.f_rctl2;
    const float em = expm1f(k.f_cs_beta * e);                       // A'(phi)/A'(phibar) - 1
    const float lv = log1pf(e * k.f_cs_rphibar);                    // log(phi/phibar)
    const float vm = expm1f(-k.f_cs_a1 * lv);                       // V'(phi)/V'(phibar) - 1
    const float rho = dval + 1.0f;
    const float A_phi = k.f_cs_Aphibar * (em + 1.0f);
    const float V_phi = k.f_cs_Vphibar * (vm + 1.0f);
    L = L - k.f_cs_fct1 * (k.f_cs_Aphibar * fmaf(em, rho, dval));
    L = L - k.f_cs_Vphibar * vm;
    const float A_pp = k.f_cs_beta * A_phi * k.f_rctl2;
    const float V_pp = -k.f_cs_a1 * V_phi * k.f_rctl2 * __expf(-lv) * k.f_cs_rphibar;   // / phi
    const float dL = -6.0f * k.f_rdx2 - k.f_cs_fct1 * rho * A_pp - V_pp;
    return uc - L / dL;
}

template <int MODEL, bool MIX = false>
__device__ __forceinline__ float sweep_smem(const float* __restrict__ Sm, const float* __restrict__ S0,
                                            const float* __restrict__ Sp, int p, double dval, double tval, bool l0,
                                            const LevelConsts& kc) {
    if (MIX && MODEL == MGG_MODEL_CSF) return csf_sweep_f32(Sm, S0, Sp, p, (float)dval, (float)tval, l0, kc);
    if (MIX && MODEL == MGG_MODEL_DGP) return dgp_sweep_f32(Sm, S0, Sp, p, (float)dval, (float)tval, l0, kc);
    if (MIX && MODEL == MGG_MODEL_KMOUFLAGE) {
        float qs;
        const float src = kmf_src_f32(nb19_smem(Sm, S0, Sp, p), (float)dval, kc, qs);
        const float Q = l0 ? qs : fmaf(-(float)tval, kc.f_km_dx2ctl, qs);
        return (Q - src * kc.f_km_dx2ctl) * (1.0f / 6.0f);
    }
    if (MODEL == MGG_MODEL_DGP) {
        double L = op_smem<MGG_MODEL_DGP, 0>(Sm, S0, Sp, p, dval, kc);
        if (!l0) L = L - tval;
        return (float)((double)S0[p] - L * kc.dg_rdLphi);
    } else if (MODEL == MGG_MODEL_KMOUFLAGE) {
        float qs;
        const double src = kmf_src(nb19_smem(Sm, S0, Sp, p), dval, kc.r4dx2, kc.rdx4, kc, qs);
        const double Q = l0 ? (double)qs : -tval * kc.km_dx2ctl + (double)qs;
        const double P = src * kc.km_dx2ctl;
        return (float)((Q - P) * (1.0 / 6.0));
    } else {   // csf
        const float uc = S0[p];
        const float xu = S0[p + 1], xl = S0[p - 1], yu = S0[p + OP_PX], yl = S0[p - OP_PX], zu = Sp[p], zl = Sm[p];
        double L;
        if (l0) {
            float s = xu;
            s = s + xl; s = s + yu; s = s + yl; s = s + zu; s = s + zl;
            L = (double)s - (double)uc * 6.0;
        } else {
            L = -tval * kc.dx2 + (double)xu;
            L = L + (double)xl; L = L + (double)yu; L = L + (double)yl;
            L = L + (double)zu; L = L + (double)zl; L = L - (double)uc * 6.0;
        }
        double phi, A_phi, V_phi;
        csf_phi((double)uc, kc, phi, A_phi, V_phi);
        const double rho = dval + 1.0;
        const double A_pp = kc.cs_beta * A_phi * kc.rctl2;
        const double V_pp = -(1.0 + kc.cs_alpha) * V_phi * kc.rctl2 / phi;
        L = L * kc.rdx2;
        L = L - kc.cs_fct1 * (A_phi * rho - kc.cs_Aphibar);
        L = L - (V_phi - kc.cs_Vphibar);
        const double dL = -6.0 * kc.rdx2 - kc.cs_fct1 * rho * A_pp - V_pp;
        return (float)((double)uc - L / dL);
    }
}

// Precision form: the operator of the other models at one cell in FP32 (the
// residual / right-hand side forms of the sweeps above); tval is subtracted
// first for the csf coarse residual, as the reference does.
template <int MODEL>
__device__ __forceinline__ float op_f32(const float* __restrict__ Sm, const float* __restrict__ S0,
                                        const float* __restrict__ Sp, int p, float dval, float tval, bool res,
                                        const LevelConsts& k) {
    const float uc = S0[p];
    if (MODEL == MGG_MODEL_DGP) return dgp_L_f32(Sm, S0, Sp, p, dval, k);
    if (MODEL == MGG_MODEL_KMOUFLAGE) {
        float qs;
        const float src = kmf_src_f32(nb19_smem(Sm, S0, Sp, p), dval, k, qs);
        return fmaf(fmaf(-6.0f, uc, qs) * k.f_rdx2, k.f_ctl, -src);
    }
    float sn = S0[p + 1];
    sn = sn + S0[p - 1]; sn = sn + S0[p + OP_PX]; sn = sn + S0[p - OP_PX]; sn = sn + Sp[p]; sn = sn + Sm[p];
    const float lap = fmaf(-6.0f, uc, sn) * k.f_rdx2;
    if (MODEL == MGG_MODEL_CSF) return (res ? lap - tval : lap) - csf_terms_f32(uc, dval, k);
    // symmetron
    return lap - k.f_sy_f2r * fmaf(fmaf(k.f_sy_fct1, dval + 1.0f, -1.0f), uc, uc * uc * uc);
}

template <int MODEL, int FRN, int MODE, bool MIX = false>
__global__ void __launch_bounds__(OP_T) k_march_op(const float* __restrict__ u, const float* __restrict__ d,
                                                   const float* __restrict__ aux, float* __restrict__ out, int n,
                                                   int cz, LevelConsts kc, double* __restrict__ part, int colour = 0) {
    __shared__ __align__(16) float S[3 * OP_PLANE];
    const int x0 = blockIdx.x * OP_X, y0 = blockIdx.y * OP_Y, kbeg = blockIdx.z * cz;
    const int nm = n - 1;
    const int plane = n * n;   // offsets fit 32 bits: n^3 <= 2^30
    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    // float2 pairs of the padded plane (x from x0 - 2, y from y0 - 1): periodic offsets
    constexpr int NPL = (OP_PLANE / 2 + OP_T - 1) / OP_T;
    int pxy[NPL], sxy[NPL];
#pragma unroll
    for (int i = 0; i < NPL; ++i) {
        const int e = min(tid + i * OP_T, OP_PLANE / 2 - 1);
        const int yy = e / (OP_PX / 2), xx = 2 * (e - yy * (OP_PX / 2));
        pxy[i] = ((x0 + xx - 2) & nm) + n * ((y0 + yy - 1) & nm);
        sxy[i] = yy * OP_PX + xx;
    }
    auto load_plane = [&](int z, int slot) {
        float* P = S + slot * OP_PLANE;
        const float* uz = u + (z & nm) * plane;
#pragma unroll
        for (int i = 0; i < NPL; ++i)
            if (tid + i * OP_T < OP_PLANE / 2)
                *reinterpret_cast<float2*>(P + sxy[i]) = __ldg(reinterpret_cast<const float2*>(uz + pxy[i]));
    };
    // Plane z+1 goes to the slot of plane z-2 before plane z is computed.  The
    // precision-form level-0 norm (PF) instead fetches plane z+2 into registers
    // while plane z is computed and stores it into the slot of plane z-1 (the
    // other instantiations are faster with the direct loads).
    constexpr bool PF = MIX && MODE == OPM_NORM;
    load_plane(kbeg - 1, 0);
    load_plane(kbeg, 1);
    if constexpr (PF) load_plane(kbeg + 1, 2);
    double acc = 0.0;
    const int p = (ty + 1) * OP_PX + (tx + 2);
    const int gxy = (x0 + tx) + n * (y0 + ty);
    float2 pre[NPL];
    // one plane z; the slots of planes z-1, z, z+1 are (J + 0, 1, 2) mod 3 with
    // J = z - kbeg (compile-time in the prefetching loop, three planes per iteration)
    auto plane_step = [&](auto jc, int z) {
        const int J = decltype(jc)::value < 0 ? z - kbeg : decltype(jc)::value;
        const bool fetch = PF && z + 2 <= kbeg + cz;
        if (fetch) {
            const float* uz = u + ((z + 2) & nm) * plane;
#pragma unroll
            for (int i = 0; i < NPL; ++i)
                if (tid + i * OP_T < OP_PLANE / 2) pre[i] = __ldg(reinterpret_cast<const float2*>(uz + pxy[i]));
        }
        if (!PF) load_plane(z + 1, (J + 2) % 3);
        __syncthreads();
        const float* Sm = S + (J % 3) * OP_PLANE;
        const float* S0 = S + ((J + 1) % 3) * OP_PLANE;
        const float* Sp = S + ((J + 2) % 3) * OP_PLANE;
        const int g = (z & nm) * plane + gxy;
        if (MODE == OPM_SWEEP) {
            // cells of the colour in this row: x = 2 (tx + 32 c) + par; the partner
            // x ^ 1 keeps its value (sweep src -> dst)
            const int par = (x0 + y0 + ty + z + colour) & 1;
            const int gr = (z & nm) * plane + x0 + n * (y0 + ty), pr = (ty + 1) * OP_PX + 2;
#pragma unroll
            for (int c = 0; c < OP_CPT / 2; ++c) {
                const int xc = 2 * (tx + 32 * c) + par, xo = xc ^ 1;
                const double tv = aux ? (double)__ldg(aux + gr + xc) : 0.0;
                out[gr + xc] = sweep_smem<MODEL, MIX>(Sm, S0, Sp, pr + xc, (double)__ldg(d + gr + xc), tv, aux == nullptr, kc);
                out[gr + xo] = S0[pr + xo];
            }
        } else {
#pragma unroll
            for (int c = 0; c < OP_CPT; ++c) {
                if (MIX && MODEL != MGG_MODEL_FR) {   // precision form, other models
                    const int q = p + 32 * c;
                    const float dv = __ldg(d + g + 32 * c);
                    if (MODEL == MGG_MODEL_CSF && MODE == OPM_RES) {
                        out[g + 32 * c] = op_f32<MODEL>(Sm, S0, Sp, q, dv, __ldg(aux + g + 32 * c), true, kc);
                        continue;
                    }
                    const float OPf = op_f32<MODEL>(Sm, S0, Sp, q, dv, 0.0f, false, kc);
                    if (MODE == OPM_NORM) acc += (double)(OPf * OPf);
                    else out[g + 32 * c] = OPf - __ldg(aux + g + 32 * c);
                    continue;
                }
                if (MIX && MODEL == MGG_MODEL_FR && FRN == 1) {   // precision form
                    const int q = p + 32 * c;
                    const float nxu = S0[q + 1], nxl = S0[q - 1], nyu = S0[q + OP_PX], nyl = S0[q - OP_PX];
                    float sn = nxu * nxu;
                    sn = sn + nxl * nxl; sn = sn + nyu * nyu; sn = sn + nyl * nyl;
                    sn = sn + Sp[q] * Sp[q]; sn = sn + Sm[q] * Sm[q];
                    const float OPf = fr1_op_f32(sn, S0[q], __ldg(d + g + 32 * c), kc);
                    if (MODE == OPM_NORM) acc += (double)OPf * (double)OPf;
                    else out[g + 32 * c] = OPf - __ldg(aux + g + 32 * c);
                    continue;
                }
                if (MODEL == MGG_MODEL_CSF && MODE == OPM_RES) {   // tau first (PMP2MGsolver_csf.f90:179-353)
                    const int q = p + 32 * c;
                    float sn = S0[q + 1];
                    sn = sn + S0[q - 1]; sn = sn + S0[q + OP_PX]; sn = sn + S0[q - OP_PX]; sn = sn + Sp[q]; sn = sn + Sm[q];
                    out[g + 32 * c] = (float)csf_res(S0[q], sn, (double)__ldg(d + g + 32 * c),
                                                     (double)__ldg(aux + g + 32 * c), kc);
                    continue;
                }
                const double OP = op_smem<MODEL, FRN>(Sm, S0, Sp, p + 32 * c, (double)__ldg(d + g + 32 * c), kc);
                if (MODE == OPM_NORM) {
                    if (MODEL == MGG_MODEL_FR) acc += OP * OP;
                    else { const float r = (float)OP; acc += (double)(r * r); }
                } else {
                    out[g + 32 * c] = (float)(OP - (double)__ldg(aux + g + 32 * c));
                }
            }
        }
        __syncthreads();
        if (fetch) {   // plane z+2 replaces plane z-1
            float* P = S + (J % 3) * OP_PLANE;
#pragma unroll
            for (int i = 0; i < NPL; ++i)
                if (tid + i * OP_T < OP_PLANE / 2) *reinterpret_cast<float2*>(P + sxy[i]) = pre[i];
        }
    };
    if constexpr (PF) {
        for (int z = kbeg; z < kbeg + cz; z += 3) {
            plane_step(std::integral_constant<int, 0>{}, z);
            if (z + 1 >= kbeg + cz) break;
            plane_step(std::integral_constant<int, 1>{}, z + 1);
            if (z + 2 >= kbeg + cz) break;
            plane_step(std::integral_constant<int, 2>{}, z + 2);
        }
    } else {
        for (int z = kbeg; z < kbeg + cz; ++z) plane_step(std::integral_constant<int, -1>{}, z);
    }
    if (MODE == OPM_NORM) {
        acc = block_sum_fixed(acc);
        if (tid == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = acc;
    }
}

// --------------------------------------------------------- residuals ------
// Level 0: per-block partial of the squared residual (no field written).
// Level > 0: writes the coarse residual (section 6).
// Cells first, first + stride, ... of the residual; returns this thread's sum of
// squares (level 0) or writes res (level > 0).
template <int MODEL, int FRN, bool L0>
__device__ __forceinline__ double resid_cells(const float* __restrict__ u, const float* __restrict__ d,
                                              const float* __restrict__ tau, float* __restrict__ res, int n,
                                              const LevelConsts& kc, uint32_t first, uint32_t stride) {
    const uint32_t total = (uint32_t)n * n * n;
    double acc = 0.0;
    for (uint32_t idx = first; idx < total; idx += stride) {
        int i, j, k;
        decode3(idx, n, i, j, k);
        const Nb q = nb6(i, j, k, n);
        double OP;
        if (MODEL == MGG_MODEL_FR) OP = fr_op<FRN>(u, q, (double)d[q.c], kc);
        else if (MODEL == MGG_MODEL_DGP) OP = dgp_op(u, q, i, j, k, n, (double)d[q.c], kc);
        else if (MODEL == MGG_MODEL_KMOUFLAGE) OP = kmf_op(nb19_global(u, i, j, k, n), (double)d[q.c], kc);
        else if (MODEL == MGG_MODEL_CSF) {
            float s = u[q.xu];
            s = s + u[q.xl]; s = s + u[q.yu]; s = s + u[q.yl]; s = s + u[q.zu]; s = s + u[q.zl];
            if (L0) OP = csf_op(u[q.c], s, (double)d[q.c], kc);
            else { res[q.c] = (float)csf_res(u[q.c], s, (double)d[q.c], (double)tau[q.c], kc); continue; }
        } else OP = sym_op(u, q, (double)d[q.c], kc);
        if (L0) {
            if (MODEL == MGG_MODEL_FR) acc += OP * OP;                       // (400)
            else { const float r = (float)OP; acc += (double)(r * r); }     // FI3**2 in Real*4
        } else {
            res[q.c] = (float)(OP - (double)tau[q.c]);
        }
    }
    return acc;
}

template <int MODEL, int FRN, bool L0>
__global__ void k_resid(const float* __restrict__ u, const float* __restrict__ d, const float* __restrict__ tau,
                        float* __restrict__ res, int n, LevelConsts kc, double* __restrict__ part) {
    double acc = resid_cells<MODEL, FRN, L0>(u, d, tau, res, n, kc, blockIdx.x * blockDim.x + threadIdx.x,
                                             gridDim.x * blockDim.x);
    if (L0) {
        acc = block_sum_fixed(acc);
        if (threadIdx.x == 0) part[blockIdx.x] = acc;
    }
}

// ---------------------------------------------------------- restrict ------
__device__ __forceinline__ int64_t cidx(int i, int j, int k, int n) { return i + (int64_t)n * (j + (int64_t)n * k); }

// Level 0 -> 1: the restricted residual is recomputed from the fine field
// (PMP2MGsolver_*.f90 restrict_residual at ilevel = 1), together with the
// 8-child averages of field and density (PMP2extradof.f90:1208-1217, 1303-1314).
// One coarse cell from an accessor U(x, y, z) of the fine field at offsets
// x, y, z in [-1, 2] from its first child and Dn(x, y, z) of the fine density
// at the children (x, y, z in {0, 1}); children in the order x, then y, then z.
template <int MODEL, int FRN, bool MIX, class UA, class DA>
__device__ __forceinline__ void restrict1_cell(const UA& U, const DA& Dn, const LevelConsts& kc, float& rr_out,
                                               float& ru_out, float& dc_out) {
    if (MIX && MODEL == MGG_MODEL_FR && FRN == 1) {
        // Precision form: the restricted fine residual in FP32.  The 24 outer
        // and 8 inner u^2 enter with weights summing to zero, so each is taken
        // relative to the first child's u^2 (one FMA each): the cancellation of
        // the Laplacian is carried without loss.
        float Pu = U(0, 0, 0), Pd = Dn(0, 0, 0);
        float Q = -8.0f * kc.f_r2;
        const float c0 = U(0, 0, 0) * U(0, 0, 0);
        float inner = 0.0f;
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int x = m & 1, y = (m >> 1) & 1, z = m >> 2;
            const float uv = U(x, y, z), dv = Dn(x, y, z);
            if (m) { Pu += uv; Pd += dv; }
            Q += fmaf(kc.f_r1, dv, (float)kc.fr_r4 * __frcp_rn(uv));
            inner += fmaf(uv, uv, -c0);
        }
        auto W = [&](int x, int y, int z) { const float v = U(x, y, z); return fmaf(v, v, -c0); };
        float P = -3.0f * inner;
        P += ((W(-1, 0, 0) + W(-1, 1, 0)) + (W(-1, 0, 1) + W(-1, 1, 1))) + ((W(2, 0, 0) + W(2, 1, 0)) + (W(2, 0, 1) + W(2, 1, 1)));
        P += ((W(0, -1, 0) + W(1, -1, 0)) + (W(0, -1, 1) + W(1, -1, 1))) + ((W(0, 2, 0) + W(1, 2, 0)) + (W(0, 2, 1) + W(1, 2, 1)));
        P += ((W(0, 0, -1) + W(1, 0, -1)) + (W(0, 1, -1) + W(1, 1, -1))) + ((W(0, 0, 2) + W(1, 0, 2)) + (W(0, 1, 2) + W(1, 1, 2)));
        rr_out = fmaf(P, (float)(kc.fr_r3 * kc.dx2), Q) * 0.125f;
        ru_out = Pu * 0.125f;
        dc_out = Pd * 0.125f;
        return;
    }
    double Pu = (double)U(0, 0, 0), Pd = (double)Dn(0, 0, 0);
#pragma unroll
    for (int m = 1; m < 8; ++m) {
        Pu = Pu + (double)U(m & 1, (m >> 1) & 1, m >> 2);
        Pd = Pd + (double)Dn(m & 1, (m >> 1) & 1, m >> 2);
    }
    double rrv;
    if (MODEL == MGG_MODEL_FR) {   // PMP2MGsolver_fR.f90:607-653
        double Q = -8.0 * kc.fr_r2;
#pragma unroll
        for (int m = 0; m < 8; ++m) {
            const int x = m & 1, y = (m >> 1) & 1, z = m >> 2;
            Q = Q + kc.fr_r1 * (double)Dn(x, y, z) + div_by(kc.fr_r4, U(x, y, z));
        }
        float s8 = upow<FRN>(U(0, 0, 0));
#pragma unroll
        for (int m = 1; m < 8; ++m) s8 = s8 + upow<FRN>(U(m & 1, (m >> 1) & 1, m >> 2));
        double P = -3.0 * (double)s8;
        auto W = [&](int x, int y, int z) { return (double)upow<FRN>(U(x, y, z)); };
        P = P + W(-1, 0, 0) + W(-1, 1, 0) + W(-1, 0, 1) + W(-1, 1, 1);
        P = P + W(2, 0, 0) + W(2, 1, 0) + W(2, 0, 1) + W(2, 1, 1);
        P = P + W(0, -1, 0) + W(1, -1, 0) + W(0, -1, 1) + W(1, -1, 1);
        P = P + W(0, 2, 0) + W(1, 2, 0) + W(0, 2, 1) + W(1, 2, 1);
        P = P + W(0, 0, -1) + W(1, 0, -1) + W(0, 1, -1) + W(1, 1, -1);
        P = P + W(0, 0, 2) + W(1, 0, 2) + W(0, 1, 2) + W(1, 1, 2);
        const double fct3 = kc.fr_r3 * kc.dx2;   // fine spacing dx = 1
        rrv = (P * fct3 + Q) / 8.0;
    } else {
        // Laplacian part identical for the other models; the rest per child
        double Q;
        if (MODEL == MGG_MODEL_DGP) {   // PMP2MGsolver_DGP.f90:467-716, Eq. (B1) form
            Q = -8.0 * kc.dg_fct2;
#pragma unroll 1
            for (int m = 0; m < 8; ++m) {
                const int a = m & 1, b = (m >> 1) & 1, c = m >> 2;
                const float X = U(a + 1, b, c) + U(a - 1, b, c);
                const float Y = U(a, b + 1, c) + U(a, b - 1, c);
                const float Z = U(a, b, c + 1) + U(a, b, c - 1);
                double Sg = kc.dg_fct1 * (double)Dn(a, b, c);
                Sg = Sg + (double)X * (2.0 * (double)X - (double)Y - (double)Z) * (1.0 / 3.0) +
                     (double)Y * (2.0 * (double)Y - (double)X - (double)Z) * (1.0 / 3.0) +
                     (double)Z * (2.0 * (double)Z - (double)X - (double)Y) * (1.0 / 3.0);
                const float dxy = (U(a + 1, b + 1, c) + U(a - 1, b - 1, c)) - (U(a + 1, b - 1, c) + U(a - 1, b + 1, c));
                const float dxz = (U(a + 1, b, c + 1) + U(a - 1, b, c - 1)) - (U(a + 1, b, c - 1) + U(a - 1, b, c + 1));
                const float dyz = (U(a, b + 1, c + 1) + U(a, b - 1, c - 1)) - (U(a, b + 1, c - 1) + U(a, b - 1, c + 1));
                Sg = Sg + (double)(dxy * dxy) * 0.125 + (double)(dxz * dxz) * 0.125 + (double)(dyz * dyz) * 0.125;
                Q = Q - kc.dg_fct3 * sqrt(kc.dg_alpha * kc.dg_alpha + 8.0 / 3.0 * Sg);
            }
        } else if (MODEL == MGG_MODEL_KMOUFLAGE) {   // PMP2MGsolver_kmf.f90:507-1067
            Q = 0.0;
#pragma unroll 1
            for (int m = 0; m < 8; ++m) {
                const int a = m & 1, b = (m >> 1) & 1, c = m >> 2;
                Nb19 v;
                v.c = U(a, b, c);
                v.xu = U(a + 1, b, c); v.xl = U(a - 1, b, c); v.yu = U(a, b + 1, c); v.yl = U(a, b - 1, c);
                v.zu = U(a, b, c + 1); v.zl = U(a, b, c - 1);
                v.xyPP = U(a + 1, b + 1, c); v.xyMM = U(a - 1, b - 1, c); v.xyPM = U(a + 1, b - 1, c); v.xyMP = U(a - 1, b + 1, c);
                v.xzPP = U(a + 1, b, c + 1); v.xzMM = U(a - 1, b, c - 1); v.xzPM = U(a + 1, b, c - 1); v.xzMP = U(a - 1, b, c + 1);
                v.yzPP = U(a, b + 1, c + 1); v.yzMM = U(a, b - 1, c - 1); v.yzPM = U(a, b + 1, c - 1); v.yzMP = U(a, b - 1, c + 1);
                float qs;
                Q = Q + kmf_src(v, (double)Dn(a, b, c), 0.25, 1.0, kc, qs);
            }
        } else if (MODEL == MGG_MODEL_CSF) {   // PMP2MGsolver_csf.f90:355-572
            Q = 0.0;
#pragma unroll 1
            for (int m = 0; m < 8; ++m) {
                const int a = m & 1, b = (m >> 1) & 1, c = m >> 2;
                double phi, A_phi, V_phi;
                csf_phi((double)U(a, b, c), kc, phi, A_phi, V_phi);
                Q = Q + kc.cs_fct1 * (A_phi * ((double)Dn(a, b, c) + 1.0) - kc.cs_Aphibar) + (V_phi - kc.cs_Vphibar);
            }
        } else {   // PMP2MGsolver_sym.f90:329-352
            Q = 0.0;
#pragma unroll
            for (int m = 0; m < 8; ++m) {
                const int a = m & 1, b = (m >> 1) & 1, c = m >> 2;
                const float uq = U(a, b, c);
                Q = Q + kc.sy_f2r * (kc.sy_fct1 * ((double)Dn(a, b, c) + 1.0) - 1.0) * (double)uq +
                    kc.sy_f2r * (double)(uq * uq * uq);
            }
        }
        double P = 0.0;
#pragma unroll
        for (int m = 0; m < 8; ++m) P = P - 3.0 * (double)U(m & 1, (m >> 1) & 1, m >> 2);
        P = P + U(-1, 0, 0); P = P + U(-1, 1, 0); P = P + U(-1, 0, 1); P = P + U(-1, 1, 1);
        P = P + U(2, 0, 0); P = P + U(2, 1, 0); P = P + U(2, 0, 1); P = P + U(2, 1, 1);
        P = P + U(0, -1, 0); P = P + U(1, -1, 0); P = P + U(0, -1, 1); P = P + U(1, -1, 1);
        P = P + U(0, 2, 0); P = P + U(1, 2, 0); P = P + U(0, 2, 1); P = P + U(1, 2, 1);
        P = P + U(0, 0, -1); P = P + U(1, 0, -1); P = P + U(0, 1, -1); P = P + U(1, 1, -1);
        P = P + U(0, 0, 2); P = P + U(1, 0, 2); P = P + U(0, 1, 2); P = P + U(1, 1, 2);
        if (MODEL == MGG_MODEL_DGP) P = P / 1.0 + Q;
        else if (MODEL == MGG_MODEL_KMOUFLAGE) P = P / 1.0 * kc.ctl - Q;
        else P = P / 1.0 - Q;
        rrv = P / 8.0;
    }
    rr_out = (float)rrv;
    ru_out = (float)(Pu / 8.0);
    dc_out = (float)(Pd / 8.0);
}

// grid-stride version (small levels): periodic fine indices
template <int MODEL, int FRN>
__global__ void k_restrict1(const float* __restrict__ fi, const float* __restrict__ fi2, int Nf,
                            float* __restrict__ rr, float* __restrict__ ru, float* __restrict__ uc,
                            float* __restrict__ dc, LevelConsts kc) {
    const int n = Nf >> 1, fm = Nf - 1;
    const uint32_t total = (uint32_t)n * n * n;
    for (uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += gridDim.x * blockDim.x) {
        int i, j, k;
        decode3(idx, n, i, j, k);
        const int a0 = 2 * i, b0 = 2 * j, c0 = 2 * k;
        auto U = [&](int x, int y, int z) { return fi2[cidx((a0 + x) & fm, (b0 + y) & fm, (c0 + z) & fm, Nf)]; };
        auto Dn = [&](int x, int y, int z) { return fi[cidx(a0 + x, b0 + y, c0 + z, Nf)]; };
        float r, u, dd;
        restrict1_cell<MODEL, FRN, false>(U, Dn, kc, r, u, dd);
        rr[idx] = r;
        ru[idx] = u;
        uc[idx] = u;
        dc[idx] = dd;
    }
}

// Marching version: a block owns RS_CX x RS_CY coarse cells and a chunk of
// coarse planes; the fine field of the four fine planes 2k-1 .. 2k+2 (with a
// 1-cell x-y halo) sits in a shared-memory ring, so each fine value comes from
// DRAM once.  Same arithmetic as k_restrict1.
constexpr int RS_CX = 32, RS_CY = 8, RS_FX = 2 * RS_CX + 2, RS_FY = 2 * RS_CY + 2, RS_FPL = RS_FX * RS_FY;

// five blocks (40 warps) per SM; the 19-point k-mouflage needs more registers; the
// precision form's f(R) n = 1 restriction at seven blocks (32 registers): 0.546 ->
// 0.455 ms per launch at 1024^3 against five (48 registers); six 0.502
template <int MODEL, int FRN, bool MIX>
constexpr int rs_min_blocks() {
    return MODEL == MGG_MODEL_KMOUFLAGE ? 3 : (MIX && MODEL == MGG_MODEL_FR && FRN == 1 ? 7 : 5);
}

template <int MODEL, int FRN, bool MIX = false>
__global__ void __launch_bounds__(RS_CX * RS_CY, rs_min_blocks<MODEL, FRN, MIX>()) k_restrict1_march(const float* __restrict__ fi,
                                                                   const float* __restrict__ fi2, int Nf,
                                                                   float* __restrict__ rr, float* __restrict__ ru,
                                                                   float* __restrict__ uc, float* __restrict__ dc,
                                                                   int czc, LevelConsts kc) {
    __shared__ float SU[4 * RS_FPL];
    const int n = Nf >> 1, fm = Nf - 1;
    const int cx0 = blockIdx.x * RS_CX, cy0 = blockIdx.y * RS_CY, kbeg = blockIdx.z * czc;
    const int fx0 = 2 * cx0 - 1, fy0 = 2 * cy0 - 1;
    const int tid = threadIdx.x, tx = tid & (RS_CX - 1), ty = tid / RS_CX;
    const int fplane = Nf * Nf;   // offsets fit 32 bits: Nf^3 <= 2^30
    constexpr int NLD = (RS_FPL + RS_CX * RS_CY - 1) / (RS_CX * RS_CY);
    int pxy[NLD];
#pragma unroll
    for (int t = 0; t < NLD; ++t) {
        const int e = min(tid + t * RS_CX * RS_CY, RS_FPL - 1);
        const int yy = e / RS_FX, xx = e - yy * RS_FX;
        pxy[t] = ((fx0 + xx) & fm) + Nf * ((fy0 + yy) & fm);
    }
    auto load = [&](int fz) {
        const float* src = fi2 + (fz & fm) * fplane;
        float* dst = SU + (fz & 3) * RS_FPL;
#pragma unroll
        for (int t = 0; t < NLD; ++t) {
            const int e = tid + t * RS_CX * RS_CY;
            if (e < RS_FPL) dst[e] = __ldg(src + pxy[t]);
        }
    };
    for (int fz = 2 * kbeg - 1; fz <= 2 * kbeg + 2; ++fz) load(fz);
    __syncthreads();
    const int lp = (2 * ty + 1) * RS_FX + 2 * tx + 1;              // first child in the plane tile
    const int dxy = 2 * (cx0 + tx) + Nf * (2 * (cy0 + ty));         // first child in a fine plane
    for (int k = kbeg; k < kbeg + czc; ++k) {
        const int fz0 = 2 * k;
        auto U = [&](int x, int y, int z) { return SU[((fz0 + z) & 3) * RS_FPL + lp + y * RS_FX + x]; };
        auto Dn = [&](int x, int y, int z) { return __ldg(fi + (fz0 + z) * fplane + dxy + y * Nf + x); };
        float r, u, dd;
        restrict1_cell<MODEL, FRN, MIX>(U, Dn, kc, r, u, dd);
        const int64_t o = (int64_t)(cx0 + tx) + (int64_t)n * ((cy0 + ty) + (int64_t)n * k);
        rr[o] = r;
        ru[o] = u;
        uc[o] = u;
        dc[o] = dd;
        __syncthreads();
        if (k + 1 < kbeg + czc) {   // planes 2k+3, 2k+4 replace 2k-1, 2k
            load(fz0 + 3);
            load(fz0 + 4);
        }
        __syncthreads();
    }
}

// level l-1 -> l (l >= 2): 8-child averages of residual, field and density
__device__ __forceinline__ void restrict_cells(const float* __restrict__ resf, const float* __restrict__ uf,
                                               const float* __restrict__ df, int n, float* __restrict__ rr,
                                               float* __restrict__ ru, float* __restrict__ uc, float* __restrict__ dc,
                                               uint32_t first, uint32_t stride) {
    const int nf = 2 * n;
    const uint32_t total = (uint32_t)n * n * n;
    for (uint32_t idx = first; idx < total; idx += stride) {
        int i, j, k;
        decode3(idx, n, i, j, k);
        const int64_t ch[8] = {cidx(2 * i, 2 * j, 2 * k, nf),         cidx(2 * i + 1, 2 * j, 2 * k, nf),
                               cidx(2 * i, 2 * j + 1, 2 * k, nf),     cidx(2 * i + 1, 2 * j + 1, 2 * k, nf),
                               cidx(2 * i, 2 * j, 2 * k + 1, nf),     cidx(2 * i + 1, 2 * j, 2 * k + 1, nf),
                               cidx(2 * i, 2 * j + 1, 2 * k + 1, nf), cidx(2 * i + 1, 2 * j + 1, 2 * k + 1, nf)};
        double Pr = (double)resf[ch[0]], Pu = (double)uf[ch[0]], Pd = (double)df[ch[0]];
#pragma unroll
        for (int m = 1; m < 8; ++m) {
            Pr = Pr + (double)resf[ch[m]];
            Pu = Pu + (double)uf[ch[m]];
            Pd = Pd + (double)df[ch[m]];
        }
        rr[idx] = (float)(Pr / 8.0);
        ru[idx] = (float)(Pu / 8.0);
        uc[idx] = (float)(Pu / 8.0);
        dc[idx] = (float)(Pd / 8.0);
    }
}

__global__ void k_restrict(const float* __restrict__ resf, const float* __restrict__ uf, const float* __restrict__ df,
                           int n, float* __restrict__ rr, float* __restrict__ ru, float* __restrict__ uc,
                           float* __restrict__ dc) {
    restrict_cells(resf, uf, df, n, rr, ru, uc, dc, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// --------------------------------------------------------------- rhs ------
template <int MODEL, int FRN>
__device__ __forceinline__ void rhs_cells(const float* __restrict__ ru, const float* __restrict__ d,
                                          const float* __restrict__ rr, float* __restrict__ tau, int n,
                                          const LevelConsts& kc, uint32_t first, uint32_t stride) {
    const uint32_t total = (uint32_t)n * n * n;
    for (uint32_t idx = first; idx < total; idx += stride) {
        int i, j, k;
        decode3(idx, n, i, j, k);
        const Nb q = nb6(i, j, k, n);
        double OP;
        if (MODEL == MGG_MODEL_FR) OP = fr_op<FRN>(ru, q, (double)d[q.c], kc);
        else if (MODEL == MGG_MODEL_DGP) OP = dgp_op(ru, q, i, j, k, n, (double)d[q.c], kc);
        else if (MODEL == MGG_MODEL_KMOUFLAGE) OP = kmf_op(nb19_global(ru, i, j, k, n), (double)d[q.c], kc);
        else if (MODEL == MGG_MODEL_CSF) {
            float s = ru[q.xu];
            s = s + ru[q.xl]; s = s + ru[q.yu]; s = s + ru[q.yl]; s = s + ru[q.zu]; s = s + ru[q.zl];
            OP = csf_op(ru[q.c], s, (double)d[q.c], kc);
        } else OP = sym_op(ru, q, (double)d[q.c], kc);
        tau[q.c] = (float)(OP - (double)rr[q.c]);
    }
}

template <int MODEL, int FRN>
__global__ void k_rhs(const float* __restrict__ ru, const float* __restrict__ d, const float* __restrict__ rr,
                      float* __restrict__ tau, int n, LevelConsts kc) {
    rhs_cells<MODEL, FRN>(ru, d, rr, tau, n, kc, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// ------------------------------------------------------- prolongation -----
// correct_solution (PMP2extradof.f90:1361-1578) as a gather over fine cells:
// fine cell (i,j,k) has parent (i/2,j/2,k/2) and son bits (i&1,j&1,k&1); its
// 8 coarse contributors and weights follow the reference's ccc/bbb tables.
__device__ __forceinline__ void prolong_cells(float* __restrict__ uf, const float* __restrict__ uc,
                                              const float* __restrict__ ruc, int nf, int model, double phibar,
                                              double ctl2, uint32_t first, uint32_t stride) {
    const int n = nf >> 1;
    const uint32_t total = (uint32_t)nf * nf * nf;
    const double a = 1.0 / 64.0, b = 3.0 * a, c = 9.0 * a, dd = 27.0 * a;
    const double bbb[8] = {a, b, b, c, b, c, c, dd};
    for (uint32_t idx = first; idx < total; idx += stride) {
        int i, j, k;
        decode3(idx, nf, i, j, k);
        const int pi = i >> 1, pj = j >> 1, pk = k >> 1;
        const int sx = i & 1, sy = j & 1, sz = k & 1;
        const int fx = sx ? (pi + 1 == n ? 0 : pi + 1) : (pi == 0 ? n - 1 : pi - 1);
        const int fy = sy ? (pj + 1 == n ? 0 : pj + 1) : (pj == 0 ? n - 1 : pj - 1);
        const int fz = sz ? (pk + 1 == n ? 0 : pk + 1) : (pk == 0 ? n - 1 : pk - 1);
        double P = 0.0;
#pragma unroll
        for (int ind = 0; ind < 8; ++ind) {
            const int xi = (ind & 1) ? pi : fx, yj = (ind & 2) ? pj : fy, zk = (ind & 4) ? pk : fz;
            const int64_t q = cidx(xi, yj, zk, n);
            P = P + bbb[ind] * (double)uc[q];
            P = P - bbb[ind] * (double)ruc[q];
        }
        const double tmpt = (double)uf[idx] + P;
        if (model == MGG_MODEL_FR || model == MGG_MODEL_SYMMETRON) {
            if (tmpt > 0.0) uf[idx] = (float)tmpt;
        } else if (model == MGG_MODEL_CSF) {
            if (phibar + tmpt / ctl2 > 0.0) uf[idx] = (float)tmpt;
        } else {
            uf[idx] = (float)tmpt;
        }
    }
}

__global__ void k_prolong(float* __restrict__ uf, const float* __restrict__ uc, const float* __restrict__ ruc,
                          int nf, int model, double phibar, double ctl2) {
    prolong_cells(uf, uc, ruc, nf, model, phibar, ctl2, blockIdx.x * blockDim.x + threadIdx.x, gridDim.x * blockDim.x);
}

// Prolongation over a block of fine cells: a block owns a PR_X x PR_Y fine tile
// and a chunk of czf <= PR_CZF fine planes.  It first stages the coarse U and
// R u values the chunk needs (PR_X/2 x PR_Y/2 parents + 1-cell halo, czf/2 + 2
// planes) in shared memory; then each thread walks four consecutive fine cells
// of one row (a float4 of the fine field) up the chunk with no further
// barrier.  Same contributors, weights and summation order as k_prolong.
constexpr int PR_X = 128, PR_Y = 8, PR_CX = PR_X / 2 + 2, PR_CY = PR_Y / 2 + 2, PR_CPLANE = PR_CX * PR_CY;
constexpr int PR_CZF = 16, PR_CPL = PR_CZF / 2 + 2, PR_T = PR_X / 4 * PR_Y;

// MIX (precision form): the correction sum_i w_i (U_i - Ru_i) in FP32 from the
// staged differences U - Ru (exact when the two are within a factor of two,
// as they are where the correction is small), same contributors and order.
// The precision form at six blocks per SM (40 registers): 0.396 -> 0.362 ms per
// launch at 1024^3 against the unbounded 52 registers; five 0.371.  The plain
// form keeps its registers (its FP64 correction spills at 40).
template <bool MIX = false>
__global__ void __launch_bounds__(PR_T, MIX ? 6 : 1) k_prolong_march(float* __restrict__ uf, const float* __restrict__ uc,
                                                        const float* __restrict__ ruc, int nf, int czf, int model,
                                                        double phibar, double ctl2) {
    __shared__ float SU[PR_CPL * PR_CPLANE], SR[MIX ? 1 : PR_CPL * PR_CPLANE];
    const int n = nf >> 1, nm = n - 1;
    const int x0 = blockIdx.x * PR_X, y0 = blockIdx.y * PR_Y, zbeg = blockIdx.z * czf;
    const int cx0 = x0 >> 1, cy0 = y0 >> 1, cbeg = zbeg >> 1;
    const int tid = threadIdx.x;
    const int cplane = n * n;   // offsets fit 32 bits
    const int npl = czf / 2 + 2;   // coarse planes cbeg-1 .. cbeg+czf/2
    for (int e = tid; e < npl * PR_CPLANE; e += PR_T) {
        const int pl = e / PR_CPLANE, r = e - pl * PR_CPLANE;
        const int yy = r / PR_CX, xx = r - yy * PR_CX;
        const int g = ((cx0 + xx - 1) & nm) + n * ((cy0 + yy - 1) & nm) + ((cbeg - 1 + pl) & nm) * cplane;
        if (MIX) {
            SU[e] = __ldg(uc + g) - __ldg(ruc + g);
        } else {
            SU[e] = __ldg(uc + g);
            SR[e] = __ldg(ruc + g);
        }
    }
    __syncthreads();
    const double a = 1.0 / 64.0, b = 3.0 * a, c = 9.0 * a, dd = 27.0 * a;
    const double bbb[8] = {a, b, b, c, b, c, c, dd};
    const int tx = tid & (PR_X / 4 - 1), ty = tid / (PR_X / 4);
    const int fx = x0 + 4 * tx, fy = y0 + ty;
    const int sy = fy & 1;
    const int lpy = (fy >> 1) - cy0 + 1, oy = sy ? 1 : -1;
    const int lcx = 2 * tx + 1;   // local coarse column of the parent of fine x = 4 tx
    const int64_t nnf = nf;
    float* row = uf + (int64_t)fx + nnf * (int64_t)fy;
    for (int fzl = 0; fzl < czf; ++fzl) {
        const int sc = (fzl >> 1) + 1, so = (fzl & 1) ? sc + 1 : sc - 1;   // coarse plane pk, pk +/- 1
        float4* q4 = reinterpret_cast<float4*>(row + nnf * nnf * (int64_t)(zbeg + fzl));
        float4 v = *q4;
        float o[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int lpx = lcx + (j >> 1), ox = (j & 1) ? 1 : -1;
            if (MIX) {
                constexpr float wf[8] = {1.f / 64, 3.f / 64, 3.f / 64, 9.f / 64, 3.f / 64, 9.f / 64, 9.f / 64, 27.f / 64};
                float Pf = 0.0f;
#pragma unroll
                for (int ind = 0; ind < 8; ++ind) {
                    const int s = (ind & 4) ? sc : so;
                    const int q = s * PR_CPLANE + ((ind & 2) ? lpy : lpy + oy) * PR_CX + ((ind & 1) ? lpx : lpx + ox);
                    Pf = fmaf(wf[ind], SU[q], Pf);
                }
                const float t = o[j] + Pf;
                if (model == MGG_MODEL_FR || model == MGG_MODEL_SYMMETRON) {
                    if (t > 0.0f) o[j] = t;
                } else if (model == MGG_MODEL_CSF) {
                    if (phibar + (double)t / ctl2 > 0.0) o[j] = t;
                } else {
                    o[j] = t;
                }
                continue;
            }
            double P = 0.0;
#pragma unroll
            for (int ind = 0; ind < 8; ++ind) {
                const int s = (ind & 4) ? sc : so;
                const int q = s * PR_CPLANE + ((ind & 2) ? lpy : lpy + oy) * PR_CX + ((ind & 1) ? lpx : lpx + ox);
                P = P + bbb[ind] * (double)SU[q];
                P = P - bbb[ind] * (double)SR[q];
            }
            const double tmpt = (double)o[j] + P;
            if (model == MGG_MODEL_FR || model == MGG_MODEL_SYMMETRON) {
                if (tmpt > 0.0) o[j] = (float)tmpt;
            } else if (model == MGG_MODEL_CSF) {
                if (phibar + tmpt / ctl2 > 0.0) o[j] = (float)tmpt;
            } else {
                o[j] = (float)tmpt;
            }
        }
        *q4 = make_float4(o[0], o[1], o[2], o[3]);
    }
}

__global__ void k_fill(float* __restrict__ f, int64_t n, float v) {
    const int64_t n4 = n >> 2, stride = (int64_t)gridDim.x * blockDim.x;
    float4* f4 = reinterpret_cast<float4*>(f);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) f4[q] = make_float4(v, v, v, v);
    for (int64_t q = 4 * n4 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride) f[q] = v;
}
// f *= s in Real*4 (each value rounded once); 16-byte accesses, scalar tail
__global__ void k_scale(float* __restrict__ f, int64_t n, double s) {
    const int64_t n4 = n >> 2, stride = (int64_t)gridDim.x * blockDim.x;
    float4* f4 = reinterpret_cast<float4*>(f);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
        float4 v = f4[q];
        v.x = (float)((double)v.x * s); v.y = (float)((double)v.y * s);
        v.z = (float)((double)v.z * s); v.w = (float)((double)v.w * s);
        f4[q] = v;
    }
    for (int64_t q = 4 * n4 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride)
        f[q] = (float)((double)f[q] * s);
}
// two rescalings in one pass, each rounded to Real*4 as two separate passes would
__device__ __forceinline__ float scale2_one(float v, double s1, double s2) {
    return (float)((double)(float)((double)v * s1) * s2);
}
__global__ void k_scale2(float* __restrict__ f, int64_t n, double s1, double s2) {
    const int64_t n4 = n >> 2, stride = (int64_t)gridDim.x * blockDim.x;
    float4* f4 = reinterpret_cast<float4*>(f);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += stride) {
        float4 v = f4[q];
        v.x = scale2_one(v.x, s1, s2); v.y = scale2_one(v.y, s1, s2);
        v.z = scale2_one(v.z, s1, s2); v.w = scale2_one(v.w, s1, s2);
        f4[q] = v;
    }
    for (int64_t q = 4 * n4 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += stride)
        f[q] = scale2_one(f[q], s1, s2);
}

int grid_for(int64_t work, int threads = 256) {
    int64_t b = (work + threads - 1) / threads;
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return (int)b;
}

// ============================================================ driver ======
// ------------------------------------------------------------- autotuner ----
// The plane chunk of the marching kernels -- how many planes one block marches
// over, i.e. the trade between halo re-reads and the number of blocks -- is
// picked per device, kernel variant and level size by timing the candidates
// the first time that combination runs outside a CUDA-graph capture (the first
// solve of a context runs eagerly for this).  The choice is cached for the
// process.  Only kernels whose output does not depend on the chunk (every cell
// gets the same arithmetic) and that can be re-run in place are tuned: the
// fused smoother, the marching colour sweeps, the coarse residual and FAS
// right-hand side, and the level-1 restriction.  The level-0 residual norm is
// not (its block partial sums set the reduction order), nor the prolongation
// (it updates the field in place).  A candidate replaces the default only when
// it is at least 3 % faster.
enum TuneKind { TK_FUSED = 1, TK_SWEEP, TK_MARCH, TK_RESTRICT1 };

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tune;   // (device, kind, n, variant) -> chunk

// MGG_CHUNK=<k> in the environment forces chunk k wherever it is a candidate
// (tests use it to check that results do not depend on the chunk)
int forced_chunk() {
    static const int forced = [] {
        const char* e = std::getenv("MGG_CHUNK");
        return e ? std::atoi(e) : 0;
    }();
    return forced;
}

template <class F>
int tune_chunk(Ctx& c, int kind, int n, int variant, int dflt, const std::vector<int>& cands, F&& launch) {
    const int f = forced_chunk();
    if (f > 0) {
        for (int cz : cands)
            if (cz == f && f <= n && n % f == 0) return f;
    }
    const auto key = std::make_tuple(c.cfg.device, kind, n, variant);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune.find(key);
    if (it != g_tune.end()) return it->second;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    MGG_CUDA(cudaStreamIsCapturing(c.stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return dflt;
    cudaEvent_t a, b;
    MGG_CUDA(cudaEventCreate(&a));
    MGG_CUDA(cudaEventCreate(&b));
    auto time_of = [&](int cz) {
        launch(cz);   // warm-up
        MGG_CUDA(cudaEventRecord(a, c.stream));
        launch(cz);
        launch(cz);
        MGG_CUDA(cudaEventRecord(b, c.stream));
        MGG_CUDA(cudaEventSynchronize(b));
        float ms = 0.f;
        MGG_CUDA(cudaEventElapsedTime(&ms, a, b));
        return ms;
    };
    int best = dflt;
    float best_ms = time_of(dflt);
    for (int cz : cands) {
        if (cz == dflt || cz > n || n % cz) continue;
        const float ms = time_of(cz);
        if (ms < 0.97f * best_ms) {
            best_ms = ms;
            best = cz;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    g_tune[key] = best;
    return best;
}

// ---------------------------------------------------- small levels --------
// The cycle below a level of at most 16^3 cells (MGG_COARSE_N sets the size;
// 0 turns it off) in one launch of one block: the host lists the level
// operations in the order vcycle / fcycle / wcycle issue them (the colour
// sweeps of the smoothing, the residual, the restriction, the FAS right-hand
// side, the correction), and the block makes one pass over the level's cells
// per operation with the per-cell code of the separate kernels, a block
// barrier between passes.  Those levels are a few thousand cells; as separate
// launches they cost tens of launch latencies per cycle and left the GPU idle.
constexpr int CC_T = 512, CC_MAXOPS = 384, CC_MAXLEV = 6;
enum : uint8_t { CO_RED = 0, CO_BLACK = 1, CO_RESID, CO_RESTRICT, CO_RHS, CO_PROLONG };
struct CoarseLev {
    int n;
    float *u, *d, *tau, *res, *rr, *ru, *snap;
};
struct CoarseArgs {
    int nops;
    uint8_t op[CC_MAXOPS], lev[CC_MAXOPS];   // lev: level index relative to L[0]
    CoarseLev L[CC_MAXLEV];
    LevelConsts K[CC_MAXLEV];
};

// one colour sweep of a level > 0 (as Solver::relax below the marching sizes)
template <int MODEL, int FRN>
__device__ __forceinline__ void coarse_relax(const CoarseLev& L, const LevelConsts& k, int colour, uint32_t t,
                                             uint32_t st) {
    if (MODEL == MGG_MODEL_FR) {
        relax_fr_cells<FRN, false>(L.u, L.d, L.tau, L.n, colour, k, t, st);
    } else if (MODEL == MGG_MODEL_DGP || MODEL == MGG_MODEL_KMOUFLAGE) {
        float* dst = colour == 0 ? L.snap : L.u;
        const float* src = colour == 0 ? L.u : L.snap;
        if (MODEL == MGG_MODEL_DGP) relax_dgp_cells<false>(dst, src, L.d, L.tau, L.n, colour, k, t, st);
        else relax_kmf_cells<false>(dst, src, L.d, L.tau, L.n, colour, k, t, st);
    } else if (MODEL == MGG_MODEL_CSF) {
        relax_csf_cells<false>(L.u, L.d, L.tau, L.n, colour, k, t, st);
    } else {
        relax_sym_cells<false>(L.u, L.d, L.tau, L.n, colour, k, t, st);
    }
}

template <int MODEL, int FRN>
__global__ void __launch_bounds__(CC_T) k_coarse_cycle(const __grid_constant__ CoarseArgs a) {
    const uint32_t t = threadIdx.x, st = blockDim.x;
    for (int o = 0; o < a.nops; ++o) {
        const int l = a.lev[o], op = a.op[o];
        const CoarseLev& L = a.L[l];
        if (op <= CO_BLACK) {
            coarse_relax<MODEL, FRN>(L, a.K[l], op, t, st);
        } else if (op == CO_RESID) {
            resid_cells<MODEL, FRN, false>(L.u, L.d, L.tau, L.res, L.n, a.K[l], t, st);
        } else if (op == CO_RESTRICT) {   // level l -> l + 1
            const CoarseLev& C = a.L[l + 1];
            restrict_cells(L.res, L.u, L.d, C.n, C.rr, C.ru, C.u, C.d, t, st);
        } else if (op == CO_RHS) {
            rhs_cells<MODEL, FRN>(L.ru, L.d, L.rr, L.tau, L.n, a.K[l], t, st);
        } else {   // CO_PROLONG: correct level l from level l + 1
            const CoarseLev& C = a.L[l + 1];
            prolong_cells(L.u, C.u, C.ru, L.n, MODEL, a.K[l + 1].phibar, a.K[l + 1].ctl2, t, st);
        }
        __syncthreads();
    }
}

// size limit of the one-block cycle (cells per edge)
int coarse_max_n() {
    static const int v = [] {
        const char* e = std::getenv("MGG_COARSE_N");
        return e ? std::atoi(e) : 16;
    }();
    return v;
}

struct Solver {
    Ctx& c;
    int model, frn;
    explicit Solver(Ctx& c_) : c(c_), model(c_.cfg.mg_model), frn(c_.cfg.fr_n) {}

    float* U(int l) { return l == 0 ? c.fi2 : c.lev[l].u; }
    float* D(int l) { return l == 0 ? c.fi : c.lev[l].d; }

    void relax(int l, int colour) {
        const LevelConsts k = make_consts(c, l);
        const int n = k.n;
        const int64_t work = (int64_t)n * n * (n / 2);
        const int g = grid_for(work);
        float* u = U(l);
        const float* d = D(l);
        const float* tau = l > 0 ? c.lev[l].tau : nullptr;
        ProfScope ps(c, l == 0 ? K_MG_SMOOTH0 : K_MG_SMOOTH,
                     10.0 * (double)n * n * n / 2.0 + (l > 0 ? 2.0 * (double)n * n * n : 0.0));
        if (model == MGG_MODEL_FR) {
            if (l == 0) {
                if (frn == 0) k_relax_fr<0, true><<<g, 256, 0, c.stream>>>(u, d, tau, n, colour, k);
                else if (frn == 1) k_relax_fr<1, true><<<g, 256, 0, c.stream>>>(u, d, tau, n, colour, k);
                else k_relax_fr<2, true><<<g, 256, 0, c.stream>>>(u, d, tau, n, colour, k);
            } else {
                if (frn == 0) k_relax_fr<0, false><<<g, 256, 0, c.stream>>>(u, d, tau, n, colour, k);
                else if (frn == 1) k_relax_fr<1, false><<<g, 256, 0, c.stream>>>(u, d, tau, n, colour, k);
                else k_relax_fr<2, false><<<g, 256, 0, c.stream>>>(u, d, tau, n, colour, k);
            }
        } else if ((model == MGG_MODEL_DGP || model == MGG_MODEL_KMOUFLAGE || model == MGG_MODEL_CSF) &&
                   march_ok(n)) {
            // marching colour sweep src -> dst (red U -> snap, black snap -> U)
            float* snap = c.lev[l].snap;
            float* dst = colour == 0 ? snap : u;
            const float* src = colour == 0 ? u : snap;
            const bool mix = c.cfg.precision == MGG_PREC_MIXED;
#define SWEEP(M, X) k_march_op<M, 0, OPM_SWEEP, X><<<dim3(n / OP_X, n / OP_Y, n / cz), OP_T, 0, c.stream>>>(src, d, tau, dst, n, cz, k, c.red_partial, colour)
            auto launch = [&](int cz) {
                if (model == MGG_MODEL_DGP) { if (mix) SWEEP(MGG_MODEL_DGP, true); else SWEEP(MGG_MODEL_DGP, false); }
                else if (model == MGG_MODEL_KMOUFLAGE) { if (mix) SWEEP(MGG_MODEL_KMOUFLAGE, true); else SWEEP(MGG_MODEL_KMOUFLAGE, false); }
                else { if (mix) SWEEP(MGG_MODEL_CSF, true); else SWEEP(MGG_MODEL_CSF, false); }
                MGG_CHECK_LAUNCH();
            };
#undef SWEEP
            launch(tune_chunk(c, TK_SWEEP, n, model * 2 + (mix ? 1 : 0), march_cz(n), {8, 16, 32, 64}, launch));
        } else if (model == MGG_MODEL_DGP || model == MGG_MODEL_KMOUFLAGE) {
            // same-colour diagonal neighbours read the field as it was before this
            // sweep: red U -> snap, black snap -> U (relax is called in red/black pairs)
            float* snap = c.lev[l].snap;
            float* dst = colour == 0 ? snap : u;
            const float* src = colour == 0 ? u : snap;
            const int ga = g;
            if (model == MGG_MODEL_DGP) {
                if (l == 0) k_relax_dgp<true><<<ga, 256, 0, c.stream>>>(dst, src, d, tau, n, colour, k);
                else k_relax_dgp<false><<<ga, 256, 0, c.stream>>>(dst, src, d, tau, n, colour, k);
            } else {
                if (l == 0) k_relax_kmf<true><<<ga, 256, 0, c.stream>>>(dst, src, d, tau, n, colour, k);
                else k_relax_kmf<false><<<ga, 256, 0, c.stream>>>(dst, src, d, tau, n, colour, k);
            }
        } else if (model == MGG_MODEL_CSF) {
            if (l == 0) k_relax_csf<true><<<g, 256, 0, c.stream>>>(u, d, tau, n, colour, k);
            else k_relax_csf<false><<<g, 256, 0, c.stream>>>(u, d, tau, n, colour, k);
        } else {
            if (l == 0) k_relax_sym<true><<<g, 256, 0, c.stream>>>(u, d, tau, n, colour, k);
            else k_relax_sym<false><<<g, 256, 0, c.stream>>>(u, d, tau, n, colour, k);
        }
        MGG_CHECK_LAUNCH();
    }

    // one red+black iteration in a single fused sweep (7-point models, n >= 64)
    bool fused_ok(int l) const {
        const int n = c.N >> l;
        return (model == MGG_MODEL_FR || model == MGG_MODEL_SYMMETRON) && n >= FB_X && c.lev[l].snap != nullptr;
    }
    void fused_pass(int l, const float* uin, float* uout) {
        const LevelConsts k = make_consts(c, l);
        const int n = k.n;
        const bool mix = c.cfg.precision == MGG_PREC_MIXED;
        const int cz = tune_chunk(c, TK_FUSED, n, model * 100 + frn * 10 + (l == 0 ? 2 : 0) + (mix ? 1 : 0),
                                  n >= 256 ? 64 : (n >= 128 ? 32 : 16), {16, 32, 64, 128},
                                  [&](int z) { fused_launch(l, k, uin, uout, z); });
        fused_launch(l, k, uin, uout, cz, true);
    }
    void fused_launch(int l, const LevelConsts& k, const float* uin, float* uout, int cz, bool profile = false) {
        const int n = k.n;
        dim3 grid(n / FB_X, n / FB_Y, n / cz);
        const float* d = D(l);
        const float* tau = l > 0 ? c.lev[l].tau : nullptr;
        ProfScope ps(c, profile ? (l == 0 ? K_MG_SMOOTH0 : K_MG_SMOOTH) : -1,
                     12.0 * (double)n * n * n + (l > 0 ? 4.0 * (double)n * n * n : 0.0));
#define FUSED(M, F, L0) k_smooth_fused<M, F, L0><<<grid, FB_THREADS, FB_SMEM, c.stream>>>(uin, uout, d, tau, n, cz, k)
#define FUSEDX(M, F, L0) k_smooth_fused<M, F, L0, true><<<grid, FB_THREADS, FB_SMEM, c.stream>>>(uin, uout, d, tau, n, cz, k)
        if (model == MGG_MODEL_FR && c.cfg.precision == MGG_PREC_MIXED) {
            if (l == 0) { if (frn == 0) FUSEDX(MGG_MODEL_FR, 0, true); else if (frn == 1) FUSEDX(MGG_MODEL_FR, 1, true); else FUSEDX(MGG_MODEL_FR, 2, true); }
            else { if (frn == 0) FUSEDX(MGG_MODEL_FR, 0, false); else if (frn == 1) FUSEDX(MGG_MODEL_FR, 1, false); else FUSEDX(MGG_MODEL_FR, 2, false); }
        } else if (model == MGG_MODEL_FR) {
            if (l == 0) { if (frn == 0) FUSED(MGG_MODEL_FR, 0, true); else if (frn == 1) FUSED(MGG_MODEL_FR, 1, true); else FUSED(MGG_MODEL_FR, 2, true); }
            else { if (frn == 0) FUSED(MGG_MODEL_FR, 0, false); else if (frn == 1) FUSED(MGG_MODEL_FR, 1, false); else FUSED(MGG_MODEL_FR, 2, false); }
        } else if (c.cfg.precision == MGG_PREC_MIXED) {
            if (l == 0) FUSEDX(MGG_MODEL_SYMMETRON, 0, true);
            else FUSEDX(MGG_MODEL_SYMMETRON, 0, false);
        } else {
            if (l == 0) FUSED(MGG_MODEL_SYMMETRON, 0, true); else FUSED(MGG_MODEL_SYMMETRON, 0, false);
        }
#undef FUSED
#undef FUSEDX
        MGG_CHECK_LAUNCH();
    }

    void smooth(int l) {
        if (fused_ok(l)) {              // two iterations: field -> snapshot -> field
            fused_pass(l, U(l), c.lev[l].snap);
            fused_pass(l, c.lev[l].snap, U(l));
            return;
        }
        for (int s = 0; s < 2; ++s) {   // Nsmth = 2 (PMP2extradof.f90:361)
            relax(l, 0);                // red: M1+M2+M3 odd (1-based)
            relax(l, 1);
        }
    }

    template <bool L0>
    void launch_resid(int l, const LevelConsts& k, int g) {
        const int n = k.n;
        float* u = U(l);
        const float* d = D(l);
        const float* tau = l > 0 ? c.lev[l].tau : nullptr;
        float* res = l > 0 ? c.lev[l].res : nullptr;
        if (model == MGG_MODEL_FR) {
            if (frn == 0) k_resid<MGG_MODEL_FR, 0, L0><<<g, 256, 0, c.stream>>>(u, d, tau, res, n, k, c.red_partial);
            else if (frn == 1) k_resid<MGG_MODEL_FR, 1, L0><<<g, 256, 0, c.stream>>>(u, d, tau, res, n, k, c.red_partial);
            else k_resid<MGG_MODEL_FR, 2, L0><<<g, 256, 0, c.stream>>>(u, d, tau, res, n, k, c.red_partial);
        } else if (model == MGG_MODEL_DGP) {
            k_resid<MGG_MODEL_DGP, 0, L0><<<g, 256, 0, c.stream>>>(u, d, tau, res, n, k, c.red_partial);
        } else if (model == MGG_MODEL_KMOUFLAGE) {
            k_resid<MGG_MODEL_KMOUFLAGE, 0, L0><<<g, 256, 0, c.stream>>>(u, d, tau, res, n, k, c.red_partial);
        } else if (model == MGG_MODEL_CSF) {
            k_resid<MGG_MODEL_CSF, 0, L0><<<g, 256, 0, c.stream>>>(u, d, tau, res, n, k, c.red_partial);
        } else {
            k_resid<MGG_MODEL_SYMMETRON, 0, L0><<<g, 256, 0, c.stream>>>(u, d, tau, res, n, k, c.red_partial);
        }
        MGG_CHECK_LAUNCH();
    }

    // marching operator pass: MODE = OPM_NORM (level-0 norm partials), OPM_RES, OPM_RHS
    template <int MODE>
    void march(const LevelConsts& k, const float* u, const float* d, const float* aux, float* out, dim3 grid, int cz) {
        const int n = k.n;
#define MARCH(M, F) k_march_op<M, F, MODE><<<grid, OP_T, 0, c.stream>>>(u, d, aux, out, n, cz, k, c.red_partial)
        const bool mix = c.cfg.precision == MGG_PREC_MIXED;
#define MARCHX(M) k_march_op<M, 0, MODE, true><<<grid, OP_T, 0, c.stream>>>(u, d, aux, out, n, cz, k, c.red_partial)
        if (mix && model == MGG_MODEL_FR && frn == 1) {
            k_march_op<MGG_MODEL_FR, 1, MODE, true><<<grid, OP_T, 0, c.stream>>>(u, d, aux, out, n, cz, k, c.red_partial);
        } else if (mix && model == MGG_MODEL_DGP) MARCHX(MGG_MODEL_DGP);
        else if (mix && model == MGG_MODEL_KMOUFLAGE) MARCHX(MGG_MODEL_KMOUFLAGE);
        else if (mix && model == MGG_MODEL_CSF) MARCHX(MGG_MODEL_CSF);
        else if (mix && model == MGG_MODEL_SYMMETRON) MARCHX(MGG_MODEL_SYMMETRON);
        else if (model == MGG_MODEL_FR) {
            if (frn == 0) MARCH(MGG_MODEL_FR, 0); else if (frn == 1) MARCH(MGG_MODEL_FR, 1); else MARCH(MGG_MODEL_FR, 2);
        } else if (model == MGG_MODEL_DGP) MARCH(MGG_MODEL_DGP, 0);
        else if (model == MGG_MODEL_KMOUFLAGE) MARCH(MGG_MODEL_KMOUFLAGE, 0);
        else if (model == MGG_MODEL_CSF) MARCH(MGG_MODEL_CSF, 0);
        else MARCH(MGG_MODEL_SYMMETRON, 0);
#undef MARCH
#undef MARCHX
        MGG_CHECK_LAUNCH();
    }
    static int march_cz(int n) { return n >= 256 ? 32 : (n >= 64 ? 16 : 8); }
    int march_variant(int mode) const {
        return mode * 1000 + model * 100 + frn * 10 + (c.cfg.precision == MGG_PREC_MIXED ? 1 : 0);
    }
    bool march_ok(int n) const { return n >= OP_X; }

    // partial sums of the level-0 residual norm: one per block
    int norm0_blocks() const {
        const int n = c.N;
        if (march_ok(n)) {
            const int cz = march_cz(n);
            return (n / OP_X) * (n / OP_Y) * (n / cz);
        }
        return grid_for((int64_t)n * n * n);
    }

    // level-0 residual norm: the per-block partials and their fixed-order sum into
    // out (device), without waiting; the RMS residual is sqrt(*out / n^3)
    void norm0_async(double* out) {
        const LevelConsts k = make_consts(c, 0);
        const int n = k.n;
        const int64_t work = (int64_t)n * n * n;
        const int nb = norm0_blocks();
        ensure_partials(c, nb);
        {
            ProfScope ps(c, K_MG_RESID, 8.0 * (double)work);
            if (march_ok(n)) {
                const int cz = march_cz(n);
                march<OPM_NORM>(k, U(0), D(0), nullptr, nullptr, dim3(n / OP_X, n / OP_Y, n / cz), cz);
            } else {
                launch_resid<true>(0, k, nb);
            }
        }
        reduce_sum_blocks_async(c, nb, out);
    }

    double resid(int l) {
        const LevelConsts k = make_consts(c, l);
        const int n = k.n;
        const int64_t work = (int64_t)n * n * n;
        const int g = grid_for(work);
        if (l == 0) {
            norm0_async(c.red_out);
            MGG_CUDA(cudaMemcpyAsync(c.h_red, c.red_out, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
            MGG_CUDA(cudaStreamSynchronize(c.stream));
            return sqrt(c.h_red[0] / pow((double)n, 3));
        }
        if (march_ok(n)) {
            auto launch = [&](int z) {
                march<OPM_RES>(k, U(l), D(l), c.lev[l].tau, c.lev[l].res, dim3(n / OP_X, n / OP_Y, n / z), z);
            };
            const int zt = tune_chunk(c, TK_MARCH, n, march_variant(OPM_RES), march_cz(n), {8, 16, 32, 64}, launch);
            ProfScope ps(c, K_MG_RESID, 16.0 * (double)work);
            launch(zt);
            return 0.0;
        }
        ProfScope ps(c, K_MG_RESID, 16.0 * (double)work);
        launch_resid<false>(l, k, g);
        return 0.0;
    }

    void coarse_prepare(int l) {   // restrict residual, field, density; coarse rhs
        const int lc = l + 1;
        const LevelConsts kc = make_consts(c, lc);
        const int n = kc.n;
        const int64_t work = (int64_t)n * n * n;
        const int g = grid_for(work);
        Level& L = c.lev[lc];
        if (lc == 1 && n >= RS_CX) {
            const LevelConsts kf = make_consts(c, 0);
#define RS1(M, F) k_restrict1_march<M, F><<<grid, RS_CX * RS_CY, 0, c.stream>>>(c.fi, c.fi2, c.N, L.rr, L.ru, L.u, L.d, czc, kf)
            auto launch = [&](int czc) {
                const dim3 grid(n / RS_CX, n / RS_CY, n / czc);
                if (model == MGG_MODEL_FR && frn == 1 && c.cfg.precision == MGG_PREC_MIXED) {
                    k_restrict1_march<MGG_MODEL_FR, 1, true><<<grid, RS_CX * RS_CY, 0, c.stream>>>(c.fi, c.fi2, c.N, L.rr,
                                                                                                L.ru, L.u, L.d, czc, kf);
                } else if (model == MGG_MODEL_FR) {
                    if (frn == 0) RS1(MGG_MODEL_FR, 0); else if (frn == 1) RS1(MGG_MODEL_FR, 1); else RS1(MGG_MODEL_FR, 2);
                } else if (model == MGG_MODEL_DGP) RS1(MGG_MODEL_DGP, 0);
                else if (model == MGG_MODEL_KMOUFLAGE) RS1(MGG_MODEL_KMOUFLAGE, 0);
                else if (model == MGG_MODEL_CSF) RS1(MGG_MODEL_CSF, 0);
                else RS1(MGG_MODEL_SYMMETRON, 0);
                MGG_CHECK_LAUNCH();
            };
#undef RS1
            const int czt = tune_chunk(c, TK_RESTRICT1, n, march_variant(0), n >= 256 ? 16 : 8, {4, 8, 16, 32}, launch);
            ProfScope ps(c, K_MG_RESTRICT, 8.0 * (double)c.ncell + 16.0 * (double)work);
            launch(czt);
        } else if (lc == 1) {
            const LevelConsts kf = make_consts(c, 0);
            ProfScope ps(c, K_MG_RESTRICT, 8.0 * (double)c.ncell + 16.0 * (double)work);
            if (model == MGG_MODEL_FR) {
                if (frn == 0) k_restrict1<MGG_MODEL_FR, 0><<<g, 256, 0, c.stream>>>(c.fi, c.fi2, c.N, L.rr, L.ru, L.u, L.d, kf);
                else if (frn == 1) k_restrict1<MGG_MODEL_FR, 1><<<g, 256, 0, c.stream>>>(c.fi, c.fi2, c.N, L.rr, L.ru, L.u, L.d, kf);
                else k_restrict1<MGG_MODEL_FR, 2><<<g, 256, 0, c.stream>>>(c.fi, c.fi2, c.N, L.rr, L.ru, L.u, L.d, kf);
            } else if (model == MGG_MODEL_DGP) {
                k_restrict1<MGG_MODEL_DGP, 0><<<g, 256, 0, c.stream>>>(c.fi, c.fi2, c.N, L.rr, L.ru, L.u, L.d, kf);
            } else if (model == MGG_MODEL_KMOUFLAGE) {
                k_restrict1<MGG_MODEL_KMOUFLAGE, 0><<<g, 256, 0, c.stream>>>(c.fi, c.fi2, c.N, L.rr, L.ru, L.u, L.d, kf);
            } else if (model == MGG_MODEL_CSF) {
                k_restrict1<MGG_MODEL_CSF, 0><<<g, 256, 0, c.stream>>>(c.fi, c.fi2, c.N, L.rr, L.ru, L.u, L.d, kf);
            } else {
                k_restrict1<MGG_MODEL_SYMMETRON, 0><<<g, 256, 0, c.stream>>>(c.fi, c.fi2, c.N, L.rr, L.ru, L.u, L.d, kf);
            }
            MGG_CHECK_LAUNCH();
        } else {
            Level& F = c.lev[l];
            ProfScope ps(c, K_MG_RESTRICT, 12.0 * 8.0 * (double)work + 16.0 * (double)work);
            k_restrict<<<g, 256, 0, c.stream>>>(F.res, F.u, F.d, n, L.rr, L.ru, L.u, L.d);
            MGG_CHECK_LAUNCH();
        }
        if (march_ok(n)) {
            auto launch = [&](int z) {
                march<OPM_RHS>(kc, L.ru, L.d, L.rr, L.tau, dim3(n / OP_X, n / OP_Y, n / z), z);
            };
            const int zt = tune_chunk(c, TK_MARCH, n, march_variant(OPM_RHS), march_cz(n), {8, 16, 32, 64}, launch);
            ProfScope ps(c, K_MG_RHS, 16.0 * (double)work);
            launch(zt);
        } else {
            ProfScope ps(c, K_MG_RHS, 16.0 * (double)work);
            if (model == MGG_MODEL_FR) {
                if (frn == 0) k_rhs<MGG_MODEL_FR, 0><<<g, 256, 0, c.stream>>>(L.ru, L.d, L.rr, L.tau, n, kc);
                else if (frn == 1) k_rhs<MGG_MODEL_FR, 1><<<g, 256, 0, c.stream>>>(L.ru, L.d, L.rr, L.tau, n, kc);
                else k_rhs<MGG_MODEL_FR, 2><<<g, 256, 0, c.stream>>>(L.ru, L.d, L.rr, L.tau, n, kc);
            } else if (model == MGG_MODEL_DGP) {
                k_rhs<MGG_MODEL_DGP, 0><<<g, 256, 0, c.stream>>>(L.ru, L.d, L.rr, L.tau, n, kc);
            } else if (model == MGG_MODEL_KMOUFLAGE) {
                k_rhs<MGG_MODEL_KMOUFLAGE, 0><<<g, 256, 0, c.stream>>>(L.ru, L.d, L.rr, L.tau, n, kc);
            } else if (model == MGG_MODEL_CSF) {
                k_rhs<MGG_MODEL_CSF, 0><<<g, 256, 0, c.stream>>>(L.ru, L.d, L.rr, L.tau, n, kc);
            } else {
                k_rhs<MGG_MODEL_SYMMETRON, 0><<<g, 256, 0, c.stream>>>(L.ru, L.d, L.rr, L.tau, n, kc);
            }
            MGG_CHECK_LAUNCH();
        }
    }

    void correct(int lc) {
        const int nf = c.N >> (lc - 1);
        const int64_t work = (int64_t)nf * nf * nf;
        const LevelConsts k = make_consts(c, lc);
        ProfScope ps(c, K_MG_PROLONG, 8.0 * (double)work + 1.0 * (double)work);
        if (nf >= PR_X) {
            const int czf = PR_CZF;
            const bool mix = c.cfg.precision == MGG_PREC_MIXED;   // FP32 in the precision form
            if (mix)
                k_prolong_march<true><<<dim3(nf / PR_X, nf / PR_Y, nf / czf), PR_T, 0, c.stream>>>(
                    U(lc - 1), c.lev[lc].u, c.lev[lc].ru, nf, czf, model, k.phibar, k.ctl2);
            else
                k_prolong_march<false><<<dim3(nf / PR_X, nf / PR_Y, nf / czf), PR_T, 0, c.stream>>>(
                    U(lc - 1), c.lev[lc].u, c.lev[lc].ru, nf, czf, model, k.phibar, k.ctl2);
        } else {
            k_prolong<<<grid_for(work), 256, 0, c.stream>>>(U(lc - 1), c.lev[lc].u, c.lev[lc].ru, nf, model, k.phibar, k.ctl2);
        }
        MGG_CHECK_LAUNCH();
    }

    // The cycle below level l as one k_coarse_cycle launch, when l is the first
    // level (> 0) of at most coarse_max_n() cells per edge; type 0 V, 1 F, 2 W.
    struct OpList {
        CoarseArgs& a;
        int base;
        bool ok = true;
        void add(uint8_t op, int l) {
            if (a.nops >= CC_MAXOPS || l - base >= CC_MAXLEV) { ok = false; return; }
            a.op[a.nops] = op;
            a.lev[a.nops] = (uint8_t)(l - base);
            ++a.nops;
        }
    };
    void emit_smooth(OpList& o, int l) {
        for (int s = 0; s < 2; ++s) {
            o.add(CO_RED, l);
            o.add(CO_BLACK, l);
        }
    }
    void emit_prepare(OpList& o, int l) {   // resid(l), coarse_prepare(l) for l > 0
        o.add(CO_RESID, l);
        o.add(CO_RESTRICT, l);
        o.add(CO_RHS, l + 1);
    }
    void emit_cycle(OpList& o, int l, int type) {   // mirrors vcycle / fcycle / wcycle
        if (c.levelmax - l <= c.levelmin) { emit_smooth(o, l); return; }
        emit_smooth(o, l);
        emit_prepare(o, l);
        emit_cycle(o, l + 1, type);
        o.add(CO_PROLONG, l);
        emit_smooth(o, l);
        if (type == 0) return;
        emit_prepare(o, l);
        emit_cycle(o, l + 1, type == 1 ? 0 : 2);
        o.add(CO_PROLONG, l);
        emit_smooth(o, l);
    }
    bool coarse_cycle(int l, int type) {
        const int lim = coarse_max_n();
        const int n = c.N >> l;
        if (l < 1 || lim <= 0 || n > lim || (l > 1 && (c.N >> (l - 1)) <= lim) || n >= OP_X) return false;
        CoarseArgs a;
        memset(&a, 0, sizeof(a));
        OpList o{a, l};
        emit_cycle(o, l, type);
        if (!o.ok) return false;
        double cells = 0.0;
        for (int q = l; q <= c.levelmax && q - l < CC_MAXLEV; ++q) {
            const Level& V = c.lev[q];
            a.L[q - l] = CoarseLev{V.n, V.u, V.d, V.tau, V.res, V.rr, V.ru, V.snap};
            a.K[q - l] = make_consts(c, q);
            cells += (double)V.n * V.n * V.n;
        }
        ProfScope ps(c, K_MG_COARSE, 16.0 * 4.0 * cells);
#define CC(M, F) k_coarse_cycle<M, F><<<1, CC_T, 0, c.stream>>>(a)
        if (model == MGG_MODEL_FR) {
            if (frn == 0) CC(MGG_MODEL_FR, 0); else if (frn == 1) CC(MGG_MODEL_FR, 1); else CC(MGG_MODEL_FR, 2);
        } else if (model == MGG_MODEL_DGP) CC(MGG_MODEL_DGP, 0);
        else if (model == MGG_MODEL_KMOUFLAGE) CC(MGG_MODEL_KMOUFLAGE, 0);
        else if (model == MGG_MODEL_CSF) CC(MGG_MODEL_CSF, 0);
        else CC(MGG_MODEL_SYMMETRON, 0);
#undef CC
        MGG_CHECK_LAUNCH();
        return true;
    }

    // V_cycle (PMP2extradof.f90:352-555); the level-0 residual inside the
    // cycle only feeds the level-1 restriction, which recomputes it
    void vcycle(int l) {
        if (coarse_cycle(l, 0)) return;
        if (c.levelmax - l <= c.levelmin) { smooth(l); return; }
        smooth(l);
        if (l > 0) resid(l);
        coarse_prepare(l);
        vcycle(l + 1);
        correct(l + 1);
        smooth(l);
    }
    void fcycle(int l) {   // (563-865)
        if (coarse_cycle(l, 1)) return;
        if (c.levelmax - l <= c.levelmin) { smooth(l); return; }
        smooth(l);
        if (l > 0) resid(l);
        coarse_prepare(l);
        fcycle(l + 1);
        correct(l + 1);
        smooth(l);
        if (l > 0) resid(l);
        coarse_prepare(l);
        vcycle(l + 1);
        correct(l + 1);
        smooth(l);
    }
    void wcycle(int l) {   // (867-1165)
        if (coarse_cycle(l, 2)) return;
        if (c.levelmax - l <= c.levelmin) { smooth(l); return; }
        smooth(l);
        if (l > 0) resid(l);
        coarse_prepare(l);
        wcycle(l + 1);
        correct(l + 1);
        smooth(l);
        if (l > 0) resid(l);
        coarse_prepare(l);
        wcycle(l + 1);
        correct(l + 1);
        smooth(l);
    }

    void fill(float* f, int64_t n, float v) {
        ProfScope ps(c, K_GRID_OP, 4.0 * n);
        k_fill<<<grid_for(n), 256, 0, c.stream>>>(f, n, v);
        MGG_CHECK_LAUNCH();
    }
    void scale(float* f, int64_t n, double s) {
        ProfScope ps(c, K_GRID_OP, 8.0 * n);
        k_scale<<<grid_for(n), 256, 0, c.stream>>>(f, n, s);
        MGG_CHECK_LAUNCH();
    }
    void scale2(float* f, int64_t n, double s1, double s2) {
        ProfScope ps(c, K_GRID_OP, 8.0 * n);
        k_scale2<<<grid_for(n), 256, 0, c.stream>>>(f, n, s1, s2);
        MGG_CHECK_LAUNCH();
    }
};

double fr_ubg(const Ctx& c, double expo) {
    const mgg_config& g = c.cfg;
    const float A = c.aexpn;
    const double R_bg = 3.0 * ((double)(g.om / fcube(A)) + 4.0 * (double)g.oml);
    const double R0_bg = 3.0 * ((double)g.om + 4.0 * (double)g.oml);
    const double fR_bg = g.fr0 * pow(R0_bg / R_bg, g.fr_n + 1);
    return pow(fabs(fR_bg), expo);
}

// Largest cycle limit (iter_count_max) whose solve runs with the exit test on the
// device; a larger limit keeps the host loop.  A device-tested solve ends at the
// limit at the latest, as the host loop does.
constexpr int kDeviceLoopMax = 1024;

__global__ void k_mg_loop_reset(MgLoopState* st) {
    st->res_old_1 = 1.0e5;
    st->res_old_2 = 1.0e10;
    st->iter = 0;
    st->reason = 0;
    st->bad = 0;
}

// The exit test of scalar_field (PMP2extradof.f90:107-121) after one cycle, on the
// device, from the fixed-order sum of the level-0 squared residuals.  The double
// arithmetic is the host loop's (division and square root are correctly rounded
// on both sides), so the residuals, the cycle count and the exit reason are the
// host loop's bit for bit.  Sets the condition of the enclosing while node:
// 1 runs another cycle, 0 ends the solve.  A non-finite residual ends it too
// (and, with sticky non-null, sets bit 3 of *sticky).
__global__ void k_mg_exit(const double* __restrict__ sum, double n3, MgLoopState* st, int iter_max,
                          double res_conv, int32_t* sticky, cudaGraphConditionalHandle h) {
    const double res = sqrt(sum[0] / n3);
    const int iter = st->iter + 1;
    st->iter = iter;
    bool can_exit = false;
    int reason = 0;
    if (!isfinite(res)) {
        st->bad = 1;
        if (sticky) atomicOr(sticky, 8);
        can_exit = true;
    } else {
        if (iter <= 64) st->residual[iter - 1] = res;
        if (res <= res_conv) {
            can_exit = true;
            reason = 1;
        }
        if (iter > 2) {
            const double r1 = fabs(res / st->res_old_1 - 1.0);
            if (r1 <= 5.0e-3 || (r1 <= 1.0e-2 && fabs(st->res_old_1 / st->res_old_2 - 1.0) <= 1.0e-2)) {
                can_exit = true;
                if (!reason) reason = 2;
            }
        }
    }
    if (iter >= iter_max) {
        can_exit = true;
        if (!reason) reason = 3;
    }
    st->reason = reason;
    st->res_old_2 = st->res_old_1;
    st->res_old_1 = res;
    cudaGraphSetConditional(h, can_exit ? 0u : 1u);
}

// Copies the kernel parameters of graph src into graph dst, node by node in
// capture order.  Both must hold only kernel nodes, the same kernels with the
// same launch shapes in the same order; returns false (dst possibly partly
// updated) otherwise.
bool copy_kernel_params(cudaGraph_t src, cudaGraph_t dst) {
    size_t ns = 0, nd = 0;
    if (cudaGraphGetNodes(src, nullptr, &ns) != cudaSuccess || cudaGraphGetNodes(dst, nullptr, &nd) != cudaSuccess ||
        ns != nd || ns == 0)
        return false;
    std::vector<cudaGraphNode_t> a(ns), b(nd);
    if (cudaGraphGetNodes(src, a.data(), &ns) != cudaSuccess || cudaGraphGetNodes(dst, b.data(), &nd) != cudaSuccess)
        return false;
    for (size_t i = 0; i < ns; ++i) {
        cudaGraphNodeType ta, tb;
        if (cudaGraphNodeGetType(a[i], &ta) != cudaSuccess || cudaGraphNodeGetType(b[i], &tb) != cudaSuccess ||
            ta != cudaGraphNodeTypeKernel || tb != cudaGraphNodeTypeKernel)
            return false;
        cudaKernelNodeParams pa{}, pb{};
        if (cudaGraphKernelNodeGetParams(a[i], &pa) != cudaSuccess ||
            cudaGraphKernelNodeGetParams(b[i], &pb) != cudaSuccess)
            return false;
        if (pa.func != pb.func || pa.gridDim.x != pb.gridDim.x || pa.gridDim.y != pb.gridDim.y ||
            pa.gridDim.z != pb.gridDim.z || pa.blockDim.x != pb.blockDim.x || pa.blockDim.y != pb.blockDim.y ||
            pa.blockDim.z != pb.blockDim.z || pa.sharedMemBytes != pb.sharedMemBytes)
            return false;
        if (cudaGraphKernelNodeSetParams(b[i], &pa) != cudaSuccess) return false;
    }
    return true;
}

void mg_validate(const Ctx& c) {
    const mgg_config& g = c.cfg;
    if (g.mg_flag != 1 || !c.fi2) throw Error{MGG_ERR_STATE, "scalar_field: MG_flag is off"};
    if (g.mg_model < 1 || g.mg_model > 5) throw Error{MGG_ERR_ARG, "scalar_field: MG_model must be 1..5"};
    if ((g.mg_model == MGG_MODEL_KMOUFLAGE || g.mg_model == MGG_MODEL_CSF) && c.bgrows < 2)
        throw Error{MGG_ERR_STATE, "scalar_field: background table required for k-mouflage / csf"};
    if (g.mg_model == MGG_MODEL_FR && (g.fr_n < 0 || g.fr_n > 2))
        throw Error{MGG_ERR_UNSUPPORTED, "scalar_field: f(R) n must be 0, 1 or 2"};
    if (g.vcycle + g.fcycle + g.wcycle < 1) throw Error{MGG_ERR_ARG, "scalar_field: no cycle type selected"};
}

// initialise_extradof at the first step (PMP2extradof.f90:181-344) and the entry
// rescaling of a later step (47-80), queued; false when the step has no solve
// (the symmetron before a*, 37-41)
bool mg_enter(Ctx& c, Solver& s, int i_step) {
    const mgg_config& g = c.cfg;
    const float A = c.aexpn;
    if (i_step == 1) {
        double ubg = 0.0;
        if (g.mg_model == MGG_MODEL_FR) ubg = fr_ubg(c, 1.0 / (1.0 + (double)g.fr_n));
        else if (g.mg_model == MGG_MODEL_SYMMETRON && A > g.sym_astar) {
            const double sa = g.sym_astar / (double)A;
            ubg = sqrt(1.0 - sa * sa * sa);
        }
        s.fill(c.fi2, c.ncell, (float)ubg);
        c.fi2_pending = 0.0;
        c.have_fi2 = true;
    }
    if (g.mg_model == MGG_MODEL_SYMMETRON && A < g.sym_astar) return false;
    if (i_step > 1) {
        if (g.mg_model == MGG_MODEL_FR) {
            const double ubg = fr_ubg(c, 1.0 / (1.0 + (double)g.fr_n));
            if (c.fi2_pending != 0.0) s.scale2(c.fi2, c.ncell, c.fi2_pending, ubg);   // last exit + this entry
            else s.scale(c.fi2, c.ncell, ubg);
            c.fi2_pending = 0.0;
        }
        if (g.mg_model == MGG_MODEL_SYMMETRON) {
            const double sa = g.sym_astar / (double)A;
            s.fill(c.fi2, c.ncell, (float)sqrt(1.0 - sa * sa * sa));
        }
    }
    return true;
}

void run_cycle(const mgg_config& g, Solver& s) {
    if (g.vcycle == 1) s.vcycle(0);
    if (g.fcycle == 1) s.fcycle(0);
    if (g.wcycle == 1) s.wcycle(0);
}

// FI2 *= u_bg^-1 at the exit (PMP2extradof.f90:131-140), deferred to its next use
void mg_exit_rescale(Ctx& c) {
    const mgg_config& g = c.cfg;
    if (g.mg_model == MGG_MODEL_FR) c.fi2_pending = fr_ubg(c, -1.0 / (1.0 + (double)g.fr_n));
}

}  // namespace

int mg_device_loop_max() { return kDeviceLoopMax; }

// Whether this driver and runtime build graphs with conditional (while) nodes:
// checked once per process by building (not launching) such a graph.  Without
// them the solves keep the host loop and mgg_run_steps runs step by step.
bool mg_conditional_nodes() {
    static const bool ok = [] {
        cudaGraph_t g = nullptr;
        if (cudaGraphCreate(&g, 0) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cudaGraphConditionalHandle h;
        bool r = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
        if (r) {
            cudaGraphNodeParams p{};
            p.type = cudaGraphNodeTypeConditional;
            p.conditional.handle = h;
            p.conditional.type = cudaGraphCondTypeWhile;
            p.conditional.size = 1;
            cudaGraphNode_t node;
            r = cudaGraphAddNode(&node, g, nullptr, 0, &p) == cudaSuccess;
        }
        cudaGraphDestroy(g);
        cudaGetLastError();
        return r;
    }();
    return ok;
}

int mg_norm_partials(Ctx& c) {
    Solver s(c);
    return s.norm0_blocks();
}

bool mg_record_solve(Ctx& c, int i_step, Recorder& rec, MgLoopState* slot, int32_t* sticky) {
    mg_validate(c);
    const mgg_config& g = c.cfg;
    if (!c.mg_tuned || c.prof.on || g.iter_count_max > kDeviceLoopMax || !mg_conditional_nodes())
        throw Error{MGG_ERR_STATE, "scalar_field: a recorded solve needs a tuned context with profiling off"};
    Solver s(c);
    if (!mg_enter(c, s, i_step)) return false;
    const double n3 = pow((double)c.N, 3);
    k_mg_loop_reset<<<1, 1, 0, c.stream>>>(slot);
    MGG_CHECK_LAUNCH();
    rec.loop([&](cudaGraphConditionalHandle h) {
        run_cycle(g, s);
        s.norm0_async(c.red_out);
        k_mg_exit<<<1, 1, 0, c.stream>>>(c.red_out, n3, slot, g.iter_count_max, g.res_conv, sticky, h);
        MGG_CHECK_LAUNCH();
    });
    mg_exit_rescale(c);
    return true;
}

void mg_read_report(Ctx& c, mgg_mg_report* rep) {
    if (!c.mg_deferred) return;
    c.mg_deferred = false;
    const MgLoopState& m = c.h_step->mg;
    if (m.bad) throw Error{MGG_ERR_NUMERIC, "scalar_field: residual is not finite"};
    if (rep) {
        rep->cycles = m.iter;
        rep->exit_reason = m.reason;
        for (int i = 0; i < m.iter && i < 64; ++i) rep->residual[i] = m.residual[i];
    }
}

void mg_alloc(Ctx& c) {
    // the fused smoother's five-plane ring exceeds the 48 KB default
#define MGG_FB_ATTR(M, F, L0) \
    MGG_CUDA(cudaFuncSetAttribute(k_smooth_fused<M, F, L0>, cudaFuncAttributeMaxDynamicSharedMemorySize, FB_SMEM))
    MGG_FB_ATTR(MGG_MODEL_FR, 0, true); MGG_FB_ATTR(MGG_MODEL_FR, 0, false);
    MGG_FB_ATTR(MGG_MODEL_FR, 1, true); MGG_FB_ATTR(MGG_MODEL_FR, 1, false);
#define MGG_FB_ATTRX(M, F, L0) \
    MGG_CUDA(cudaFuncSetAttribute(k_smooth_fused<M, F, L0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, FB_SMEM))
    MGG_FB_ATTRX(MGG_MODEL_FR, 0, true); MGG_FB_ATTRX(MGG_MODEL_FR, 0, false);
    MGG_FB_ATTRX(MGG_MODEL_FR, 1, true); MGG_FB_ATTRX(MGG_MODEL_FR, 1, false);
    MGG_FB_ATTRX(MGG_MODEL_FR, 2, true); MGG_FB_ATTRX(MGG_MODEL_FR, 2, false);
    MGG_FB_ATTRX(MGG_MODEL_SYMMETRON, 0, true); MGG_FB_ATTRX(MGG_MODEL_SYMMETRON, 0, false);
#undef MGG_FB_ATTRX
    MGG_FB_ATTR(MGG_MODEL_FR, 2, true); MGG_FB_ATTR(MGG_MODEL_FR, 2, false);
    MGG_FB_ATTR(MGG_MODEL_SYMMETRON, 0, true); MGG_FB_ATTR(MGG_MODEL_SYMMETRON, 0, false);
#undef MGG_FB_ATTR
    const int N = c.N;
    int levelmax = 0;
    while ((1 << levelmax) < N) ++levelmax;
    int ngridmax = N;
    while (ngridmax % 2 == 0) ngridmax /= 2;
    int levelmin = 0;
    while ((1 << levelmin) < ngridmax) ++levelmin;
    levelmin += 1;   // PMP2extradof.f90:240-252
    c.levelmax = levelmax;
    c.levelmin = levelmin;
    if (levelmax >= 12) throw Error{MGG_ERR_ARG, "NGRID too large"};
    const bool need_snap = true;   // nDGP/k-mouflage snapshots, ping-pong of the fused sweep
    for (int l = 1; l <= levelmax; ++l) {
        Level& L = c.lev[l];
        L.n = N >> l;
        const size_t n3 = (size_t)L.n * L.n * L.n;
        float* block = nullptr;
        const int arrays = need_snap ? 7 : 6;
        MGG_CUDA(cudaMalloc(&block, sizeof(float) * n3 * arrays));
        MGG_CUDA(cudaMemset(block, 0, sizeof(float) * n3 * arrays));
        L.d = block;
        L.ru = block + n3;
        L.u = block + 2 * n3;
        L.tau = block + 3 * n3;
        L.res = block + 4 * n3;
        L.rr = block + 5 * n3;
        L.snap = need_snap ? block + 6 * n3 : nullptr;
    }
    c.lev[0].n = N;
    if (need_snap) MGG_CUDA(cudaMalloc(&c.lev[0].snap, sizeof(float) * c.ncell));
}

void fi2_materialize(Ctx& c) {
    if (c.fi2_pending == 0.0 || !c.fi2) return;
    k_scale<<<grid_for(c.ncell), 256, 0, c.stream>>>(c.fi2, c.ncell, c.fi2_pending);
    MGG_CHECK_LAUNCH();
    c.fi2_pending = 0.0;
}

void mg_scalar_field(Ctx& c, int i_step, mgg_mg_report* rep, bool defer) {
    const mgg_config& g = c.cfg;
    mg_validate(c);
    BucketScope bs(c, MGG_T_MG);
    Solver s(c);
    if (rep) memset(rep, 0, sizeof(*rep));
    c.mg_deferred = false;
    if (!mg_enter(c, s, i_step)) return;
    auto run_cycle = [&] { mgg::run_cycle(g, s); };
    // With per-kernel profiling off (after a context's first, eager solve, which
    // tunes the plane chunks), the cycles (tens to hundreds of launches, the same
    // for every cycle of this step) are captured into a CUDA graph.  Up to
    // kDeviceLoopMax cycles, the whole solve is one graph: a while node whose body
    // is a cycle, the level-0 residual norm and the exit test, so the host waits
    // once per solve (or, under mgg_step, once per step) instead of once per
    // cycle.  Above it (or without conditional graph nodes), the cycle graph is
    // replayed under the host loop.
    // Thread-local capture leaves other threads' CUDA calls alone.
    const bool graphed = !c.prof.on && c.mg_tuned;
    if (graphed && g.iter_count_max <= kDeviceLoopMax && mg_conditional_nodes()) {
        ensure_partials(c, s.norm0_blocks());   // no allocation under capture
        const double n3 = pow((double)c.N, 3);
        auto capture_body = [&](cudaGraphConditionalHandle h) {
            run_cycle();
            s.norm0_async(c.red_out);
            k_mg_exit<<<1, 1, 0, c.stream>>>(c.red_out, n3, c.mg_loop, g.iter_count_max, g.res_conv, nullptr, h);
            MGG_CHECK_LAUNCH();
        };
        // capture into body (an existing graph) or, with body null, into a new graph
        auto capture = [&](cudaGraph_t body, cudaGraphConditionalHandle h) -> cudaGraph_t {
            if (body)
                MGG_CUDA(cudaStreamBeginCaptureToGraph(c.stream, body, nullptr, nullptr, 0,
                                                       cudaStreamCaptureModeThreadLocal));
            else
                MGG_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
            cudaGraph_t ended = nullptr;
            try {
                capture_body(h);
            } catch (...) {
                cudaStreamEndCapture(c.stream, &ended);
                if (ended && !body) cudaGraphDestroy(ended);
                cudaGetLastError();
                throw;
            }
            MGG_CUDA(cudaStreamEndCapture(c.stream, &ended));
            return ended;
        };
        // Later solves of the context keep its graph: this step's cycle (whose kernel
        // constants follow the expansion factor) is captured on its own, its kernel
        // parameters are copied node by node into the kept body (same kernels, same
        // launch shapes, in capture order, else the graph is rebuilt), and the
        // executable graph is updated in place.  The while node and its condition
        // handle stay the same, so the exit test always sets its own loop's condition.
        bool reused = false;
        if (c.loop_exec) {
            cudaGraph_t fresh = capture(nullptr, c.loop_h);
            reused = copy_kernel_params(fresh, c.loop_body);
            cudaGraphDestroy(fresh);
            if (reused) {
                cudaGraphExecUpdateResultInfo info;
                reused = cudaGraphExecUpdate(c.loop_exec, c.loop_graph, &info) == cudaSuccess;
            }
            if (!reused) {
                cudaGetLastError();
                cudaGraphExecDestroy(c.loop_exec);
                cudaGraphDestroy(c.loop_graph);
                c.loop_exec = nullptr;
                c.loop_graph = nullptr;
                c.loop_body = nullptr;
            }
        }
        if (!reused) {
            cudaGraph_t outer = nullptr;
            MGG_CUDA(cudaGraphCreate(&outer, 0));
            try {
                cudaGraphConditionalHandle h;
                MGG_CUDA(cudaGraphConditionalHandleCreate(&h, outer, 1, cudaGraphCondAssignDefault));
                cudaGraphNodeParams p{};
                p.type = cudaGraphNodeTypeConditional;
                p.conditional.handle = h;
                p.conditional.type = cudaGraphCondTypeWhile;
                p.conditional.size = 1;
                cudaGraphNode_t node;
                MGG_CUDA(cudaGraphAddNode(&node, outer, nullptr, 0, &p));
                cudaGraph_t body = p.conditional.phGraph_out[0];
                capture(body, h);
                MGG_CUDA(cudaGraphInstantiate(&c.loop_exec, outer, 0));
                c.loop_graph = outer;
                c.loop_body = body;
                c.loop_h = h;
            } catch (...) {
                cudaGraphDestroy(outer);
                throw;
            }
        }
        k_mg_loop_reset<<<1, 1, 0, c.stream>>>(c.mg_loop);
        MGG_CHECK_LAUNCH();
        MGG_CUDA(cudaGraphLaunch(c.loop_exec, c.stream));
        MGG_CUDA(cudaMemcpyAsync(&c.h_step->mg, c.mg_loop, sizeof(MgLoopState), cudaMemcpyDeviceToHost, c.stream));
        c.mg_deferred = true;
        mg_exit_rescale(c);
        if (!defer) {
            MGG_CUDA(cudaStreamSynchronize(c.stream));
            mg_read_report(c, rep);
        }
        return;
    }
    if (graphed) {
        cudaGraph_t graph = nullptr;
        MGG_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
        try {
            run_cycle();
        } catch (...) {
            cudaStreamEndCapture(c.stream, &graph);
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            throw;
        }
        MGG_CUDA(cudaStreamEndCapture(c.stream, &graph));
        bool updated = false;
        if (c.mg_exec) {
            cudaGraphExecUpdateResultInfo info;
            if (cudaGraphExecUpdate(c.mg_exec, graph, &info) == cudaSuccess) {
                updated = true;
            } else {
                cudaGetLastError();
                cudaGraphExecDestroy(c.mg_exec);
                c.mg_exec = nullptr;
            }
        }
        cudaError_t e = cudaSuccess;
        if (!updated) e = cudaGraphInstantiate(&c.mg_exec, graph, 0);
        cudaGraphDestroy(graph);
        MGG_CUDA(e);
    }
    double res_old_1 = 1.0e5, res_old_2 = 1.0e10;
    int iter = 1;
    for (;;) {
        if (graphed) MGG_CUDA(cudaGraphLaunch(c.mg_exec, c.stream));
        else run_cycle();
        const double res = s.resid(0);
        if (!std::isfinite(res)) throw Error{MGG_ERR_NUMERIC, "scalar_field: residual is not finite"};
        if (rep && iter <= 64) rep->residual[iter - 1] = res;
        bool can_exit = false;
        int reason = 0;
        if (res <= g.res_conv) { can_exit = true; reason = 1; }
        if (iter > 2) {
            if (fabs(res / res_old_1 - 1.0) <= 5.0e-3) { can_exit = true; if (!reason) reason = 2; }
            if (fabs(res / res_old_1 - 1.0) <= 1.0e-2 && fabs(res_old_1 / res_old_2 - 1.0) <= 1.0e-2) {
                can_exit = true;
                if (!reason) reason = 2;
            }
        }
        if (iter >= g.iter_count_max) { can_exit = true; if (!reason) reason = 3; }
        if (can_exit) {
            mg_exit_rescale(c);
            if (rep) {
                rep->cycles = iter;
                rep->exit_reason = reason;
            }
            break;
        }
        ++iter;
        res_old_2 = res_old_1;
        res_old_1 = res;
    }
    c.mg_tuned = true;
}

}  // namespace mgg
