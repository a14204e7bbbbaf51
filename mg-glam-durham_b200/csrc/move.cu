// Kernel (c): MOVE(FactV) (PMP2main.f90:304-685) -- potential gradient at the
// 8 CIC nodes from 32 gathered FI values, CIC interpolation to the particle,
// leapfrog kick and drift, periodic wrap, and the kinetic-energy sum.
// Kernel (e): POTENT_FOR_MG (PMP2main.f90:869-1015) -- the fifth-force
// potential of FI2 added to FI.
//
// Arithmetic follows the reference: the 32 FI values are Real*4 and their
// 24 differences are taken in Real*4 (566-594), the interpolation, kick and
// drift are Real*8 (315-324), PCONST/XCONST are Real*4 expressions of AEXPN,
// ASTEP and FactV (336-338), positions and velocities are stored as Real*4.
// The sum of v^2 is reduced in a fixed order (block tree + ordered partials),
// so ENKIN is the same on every run.
#include "mgg_internal.cuh"
#include "reduce.cuh"
#include <cmath>

namespace mgg {

namespace {

struct MoveConsts {
    double pconst, xconst;
    double fric_fac;   // symmetron / k-mouflage / csf friction
    double bs_m1;      // bs_fct - 1
    int sym_fric, bg_fric;
    double astep_over_fv;
    double xn, yn;     // N+1 (Real*4 expression) and N
    double wpar;
};

__global__ void __launch_bounds__(256, 3) k_move(const float* __restrict__ fi, const float* __restrict__ fi2,
                                              float* __restrict__ xp, float* __restrict__ yp, float* __restrict__ zp,
                                              float* __restrict__ vxp, float* __restrict__ vyp,
                                              float* __restrict__ vzp, int64_t np, int N, MoveConsts k,
                                              double* __restrict__ part, const int32_t* __restrict__ skip_flags,
                                              const MgLoopState* __restrict__ skip_mg) {
    // a step whose density or transforms set an error flag, or whose multigrid solve
    // saw a non-finite residual, leaves the particles as they were (the host reports it)
    if ((skip_flags && *skip_flags) || (skip_mg && skip_mg->bad)) {
        if (threadIdx.x == 0) part[blockIdx.x] = 0.0;
        return;
    }
    double sv = 0.0;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
        double X = xp[p], Y = yp[p], Z = zp[p];
        double VVX = vxp[p], VVY = vyp[p], VVZ = vzp[p];
        int I = (int)X, J = (int)Y, K = (int)Z;
        I = I < 1 ? 1 : (I > N ? N : I);
        J = J < 1 ? 1 : (J > N ? N : J);
        K = K < 1 ? 1 : (K > N ? N : K);
        const double D1 = X - (double)(float)I, D2 = Y - (double)(float)J, D3 = Z - (double)(float)K;
        const double T1 = 1.0 - D1, T2 = 1.0 - D2, T3 = 1.0 - D3;
        const double T2T1 = T2 * T1, T2D1 = T2 * D1, D2T1 = D2 * T1, D2D1 = D2 * D1;
        // 0-based neighbour indices
        const int i = I - 1, j = J - 1, kk = K - 1;
        const int i1 = I == N ? 0 : I, j1 = J == N ? 0 : J, k1 = K == N ? 0 : K;
        const int i2 = i1 + 1 == N ? 0 : i1 + 1, j2 = j1 + 1 == N ? 0 : j1 + 1, k2 = k1 + 1 == N ? 0 : k1 + 1;
        const int i0 = i == 0 ? N - 1 : i - 1, j0 = j == 0 ? N - 1 : j - 1, k0 = kk == 0 ? N - 1 : kk - 1;
        // row offsets fit 32 bits (N^3 <= 2^30)
        auto F = [&](int a, int b, int c) -> float { return __ldg(fi + (a + N * (b + N * c))); };
        const float F111 = F(i, j, kk), F211 = F(i1, j, kk), F121 = F(i, j1, kk), F221 = F(i1, j1, kk);
        const float F112 = F(i, j, k1), F212 = F(i1, j, k1), F122 = F(i, j1, k1), F222 = F(i1, j1, k1);
        const float F113 = F(i, j, k2), F213 = F(i1, j, k2), F123 = F(i, j1, k2), F223 = F(i1, j1, k2);
        const float F110 = F(i, j, k0), F210 = F(i1, j, k0), F120 = F(i, j1, k0), F220 = F(i1, j1, k0);
        const float F311 = F(i2, j, kk), F321 = F(i2, j1, kk), F131 = F(i, j2, kk), F231 = F(i1, j2, kk);
        const float F312 = F(i2, j, k1), F322 = F(i2, j1, k1), F132 = F(i, j2, k1), F232 = F(i1, j2, k1);
        const float F011 = F(i0, j, kk), F021 = F(i0, j1, kk), F101 = F(i, j0, kk), F201 = F(i1, j0, kk);
        const float F012 = F(i0, j, k1), F022 = F(i0, j1, k1), F102 = F(i, j0, k1), F202 = F(i1, j0, k1);
        const double GX111 = (double)(F211 - F011), GX211 = (double)(F311 - F111), GX121 = (double)(F221 - F021),
                     GX221 = (double)(F321 - F121);
        const double GX112 = (double)(F212 - F012), GX212 = (double)(F312 - F112), GX122 = (double)(F222 - F022),
                     GX222 = (double)(F322 - F122);
        const double GY111 = (double)(F121 - F101), GY211 = (double)(F221 - F201), GY121 = (double)(F131 - F111),
                     GY221 = (double)(F231 - F211);
        const double GY112 = (double)(F122 - F102), GY212 = (double)(F222 - F202), GY122 = (double)(F132 - F112),
                     GY222 = (double)(F232 - F212);
        const double GZ111 = (double)(F112 - F110), GZ211 = (double)(F212 - F210), GZ121 = (double)(F122 - F120),
                     GZ221 = (double)(F222 - F220);
        const double GZ112 = (double)(F113 - F111), GZ212 = (double)(F213 - F211), GZ122 = (double)(F123 - F121),
                     GZ222 = (double)(F223 - F221);
        const double GX = k.pconst * (T3 * (T2T1 * GX111 + T2D1 * GX211 + D2T1 * GX121 + D2D1 * GX221) +
                                      D3 * (T2T1 * GX112 + T2D1 * GX212 + D2T1 * GX122 + D2D1 * GX222));
        const double GY = k.pconst * (T3 * (T2T1 * GY111 + T2D1 * GY211 + D2T1 * GY121 + D2D1 * GY221) +
                                      D3 * (T2T1 * GY112 + T2D1 * GY212 + D2T1 * GY122 + D2D1 * GY222));
        const double GZ = k.pconst * (T3 * (T2T1 * GZ111 + T2D1 * GZ211 + D2T1 * GZ121 + D2D1 * GZ221) +
                                      D3 * (T2T1 * GZ112 + T2D1 * GZ212 + D2T1 * GZ122 + D2D1 * GZ222));
        if (k.sym_fric) {   // (613-617)
            const double f2 = (double)__ldg(fi2 + (i + N * (j + N * kk)));
            VVX = VVX + k.fric_fac * f2 * VVX * k.astep_over_fv;
            VVY = VVY + k.fric_fac * f2 * VVY * k.astep_over_fv;
            VVZ = VVZ + k.fric_fac * f2 * VVZ * k.astep_over_fv;
        }
        if (k.bg_fric) {    // (619-630)
            VVX = VVX + k.fric_fac * VVX * k.astep_over_fv;
            VVY = VVY + k.fric_fac * VVY * k.astep_over_fv;
            VVZ = VVZ + k.fric_fac * VVZ * k.astep_over_fv;
            VVX = VVX + k.bs_m1 * GX;
            VVY = VVY + k.bs_m1 * GY;
            VVZ = VVZ + k.bs_m1 * GZ;
        }
        VVX = VVX + GX;
        VVY = VVY + GY;
        VVZ = VVZ + GZ;
        X = X + VVX * k.xconst;
        Y = Y + VVY * k.xconst;
        Z = Z + VVZ * k.xconst;
        if (X < 1.0) X = X + k.yn;
        if (X >= k.xn) X = X - k.yn;
        if (Y < 1.0) Y = Y + k.yn;
        if (Y >= k.xn) Y = Y - k.yn;
        if (Z < 1.0) Z = Z + k.yn;
        if (Z >= k.xn) Z = Z - k.yn;
        sv = sv + (VVX * VVX + VVY * VVY + VVZ * VVZ) * k.wpar;
        float xf = (float)X, yf = (float)Y, zf = (float)Z;
        if ((int)xf == N + 1) xf = xf - 1.e-3f;   // (673-675)
        if ((int)yf == N + 1) yf = yf - 1.e-3f;
        if ((int)zf == N + 1) zf = zf - 1.e-3f;
        xp[p] = xf;
        yp[p] = yf;
        zp[p] = zf;
        vxp[p] = (float)VVX;
        vyp[p] = (float)VVY;
        vzp[p] = (float)VVZ;
    }
    sv = block_sum_fixed(sv);
    if (threadIdx.x == 0) part[blockIdx.x] = sv;
}

// FI += fct * FI2^(pw) with the power taken in Real*4, the sum in Real*8; with
// pre != 0, FI2 is first rescaled by pre and rounded to Real*4 (a pending
// rescaling of the scalar field, applied here instead of in its own pass)
__global__ void k_potent_mg(float* __restrict__ fi, const float* __restrict__ fi2, int64_t n4, double fct, int pw,
                            double pre) {
    float4* f4 = reinterpret_cast<float4*>(fi);
    const float4* g4 = reinterpret_cast<const float4*>(fi2);
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n4; q += (int64_t)gridDim.x * blockDim.x) {
        float4 f = f4[q];
        float4 g = __ldg(g4 + q);
        if (pre != 0.0) {
            g.x = (float)((double)g.x * pre);
            g.y = (float)((double)g.y * pre);
            g.z = (float)((double)g.z * pre);
            g.w = (float)((double)g.w * pre);
        }
        auto term = [&](float u) -> double {
            if (pw == 1) return fct * (double)u;
            if (pw == 2) return fct * (double)(u * u);
            return fct * (double)(u * u * u);
        };
        f.x = (float)((double)f.x + term(g.x));
        f.y = (float)((double)f.y + term(g.y));
        f.z = (float)((double)f.z + term(g.z));
        f.w = (float)((double)f.w + term(g.w));
        f4[q] = f;
    }
}

inline float fcube(float a) { return a * a * a; }

// background-table interpolation, first row with a_row >= a (PMP2main.f90:351-358)
double bg_interp(const std::vector<double>& t, int rows, double a, double aval, int col) {
    int ist = 0;
    while (ist < rows - 1 && t[ist * 6 + 0] < a) ++ist;
    if (ist == 0) ist = 1;
    const double* r0 = &t[(ist - 1) * 6];
    const double* r1 = &t[ist * 6];
    return r0[col] + (r1[col] - r0[col]) / (r1[0] - r0[0]) * (aval - r0[0]);
}

}  // namespace

float move_enkin(const Ctx& c, double svel) {   // (666)
    const float ah = c.aexpn + c.astep / 2.0f;
    return (float)(svel / 2.0 / (double)(ah * ah));
}

void move_particles(Ctx& c, float FactV, double* enkin, bool defer) {
    if (defer) {   // SVEL into red_out[1]; the caller reads it back with the step's other results
        move_enqueue(c, FactV, c.red_out + 1, c.d_flags, c.mg_deferred ? c.mg_loop : nullptr);
        return;
    }
    move_enqueue(c, FactV, c.red_out, nullptr, nullptr);
    MGG_CUDA(cudaMemcpyAsync(c.h_red, c.red_out, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaStreamSynchronize(c.stream));
    const float ENKIN = move_enkin(c, c.h_red[0]);
    if (!std::isfinite(ENKIN)) throw Error{MGG_ERR_NUMERIC, "move: kinetic energy is not finite"};
    if (enkin) *enkin = (double)ENKIN;
}

void move_enqueue(Ctx& c, float FactV, double* svel, const int32_t* skip_flags, const MgLoopState* skip_mg) {
    if (!c.have_particles) throw Error{MGG_ERR_STATE, "move: no particles uploaded"};
    wait_velocities(c);
    BucketScope bs(c, MGG_T_MOVE);
    const mgg_config& g = c.cfg;
    const float AEXPN = c.aexpn, ASTEP = c.astep;
    const float Om = g.om, OmL = g.oml;
    MoveConsts k{};
    k.pconst = (double)(-sqrtf(AEXPN / (Om + OmL * fcube(AEXPN))) * ASTEP * 0.5f / FactV);
    const float Ahalf = AEXPN + ASTEP / 2.0f;
    k.xconst = (double)(ASTEP / sqrtf(Ahalf * (Om + OmL * fcube(Ahalf))) / Ahalf);
    if (g.mg_model == MGG_MODEL_KMOUFLAGE) {
        const float r = 9.116748693e-5f;
        k.pconst = (double)(-sqrtf(AEXPN / (Om + r / AEXPN + (OmL - r) * fcube(AEXPN))) * ASTEP * 0.5f / FactV);
        k.xconst = (double)(ASTEP / sqrtf(Ahalf * (Om + r / Ahalf + (OmL - r) * fcube(Ahalf))) / Ahalf);
    }
    double bs_fct = 1.0;
    if (g.mg_flag == 1 && (g.mg_model == 4 || g.mg_model == 5)) {
        if (c.bgrows < 2) throw Error{MGG_ERR_STATE, "move: background table required for this model"};
        double pc = bg_interp(c.h_bg, c.bgrows, AEXPN, AEXPN, 4);
        double P = 1.0 / pc;
        k.pconst = -P * ASTEP * 0.5 / FactV;
        double xc = bg_interp(c.h_bg, c.bgrows, Ahalf, Ahalf, 4);
        xc = (double)(Ahalf * Ahalf) * xc;
        k.xconst = 1.0 / xc * ASTEP;
        bs_fct = bg_interp(c.h_bg, c.bgrows, Ahalf, AEXPN, 1);
        if (g.mg_model == 4) bs_fct = exp(g.kmf_beta * bs_fct);
        if (g.mg_model == 5 && g.csf_coupling == 1) bs_fct = exp(g.csf_beta * bs_fct);
    }
    k.fric_fac = 0.0;
    if (g.mg_flag == 1) {
        if (g.mg_model == 3 && AEXPN > g.sym_astar) {
            const double sa = g.sym_astar / (double)AEXPN;
            k.fric_fac = (double)(-9.0f * Om) * g.sym_beta * g.sym_beta * g.sym_xi * g.sym_xi * sqrt(1.0 - sa * sa * sa);
            k.sym_fric = 1;
        }
        if (g.mg_model == 4 || g.mg_model == 5) {
            const double pb = g.mg_model == 4 ? g.kmf_beta : g.csf_beta;
            double f = bg_interp(c.h_bg, c.bgrows, AEXPN, AEXPN, 2);
            f = f / (double)AEXPN;
            k.fric_fac = -f * pb;
            k.bg_fric = 1;
        }
    }
    k.bs_m1 = bs_fct - 1.0;
    k.astep_over_fv = (double)ASTEP / (double)FactV;
    k.xn = (double)((float)c.N + 1.0f - 1.0e-8f);
    k.yn = (double)(float)c.N;
    k.wpar = (double)(float)((double)c.N * c.N * c.N / (double)(float)c.np);
    const int blocks = 148 * 8;
    ensure_partials(c, blocks);
    {
        ProfScope ps(c, K_MOVE, 48.0 * (double)c.np + 4.0 * (double)c.ncell);
        k_move<<<blocks, 256, 0, c.stream>>>(c.fi, c.fi2 ? c.fi2 : c.fi, c.x, c.y, c.z, c.vx, c.vy, c.vz, c.np, c.N,
                                             k, c.red_partial, skip_flags, skip_mg);
        MGG_CHECK_LAUNCH();
    }
    reduce_sum_blocks_async(c, blocks, svel);
}

void potential_mg(Ctx& c) {
    const mgg_config& g = c.cfg;
    if (!c.fi2) throw Error{MGG_ERR_STATE, "potential_mg: MG_flag is off (no FI2)"};
    BucketScope bs(c, MGG_T_FORCE);
    const float AEXPN = c.aexpn;
    const double ctilde = kCtildeC * (double)c.N / (double)g.box;
    double fct = 0.0;
    int pw = 1;
    switch (g.mg_model) {
    case 1: {
        const double R_bg = 3.0 * ((double)(g.om / fcube(AEXPN)) + 4.0 * (double)g.oml);
        const double R0_bg = 3.0 * ((double)g.om + 4.0 * (double)g.oml);
        const double fR_bg = g.fr0 * pow(R0_bg / R_bg, g.fr_n + 1);
        fct = -(ctilde * ctilde * 0.5 * fR_bg);
        pw = g.fr_n + 1;
        break;
    }
    case 2: fct = 0.5; pw = 1; break;
    case 3:
        fct = 3.0 * g.sym_xi * g.sym_xi * (double)g.om * g.sym_beta * g.sym_beta * ctilde * ctilde /
              (g.sym_astar * g.sym_astar * g.sym_astar);
        pw = 2;
        break;
    case 4: fct = g.kmf_beta * ctilde; pw = 1; break;
    case 5: fct = g.csf_coupling == 1 ? g.csf_beta : 0.0; pw = 1; break;
    default: throw Error{MGG_ERR_UNSUPPORTED, "potential_mg: unknown MG_model"};
    }
    ProfScope ps(c, K_POTENT_MG, 12.0 * (double)c.ncell);
    k_potent_mg<<<148 * 16, 256, 0, c.stream>>>(c.fi, c.fi2, c.ncell / 4, fct, pw, c.fi2_pending);
    MGG_CHECK_LAUNCH();
}

}  // namespace mgg
