// Synthetic initial conditions on the device, in the role of PMP2start
// (PMP2start.f90:265-460, 797-873): a Gaussian random field on the NROW^3
// particle lattice, coloured by a BBKS P(k) normalised to sigma8 and scaled by
// the linear growth factor, turned into a Zel'dovich displacement with the same
// Stockham FFT as the Poisson solve.  Positions and velocities follow BLOCKS
// (PMP2start.f90:397-460): lattice point Q = QFACT*(ip-1) + 1, shift 0.5,
// x = Q + d + 0.5, v = d * (AEXPV/AEXPN) sqrt(AEXPV) sqrt(Om + OmL AEXPV^3)
// with AEXPV = AEXPN - ASTEP/2 (the ratio VCONS/XCONS of PMP2start.f90:836-837),
// and the same periodic wrap.
//
// The random numbers come from a counter-based generator (splitmix64 of the
// seed and the lattice index, Box-Muller), so a seed gives the same field on
// every device and launch shape.  The reference's RANLUX stream is not
// reproduced; P(k) is the reference's BBKS form with the Nyquist cut of TRUNF
// (PMP2start.f90:37-46).
#include "mgg_internal.cuh"
#include "fft.cuh"
#include <cmath>

namespace mgg {

namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__global__ void k_white_noise(float* __restrict__ f, int64_t n, uint64_t seed) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t h = splitmix64(seed ^ splitmix64((uint64_t)q));
        const double u1 = ((double)(h >> 11) + 1.0) * (1.0 / 9007199254740993.0);   // (0,1]
        const uint64_t h2 = splitmix64(h);
        const double u2 = (double)(h2 >> 11) * (1.0 / 9007199254740992.0);
        f[q] = (float)(sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2));
    }
}

__global__ void k_ic_place(const float* __restrict__ d, int nrow, int ngrid, int comp, double vfac,
                           float* __restrict__ pos, float* __restrict__ vel) {
    const int64_t np = (int64_t)nrow * nrow * nrow;
    const float qfact = (float)ngrid / (float)nrow;
    const float XMAX = (float)ngrid + 1.0f, XSHF = (float)ngrid;
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
        const int ip = (int)(p % nrow), jp = (int)((p / nrow) % nrow), kp = (int)(p / ((int64_t)nrow * nrow));
        const int a = comp == 0 ? ip : (comp == 1 ? jp : kp);
        const float Q = qfact * (float)a + 1.0f;
        const float disp = d[p];
        float x = Q + disp + 0.5f;
        if (x > XMAX) x = x - XSHF;
        if (x <= 1.0f) x = x + XSHF;
        if (x >= XMAX) x = x - 1.e-3f;
        if (x >= XMAX) x = x - 1.e-3f;
        pos[p] = x;
        vel[p] = (float)((double)disp * vfac);
    }
}

// ---- host cosmology -------------------------------------------------------
struct Cosmo {
    double om, oml, omb, h, ns;
    double gamma;   // BBKS shape, Sugiyama (1995) baryon correction
    double amp = 1.0;
    double T(double k) const {   // k in h/Mpc
        const double q = k / gamma;
        if (q <= 0) return 1.0;
        const double t = log(1.0 + 2.34 * q) / (2.34 * q);
        const double p = 1.0 + 3.89 * q + pow(16.1 * q, 2) + pow(5.46 * q, 3) + pow(6.71 * q, 4);
        return t * pow(p, -0.25);
    }
    double P(double k) const { return amp * pow(k, ns) * T(k) * T(k); }
    double sigma_R(double R) const {
        // sigma^2 = 1/(2 pi^2) int k^2 P(k) W^2(kR) dk, log-spaced Simpson
        const int n = 4000;
        const double lk0 = log(1e-5), lk1 = log(1e3);
        const double hstep = (lk1 - lk0) / n;
        double s = 0.0;
        for (int i = 0; i <= n; ++i) {
            const double k = exp(lk0 + i * hstep);
            const double x = k * R;
            const double W = x < 1e-4 ? 1.0 - x * x / 10.0 : 3.0 * (sin(x) - x * cos(x)) / (x * x * x);
            const double f = k * k * k * P(k) * W * W;
            const double w = (i == 0 || i == n) ? 1.0 : (i % 2 ? 4.0 : 2.0);
            s += w * f;
        }
        s *= hstep / 3.0;
        return sqrt(s / (2.0 * M_PI * M_PI));
    }
    double E(double a) const { return sqrt(om / (a * a * a) + oml + (1.0 - om - oml) / (a * a)); }
    double growth(double a) const {   // D(a) = 5 om / 2 E(a) int_0^a da' / (a' E(a'))^3
        const int n = 2000;
        double s = 0.0;
        for (int i = 1; i <= n; ++i) {
            const double x = a * (i - 0.5) / n;
            const double e = x * E(x);
            s += 1.0 / (e * e * e);
        }
        s *= a / n;
        return 2.5 * om * E(a) * s;
    }
};

}  // namespace

void make_ics(Ctx& c, const mgg_ic_params& ic) {
    wait_velocities(c);
    const mgg_config& g = c.cfg;
    const int nrow = g.nrow;
    if (nrow < 16 || (nrow & (nrow - 1)) || nrow > c.N)
        throw Error{MGG_ERR_ARG, "make_ics: NROW must be a power of two in [16, NGRID]"};
    const int64_t nc = (int64_t)nrow * nrow * nrow;
    Cosmo cm;
    cm.om = g.om;
    cm.oml = g.oml;
    cm.omb = g.omb;
    cm.h = ic.hubble;
    cm.ns = ic.ns;
    cm.gamma = cm.om * cm.h * exp(-cm.omb * (1.0 + sqrt(2.0 * cm.h) / cm.om));
    cm.amp = 1.0;
    const double s8 = cm.sigma_R(8.0);
    cm.amp = (ic.sigma8 / s8) * (ic.sigma8 / s8);
    const double D = cm.growth(ic.aexpn) / cm.growth(1.0);
    // plan for the NROW lattice
    FftPlan p;
    p.n = nrow;
    p.nxp = ((nrow / 2 + 1) + 15) / 16 * 16;
    std::vector<float2> tw(nrow);
    for (int k = 0; k < nrow; ++k) {
        const double a = -2.0 * M_PI * (double)k / (double)nrow;
        tw[k] = make_float2((float)cos(a), (float)sin(a));
    }
    float2* dtw = nullptr;
    float* dtk = nullptr;
    MGG_CUDA(cudaMalloc(&dtw, sizeof(float2) * nrow));
    MGG_CUDA(cudaMemcpyAsync(dtw, tw.data(), sizeof(float2) * nrow, cudaMemcpyHostToDevice, c.stream));
    p.tw = dtw;
    // displacement amplitude per integer |m|^2 (grid units of the PM mesh):
    //   tk = 2 * sqrt(P(k) / (V Nc)) * D * N / (2 pi),  k = 2 pi |m| / Box, 0 for |m| >= NROW/2
    const int m2max = 3 * (nrow / 2) * (nrow / 2);
    std::vector<float> tk(m2max + 1, 0.f);
    const double V = (double)g.box * g.box * g.box;
    for (int m2 = 1; m2 <= m2max; ++m2) {
        const double wk = sqrt((double)m2);
        if (wk >= (double)(nrow / 2)) continue;
        const double k = 2.0 * M_PI * wk / (double)g.box;
        tk[m2] = (float)(2.0 * sqrt(cm.P(k) / (V * (double)nc)) * D * (double)c.N / (2.0 * M_PI));
    }
    MGG_CUDA(cudaMalloc(&dtk, sizeof(float) * (m2max + 1)));
    MGG_CUDA(cudaMemcpyAsync(dtk, tk.data(), sizeof(float) * (m2max + 1), cudaMemcpyHostToDevice, c.stream));
    // buffers: noise / displacement on FI (>= NROW^3 floats), spectra inside cbuf
    float* real = c.fi;
    float2* spec = c.cbuf;
    float2* work = c.cbuf + (size_t)p.nxp * nrow * nrow;
    float2* own_work = nullptr;
    if (2 * (size_t)p.nxp * nrow * nrow > (size_t)c.nxp * c.N * c.N) {
        MGG_CUDA(cudaMalloc(&own_work, sizeof(float2) * (size_t)p.nxp * nrow * nrow));
        work = own_work;
    }
    {
        ProfScope ps(c, K_IC, 4.0 * nc);
        k_white_noise<<<148 * 8, 256, 0, c.stream>>>(real, nc, ic.seed);
        MGG_CHECK_LAUNCH();
    }
    LineExtra ex;
    fft_x_r2c(p, real, spec, c.stream);
    fft_lines(p, spec, 1, LM_FWD, ex, c.stream);
    fft_lines(p, spec, 2, LM_FWD, ex, c.stream);
    const float AEXPN = ic.aexpn, ASTEP = ic.astep;
    const float AEXPV = AEXPN - ASTEP / 2.0f;
    const double vfac = (double)(AEXPV / AEXPN) * sqrt((double)AEXPV) * sqrt((double)(g.om + g.oml * AEXPV * AEXPV * AEXPV));
    float* pos[3] = {c.x, c.y, c.z};
    float* vel[3] = {c.vx, c.vy, c.vz};
    for (int comp = 0; comp < 3; ++comp) {
        LineExtra ed;
        ed.src = spec;
        ed.tk = dtk;
        ed.comp = comp;
        fft_lines(p, work, 2, LM_DISP, ed, c.stream);
        fft_lines(p, work, 1, LM_INV, ex, c.stream);
        fft_x_c2r(p, work, real, c.stream);
        ProfScope ps(c, K_IC, 12.0 * nc);
        k_ic_place<<<148 * 8, 256, 0, c.stream>>>(real, nrow, c.N, comp, vfac, pos[comp], vel[comp]);
        MGG_CHECK_LAUNCH();
    }
    MGG_CUDA(cudaStreamSynchronize(c.stream));
    MGG_CUDA(cudaFree(dtw));
    MGG_CUDA(cudaFree(dtk));
    if (own_work) MGG_CUDA(cudaFree(own_work));
    c.have_particles = true;
    c.aexpn = AEXPN;
    c.astep = ASTEP;
}

}  // namespace mgg
