// Analysis after the step: the redshift-space power spectrum multipoles of
// GetPower(1) (PMP2mod_power.f90:20-108 with DENSITrsd, PMP2mod_density.f90:
// 407-557) and the density PDFs of DensDistr (PMP2mod_density.f90:1041-1126)
// on the NGRID/2^l meshes that Analysis uses (PMP2mod_analyze.f90:44-86).
//
// Both need the CIC density of rescaled (and, in redshift space, displaced)
// particle positions on a coarser mesh.  k_rsd_positions forms those positions
// with the reference's Real*4 expressions; the deterministic CIC of the PM step
// (cic_grid) deposits them.  The reference computes the density and the FFT
// twice per line of sight (once for the monopole, once for the quadrupole);
// here one spectrum feeds both sums (LineExtra::quad).
//
// Only sigv = 0 is restated: the extra velocity dispersion vv of dense
// particles is zero, as it is when Setup.dat's sigv is 0 (its random numbers
// come from the reference's RANLUX pages, which this library does not carry).
#include "mgg_internal.cuh"
#include "reduce.cuh"

#include <cmath>

namespace mgg {

namespace {

// Positions of DENSITrsd(iSwitch, NGRID_old) on the ng mesh: X = (XPAR-1)*Xscale+1
// in Real*4; for iSwitch = 1, 2, 3 the axes rotate so that the displaced axis is
// the third and it moves by (V*Xscale + vv)*factor, vv = 0 (PMP2mod_density.f90:
// 466-496).  The periodic wrap (497-503) is exact for X >= ng+1; for X < 1 the
// reference adds ng in Real*8, here in FP32 (the result rounds to the FP32 grid
// of [ng, ng+1); a sum that rounds up to ng+1 is the periodic image X = 1).
__global__ void k_rsd_positions(const float* __restrict__ x, const float* __restrict__ y,
                                const float* __restrict__ z, const float* __restrict__ vx,
                                const float* __restrict__ vy, const float* __restrict__ vz, int64_t np, int iswitch,
                                float xscale, float factor, int ng, float* __restrict__ ox, float* __restrict__ oy,
                                float* __restrict__ oz) {
    const float top = (float)ng + 1.0f, fng = (float)ng;
    auto scaled = [&](float p) { return __fadd_rn(__fmul_rn(__fsub_rn(p, 1.0f), xscale), 1.0f); };
    auto shift = [&](float v) { return __fmul_rn(__fadd_rn(__fmul_rn(v, xscale), 0.0f), factor); };
    auto wrap = [&](float v) {
        if (v >= top) v = __fsub_rn(v, fng);
        if (v < 1.0f) {
            v = __fadd_rn(v, fng);
            if (v >= top) v = 1.0f;
        }
        return v;
    };
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < np; p += (int64_t)gridDim.x * blockDim.x) {
        const float px = scaled(__ldg(x + p)), py = scaled(__ldg(y + p)), pz = scaled(__ldg(z + p));
        float X = px, Y = py, Z = pz;
        if (iswitch == 1) {
            Z = __fadd_rn(px, shift(__ldg(vx + p)));
            Y = py;
            X = pz;
        } else if (iswitch == 2) {
            Z = __fadd_rn(py, shift(__ldg(vy + p)));
            Y = pz;
        } else if (iswitch == 3) {
            Z = __fadd_rn(pz, shift(__ldg(vz + p)));
        }
        ox[p] = wrap(X);
        oy[p] = wrap(Y);
        oz[p] = wrap(Z);
    }
}

// DensDistr bins: i = floor(log10(1 + delta) / 0.001), clamped to [-2001, 2001]
// (iMin = log10(0.01)/dlog - 1, iMax = log10(100)/dlog + 1); the Real*4 LOG10 is
// taken as the correctly rounded FP32 log10 (FP64 log10 rounded to FP32); an
// empty cell (1 + delta = 0) goes to iMin.
constexpr int kPdfMin = -2001, kPdfBins = MGG_PDF_BINS, kPdfThreads = 512;

__device__ __forceinline__ int pdf_bin(float v) {
    if (!(v > 0.0f)) return 0;
    const double l = (double)(float)log10((double)v);
    const double f = floor(l / 0.001);
    const int i = f < (double)kPdfMin ? kPdfMin : (f > (double)(kPdfMin + kPdfBins - 1) ? kPdfMin + kPdfBins - 1 : (int)f);
    return i - kPdfMin;
}

// Per-bin cell counts and sums of 1 + delta (shared-memory histograms, then one
// global atomic per non-empty bin and block), and per-block partial sums of
// 1 + delta and (1 + delta)^2 (Real*4 square, as (FI+1.)**2) in a fixed order.
// The per-bin FP64 sums add FP32 values that lie within 0.001 dex of each other,
// so they are exact -- and the result independent of the order -- while a bin
// holds fewer than 2^29 cells.
__global__ void __launch_bounds__(kPdfThreads) k_density_pdf(const float* __restrict__ fi, int64_t n,
                                                             unsigned long long* __restrict__ cnt,
                                                             double* __restrict__ den, double* __restrict__ part) {
    __shared__ unsigned int sc[kPdfBins];
    __shared__ double sd[kPdfBins];
    for (int b = threadIdx.x; b < kPdfBins; b += kPdfThreads) {
        sc[b] = 0u;
        sd[b] = 0.0;
    }
    __syncthreads();
    double s1 = 0.0, s2 = 0.0;
    for (int64_t q = (int64_t)blockIdx.x * kPdfThreads + threadIdx.x; q < n; q += (int64_t)gridDim.x * kPdfThreads) {
        const float v = __fadd_rn(__ldg(fi + q), 1.0f);
        s1 += (double)v;
        s2 += (double)__fmul_rn(v, v);
        const int b = pdf_bin(v);
        atomicAdd(sc + b, 1u);
        atomicAdd(sd + b, (double)v);
    }
    __syncthreads();
    for (int b = threadIdx.x; b < kPdfBins; b += kPdfThreads)
        if (sc[b]) {
            atomicAdd(cnt + b, (unsigned long long)sc[b]);
            atomicAdd(den + b, sd[b]);
        }
    s1 = block_sum_fixed(s1);
    if (threadIdx.x == 0) part[blockIdx.x] = s1;
    s2 = block_sum_fixed(s2);
    if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = s2;
}

// three position arrays of np floats, stream-ordered
struct PosScratch {
    Ctx& c;
    float* p = nullptr;
    explicit PosScratch(Ctx& c_) : c(c_) {
        MGG_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&p), sizeof(float) * 3 * (size_t)c.np, c.stream));
    }
    ~PosScratch() {
        if (p) cudaFreeAsync(p, c.stream);
    }
    float* x() { return p; }
    float* y() { return p + c.np; }
    float* z() { return p + 2 * c.np; }
};

void rsd_positions(Ctx& c, PosScratch& s, int iswitch, int ng, float factor) {
    const float xscale = (float)ng / (float)c.N;   // Xscale = Float(NGRID)/NGRID_old (Real*4)
    const int blocks = (int)std::min<int64_t>(div_up(c.np, 256), 148 * 16);
    ProfScope ps(c, K_GRID_OP, (iswitch ? 16.0 : 12.0) * c.np + 12.0 * c.np);
    k_rsd_positions<<<blocks, 256, 0, c.stream>>>(c.x, c.y, c.z, c.vx, c.vy, c.vz, c.np, iswitch, xscale, factor, ng,
                                                  s.x(), s.y(), s.z());
    MGG_CHECK_LAUNCH();
}

void check_positions(Ctx& c) {
    int32_t h = 0;
    MGG_CUDA(cudaMemcpyAsync(&h, c.d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaStreamSynchronize(c.stream));
    if (h & 1) {   // bit 0: a position outside the box
        MGG_CUDA(cudaMemsetAsync(c.d_flags, 0, sizeof(int32_t), c.stream));
        throw Error{MGG_ERR_NUMERIC, "analysis: a particle position is outside [1, NGRID+1)"};
    }
}

}  // namespace

void power_rsd(Ctx& c, int nbins, double* k, double* nm, double* preal, double* p0, double* p2) {
    if (!c.have_particles) throw Error{MGG_ERR_STATE, "power_rsd: no particles uploaded"};
    const int ng = c.N / 2;
    if (ng < 16) throw Error{MGG_ERR_ARG, "power_rsd: NGRID must be at least 32"};
    if (nbins < 1 || nbins > ng / 2) throw Error{MGG_ERR_ARG, "power_rsd: nbins must be in [1, NGRID/4]"};
    BucketScope bs(c, MGG_T_POWER);
    wait_velocities(c);
    if (!c.tw_h) c.tw_h = make_twiddles(ng);
    if (!c.tw64_h) c.tw64_h = make_twiddles64(ng);
    if (!c.pk_logbin_h) c.pk_logbin_h = make_logbins(ng);
    // factor = sqrt(AEXPN/(Om+AEXPN**3*OmL))/AEXPN in Real*4 (PMP2mod_density.f90:436)
    const float A = c.aexpn, om = c.cfg.om, oml = c.cfg.oml;
    const float factor = std::sqrt(A / (om + A * A * A * oml)) / A;
    PosScratch s(c);
    PkBins b[4];
    for (int sw = 0; sw <= 3; ++sw) {
        rsd_positions(c, s, sw, ng, factor);
        cic_grid(c, s.x(), s.y(), s.z(), ng, c.fi);
        power_bins(c, c.fi, ng, c.tw_h, c.cfg.precision == MGG_PREC_PLAIN ? c.tw64_h : nullptr, c.pk_logbin_h,
                   sw > 0, b[sw]);
    }
    check_positions(c);
    for (int I = 1; I <= nbins; ++I) {
        if (k) k[I - 1] = b[0].k[I];
        if (nm) nm[I - 1] = b[0].n[I];
        if (preal) preal[I - 1] = b[0].p[I];
        // P0 = (Pk(I,2)+Pk(I,4)+Pk(I,6))/3., P2 = (Pk(I,1)+Pk(I,3)+Pk(I,5))/3. in Real*4 (PMP2mod_power.f90:94-95)
        const float s0 = ((float)b[1].p[I] + (float)b[2].p[I]) + (float)b[3].p[I];
        const float s2 = ((float)b[1].q[I] + (float)b[2].q[I]) + (float)b[3].q[I];
        if (p0) p0[I - 1] = s0 / 3.0f;
        if (p2) p2[I - 1] = s2 / 3.0f;
    }
}

void density_pdf(Ctx& c, int level, int64_t* ncells, double* den, double* stats) {
    if (level < 0 || level > 4) throw Error{MGG_ERR_ARG, "density_pdf: level must be in [0, 4]"};
    const int ng = c.N >> level;
    if (ng < 8) throw Error{MGG_ERR_ARG, "density_pdf: NGRID/2^level must be at least 8"};
    BucketScope bs(c, MGG_T_POWER);
    if (level > 0) {
        // DENSITrsd(0, NGRID_old) on the coarser mesh (PMP2mod_analyze.f90:57-86)
        if (!c.have_particles) throw Error{MGG_ERR_STATE, "density_pdf: no particles uploaded"};
        PosScratch s(c);
        rsd_positions(c, s, 0, ng, 0.0f);
        cic_grid(c, s.x(), s.y(), s.z(), ng, c.fi);
        check_positions(c);
    }
    const int64_t n = (int64_t)ng * ng * ng;
    const int blocks = 148 * 4;
    ensure_partials(c, 2 * blocks);
    unsigned long long* dcnt = nullptr;
    double* dden = nullptr;
    MGG_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dcnt), sizeof(unsigned long long) * kPdfBins, c.stream));
    MGG_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dden), sizeof(double) * kPdfBins, c.stream));
    MGG_CUDA(cudaMemsetAsync(dcnt, 0, sizeof(unsigned long long) * kPdfBins, c.stream));
    MGG_CUDA(cudaMemsetAsync(dden, 0, sizeof(double) * kPdfBins, c.stream));
    {
        ProfScope ps(c, K_GRID_OP, 4.0 * (double)n);
        k_density_pdf<<<blocks, kPdfThreads, 0, c.stream>>>(c.fi, n, dcnt, dden, c.red_partial);
        MGG_CHECK_LAUNCH();
    }
    std::vector<unsigned long long> hc(kPdfBins);
    std::vector<double> hp(2 * blocks);
    MGG_CUDA(cudaMemcpyAsync(hc.data(), dcnt, sizeof(unsigned long long) * kPdfBins, cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaMemcpyAsync(den, dden, sizeof(double) * kPdfBins, cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaMemcpyAsync(hp.data(), c.red_partial, sizeof(double) * 2 * blocks, cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaFreeAsync(dcnt, c.stream));
    MGG_CUDA(cudaFreeAsync(dden, c.stream));
    MGG_CUDA(cudaStreamSynchronize(c.stream));
    for (int b = 0; b < kPdfBins; ++b) ncells[b] = (int64_t)hc[b];
    double s1 = 0.0, s2 = 0.0;
    for (int b = 0; b < blocks; ++b) {
        s1 += hp[b];
        s2 += hp[blocks + b];
    }
    // Total = FLOAT(NGRID)**3 (Real*4); DENM = SUM1/Total, DELR = sqrt(SUM2/Total - DENM**2)
    const float total = (float)ng * (float)ng * (float)ng;
    const double denm = s1 / (double)total;
    stats[0] = std::sqrt(s2 / (double)total - denm * denm);
    stats[1] = denm;
}

}  // namespace mgg
