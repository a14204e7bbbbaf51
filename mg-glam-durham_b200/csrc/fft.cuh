// Stockham FFT building blocks shared by the Poisson solve, P(k) and the
// initial-condition generator.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace mgg {

// A 3-D real <-> half-complex transform of an n^3 grid.
//   real grid : n^3 floats, x fastest
//   spectrum  : float2 [kz][ky][kx], kx in [0, n/2], row pitch nxp >= n/2+1
struct FftPlan {
    int n = 0;
    int nxp = 0;
    const float2* tw = nullptr;   // exp(-2 pi i k / n), k < n
    const double2* tw64 = nullptr;   // the same in FP64; when set, the lines are computed in FP64
                                     // (stored as FP32 between passes, as FFTPACK5 in the reference)
    // tensor maps (CUtensorMap) of the context's spectrum for the TMA-staged y / z
    // passes (FP32 lines, n >= 256), per pencil width (8, 4 kx columns) and axis
    // (y, z); null: the passes load their pencils directly
    const void* tmap[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};
    int tile_tx[5] = {8, 8, 8, 8, 8};   // pencil width of the staged pass of each LineMode
    int32_t* flags = nullptr;        // bit 2: a staged pencil copy did not complete
};

enum LineMode : int {
    LM_FWD = 0,      // forward transform along the axis
    LM_INV = 1,      // inverse (unnormalised) transform along the axis
    LM_GREEN = 2,    // forward, multiply by the Poisson kernel, inverse (z axis)
    LM_POWER = 3,    // forward, then accumulate |F|^2 into P(k) bins (z axis)
    LM_DISP = 4,     // Zel'dovich displacement component: multiply, inverse (z axis)
};

struct LineExtra {
    // LM_GREEN
    const double* green = nullptr;   // G(k) per complex index, length n
    double green_scale = 0.0;        // trfi * 2 / n^3
    // LM_POWER
    const uint8_t* logbin = nullptr;        // log bin per integer |k|^2
    unsigned long long* hist = nullptr;     // [3][n+1] fixed-point sums (linear, log, quadrupole)
    double amp_scale = 0.0;                 // fixed-point scale * 1/n^6
    int quad = 0;                           // also the P2(mu)-weighted linear sums (hist[2][..])
    // LM_DISP
    const float2* src = nullptr;     // forward spectrum to read (not overwritten)
    const float* tk = nullptr;       // transfer amplitude per integer |k|^2
    int comp = 0;                    // displacement component 0,1,2
};

// Real rows (n floats each) -> half spectrum rows (pitch nxp); rows = n*n
void fft_x_r2c(const FftPlan& p, const float* in, float2* out, cudaStream_t s);
// Half spectrum rows -> real rows; output is (n/2) * (unnormalised inverse)
void fft_x_c2r(const FftPlan& p, const float2* in, float* out, cudaStream_t s);
// Transform every y line (axis = 1) or z line (axis = 2) of the half spectrum
void fft_lines(const FftPlan& p, float2* buf, int axis, int mode, const LineExtra& ex, cudaStream_t s);
void fft_set_attributes();

}  // namespace mgg
