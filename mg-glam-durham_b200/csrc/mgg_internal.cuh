// Internal declarations shared by the sm_100a translation units of the
// MG-GLAM particle-mesh step.  Nothing here is part of the public C ABI
// (include/mgglam.h).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/mgglam.h"

namespace mgg {

// ---- error handling -------------------------------------------------------
struct Error {
    int code;
    std::string msg;
};

#define MGG_CUDA(call)                                                                        \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            throw ::mgg::Error{MGG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)}; \
    } while (0)

#define MGG_CHECK_LAUNCH() MGG_CUDA(cudaGetLastError())

// ---- kernel classes for the launch profile --------------------------------
enum KernelId : int {
    K_CIC_COUNT = 0,
    K_CIC_SCATTER,
    K_CIC_DEPOSIT,
    K_SCAN,
    K_FFT_X_R2C,
    K_FFT_Y,
    K_FFT_Z_GREEN,
    K_FFT_X_C2R,
    K_FFT_Z_POWER,
    K_POWER_FINISH,
    K_MOVE,
    K_POTENT_MG,
    K_MG_SMOOTH,
    K_MG_RESID,
    K_MG_RESTRICT,
    K_MG_RHS,
    K_MG_PROLONG,
    K_MG_REDUCE,
    K_GRID_OP,
    K_IC,
    K_MG_SMOOTH0,   // the smoother on the finest level (the PM grid)
    K_MG_COARSE,    // the cycle on the small levels, one launch
    K_NUM
};
extern const char* kKernelNames[K_NUM];

struct Level {
    int n = 0;
    float* d = nullptr;    // restricted density (section 2 of FI3)
    float* ru = nullptr;   // restricted fine solution, frozen (section 3)
    float* u = nullptr;    // working coarse solution (section 4)
    float* tau = nullptr;  // FAS right-hand side (section 5)
    float* res = nullptr;  // coarse residual (section 6)
    float* rr = nullptr;   // restricted residual (section 1)
    float* snap = nullptr; // ping-pong copy for models whose stencil reads same-colour cells
};

// State of a multigrid solve whose exit test (PMP2extradof.f90:107-121) runs on
// the device after every cycle: the last two residuals, the residual of each
// cycle, the cycles run, the exit reason, and whether a residual was not finite.
struct MgLoopState {
    double res_old_1, res_old_2;
    double residual[64];
    int32_t iter, reason, bad, pad;
};

// Pinned host copy of what one mgg_step reads back at its end, in one
// synchronisation: the multigrid state, the device error flags and the
// kinetic-energy sum of MOVE.
struct StepReadback {
    MgLoopState mg;
    double svel;
    int32_t flags, pad;
};

struct Ctx;

// Launch profile: events bracket launches when enabled.
struct Profiler {
    bool on = false;
    int64_t launches[K_NUM] = {};
    double ms[K_NUM] = {};
    double bytes[K_NUM] = {};
    // pending event pairs (resolved lazily)
    struct Pending {
        int id;
        cudaEvent_t a, b;
        double bytes;
    };
    std::vector<Pending> pending;
    std::vector<cudaEvent_t> pool;
};

// bucket timers (TimingMain layout)
struct BucketTimer {
    double ms[MGG_T_NBUCKETS] = {};
    struct Pending {
        int id;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending;
};

struct Ctx {
    mgg_config cfg{};
    int dev = 0;
    cudaStream_t stream = nullptr;
    // velocity upload of mgg_step_host, overlapped with the step up to MOVE
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t vel_ready = nullptr;   // last velocity copy on copy_stream (upload or download)
    cudaEvent_t moved = nullptr;       // positions downloaded (start of the pipelined velocity download)
    bool vel_pending = false;
    float aexpn = 0.f, astep = 0.f;
    int N = 0;
    int64_t ncell = 0;
    int64_t np = 0;
    bool have_particles = false;
    bool have_fi2 = false;

    // grids
    float* fi = nullptr;
    float* fi2 = nullptr;

    // multigrid arena
    int levelmax = 0, levelmin = 0;
    Level lev[12];

    // FFT workspace: complex half spectrum, padded row pitch nxp (float2 units)
    float2* cbuf = nullptr;
    int nxp = 0;
    float2* tw_n = nullptr;     // exp(-2 pi i k / N), k < N
    float2* tw_h = nullptr;     // exp(-2 pi i k / (N/2)), k < N/2 (analysis on the NGRID/2 mesh, at first use)
    // tensor maps (CUtensorMap, 128 bytes each) of cbuf for the TMA-staged y / z
    // passes: [pencil width 8, 4][axis y, z]
    alignas(64) unsigned char tmap[2][2][128] = {};
    bool tmaps = false;
    double2* tw64_n = nullptr;  // the same tables in FP64: the plain path's transforms compute in FP64
    double2* tw64_h = nullptr;  //   (FFTPACK5's real(kind=8)); tw64_h at first use
    uint8_t* pk_logbin_h = nullptr;   // log bins of the NGRID/2 mesh (at first use)
    double* green = nullptr;    // 1-D Green's function G(k) = 2 cos(2 pi k / N) for complex index k
    uint8_t* pk_logbin = nullptr;   // log bin per integer |k|^2 (power spectrum)

    // particles (SoA)
    float *x = nullptr, *y = nullptr, *z = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr;

    // CIC scratch
    uint32_t* cic_rowcnt = nullptr;    // N^2 (+1) counts
    uint32_t* cic_rowstart = nullptr;  // N^2 + 1 exclusive prefix
    uint32_t* cic_slot = nullptr;      // per particle slot within its row
    float4* cic_rec = nullptr;         // row-bucketed particle positions
    int cic_last_n = 0;                // mesh size of the last deposit (its keys are in the scratch)
    uint32_t* scan_tmp = nullptr;      // block sums for the scan
    int32_t* d_flags = nullptr;        // device error flags

    // reductions
    double* red_partial = nullptr;     // per-block partial sums
    int red_capacity = 0;
    double* red_out = nullptr;         // device result slots
    double* h_red = nullptr;           // pinned host mirror
    unsigned long long* pk_hist = nullptr;   // fixed-point P(k) histograms

    // background table (k-mouflage / coupled scalar field)
    double* bg = nullptr;
    int bgrows = 0;
    std::vector<double> h_bg;

    Profiler prof;
    cudaGraphExec_t mg_exec = nullptr;   // captured MG cycle of the current step
    // exit test of a graphed multigrid solve, run on the device (device state and its
    // pinned host mirror); mg_deferred: a solve's report is still to be read from it
    MgLoopState* mg_loop = nullptr;
    StepReadback* h_step = nullptr;
    bool mg_deferred = false;
    // the graphed solve, kept for the context's later solves: the graph (a while
    // node), its cycle body, the executable graph and the node's condition handle
    cudaGraph_t loop_graph = nullptr;
    cudaGraph_t loop_body = nullptr;
    cudaGraphExec_t loop_exec = nullptr;
    cudaGraphConditionalHandle loop_h = 0;
    // mgg_run_steps: while a run's graph is recorded, the bucket timers stay off;
    // one result slot per step of the run (device) and their pinned host copy
    bool recording = false;
    bool stepped = false;   // a main-loop step has run (its transforms tuned the pencil width)
    StepReadback* run_slots = nullptr;
    StepReadback* h_run_slots = nullptr;
    int run_cap = 0;
    bool mg_tuned = false;               // one eager solve has run (chunk sizes tuned)
    // f(R): the exit rescaling FI2 *= u_bg^-1 of scalar_field, not yet applied
    // to the array (0 = none); POTENT_FOR_MG applies it on the fly, the next
    // scalar_field together with its own rescaling, a download materialises it
    double fi2_pending = 0.0;
    BucketTimer buckets;
    cudaEvent_t tstart = nullptr, tstop = nullptr;
    std::string err;
};

// ---- profiling helpers ----------------------------------------------------
void prof_begin(Ctx& c, int id, cudaEvent_t* a);
void prof_end(Ctx& c, int id, cudaEvent_t a, double bytes);

struct ProfScope {
    Ctx& c;
    int id;
    double bytes;
    cudaEvent_t a = nullptr;
    ProfScope(Ctx& c_, int id_, double bytes_) : c(c_), id(id_), bytes(bytes_) { prof_begin(c, id, &a); }
    ~ProfScope() noexcept(false) { prof_end(c, id, a, bytes); }
};

struct BucketScope {
    Ctx& c;
    int id;
    cudaEvent_t a = nullptr, b = nullptr;
    BucketScope(Ctx& c_, int id_);
    ~BucketScope() noexcept(false);
};

// Builds one CUDA graph out of segments captured on the context stream (each
// appended as a child-graph node) and while nodes whose bodies are captured in
// turn, all in one dependency chain.  The caller instantiates graph.
struct Recorder {
    Ctx& c;
    cudaGraph_t graph = nullptr;
    cudaGraphNode_t last = nullptr;
    bool capturing = false;
    bool into_body = false;   // the open capture fills a while node's body (owned by graph)
    explicit Recorder(Ctx& c_) : c(c_) {
        if (cudaGraphCreate(&graph, 0) != cudaSuccess) throw Error{MGG_ERR_CUDA, "graph create"};
    }
    ~Recorder() {
        abort();
        if (graph) cudaGraphDestroy(graph);
    }
    // ends an open capture (after an error), leaving the stream usable
    void abort() {
        if (!capturing) return;
        cudaGraph_t g = nullptr;
        cudaStreamEndCapture(c.stream, &g);
        if (g && !into_body) cudaGraphDestroy(g);
        cudaGetLastError();
        capturing = false;
        into_body = false;
    }
    void begin() {
        MGG_CUDA(cudaStreamBeginCapture(c.stream, cudaStreamCaptureModeThreadLocal));
        capturing = true;
    }
    void end() {
        cudaGraph_t seg = nullptr;
        capturing = false;
        MGG_CUDA(cudaStreamEndCapture(c.stream, &seg));
        size_t n = 0;
        cudaError_t e = cudaGraphGetNodes(seg, nullptr, &n);
        cudaGraphNode_t node = nullptr;
        if (e == cudaSuccess && n > 0) e = cudaGraphAddChildGraphNode(&node, graph, last ? &last : nullptr, last ? 1 : 0, seg);
        cudaGraphDestroy(seg);
        MGG_CUDA(e);
        if (node) last = node;
    }
    // Closes the open segment, appends a while node whose condition is 1 at each
    // launch, captures its body with body(handle), and opens the next segment.
    template <class F>
    void loop(F&& body) {
        end();
        cudaGraphConditionalHandle h;
        MGG_CUDA(cudaGraphConditionalHandleCreate(&h, graph, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams p{};
        p.type = cudaGraphNodeTypeConditional;
        p.conditional.handle = h;
        p.conditional.type = cudaGraphCondTypeWhile;
        p.conditional.size = 1;
        cudaGraphNode_t node;
        MGG_CUDA(cudaGraphAddNode(&node, graph, last ? &last : nullptr, last ? 1 : 0, &p));
        last = node;
        MGG_CUDA(cudaStreamBeginCaptureToGraph(c.stream, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                               cudaStreamCaptureModeThreadLocal));
        capturing = true;
        into_body = true;
        body(h);
        cudaGraph_t ended = nullptr;
        capturing = false;
        into_body = false;
        MGG_CUDA(cudaStreamEndCapture(c.stream, &ended));
        begin();
    }
};

// Make the context stream wait for a velocity upload still in flight.
inline void wait_velocities(Ctx& c) {
    if (!c.vel_pending) return;
    if (cudaStreamWaitEvent(c.stream, c.vel_ready, 0) != cudaSuccess) throw Error{MGG_ERR_CUDA, "velocity upload"};
    c.vel_pending = false;
}

// ---- translation-unit entry points ----------------------------------------
// cic.cu
void cic_alloc(Ctx& c);
void cic_density(Ctx& c);
// CIC density (FI := -1 + weights) of np = c.np particles at x, y, z (grid units of an
// ng^3 mesh, ng <= NGRID) into out, with the context's sort scratch
void cic_grid(Ctx& c, const float* x, const float* y, const float* z, int ng, float* out);
void density_noalloc(const float* x, const float* y, const float* z, int64_t np, int ngrid, float* fi,
                     cudaStream_t stream);
// integer keys of the last deposit on the NGRID mesh (row counts, offsets, per-cell counts)
void cic_keys(Ctx& c, uint32_t* rowcnt, uint32_t* rowstart, uint32_t* cellcnt);
// fft.cu
void fft_alloc(Ctx& c);
void poisson_solve(Ctx& c);
void power_spectrum(Ctx& c, int nbins, double* k, double* nm, double* pk, double* kl, double* nl, double* pl);
// per-bin P(k) of a real n^3 grid (bins 1..n/2; index 0 unused): monopole k, modes, P,
// log bins, and with quad the quadrupole about the z axis
struct PkBins {
    std::vector<double> k, n, p, kl, nl, pl, q;
};
// tw64 != nullptr: FP64 line arithmetic (the plain path)
void power_bins(Ctx& c, const float* grid, int n, const float2* tw, const double2* tw64, const uint8_t* logbin,
                bool quad, PkBins& out);
int fft_pitch(int n);
float2* make_twiddles(int n);
double2* make_twiddles64(int n);
uint8_t* make_logbins(int n);
// analysis.cu
void power_rsd(Ctx& c, int nbins, double* k, double* nm, double* preal, double* p0, double* p2);
void density_pdf(Ctx& c, int level, int64_t* ncells, double* den, double* stats);
// move.cu
// defer: the kinetic-energy sum stays on the device (StepReadback::svel, read by
// the caller's synchronisation), and MOVE is skipped on the device when the step's
// device flags are set or its multigrid solve saw a non-finite residual
void move_particles(Ctx& c, float factv, double* enkin, bool defer = false);
// MOVE queued with its velocity sum into svel (device); skipped on the device when
// *skip_flags != 0 or skip_mg->bad (either may be null)
void move_enqueue(Ctx& c, float factv, double* svel, const int32_t* skip_flags, const MgLoopState* skip_mg);
float move_enkin(const Ctx& c, double svel);   // ENKIN of PMP2main.f90:666 from the velocity sum
void potential_mg(Ctx& c);
// mg.cu
void mg_alloc(Ctx& c);
// defer: a graphed solve (exit test on the device) is left running and its report
// is read by mg_read_report after the caller's synchronisation
void mg_scalar_field(Ctx& c, int i_step, mgg_mg_report* rep, bool defer = false);
void mg_read_report(Ctx& c, mgg_mg_report* rep);   // from h_step->mg; throws on a non-finite residual
// scalar_field(i_step) recorded into a run's graph: the entry work in the open
// segment, the cycles as a while node with its exit test writing *slot (and
// setting bit 3 of *sticky on a non-finite residual).  Needs a tuned context
// (one eager solve) and iter_count_max <= mg_device_loop_max().  Returns false
// when the step has no solve (symmetron before a*).
bool mg_record_solve(Ctx& c, int i_step, Recorder& rec, MgLoopState* slot, int32_t* sticky);
int mg_device_loop_max();
bool mg_conditional_nodes();   // graphs with while nodes can be built here
int mg_norm_partials(Ctx& c);   // partial sums of the level-0 residual norm
void fi2_materialize(Ctx& c);   // apply a pending FI2 rescaling to the array
// ic.cu
void make_ics(Ctx& c, const mgg_ic_params& p);
// background.cu
int background_table(mgg_config& c, double hubble, double* table, int capacity, int* rows, double* lambda_out);
// reduce.cu helpers
double reduce_sum_blocks(Ctx& c, int nblocks);   // sums red_partial[0..nblocks) on device, fixed order
void reduce_sum_blocks_async(Ctx& c, int nblocks, double* out);   // the same sum into device memory, no wait
void scan_exclusive(Ctx& c, const uint32_t* in, uint32_t* out, int64_t n);
void ensure_partials(Ctx& c, int n);

// common constants
constexpr double kCtildeC = 2.99792458e3;

inline int div_up(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

}  // namespace mgg
