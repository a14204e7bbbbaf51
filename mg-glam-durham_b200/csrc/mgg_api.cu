// C ABI of the B200 particle-mesh step (include/mgglam.h).  Every entry point
// validates its arguments, runs its work on the context's CUDA stream and turns
// any failure into a status code plus a message readable with mgg_last_error;
// nothing aborts the process and nothing falls back to the CPU.
#include "mgg_internal.cuh"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

namespace mgg {

const char* kKernelNames[K_NUM] = {
    "cic_count",   "cic_scatter", "cic_deposit", "scan",       "fft_x_r2c",   "fft_y",      "fft_z_green",
    "fft_x_c2r",   "fft_z_power", "power_finish", "move",      "potent_mg",   "mg_smooth",  "mg_resid",
    "mg_restrict", "mg_rhs",      "mg_prolong",  "mg_reduce",  "grid_op",     "ic",         "mg_smooth_l0",
    "mg_coarse"};

static cudaEvent_t new_event() {
    cudaEvent_t e;
    MGG_CUDA(cudaEventCreate(&e));
    return e;
}

static void resolve_profile(Ctx& c) {
    for (auto& p : c.prof.pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            c.prof.launches[p.id] += 1;
            c.prof.ms[p.id] += ms;
            c.prof.bytes[p.id] += p.bytes;
        }
        c.prof.pool.push_back(p.a);
        c.prof.pool.push_back(p.b);
    }
    c.prof.pending.clear();
}

void prof_begin(Ctx& c, int id, cudaEvent_t* a) {
    if (!c.prof.on || id < 0) return;   // id < 0: a launch that is not profiled
    if (c.prof.pool.empty()) *a = new_event();
    else { *a = c.prof.pool.back(); c.prof.pool.pop_back(); }
    MGG_CUDA(cudaEventRecord(*a, c.stream));
}

void prof_end(Ctx& c, int id, cudaEvent_t a, double bytes) {
    if (!c.prof.on || !a || id < 0) return;
    if (std::uncaught_exceptions() > 0) return;
    cudaEvent_t b;
    if (c.prof.pool.empty()) b = new_event();
    else { b = c.prof.pool.back(); c.prof.pool.pop_back(); }
    MGG_CUDA(cudaEventRecord(b, c.stream));
    c.prof.pending.push_back({id, a, b, bytes});
    if (c.prof.pending.size() > 8192) resolve_profile(c);
}

static void resolve_buckets(Ctx& c) {
    for (auto& p : c.buckets.pending) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess)
            c.buckets.ms[p.id] += ms;
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
    }
    c.buckets.pending.clear();
}

BucketScope::BucketScope(Ctx& c_, int id_) : c(c_), id(id_) {
    if (c.recording) return;   // no events inside a recorded graph
    a = new_event();
    MGG_CUDA(cudaEventRecord(a, c.stream));
}

BucketScope::~BucketScope() noexcept(false) {
    if (!a) return;
    if (std::uncaught_exceptions() > 0) {
        cudaEventDestroy(a);
        return;
    }
    b = new_event();
    MGG_CUDA(cudaEventRecord(b, c.stream));
    c.buckets.pending.push_back({id, a, b});
    if (c.buckets.pending.size() > 1024) resolve_buckets(c);
}

// error of the device flags h (read from c.d_flags); clears the flags on the device
static void raise_flags(Ctx& c, int32_t h) {
    if (h & 4) {   // bit 2: a staged FFT pencil copy did not complete within its bound
        MGG_CUDA(cudaMemsetAsync(c.d_flags, 0, sizeof(int32_t), c.stream));
        throw Error{MGG_ERR_CUDA, "fft: a staged pencil copy did not complete (an earlier potential or P(k) is void)"};
    }
    if (h & 1) {   // bit 0: CIC clamped a position
        MGG_CUDA(cudaMemsetAsync(c.d_flags, 0, sizeof(int32_t), c.stream));
        throw Error{MGG_ERR_NUMERIC, "density: particle position outside [1, NGRID+1) (clamped)"};
    }
    if (h & 8) {   // bit 3: a recorded solve saw a non-finite residual
        MGG_CUDA(cudaMemsetAsync(c.d_flags, 0, sizeof(int32_t), c.stream));
        throw Error{MGG_ERR_NUMERIC, "scalar_field: residual is not finite"};
    }
}

static void check_flags(Ctx& c) {
    int32_t h = 0;
    MGG_CUDA(cudaMemcpyAsync(&h, c.d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaStreamSynchronize(c.stream));
    raise_flags(c, h);
}

static void free_all(Ctx& c) {
    auto F = [](void* p) { if (p) cudaFree(p); };
    F(c.fi); F(c.fi2); F(c.cbuf); F(c.tw_n); F(c.tw_h); F(c.tw64_n); F(c.tw64_h); F(c.green); F(c.pk_logbin); F(c.pk_logbin_h); F(c.pk_hist);
    F(c.x); F(c.y); F(c.z); F(c.vx); F(c.vy); F(c.vz);
    F(c.cic_rowcnt); F(c.cic_rowstart); F(c.cic_slot); F(c.cic_rec); F(c.scan_tmp); F(c.d_flags);
    F(c.red_partial); F(c.red_out); F(c.bg); F(c.mg_loop); F(c.run_slots);
    for (int l = 1; l < 12; ++l) F(c.lev[l].d);
    F(c.lev[0].snap);
    if (c.h_red) cudaFreeHost(c.h_red);
    if (c.h_step) cudaFreeHost(c.h_step);
    if (c.h_run_slots) cudaFreeHost(c.h_run_slots);
    if (c.mg_exec) cudaGraphExecDestroy(c.mg_exec);
    if (c.loop_exec) cudaGraphExecDestroy(c.loop_exec);
    if (c.loop_graph) cudaGraphDestroy(c.loop_graph);
    c.loop_exec = nullptr;
    c.loop_graph = nullptr;
    if (c.copy_stream) cudaStreamSynchronize(c.copy_stream), cudaStreamDestroy(c.copy_stream);
    if (c.vel_ready) cudaEventDestroy(c.vel_ready);
    if (c.moved) cudaEventDestroy(c.moved);
    c.copy_stream = nullptr;
    c.vel_ready = nullptr;
    c.moved = nullptr;
    c.mg_exec = nullptr;
    resolve_profile(c);
    for (auto e : c.prof.pool) cudaEventDestroy(e);
    resolve_buckets(c);
    if (c.tstart) cudaEventDestroy(c.tstart);
    if (c.tstop) cudaEventDestroy(c.tstop);
    if (c.stream) cudaStreamDestroy(c.stream);
}

}  // namespace mgg

using namespace mgg;

struct mgg_ctx {
    Ctx c;
};

static std::mutex g_err_mu;
static std::string g_last_create_error;

template <class F>
static int guarded(mgg_ctx* ctx, F&& f) {
    if (!ctx) return MGG_ERR_ARG;
    try {
        MGG_CUDA(cudaSetDevice(ctx->c.dev));
        f(ctx->c);
        ctx->c.err.clear();
        return MGG_OK;
    } catch (const Error& e) {
        ctx->c.err = e.msg;
        return e.code;
    } catch (const std::bad_alloc&) {
        ctx->c.err = "host allocation failed";
        return MGG_ERR_NOMEM;
    } catch (...) {
        ctx->c.err = "unknown error";
        return MGG_ERR_CUDA;
    }
}

static bool is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

extern "C" {

const char* mgg_version(void) { return "mgglam-b200 0.1 (sm_100a)"; }

int mgg_create(const mgg_config* cfg, mgg_ctx** out) {
    auto fail = [](int code, const std::string& m) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_last_create_error = m;
        return code;
    };
    if (!cfg || !out) return fail(MGG_ERR_ARG, "mgg_create: null argument");
    *out = nullptr;
    if (!is_pow2(cfg->ngrid) || cfg->ngrid < 16 || cfg->ngrid > 1024)
        return fail(MGG_ERR_ARG, "mgg_create: NGRID must be a power of two in [16, 1024]");
    if (cfg->nrow < 1 || (int64_t)cfg->nrow * cfg->nrow * cfg->nrow >= (int64_t)1 << 31)
        return fail(MGG_ERR_ARG, "mgg_create: NROW out of range");
    if (!(cfg->box > 0.f) || !(cfg->om > 0.f)) return fail(MGG_ERR_ARG, "mgg_create: Box and Om must be positive");
    if (cfg->precision != MGG_PREC_PLAIN && cfg->precision != MGG_PREC_MIXED)
        return fail(MGG_ERR_ARG, "mgg_create: precision must be MGG_PREC_PLAIN or MGG_PREC_MIXED");
    if (cfg->mg_flag == 1) {
        if (cfg->mg_model < 1 || cfg->mg_model > 5) return fail(MGG_ERR_UNSUPPORTED, "mgg_create: unknown MG_model");
        if (cfg->mg_model == MGG_MODEL_KMOUFLAGE && cfg->kmf_born_infeld)
            return fail(MGG_ERR_UNSUPPORTED, "mgg_create: Born-Infeld k-mouflage is not supported (as in the reference)");
        if (cfg->mg_model == MGG_MODEL_CSF && (cfg->csf_coupling != 1 || cfg->csf_potential != 1))
            return fail(MGG_ERR_UNSUPPORTED, "mgg_create: csf needs exponential coupling and inverse power-law potential");
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(MGG_ERR_NO_DEVICE, "mgg_create: no CUDA device");
    if (cfg->device < 0 || cfg->device >= ndev) return fail(MGG_ERR_ARG, "mgg_create: bad device ordinal");
    mgg_ctx* ctx = new (std::nothrow) mgg_ctx();
    if (!ctx) return fail(MGG_ERR_NOMEM, "mgg_create: host allocation failed");
    Ctx& c = ctx->c;
    try {
        c.cfg = *cfg;
        c.dev = cfg->device;
        MGG_CUDA(cudaSetDevice(c.dev));
        cudaDeviceProp prop;
        MGG_CUDA(cudaGetDeviceProperties(&prop, c.dev));
        if (prop.major < 10) throw Error{MGG_ERR_NO_DEVICE, "mgg_create: this library is built for sm_100a (B200)"};
        MGG_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
        c.N = cfg->ngrid;
        c.ncell = (int64_t)c.N * c.N * c.N;
        c.np = (int64_t)cfg->nrow * cfg->nrow * cfg->nrow;
        auto alloc = [&](float** p, int64_t n) {
            cudaError_t e = cudaMalloc(p, sizeof(float) * n);
            if (e != cudaSuccess) {
                cudaGetLastError();
                throw Error{MGG_ERR_NOMEM, std::string("mgg_create: device allocation failed: ") + cudaGetErrorString(e)};
            }
        };
        alloc(&c.fi, c.ncell);
        MGG_CUDA(cudaMemsetAsync(c.fi, 0, sizeof(float) * c.ncell, c.stream));
        if (cfg->mg_flag == 1) {
            alloc(&c.fi2, c.ncell);
            MGG_CUDA(cudaMemsetAsync(c.fi2, 0, sizeof(float) * c.ncell, c.stream));
            mg_alloc(c);
        }
        alloc(&c.x, c.np); alloc(&c.y, c.np); alloc(&c.z, c.np);
        alloc(&c.vx, c.np); alloc(&c.vy, c.np); alloc(&c.vz, c.np);
        fft_alloc(c);
        cic_alloc(c);
        MGG_CUDA(cudaMalloc(&c.scan_tmp, sizeof(uint32_t) * 3 * 2048));
        MGG_CUDA(cudaMalloc(&c.d_flags, sizeof(int32_t)));
        MGG_CUDA(cudaMemset(c.d_flags, 0, sizeof(int32_t)));
        MGG_CUDA(cudaMalloc(&c.red_out, sizeof(double) * 4));
        MGG_CUDA(cudaMallocHost(&c.h_red, sizeof(double) * 4));
        MGG_CUDA(cudaMalloc(&c.mg_loop, sizeof(MgLoopState)));
        MGG_CUDA(cudaMemset(c.mg_loop, 0, sizeof(MgLoopState)));
        MGG_CUDA(cudaMallocHost(&c.h_step, sizeof(StepReadback)));
        std::memset(c.h_step, 0, sizeof(StepReadback));
        ensure_partials(c, 148 * 16);
        MGG_CUDA(cudaEventCreate(&c.tstart));
        MGG_CUDA(cudaEventCreate(&c.tstop));
        MGG_CUDA(cudaStreamSynchronize(c.stream));
    } catch (const Error& e) {
        free_all(c);
        delete ctx;
        return fail(e.code, e.msg);
    }
    *out = ctx;
    return MGG_OK;
}

int mgg_get_config(const mgg_ctx* ctx, mgg_config* cfg) {
    if (!ctx || !cfg) return MGG_ERR_ARG;
    *cfg = ctx->c.cfg;
    return MGG_OK;
}

int mgg_reconfigure(mgg_ctx* ctx, const mgg_config* cfg) {
    return guarded(ctx, [&](Ctx& c) {
        if (!cfg) throw Error{MGG_ERR_ARG, "reconfigure: null config"};
        if (cfg->ngrid != c.cfg.ngrid || cfg->nrow != c.cfg.nrow || cfg->mg_flag != c.cfg.mg_flag ||
            cfg->device != c.cfg.device)
            throw Error{MGG_ERR_ARG, "reconfigure: NGRID, NROW, MG_flag and device must stay the same"};
        if (!(cfg->box > 0.f) || !(cfg->om > 0.f)) throw Error{MGG_ERR_ARG, "reconfigure: Box and Om must be positive"};
        if (cfg->precision != MGG_PREC_PLAIN && cfg->precision != MGG_PREC_MIXED)
            throw Error{MGG_ERR_ARG, "reconfigure: precision must be MGG_PREC_PLAIN or MGG_PREC_MIXED"};
        if (cfg->mg_flag == 1) {
            if (cfg->mg_model < 1 || cfg->mg_model > 5) throw Error{MGG_ERR_UNSUPPORTED, "reconfigure: unknown MG_model"};
            if (cfg->mg_model == MGG_MODEL_KMOUFLAGE && cfg->kmf_born_infeld)
                throw Error{MGG_ERR_UNSUPPORTED, "reconfigure: Born-Infeld k-mouflage is not supported"};
            if (cfg->mg_model == MGG_MODEL_CSF && (cfg->csf_coupling != 1 || cfg->csf_potential != 1))
                throw Error{MGG_ERR_UNSUPPORTED, "reconfigure: csf needs exponential coupling and power-law potential"};
        }
        MGG_CUDA(cudaStreamSynchronize(c.stream));
        c.cfg = *cfg;
        c.have_particles = false;
        c.have_fi2 = false;
        c.fi2_pending = 0.0;
        c.bgrows = 0;
        c.h_bg.clear();
        c.mg_tuned = false;   // the next solve runs eagerly (chunk sizes of a new model are tuned)
    });
}

int64_t mgg_box_bytes(const mgg_config* cfg) {
    if (!cfg || cfg->ngrid < 2 || cfg->nrow < 1) return 0;
    const int64_t N = cfg->ngrid, n3 = N * N * N, np = (int64_t)cfg->nrow * cfg->nrow * cfg->nrow;
    const int64_t nxp = ((N / 2 + 1) + 15) / 16 * 16;
    int64_t b = 4 * n3;                           // FI
    if (cfg->mg_flag == 1) b += 12 * n3;         // FI2, snapshot, level arena (7 arrays x n^3/7)
    b += 24 * np;                                 // particles
    b += 8 * N * N * nxp;                         // half spectrum
    b += 8 * (N * N + 1) + 20 * np;               // CIC rows, slots, records
    return b + (8 << 20);                         // tables, partials, stream
}

int mgg_destroy(mgg_ctx* ctx) {
    if (!ctx) return MGG_ERR_ARG;
    cudaSetDevice(ctx->c.dev);
    if (ctx->c.stream) cudaStreamSynchronize(ctx->c.stream);
    free_all(ctx->c);
    delete ctx;
    return MGG_OK;
}

const char* mgg_last_error(const mgg_ctx* ctx) {
    if (!ctx) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        return g_last_create_error.c_str();
    }
    return ctx->c.err.c_str();
}

int mgg_set_time(mgg_ctx* ctx, float aexpn, float astep) {
    return guarded(ctx, [&](Ctx& c) {
        if (!(aexpn > 0.f)) throw Error{MGG_ERR_ARG, "set_time: AEXPN must be positive"};
        c.aexpn = aexpn;
        c.astep = astep;
    });
}

int mgg_upload_particles(mgg_ctx* ctx, const float* x, const float* y, const float* z, const float* vx,
                         const float* vy, const float* vz, int64_t n) {
    return guarded(ctx, [&](Ctx& c) {
        if (n != c.np) throw Error{MGG_ERR_ARG, "upload_particles: n must equal NROW^3"};
        if (!x || !y || !z || !vx || !vy || !vz) throw Error{MGG_ERR_ARG, "upload_particles: null pointer"};
        wait_velocities(c);
        const size_t b = sizeof(float) * n;
        MGG_CUDA(cudaMemcpyAsync(c.x, x, b, cudaMemcpyHostToDevice, c.stream));
        MGG_CUDA(cudaMemcpyAsync(c.y, y, b, cudaMemcpyHostToDevice, c.stream));
        MGG_CUDA(cudaMemcpyAsync(c.z, z, b, cudaMemcpyHostToDevice, c.stream));
        MGG_CUDA(cudaMemcpyAsync(c.vx, vx, b, cudaMemcpyHostToDevice, c.stream));
        MGG_CUDA(cudaMemcpyAsync(c.vy, vy, b, cudaMemcpyHostToDevice, c.stream));
        MGG_CUDA(cudaMemcpyAsync(c.vz, vz, b, cudaMemcpyHostToDevice, c.stream));
        MGG_CUDA(cudaStreamSynchronize(c.stream));
        c.have_particles = true;
    });
}

int mgg_download_particles(mgg_ctx* ctx, float* x, float* y, float* z, float* vx, float* vy, float* vz, int64_t n) {
    return guarded(ctx, [&](Ctx& c) {
        if (n != c.np) throw Error{MGG_ERR_ARG, "download_particles: n must equal NROW^3"};
        if (!c.have_particles) throw Error{MGG_ERR_STATE, "download_particles: no particles"};
        wait_velocities(c);
        const size_t b = sizeof(float) * n;
        if (x) MGG_CUDA(cudaMemcpyAsync(x, c.x, b, cudaMemcpyDeviceToHost, c.stream));
        if (y) MGG_CUDA(cudaMemcpyAsync(y, c.y, b, cudaMemcpyDeviceToHost, c.stream));
        if (z) MGG_CUDA(cudaMemcpyAsync(z, c.z, b, cudaMemcpyDeviceToHost, c.stream));
        if (vx) MGG_CUDA(cudaMemcpyAsync(vx, c.vx, b, cudaMemcpyDeviceToHost, c.stream));
        if (vy) MGG_CUDA(cudaMemcpyAsync(vy, c.vy, b, cudaMemcpyDeviceToHost, c.stream));
        if (vz) MGG_CUDA(cudaMemcpyAsync(vz, c.vz, b, cudaMemcpyDeviceToHost, c.stream));
        MGG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

// Upload, one main-loop step, download.  Positions go up on the context stream
// (the density needs them first) and velocities on the copy stream, waited for
// by MOVE.  Pipelined: the positions come back first and the call returns once
// they are on the host; the velocities follow on the copy stream, beside the
// next call's position upload (the other direction of the link), and the next
// call's velocity upload follows them on the copy stream, beside the density,
// scalar field and potential.
static int step_host(mgg_ctx* ctx, mgg_step_state* st, float* x, float* y, float* z, float* vx, float* vy, float* vz,
                     int64_t n, bool pipelined) {
    if (!st) return MGG_ERR_ARG;
    int rc = guarded(ctx, [&](Ctx& c) {
        if (n != c.np) throw Error{MGG_ERR_ARG, "step_host: n must equal NROW^3"};
        if (!x || !y || !z || !vx || !vy || !vz) throw Error{MGG_ERR_ARG, "step_host: null pointer"};
        if (!pipelined) wait_velocities(c);
        if (!c.copy_stream) {
            MGG_CUDA(cudaStreamCreateWithFlags(&c.copy_stream, cudaStreamNonBlocking));
            MGG_CUDA(cudaEventCreateWithFlags(&c.vel_ready, cudaEventDisableTiming));
            MGG_CUDA(cudaEventCreateWithFlags(&c.moved, cudaEventDisableTiming));
        }
        const size_t b = sizeof(float) * n;
        MGG_CUDA(cudaMemcpyAsync(c.x, x, b, cudaMemcpyHostToDevice, c.stream));
        MGG_CUDA(cudaMemcpyAsync(c.y, y, b, cudaMemcpyHostToDevice, c.stream));
        MGG_CUDA(cudaMemcpyAsync(c.z, z, b, cudaMemcpyHostToDevice, c.stream));
        MGG_CUDA(cudaMemcpyAsync(c.vx, vx, b, cudaMemcpyHostToDevice, c.copy_stream));
        MGG_CUDA(cudaMemcpyAsync(c.vy, vy, b, cudaMemcpyHostToDevice, c.copy_stream));
        MGG_CUDA(cudaMemcpyAsync(c.vz, vz, b, cudaMemcpyHostToDevice, c.copy_stream));
        MGG_CUDA(cudaEventRecord(c.vel_ready, c.copy_stream));
        c.vel_pending = true;
        c.have_particles = true;
    });
    if (rc != MGG_OK) return rc;
    if ((rc = mgg_step(ctx, st)) != MGG_OK) {
        guarded(ctx, [&](Ctx& c) {
            wait_velocities(c);
            MGG_CUDA(cudaStreamSynchronize(c.stream));
        });
        return rc;
    }
    if (!pipelined) return mgg_download_particles(ctx, x, y, z, vx, vy, vz, n);
    return guarded(ctx, [&](Ctx& c) {
        const size_t b = sizeof(float) * n;
        // positions first, with the whole device-to-host bandwidth ...
        MGG_CUDA(cudaMemcpyAsync(x, c.x, b, cudaMemcpyDeviceToHost, c.stream));
        MGG_CUDA(cudaMemcpyAsync(y, c.y, b, cudaMemcpyDeviceToHost, c.stream));
        MGG_CUDA(cudaMemcpyAsync(z, c.z, b, cudaMemcpyDeviceToHost, c.stream));
        // ... then the velocities on the copy stream, beside the next step's position upload
        MGG_CUDA(cudaEventRecord(c.moved, c.stream));
        MGG_CUDA(cudaStreamWaitEvent(c.copy_stream, c.moved, 0));
        MGG_CUDA(cudaMemcpyAsync(vx, c.vx, b, cudaMemcpyDeviceToHost, c.copy_stream));
        MGG_CUDA(cudaMemcpyAsync(vy, c.vy, b, cudaMemcpyDeviceToHost, c.copy_stream));
        MGG_CUDA(cudaMemcpyAsync(vz, c.vz, b, cudaMemcpyDeviceToHost, c.copy_stream));
        // anything that touches the device velocities next waits for this download
        MGG_CUDA(cudaEventRecord(c.vel_ready, c.copy_stream));
        c.vel_pending = true;
        MGG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

namespace {

// ASTEP growth and FactV of the main loop (PMP2main.f90:48-52), Real*4
float grow_astep(const mgg_step_state& st, float* factv) {
    *factv = 1.0f;
    if (st.astep < st.step_factor / 1.25f * st.aexpn && st.aexpn < 0.300f) {
        *factv = 1.2f;
        return 1.5f * st.astep;
    }
    return st.astep;
}

void step_device(Ctx& c, mgg_step_state* st) {
    if (!(st->aexpn > 0.f)) throw Error{MGG_ERR_ARG, "step: AEXPN must be positive"};
    const int i_step = st->istep + 1;
    if (i_step < 1) throw Error{MGG_ERR_ARG, "step: istep must be >= 0"};
    c.aexpn = st->aexpn;
    c.astep = st->astep;
    std::memset(&st->report, 0, sizeof(st->report));
    cic_density(c);
    const bool mg = c.cfg.mg_flag == 1;
    if (mg) mg_scalar_field(c, i_step, &st->report, true);
    poisson_solve(c);
    float factv;
    const float astep = grow_astep(*st, &factv);
    if (mg) potential_mg(c);
    c.astep = astep;
    move_particles(c, factv, nullptr, true);
    StepReadback& r = *c.h_step;
    MGG_CUDA(cudaMemcpyAsync(&r.flags, c.d_flags, sizeof(int32_t), cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaMemcpyAsync(&r.svel, c.red_out + 1, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    MGG_CUDA(cudaStreamSynchronize(c.stream));
    raise_flags(c, r.flags);
    mg_read_report(c, &st->report);
    const float enkin = move_enkin(c, r.svel);
    if (!std::isfinite(enkin)) throw Error{MGG_ERR_NUMERIC, "move: kinetic energy is not finite"};
    st->ekin = (double)enkin;
    st->astep = astep;
    st->istep += 1;
    st->aexpn = st->aexpn + st->astep;   // ADDTIME (256-261)
    c.stepped = true;
}

__global__ void k_copy_flags(const int32_t* __restrict__ flags, int32_t* __restrict__ out) { *out = *flags; }

// The steps of mgg_run_steps recorded into graphs of a few steps each, launched
// back to back without waiting; the results of each step land in its slot,
// read back once at the end.
void run_steps_graphed(Ctx& c, mgg_step_state* st, int32_t nsteps, mgg_mg_report* reports, double* ekin) {
    const bool mg = c.cfg.mg_flag == 1;
    if (nsteps > c.run_cap) {
        if (c.run_slots) MGG_CUDA(cudaFree(c.run_slots));
        if (c.h_run_slots) MGG_CUDA(cudaFreeHost(c.h_run_slots));
        c.run_slots = nullptr;
        c.h_run_slots = nullptr;
        c.run_cap = 0;
        MGG_CUDA(cudaMalloc(&c.run_slots, sizeof(StepReadback) * nsteps));
        MGG_CUDA(cudaMallocHost(&c.h_run_slots, sizeof(StepReadback) * nsteps));
        c.run_cap = nsteps;
    }
    wait_velocities(c);
    if (mg) ensure_partials(c, mg_norm_partials(c));   // no allocation while recording
    // the schedule of the run (the same Real*4 arithmetic as mgg_step)
    std::vector<mgg_step_state> plan(nsteps + 1);
    std::vector<float> factv(nsteps);
    plan[0] = *st;
    for (int k = 0; k < nsteps; ++k) {
        mgg_step_state nx = plan[k];
        nx.astep = grow_astep(plan[k], &factv[k]);
        nx.istep += 1;
        nx.aexpn = nx.aexpn + nx.astep;
        plan[k + 1] = nx;
    }
    // Reads back the slots of steps [0, upto) and advances *st over the good ones;
    // throws the first failing step's error.
    auto settle = [&](int upto) {
        if (upto <= 0) return;
        MGG_CUDA(cudaMemcpyAsync(c.h_run_slots, c.run_slots, sizeof(StepReadback) * upto, cudaMemcpyDeviceToHost,
                                 c.stream));
        MGG_CUDA(cudaStreamSynchronize(c.stream));
        for (int k = 0; k < upto; ++k) {
            const StepReadback& r = c.h_run_slots[k];
            raise_flags(c, r.flags);
            mgg_mg_report rep{};
            if (mg) {   // a step without a solve (symmetron before a*) has a cleared slot
                rep.cycles = r.mg.iter;
                rep.exit_reason = r.mg.reason;
                for (int i = 0; i < r.mg.iter && i < 64; ++i) rep.residual[i] = r.mg.residual[i];
            }
            c.aexpn = plan[k].aexpn;
            c.astep = plan[k + 1].astep;
            const float en = move_enkin(c, r.svel);
            if (!std::isfinite(en)) throw Error{MGG_ERR_NUMERIC, "move: kinetic energy is not finite"};
            plan[k + 1].report = rep;
            plan[k + 1].ekin = (double)en;
            *st = plan[k + 1];
            if (reports) reports[k] = rep;
            if (ekin) ekin[k] = (double)en;
        }
    };
    // Chunks of kRunChunk steps, each recorded, instantiated and launched in turn:
    // the host records the next chunk while the device runs the last one.
    constexpr int kRunChunk = 4;
    for (int k0 = 0; k0 < nsteps; k0 += kRunChunk) {
        const int k1 = std::min(nsteps, k0 + kRunChunk);
        cudaGraphExec_t exec = nullptr;
        Recorder rec(c);
        c.recording = true;
        try {
            rec.begin();
            for (int k = k0; k < k1; ++k) {
                StepReadback* slot = c.run_slots + k;
                c.aexpn = plan[k].aexpn;
                c.astep = plan[k].astep;
                cic_density(c);
                if (!mg || !mg_record_solve(c, plan[k].istep + 1, rec, &slot->mg, c.d_flags)) {
                    MGG_CUDA(cudaMemsetAsync(&slot->mg, 0, sizeof(MgLoopState), c.stream));
                }
                poisson_solve(c);
                if (mg) potential_mg(c);
                c.astep = plan[k + 1].astep;
                // a flag set by this or an earlier step (sticky until read) stops MOVE
                move_enqueue(c, factv[k], &slot->svel, c.d_flags, nullptr);
                k_copy_flags<<<1, 1, 0, c.stream>>>(c.d_flags, &slot->flags);
                MGG_CHECK_LAUNCH();
            }
            rec.end();
            MGG_CUDA(cudaGraphInstantiate(&exec, rec.graph, 0));
            c.recording = false;
            cudaError_t e = cudaGraphLaunch(exec, c.stream);
            cudaGraphExecDestroy(exec);   // released once the launch completes
            MGG_CUDA(e);
        } catch (...) {
            // the chunks already launched have run: their steps count, the error stands
            c.recording = false;
            rec.abort();
            settle(k0);
            throw;
        }
    }
    settle(nsteps);
}

}  // namespace

// One iteration of the main loop of Program PMP (PMP2main.f90:36-60): DENSIT,
// scalar_field, POTENTfft5, the ASTEP growth and FactV (48-52, Real*4),
// POTENT_FOR_MG, MOVE and ADDTIME (256-261), queued on the context stream with
// one host synchronisation at the end.  After a context's first solve the
// multigrid exit test runs on the device; the device error flags, the solve's
// report and MOVE's kinetic-energy sum are read back together.  A step that
// fails leaves the particles and the step state as they were.
int mgg_step(mgg_ctx* ctx, mgg_step_state* st) {
    if (!st) return MGG_ERR_ARG;
    return guarded(ctx, [&](Ctx& c) { step_device(c, st); });
}

// nsteps main-loop steps queued as CUDA graphs: every step's kernels, each
// solve a while node with its exit test on the device, each step's results
// (flags, multigrid state, velocity sum) in a device slot read back once at the
// end.  A context's first steps (up to its first, eager and tuning, solve) and
// runs with profiling on, iter_count_max above the device-loop limit or no
// conditional graph nodes in this runtime go step by step.
int mgg_run_steps(mgg_ctx* ctx, mgg_step_state* st, int32_t nsteps, mgg_mg_report* reports, double* ekin) {
    if (!st || nsteps < 0) return MGG_ERR_ARG;
    return guarded(ctx, [&](Ctx& c) {
        if (!(st->aexpn > 0.f)) throw Error{MGG_ERR_ARG, "run_steps: AEXPN must be positive"};
        if (st->istep < 0) throw Error{MGG_ERR_ARG, "run_steps: istep must be >= 0"};
        int done = 0;
        const bool mg = c.cfg.mg_flag == 1;
        auto one = [&] {
            step_device(c, st);
            if (reports) reports[done] = st->report;
            if (ekin) ekin[done] = st->ekin;
            ++done;
        };
        if (c.prof.on || (mg && (c.cfg.iter_count_max > mg_device_loop_max() || !mg_conditional_nodes()))) {
            while (done < nsteps) one();
            return;
        }
        // steps run one by one until the context has stepped and solved once: the
        // first solve (eager) tunes the plane chunks, the first transforms the pencil
        // width (a symmetron run before a* has no solve until it passes a*)
        while (done < nsteps && (!c.stepped || (mg && !c.mg_tuned))) one();
        if (done < nsteps)
            run_steps_graphed(c, st, nsteps - done, reports ? reports + done : nullptr, ekin ? ekin + done : nullptr);
    });
}

int mgg_step_host(mgg_ctx* ctx, mgg_step_state* st, float* x, float* y, float* z, float* vx, float* vy, float* vz,
                  int64_t n) {
    return step_host(ctx, st, x, y, z, vx, vy, vz, n, false);
}

int mgg_step_host_pipelined(mgg_ctx* ctx, mgg_step_state* st, float* x, float* y, float* z, float* vx, float* vy,
                            float* vz, int64_t n) {
    return step_host(ctx, st, x, y, z, vx, vy, vz, n, true);
}

int mgg_density(mgg_ctx* ctx) {
    return guarded(ctx, [&](Ctx& c) {
        cic_density(c);
        check_flags(c);
    });
}

int mgg_scalar_field(mgg_ctx* ctx, int32_t i_step, mgg_mg_report* report) {
    return guarded(ctx, [&](Ctx& c) {
        if (i_step < 1) throw Error{MGG_ERR_ARG, "scalar_field: i_step starts at 1"};
        if (!(c.aexpn > 0.f)) throw Error{MGG_ERR_STATE, "scalar_field: call mgg_set_time first"};
        mg_scalar_field(c, i_step, report);
    });
}

int mgg_potential(mgg_ctx* ctx) {
    return guarded(ctx, [&](Ctx& c) {
        if (!(c.aexpn > 0.f)) throw Error{MGG_ERR_STATE, "potential: call mgg_set_time first"};
        poisson_solve(c);
    });
}

int mgg_potential_mg(mgg_ctx* ctx) {
    return guarded(ctx, [&](Ctx& c) { potential_mg(c); });
}

int mgg_move(mgg_ctx* ctx, float factv, double* enkin) {
    return guarded(ctx, [&](Ctx& c) {
        if (!(factv > 0.f)) throw Error{MGG_ERR_ARG, "move: FactV must be positive"};
        move_particles(c, factv, enkin);
    });
}

int mgg_power(mgg_ctx* ctx, int32_t recompute_density, int32_t nbins, double* k, double* nmodes, double* pk,
              double* klog, double* nmodeslog, double* pklog) {
    return guarded(ctx, [&](Ctx& c) {
        if (nbins < 1 || nbins > c.N / 2) throw Error{MGG_ERR_ARG, "power: nbins must be in [1, NGRID/2]"};
        if (recompute_density) {
            cic_density(c);
            check_flags(c);
        }
        power_spectrum(c, nbins, k, nmodes, pk, klog, nmodeslog, pklog);
    });
}

int mgg_power_rsd(mgg_ctx* ctx, int32_t nbins, double* k, double* nmodes, double* preal, double* p0, double* p2) {
    return guarded(ctx, [&](Ctx& c) { power_rsd(c, nbins, k, nmodes, preal, p0, p2); });
}

int mgg_density_pdf(mgg_ctx* ctx, int32_t level, int64_t* ncells, double* den_sum, double* stats) {
    return guarded(ctx, [&](Ctx& c) {
        if (!ncells || !den_sum || !stats) throw Error{MGG_ERR_ARG, "density_pdf: null pointer"};
        density_pdf(c, level, ncells, den_sum, stats);
    });
}

int mgg_upload_grid(mgg_ctx* ctx, int32_t which, const float* host) {
    return guarded(ctx, [&](Ctx& c) {
        if (!host) throw Error{MGG_ERR_ARG, "upload_grid: null pointer"};
        float* d = which == MGG_GRID_FI ? c.fi : (which == MGG_GRID_FI2 ? c.fi2 : nullptr);
        if (!d) throw Error{MGG_ERR_ARG, "upload_grid: unknown grid or FI2 not allocated (MG_flag off)"};
        MGG_CUDA(cudaMemcpyAsync(d, host, sizeof(float) * c.ncell, cudaMemcpyHostToDevice, c.stream));
        MGG_CUDA(cudaStreamSynchronize(c.stream));
        if (which == MGG_GRID_FI2) {
            c.have_fi2 = true;
            c.fi2_pending = 0.0;
        }
    });
}

int mgg_download_grid(mgg_ctx* ctx, int32_t which, float* host) {
    return guarded(ctx, [&](Ctx& c) {
        if (!host) throw Error{MGG_ERR_ARG, "download_grid: null pointer"};
        float* d = which == MGG_GRID_FI ? c.fi : (which == MGG_GRID_FI2 ? c.fi2 : nullptr);
        if (!d) throw Error{MGG_ERR_ARG, "download_grid: unknown grid or FI2 not allocated (MG_flag off)"};
        if (which == MGG_GRID_FI2) fi2_materialize(c);
        MGG_CUDA(cudaMemcpyAsync(host, d, sizeof(float) * c.ncell, cudaMemcpyDeviceToHost, c.stream));
        MGG_CUDA(cudaStreamSynchronize(c.stream));
    });
}

int mgg_set_background(mgg_ctx* ctx, const double* table, int32_t rows) {
    return guarded(ctx, [&](Ctx& c) {
        if (!table || rows < 2) throw Error{MGG_ERR_ARG, "set_background: need at least 2 rows"};
        c.h_bg.assign(table, table + (size_t)rows * 6);
        if (c.bg) MGG_CUDA(cudaFree(c.bg));
        c.bg = nullptr;
        MGG_CUDA(cudaMalloc(&c.bg, sizeof(double) * rows * 6));
        MGG_CUDA(cudaMemcpy(c.bg, table, sizeof(double) * rows * 6, cudaMemcpyHostToDevice));
        c.bgrows = rows;
    });
}

int mgg_background_table(mgg_config* cfg, double hubble, double* table, int32_t capacity_rows, int32_t* rows,
                         double* lambda) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    if (!cfg || !table || !rows) {
        g_last_create_error = "background_table: null argument";
        return MGG_ERR_ARG;
    }
    try {
        int r = 0;
        background_table(*cfg, hubble, table, capacity_rows, &r, lambda);
        *rows = r;
        return MGG_OK;
    } catch (const Error& e) {
        g_last_create_error = e.msg;
        return e.code;
    }
}

int mgg_density_noalloc(const float* x, const float* y, const float* z, int64_t np, int32_t ngrid, float* fi,
                        void* stream) {
    std::string msg;
    int code = MGG_OK;
    try {
        density_noalloc(x, y, z, np, ngrid, fi, static_cast<cudaStream_t>(stream));
    } catch (const Error& e) {
        code = e.code;
        msg = e.msg;
    } catch (const std::exception& e) {
        code = MGG_ERR_CUDA;
        msg = e.what();
    }
    if (code != MGG_OK) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        g_last_create_error = msg;
    }
    return code;
}

int mgg_cic_keys(mgg_ctx* ctx, uint32_t* rowcnt, uint32_t* rowstart, uint32_t* cellcnt) {
    return guarded(ctx, [&](Ctx& c) { cic_keys(c, rowcnt, rowstart, cellcnt); });
}

int mgg_synchronize(mgg_ctx* ctx) {
    return guarded(ctx, [&](Ctx& c) {
        MGG_CUDA(cudaStreamSynchronize(c.stream));
        if (c.copy_stream) MGG_CUDA(cudaStreamSynchronize(c.copy_stream));
    });
}

int mgg_timing(mgg_ctx* ctx, double* out) {
    return guarded(ctx, [&](Ctx& c) {
        if (!out) throw Error{MGG_ERR_ARG, "timing: null pointer"};
        resolve_buckets(c);
        double tot = 0.0;
        for (int i = 1; i < MGG_T_NBUCKETS; ++i) tot += c.buckets.ms[i];
        for (int i = 0; i < MGG_T_NBUCKETS; ++i) out[i] = c.buckets.ms[i];
        out[MGG_T_TOTAL] = tot;
    });
}

int mgg_profile(mgg_ctx* ctx, int32_t enable) {
    return guarded(ctx, [&](Ctx& c) { c.prof.on = enable != 0; });
}

int mgg_profile_count(void) { return K_NUM; }

int mgg_profile_read(mgg_ctx* ctx, int32_t id, const char** name, int64_t* launches, double* total_ms,
                     double* alg_bytes) {
    return guarded(ctx, [&](Ctx& c) {
        if (id < 0 || id >= K_NUM) throw Error{MGG_ERR_ARG, "profile_read: bad id"};
        resolve_profile(c);
        if (name) *name = kKernelNames[id];
        if (launches) *launches = c.prof.launches[id];
        if (total_ms) *total_ms = c.prof.ms[id];
        if (alg_bytes) *alg_bytes = c.prof.bytes[id];
    });
}

int mgg_profile_reset(mgg_ctx* ctx) {
    return guarded(ctx, [&](Ctx& c) {
        resolve_profile(c);
        for (int i = 0; i < K_NUM; ++i) {
            c.prof.launches[i] = 0;
            c.prof.ms[i] = 0;
            c.prof.bytes[i] = 0;
        }
        resolve_buckets(c);
        for (int i = 0; i < MGG_T_NBUCKETS; ++i) c.buckets.ms[i] = 0;
    });
}

int mgg_timer_start(mgg_ctx* ctx) {
    return guarded(ctx, [&](Ctx& c) { MGG_CUDA(cudaEventRecord(c.tstart, c.stream)); });
}

int mgg_timer_stop(mgg_ctx* ctx, double* ms) {
    return guarded(ctx, [&](Ctx& c) {
        wait_velocities(c);   // a pipelined velocity download still in flight counts too
        MGG_CUDA(cudaEventRecord(c.tstop, c.stream));
        MGG_CUDA(cudaEventSynchronize(c.tstop));
        float f = 0.f;
        MGG_CUDA(cudaEventElapsedTime(&f, c.tstart, c.tstop));
        if (ms) *ms = f;
    });
}

int mgg_make_ics(mgg_ctx* ctx, const mgg_ic_params* ic) {
    return guarded(ctx, [&](Ctx& c) {
        if (!ic) throw Error{MGG_ERR_ARG, "make_ics: null parameters"};
        make_ics(c, *ic);
    });
}

}  // extern "C"
