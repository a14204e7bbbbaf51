/*
 * mgglam.h -- C ABI of the B200 (sm_100a) particle-mesh step of MG-GLAM.
 *
 * One context = one simulation box resident on one GPU: the density/potential
 * grid FI, the scalar-field grid FI2, the multigrid level arena (the role of the
 * packed FI3 array), the particle arrays XPAR..VZ and the FFT workspace.  Every
 * call is asynchronous on the context's own CUDA stream unless it returns host
 * data; every call returns an int status (MGG_OK == 0) and never aborts the
 * process.  There is no CPU fallback: a context cannot be created without a
 * CUDA device and the compiled sm_100a kernels.
 *
 * The reference (chzruan/MG-GLAM-Durham, Fortran 90 + OpenMP) passes all state
 * through module globals of `Module Tools` (PMP2mod_tools.f90:8-111) and calls
 * parameterless subroutines from `Program PMP` (PMP2main.f90:17-89).  Each entry
 * point below names the subroutine it replaces; a Fortran caller binds them with
 * iso_c_binding through a module of bind(C) interfaces, one per entry point.
 *
 * Grid layout: FP32, x fastest, 0-based index i + N*(j + N*k), i.e. exactly the
 * memory order of the column-major Fortran array FI(1:N,1:N,1:N).
 * Particle layout: six FP32 arrays (SoA) in grid units, positions in [1, N+1),
 * exactly XPAR, YPAR, ZPAR, VX, VY, VZ of Module Tools.
 */
#ifndef MGGLAM_H
#define MGGLAM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define MGG_OK                 0
#define MGG_ERR_ARG            1   /* invalid argument (size, pointer, enum)  */
#define MGG_ERR_CUDA           2   /* a CUDA runtime call failed              */
#define MGG_ERR_NOMEM          3   /* device allocation refused               */
#define MGG_ERR_STATE          4   /* call out of order (e.g. no particles)   */
#define MGG_ERR_UNSUPPORTED    5   /* model/option the reference rejects too  */
#define MGG_ERR_NUMERIC        6   /* NaN/Inf in a residual or energy         */
#define MGG_ERR_NO_DEVICE      7   /* no CUDA device / kernels not loadable   */

/* ---- gravity models (MG_model, PMP2mod_tools.f90:58-62) ----------------- */
#define MGG_MODEL_FR           1   /* Hu-Sawicki f(R)                         */
#define MGG_MODEL_DGP          2   /* normal/self-accelerating branch DGP     */
#define MGG_MODEL_SYMMETRON    3
#define MGG_MODEL_KMOUFLAGE    4
#define MGG_MODEL_CSF          5   /* coupled scalar field                    */

/* ---- precision forms ---------------------------------------------------- */
#define MGG_PREC_PLAIN         0   /* FP32 storage, FP64 arithmetic where the
                                      reference computes in real*8 (the FFT
                                      lines included, FP32 between passes as
                                      FFTPACK5 stores them)                   */
#define MGG_PREC_MIXED         1   /* FP32 bulk arithmetic (smoothers, FFT);
                                      FP64 kept for the pointwise roots,
                                      norms, zero mode, P(k) sums             */

/* ---- grids addressable by upload/download ------------------------------- */
#define MGG_GRID_FI            0   /* density contrast / potential (FI)       */
#define MGG_GRID_FI2           1   /* scalar field (FI2)                      */

/* ---- TimingMain buckets (PMP2mod_tools.f90:525-547) --------------------- */
#define MGG_T_TOTAL            0
#define MGG_T_FORCE            1   /* POTENTfft5 (+ POTENT_FOR_MG)            */
#define MGG_T_MOVE             2
#define MGG_T_DENSITY          3
#define MGG_T_POWER            4
#define MGG_T_MG               8
#define MGG_T_NBUCKETS         11

/*
 * Setup.dat contents that the path reads (ReadSetup, PMP2mod_tools.f90:114-231).
 * Scalars keep the reference's kinds: real*4 cosmology, real*8 MG parameters.
 */
typedef struct mgg_config {
    int32_t ngrid;            /* NGRID (power of two, 16..1024)               */
    int32_t nrow;             /* NROW; Nparticles = NROW^3                     */
    float   box;              /* Box [Mpc/h]                                   */
    float   om, oml, omb;     /* Om, OmL, Omb                                  */
    int32_t mg_flag;          /* MG_flag: 1 = solve the scalar field           */
    int32_t mg_model;         /* MGG_MODEL_*                                   */
    int32_t vcycle, fcycle, wcycle;  /* cycle type flags (exactly one set)     */
    int32_t iter_count_max;   /* maximum number of cycles per solve            */
    double  res_conv;         /* residual RMS convergence target               */
    int32_t fr_n;             /* Hu-Sawicki n (0, 1, 2)                         */
    double  fr0;              /* f_R0 (negative)                               */
    int32_t n_branch, s_branch;
    double  h0rc;             /* H0 * r_c                                      */
    double  sym_astar, sym_xi, sym_beta;
    int32_t kmf_power_law, kmf_born_infeld, kmf_n;
    double  kmf_k0, kmf_beta, kmf_lambda;   /* kmf_lambda from the background  */
    int32_t csf_coupling, csf_potential;
    double  csf_alpha, csf_beta, csf_lambda;
    int32_t precision;        /* MGG_PREC_*                                    */
    int32_t device;           /* CUDA device ordinal                           */
} mgg_config;

/* Per-solve report of scalar_field (PMP2extradof.f90:92-128). */
typedef struct mgg_mg_report {
    int32_t cycles;           /* iter_count at exit                            */
    int32_t exit_reason;      /* 1 residual <= res_conv, 2 stagnation,
                                 3 iter_count_max reached, 0 skipped (sym a<a*) */
    double  residual[64];     /* RMS residual on the PM grid after each cycle  */
} mgg_mg_report;

typedef struct mgg_ctx mgg_ctx;

/* Allocates the device-resident state of one box (Initialize allocations,
 * PMP2main.f90:115-122; MG_scratch_ensure, PMP2mod_tools.f90:560-581). */
int mgg_create(const mgg_config* cfg, mgg_ctx** out);
int mgg_destroy(mgg_ctx* ctx);
/* Last error message of ctx (or of the last failed mgg_create when ctx==NULL). */
const char* mgg_last_error(const mgg_ctx* ctx);

/* AEXPN and ASTEP of Module Tools (PMP2mod_tools.f90:36); ADDTIME
 * (PMP2main.f90:256-283) and the step growth (PMP2main.f90:48-52) stay in the
 * driver, which sets them here before each call. */
int mgg_set_time(mgg_ctx* ctx, float aexpn, float astep);

/* Host <-> device particle copies (ReadDataPM/WriteDataPM boundaries,
 * PMP2mod_tools.f90:237-487).  n must equal NROW^3. */
int mgg_upload_particles(mgg_ctx* ctx, const float* x, const float* y, const float* z,
                         const float* vx, const float* vy, const float* vz, int64_t n);
int mgg_download_particles(mgg_ctx* ctx, float* x, float* y, float* z,
                           float* vx, float* vy, float* vz, int64_t n);

/* DENSIT (PMP2mod_density.f90:17-301): FI := density contrast by CIC.
 * Deterministic: particles are sorted by their integer cell key and each cell
 * sums its contributions in a fixed order, so FI is bit-identical run to run. */
int mgg_density(mgg_ctx* ctx);

/* scalar_field(i_step) (PMP2extradof.f90:12-178): FAS multigrid solve of the
 * scalar field FI2 for the configured model; report may be NULL.  A context's
 * first solve (and every solve while mgg_profile is on) runs the cycles
 * eagerly and tests for the exit (107-121) on the host after each cycle.
 * Later solves with iter_count_max <= 1024 run as one CUDA graph: a while
 * node whose body is a cycle, the residual norm and the exit test, which runs
 * on the device with the same arithmetic, so the report is the same.  A
 * runtime without conditional graph nodes (before CUDA 12.4) keeps the host
 * loop. */
int mgg_scalar_field(mgg_ctx* ctx, int32_t i_step, mgg_mg_report* report);

/* POTENTfft5 (PMP2main.f90:705-867): FI := Newtonian potential of FI, solved
 * with the 7-point discrete Green's function by a 3-D real FFT. */
int mgg_potential(mgg_ctx* ctx);

/* POTENT_FOR_MG (PMP2main.f90:869-1015): FI += fifth-force potential(FI2). */
int mgg_potential_mg(mgg_ctx* ctx);

/* MOVE(FactV) (PMP2main.f90:304-685): kick and drift every particle; writes
 * ENKIN (PMP2main.f90:680) to *enkin when enkin != NULL. */
int mgg_move(mgg_ctx* ctx, float factv, double* enkin);

/* GetPower(0) -> POWERfft5(0,0) (PMP2mod_power.f90:20-66, 209-463): P(k) of FI.
 * With recompute_density != 0 the CIC density is made first, as Analysis does
 * (PMP2mod_analyze.f90:96-114).  FI is overwritten, as in the reference.
 * Outputs (each nbins = NGRID/2 entries, 1-based bin I stored at [I-1]):
 *   k, nmodes, pk          linear bins  (kharm, dNharm, Pk)
 *   klog, nmodeslog, pklog log bins     (kharmLog, dNharmLog, PkLog)
 * Any output pointer may be NULL. */
int mgg_power(mgg_ctx* ctx, int32_t recompute_density, int32_t nbins,
              double* k, double* nmodes, double* pk,
              double* klog, double* nmodeslog, double* pklog);

/* GetPower(1) (PMP2mod_power.f90:20-108, with DENSITrsd, PMP2mod_density.f90:
 * 407-557) with sigv = 0 (no added velocity dispersion): on the NGRID/2 mesh,
 * P(k) of the real-space density and, with each axis in turn as the line of
 * sight, the monopole and the quadrupole of the redshift-space density (the
 * line-of-sight coordinate moved by V*Xscale*sqrt(AEXPN/(Om+AEXPN^3 OmL))/AEXPN),
 * P0 and P2 being the averages over the three axes.  Outputs (nbins <= NGRID/4
 * entries, bin I at [I-1]): k, nmodes (the NGRID/2 mesh's bins), preal, p0, p2
 * (the columns Preal, P0_redshift, P2_redshift of PowerDM.Z files).  Uses the
 * positions and velocities on the device; FI is overwritten (the reference
 * reallocates it).  No counterpart for sigv > 0. */
int mgg_power_rsd(mgg_ctx* ctx, int32_t nbins, double* k, double* nmodes,
                  double* preal, double* p0, double* p2);

/* DensDistr (PMP2mod_density.f90:1041-1126): the PDF of 1 + delta in bins of
 * 0.001 dex, i = -2001..2001 stored at [i + 2001] (MGG_PDF_BINS entries).
 * level 0: FI as it stands (the density after mgg_density); level 1..4: the
 * CIC density of the particles on the NGRID/2^level mesh (DENSITrsd(0), as
 * Analysis does, PMP2mod_analyze.f90:44-86), which overwrites FI.
 * ncells: cells per bin; den_sum: sum of 1 + delta per bin (the reference
 * prints den_sum/ncells); stats[0] = RMS of 1 + delta, stats[1] = its mean. */
#define MGG_PDF_BINS 4003
int mgg_density_pdf(mgg_ctx* ctx, int32_t level, int64_t* ncells, double* den_sum, double* stats);

/* Grid copies for tests, MG_test fields and analysis (which = MGG_GRID_*). */
int mgg_upload_grid(mgg_ctx* ctx, int32_t which, const float* host);
int mgg_download_grid(mgg_ctx* ctx, int32_t which, float* host);

/* k-mouflage / coupled-scalar-field background table BackgroundEvolution
 * (PMP2mod_MGbackground.f90:469-731), computed on the host: rows x 6, row-major
 * (a, phi, dphi/dN, -, H/H0, -) as in the reference's column order. */
int mgg_set_background(mgg_ctx* ctx, const double* table, int32_t rows);

/* Background cosmology of the k-mouflage / coupled-scalar-field models, computed
 * on the host (Fix_Parameter_lambda + extradof_ini_background,
 * PMP2mod_MGbackground.f90:37-185, 469-731): fills table (row-major, 6 columns,
 * capacity_rows >= 100020), returns the row count, and -- as the reference does
 * with Module Tools -- stores the shooting solution lambda into cfg->kmf_lambda
 * or cfg->csf_lambda (also returned in *lambda).  Needs no device; on failure
 * mgg_last_error(NULL) holds the message. */
int mgg_background_table(mgg_config* cfg, double hubble, double* table, int32_t capacity_rows,
                         int32_t* rows, double* lambda);

/* CIC density of caller-owned device arrays with no device allocation.  This
 * entry point has no counterpart in the reference.  It is for callers that
 * cannot call cudaMalloc -- a host whose device memory all comes from its own
 * pool or arena, or code that must not allocate (and so possibly synchronise
 * the device) in the middle of its work.  x, y, z: np positions in [1, NGRID+1)
 * (the reference's convention) on the current device; fi: NGRID^3 floats on
 * the current device, overwritten with delta = rho/rho_mean - 1, bit-identical
 * to mgg_density for the same particles.  Scratch is one fixed array of about
 * 40.5 MiB in device memory that every GPU loading this library holds until the
 * process exits; sizes beyond it are rejected: NGRID a power of two in
 * [16, 256], 1 <= np <= 2097152 (2^21).  The first call on a device does a
 * one-time set-up with that device current (it looks up the scratch array's
 * device address and keeps it for the life of the process, so a
 * cudaDeviceReset between calls is not supported).  Runs on stream (NULL =
 * the default stream), which must belong to the current device, and returns
 * after the grid is complete: it waits on the host for its own result, so it
 * can never be called while the stream is being captured (MGG_ERR_STATE, with
 * no work queued).  All calls share the scratch array, which keeps the last
 * call's contents: calls that overlap on the GPU (other threads or streams)
 * race.  On failure mgg_last_error(NULL) holds the message. */
int mgg_density_noalloc(const float* x, const float* y, const float* z, int64_t np, int32_t ngrid,
                        float* fi, void* stream);

/* Integer keys of the last CIC deposit on the NGRID mesh (mgg_density, mgg_power
 * with recompute_density), for tests and diagnostics.  The reference forms the
 * same keys I = INT(X), J = INT(Y), K = INT(Z) of every particle in DENSIT
 * (PMP2mod_density.f90:235-248).  rowcnt[r] (NGRID^2 entries): particles of row
 * r = (J-1) + NGRID (K-1); rowstart (NGRID^2 + 1 entries): exclusive offsets of
 * the row buckets the positions were sorted into; cellcnt[(I-1) + NGRID r]
 * (NGRID^3 entries): particles per cell, recounted from the positions in each
 * row bucket (a temporary device array of NGRID^3 counts is allocated for it).
 * Any pointer may be NULL.  MGG_ERR_STATE when an analysis call deposited on
 * another mesh since the last density. */
int mgg_cic_keys(mgg_ctx* ctx, uint32_t* rowcnt, uint32_t* rowstart, uint32_t* cellcnt);

/* Wait for all work queued on the context's streams (and the host copies of
 * mgg_step_host_pipelined). */
int mgg_synchronize(mgg_ctx* ctx);

/* Device time per TimingMain bucket (MGG_T_*), cumulative ms, measured with CUDA
 * events on the context's stream; out must hold MGG_T_NBUCKETS doubles. */
int mgg_timing(mgg_ctx* ctx, double* out);

/* Per-kernel launch profile.  With enable != 0, every kernel launch of the
 * context is bracketed by CUDA events on its stream.  mgg_profile_read returns,
 * for kernel class id (0 <= id < mgg_profile_count()), its name, the number of
 * launches, the summed device ms and the summed algorithmic bytes. */
int mgg_profile(mgg_ctx* ctx, int32_t enable);
int mgg_profile_count(void);
int mgg_profile_read(mgg_ctx* ctx, int32_t id, const char** name,
                     int64_t* launches, double* total_ms, double* alg_bytes);
int mgg_profile_reset(mgg_ctx* ctx);

/* Device timer on the context's stream: mgg_timer_stop synchronises the stream
 * (after a velocity download of mgg_step_host_pipelined still in flight) and
 * returns the elapsed device ms since the matching mgg_timer_start. */
int mgg_timer_start(mgg_ctx* ctx);
int mgg_timer_stop(mgg_ctx* ctx, double* ms);

/* Synthetic initial conditions made on the device (the role of PMP2start,
 * PMP2start.f90:797-873): Zel'dovich displacement of a Gaussian random field with
 * a BBKS P(k) normalised to sigma8, growth-scaled to AEXPN, on the NROW^3
 * lattice.  The random field comes from a counter-based generator keyed by seed,
 * so the same seed gives the same particles on any device. */
typedef struct mgg_ic_params {
    uint64_t seed;
    double   sigma8, hubble, ns;   /* P(k) = A k^ns T_BBKS(k)^2, sigma8-normalised */
    float    aexpn, astep;         /* initial expansion factor and step            */
} mgg_ic_params;
int mgg_make_ics(mgg_ctx* ctx, const mgg_ic_params* ic);

/* ---------------------------------------------------------------------------
 * Forms beside the routine-by-routine drop-in path.
 * ------------------------------------------------------------------------- */

/* Module Tools time-stepping state of one box (PMP2mod_tools.f90:36,
 * PMP2main.f90:124): AEXPN, ASTEP, StepFactor = ASTEP0/AEXPN0, ISTEP, plus
 * the outputs of the last step (MOVE's ENKIN, scalar_field's report). */
typedef struct mgg_step_state {
    float   aexpn, astep, step_factor;
    int32_t istep;
    double  ekin;
    mgg_mg_report report;
} mgg_step_state;

/* One iteration of the main loop of Program PMP (PMP2main.f90:36-60):
 * DENSIT, scalar_field(ISTEP+1) when MG_flag = 1, POTENTfft5, the ASTEP
 * growth and FactV rule (48-52), POTENT_FOR_MG, MOVE, ADDTIME (256-261).
 * The whole step is queued on the context's stream and the call waits for
 * the device once, at its end: after a context's first multigrid solve, the
 * solve's exit test runs on the device (see mgg_scalar_field).  On failure the
 * particles and *st are left as they were. */
int mgg_step(mgg_ctx* ctx, mgg_step_state* st);

/* nsteps iterations of mgg_step (the main loop, PMP2main.f90:36-81) queued as
 * CUDA graphs of four steps each, launched back to back (the host records the
 * next while the device runs the last): every step's kernels, each multigrid
 * solve a while node with its exit test on the device, and each step's results
 * (error flags, solve report, kinetic-energy sum) in device memory, read back
 * once after the last step.  No host round trip between the steps.  reports[nsteps] and ekin[nsteps] receive each step's report and
 * ENKIN (either may be NULL); *st is advanced as by nsteps calls of mgg_step,
 * with the same results bit for bit.  A context's first steps, up to and
 * including its first multigrid solve, run one by one (that solve and the
 * first transforms tune the launch shapes), and so do all steps with profiling
 * on, iter_count_max above 1024 or a runtime without conditional graph
 * nodes.  If a step fails,
 * the later steps leave the particles alone, *st is the state after the last
 * good step, and the call returns that step's error; the scalar field is then
 * not meaningful. */
int mgg_run_steps(mgg_ctx* ctx, mgg_step_state* st, int32_t nsteps, mgg_mg_report* reports, double* ekin);

/* mgg_step with the particles in host memory: uploads them, runs the step and
 * downloads the result into the same arrays.  The velocities are copied on a
 * second stream while the density, scalar field and potential are computed,
 * and MOVE waits for them, so their transfer is hidden behind the step. */
int mgg_step_host(mgg_ctx* ctx, mgg_step_state* st, float* x, float* y, float* z, float* vx, float* vy, float* vz,
                  int64_t n);

/* mgg_step_host for a driver that steps the same host arrays again and again:
 * the same copies and the same step, but the call returns as soon as the
 * positions are back in x, y, z, and the velocities follow to vx, vy, vz in the
 * background (on a second stream), beside the next call's position upload.  The
 * next call's velocity upload reads vx, vy, vz only after that download has
 * finished, and it overlaps the next step's density, scalar field and
 * potential.  The host
 * velocity arrays are complete after mgg_synchronize(ctx), and must not be
 * read or written before it.  Same result as mgg_step_host. */
int mgg_step_host_pipelined(mgg_ctx* ctx, mgg_step_state* st, float* x, float* y, float* z, float* vx, float* vy,
                            float* vz, int64_t n);

/* Batched form: one main-loop step of each of n boxes, run concurrently (one
 * host thread and one stream per box) so that their kernels overlap on the
 * device.  Each box's result is the one mgg_step gives it alone.  Returns
 * the first failing box's status; mgg_last_error(ctxs[i]) names the error. */
int mgg_step_batch(mgg_ctx* const* ctxs, mgg_step_state* states, int32_t n);

/* The configuration the context was created (or last reconfigured) with. */
int mgg_get_config(const mgg_ctx* ctx, mgg_config* cfg);

/* Rebind a context to another box of the same NGRID, NROW, MG_flag and
 * device (other model parameters or cosmology), keeping its device memory.
 * Particles, FI2 and the background table must be set again. */
int mgg_reconfigure(mgg_ctx* ctx, const mgg_config* cfg);

/* Device bytes one context of this configuration holds (estimate used for
 * admission by the server). */
int64_t mgg_box_bytes(const mgg_config* cfg);

/* Serving form: a device-resident request loop.  Each request is one box:
 * synthetic ICs, nsteps main-loop steps, then P(k) of the final density.
 * Requests are admitted in arrival order while the device-memory budget and
 * the slot count allow, run concurrently (own host thread, stream and
 * context each; contexts of finished requests are reused by later requests
 * of the same sizes), and keep particles and fields on the device between
 * steps.  k-mouflage / csf requests get their background table from the
 * host solver, cached per parameter set. */
typedef struct mgg_server mgg_server;
typedef struct mgg_request {
    mgg_config    cfg;
    mgg_ic_params ic;      /* ic.aexpn / ic.astep: AEXPN0 and ASTEP0        */
    int32_t       nsteps;
} mgg_request;
typedef struct mgg_result_info {
    int32_t status;        /* MGG_OK or the failing call's code             */
    int32_t nbins;         /* P(k) bins written (NGRID/2)                   */
    float   aexpn;         /* expansion factor at the end                   */
    int32_t steps;         /* steps run                                     */
    int64_t cycles;        /* MG cycles run                                 */
    double  ekin;          /* ENKIN of the last step                        */
    double  t_submit_ms, t_admit_ms, t_done_ms;   /* since the server start  */
} mgg_result_info;
int mgg_server_create(int32_t device, double hbm_budget_gb, int32_t max_active, mgg_server** out);
int mgg_server_submit(mgg_server* srv, const mgg_request* req, int64_t* id);
/* Blocks until request id is done; copies min(capacity, nbins) P(k) bins
 * (k, Nmodes, P as mgg_power) and the result record.  Each id is waited once. */
int mgg_server_wait(mgg_server* srv, int64_t id, mgg_result_info* info, double* k, double* nmodes, double* pk,
                    int32_t capacity);
/* Waits for running requests, frees every context. */
int mgg_server_destroy(mgg_server* srv);
const char* mgg_server_error(const mgg_server* srv, int64_t id);

/* ---------------------------------------------------------------------------
 * PM snapshot files of the reference (ReadDataPM / WriteDataPM,
 * PMP2mod_tools.f90:237-487), big-endian as written by `-convert big_endian`:
 *   PMcrd.DAT (moment < 0) or PMcrd.NNNN.DAT: one sequential unformatted
 *     record (4-byte length markers) holding the header below, 529 bytes;
 *   PMcrs<i>.DAT or PMcrs<i>.NNNN.DAT: direct-access records of 1024^2
 *     particles, x(1024^2) y z vx vy vz as Real*4, at most 512 records per
 *     file; the last record is padded to full length (with zeros here).
 * Positions are in grid units [1, NGRID+1); on reading, a coordinate with
 * INT(x) = NGRID+1 is moved down by 1e-3 as the reference does.
 * ------------------------------------------------------------------------- */
typedef struct mgg_pm_header {
    char    header[45];
    float   aexpn, aexp0, amplt, astep;
    int32_t istep;
    float   partw, tintg, ekin, ekin1, ekin2, au0, aeu0;
    int32_t nrow, ngrid, nrealization, nseed;
    float   om, oml, hubble;
    int64_t nparticles;
    float   extras[100];      /* extras[99] = Box                          */
} mgg_pm_header;
int mgg_pm_write(const char* dir, int32_t moment, const mgg_pm_header* h, const float* x, const float* y,
                 const float* z, const float* vx, const float* vy, const float* vz);
int mgg_pm_read_header(const char* dir, int32_t moment, mgg_pm_header* h);
/* Message of the last failing mgg_pm_* call. */
const char* mgg_pm_last_error(void);
/* Reads h->nparticles particles (capacity checked). */
int mgg_pm_read(const char* dir, int32_t moment, mgg_pm_header* h, float* x, float* y, float* z, float* vx,
                float* vy, float* vz, int64_t capacity);

/* Library version string. */
const char* mgg_version(void);

#ifdef __cplusplus
}
#endif
#endif /* MGGLAM_H */
