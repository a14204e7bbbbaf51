// pmp_main: a C++ restatement of the reference driver `Program PMP`
// (PMP2main.f90:17-89) over the C ABI of libmgglam_b200.so.
//
//   pmp_main Setup.dat NSTEPS [--seed S] [--realization R] [--device D]
//
// Reads a reference-format Setup.dat (ReadSetup, PMP2mod_tools.f90:114-231),
// builds the time-step table of Initialize (PMP2main.f90:154-184), makes the
// initial conditions on the device (the role of PMP2start), runs the main loop
// with DENSIT / scalar_field / POTENTfft5 / POTENT_FOR_MG / MOVE / ADDTIME on
// the GPU, writes PowerDM.R.<ISTEP>.<Nrealization>.dat at the analysis moments
// (GetPower, PMP2mod_power.f90:40-53) and appends timing.log rows in the
// TimingMain layout (PMP2mod_tools.f90:525-547), in minutes of device time.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/mgglam.h"

namespace {

struct Setup {
    std::string header;
    float aexpn0 = 0, astep0 = 0, amplt = 0, box = 0, sigma8 = 0, hubble = 0, om = 0, oml = 0, omb = 0;
    int nrow = 0, ngrid = 0, nseed = 0;
    float zinit = 0, zfinal = 0;
    std::vector<float> zout;
    int ncheckpoint = 20, isave = 0, ipower = 1;
    int mg_flag = 0, mg_test = 0, mg_model = 1, vcycle = 1, fcycle = 0, wcycle = 0, iter_count_max = 4;
    double res_conv = 1e-8;
    int fr_n = 1;
    double fr0 = -1e-5;
    int n_branch = 0, s_branch = 0;
    double h0rc = 1.0, sym_astar = 0.5, sym_xi = 1e-3, sym_beta = 0.1;
    int power_law = 1, born_infeld = 0, kmf_n = 3;
    double kmf_k0 = 1.0, kmf_beta = 0.1;
    int csf_coupling = 1, csf_potential = 1;
    double csf_alpha = 0.1, csf_beta = -0.2;
};

// Fortran list-directed reading: one value per READ(11,*) taken from the next
// line; D exponents accepted.
struct Reader {
    std::vector<std::string> lines;
    size_t pos = 0;
    bool ok = true;
    explicit Reader(const char* path) {
        std::ifstream f(path);
        if (!f) { ok = false; return; }
        std::string l;
        while (std::getline(f, l)) lines.push_back(l);
    }
    std::string line() { return pos < lines.size() ? lines[pos++] : std::string(); }
    static std::string fix(std::string t) {
        for (auto& ch : t) if (ch == 'D' || ch == 'd') ch = 'E';
        return t;
    }
    std::string token() {
        std::string l = line();
        std::istringstream is(l);
        std::string t;
        is >> t;
        return t;
    }
    double num() { return std::atof(fix(token()).c_str()); }
    int inum() { return (int)std::lround(num()); }
    std::vector<double> nums(int n) {   // list-directed read of n values over lines
        std::vector<double> v;
        while ((int)v.size() < n && pos < lines.size()) {
            std::istringstream is(line());
            std::string t;
            while ((int)v.size() < n && is >> t) v.push_back(std::atof(fix(t).c_str()));
        }
        return v;
    }
};

bool read_setup(const char* path, Setup& s) {
    Reader r(path);
    if (!r.ok) return false;
    r.line();
    s.header = r.token();
    s.aexpn0 = (float)r.num();
    s.astep0 = (float)r.num();
    s.amplt = (float)r.num();
    s.box = (float)r.num();
    s.sigma8 = (float)r.num();
    s.hubble = (float)r.num();
    s.om = (float)r.num();
    s.oml = (float)r.num();
    s.omb = (float)r.num();
    s.nrow = r.inum();
    s.ngrid = r.inum();
    s.nseed = r.inum();
    r.num();   // Cell
    r.num();   // aMass
    s.zinit = (float)r.num();
    s.zfinal = (float)r.num();
    r.num();   // DensThr
    r.num();   // sigV
    const int nout = r.inum();
    for (double z : r.nums(nout)) s.zout.push_back((float)z);
    const int nbias = r.inum();
    for (int i = 0; i < nbias; ++i) r.num();
    s.ncheckpoint = r.inum();
    s.isave = r.inum();
    s.ipower = r.inum();
    for (int i = 0; i < 6; ++i) r.inum();   // iPowerRSD .. iBDM
    r.line();
    s.mg_flag = r.inum();
    s.mg_test = r.inum();
    s.mg_model = r.inum();
    s.vcycle = r.inum();
    s.fcycle = r.inum();
    s.wcycle = r.inum();
    s.iter_count_max = r.inum();
    s.res_conv = r.num();
    r.line();
    s.fr_n = r.inum();
    s.fr0 = r.num();
    r.line();
    s.n_branch = r.inum();
    s.s_branch = r.inum();
    s.h0rc = r.num();
    r.line();
    s.sym_astar = r.num();
    s.sym_xi = r.num();
    s.sym_beta = r.num();
    r.line();
    s.power_law = r.inum();
    s.born_infeld = r.inum();
    s.kmf_n = r.inum();
    s.kmf_k0 = r.num();
    s.kmf_beta = r.num();
    r.line();
    s.csf_coupling = r.inum();
    s.csf_potential = r.inum();
    s.csf_alpha = r.num();
    s.csf_beta = r.num();
    return true;
}

#define CHECK(call)                                                                  \
    do {                                                                             \
        int rc_ = (call);                                                            \
        if (rc_ != MGG_OK) {                                                         \
            std::fprintf(stderr, "%s failed (%d): %s\n", #call, rc_, mgg_last_error(ctx)); \
            std::exit(1);                                                            \
        }                                                                            \
    } while (0)

}  // namespace

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s Setup.dat NSTEPS [--seed S] [--realization R] [--device D]\n", argv[0]);
        return 2;
    }
    Setup s;
    if (!read_setup(argv[1], s)) {
        std::fprintf(stderr, " Error: File %s not found. Run PMP2init.exe\n", argv[1]);
        return 1;
    }
    const int nsteps = std::atoi(argv[2]);
    uint64_t seed = (uint64_t)s.nseed;
    int nreal = 1, device = 0;
    for (int i = 3; i + 1 < argc; i += 2) {
        if (!std::strcmp(argv[i], "--seed")) seed = std::strtoull(argv[i + 1], nullptr, 10);
        if (!std::strcmp(argv[i], "--realization")) nreal = std::atoi(argv[i + 1]);
        if (!std::strcmp(argv[i], "--device")) device = std::atoi(argv[i + 1]);
    }
    mgg_config cfg{};
    cfg.ngrid = s.ngrid;
    cfg.nrow = s.nrow;
    cfg.box = s.box;
    cfg.om = s.om;
    cfg.oml = s.oml;
    cfg.omb = s.omb;
    cfg.mg_flag = s.mg_flag;
    cfg.mg_model = s.mg_model;
    cfg.vcycle = s.vcycle;
    cfg.fcycle = s.fcycle;
    cfg.wcycle = s.wcycle;
    cfg.iter_count_max = s.iter_count_max;
    cfg.res_conv = s.res_conv;
    cfg.fr_n = s.fr_n;
    cfg.fr0 = s.fr0;
    cfg.n_branch = s.n_branch;
    cfg.s_branch = s.s_branch;
    cfg.h0rc = s.h0rc;
    cfg.sym_astar = s.sym_astar;
    cfg.sym_xi = s.sym_xi;
    cfg.sym_beta = s.sym_beta;
    cfg.kmf_power_law = s.power_law;
    cfg.kmf_born_infeld = s.born_infeld;
    cfg.kmf_n = s.kmf_n;
    cfg.kmf_k0 = s.kmf_k0;
    cfg.kmf_beta = s.kmf_beta;
    cfg.csf_coupling = s.csf_coupling;
    cfg.csf_potential = s.csf_potential;
    cfg.csf_alpha = s.csf_alpha;
    cfg.csf_beta = s.csf_beta;
    cfg.device = device;
    mgg_ctx* ctx = nullptr;
    if (mgg_create(&cfg, &ctx) != MGG_OK) {
        std::fprintf(stderr, "mgg_create: %s\n", mgg_last_error(nullptr));
        return 1;
    }
    // time-step table (PMP2main.f90:154-184), Real*4 arithmetic
    const float step_factor = s.astep0 / s.aexpn0;
    std::vector<float> alist(1, s.aexpn0);
    {
        float da = s.astep0, a = s.aexpn0;
        for (;;) {
            if (da < step_factor / 1.25f * a && a < 0.300f) da = 1.5f * da;
            a = a + da;
            alist.push_back(a);
            if (alist.size() > 2001) { std::fprintf(stderr, "Too many timesteps\n"); return 1; }
            if (a >= 1.0f) break;
        }
    }
    const int ntotal = (int)alist.size() - 1;
    std::vector<int> nlist(alist.size() + 1, 0);
    for (float z : s.zout) {
        const float a = 1.0f / (1.0f + z);
        int j = 1;
        for (j = 1; j <= ntotal; ++j) if (a < alist[j]) break;
        if (j > ntotal) j = ntotal;
        const float da1 = alist[j] - a, da0 = a - alist[j - 1];
        if (da1 < da0) nlist[j] = 1; else nlist[j - 1] = 1;
    }
    float AEXPN = s.aexpn0, ASTEP = s.astep0;
    int ISTEP = 0;
    const int64_t npart = (int64_t)s.nrow * s.nrow * s.nrow;
    std::vector<float> px(npart), py(npart), pz(npart), pvx(npart), pvy(npart), pvz(npart);
    // WriteDataPM (PMP2mod_tools.f90:381-487): download the particles and write PM files
    auto write_pm = [&](int moment, double ekin) {
        CHECK(mgg_download_particles(ctx, px.data(), py.data(), pz.data(), pvx.data(), pvy.data(), pvz.data(), npart));
        mgg_pm_header h{};
        std::memset(h.header, ' ', sizeof(h.header));
        std::memcpy(h.header, s.header.data(), std::min<size_t>(s.header.size(), sizeof(h.header)));
        h.aexpn = AEXPN; h.aexp0 = s.aexpn0; h.astep = ASTEP; h.istep = ISTEP;
        h.partw = (float)s.ngrid * (float)s.ngrid * (float)s.ngrid / (float)npart;
        h.ekin = (float)ekin;
        h.nrow = s.nrow; h.ngrid = s.ngrid; h.nrealization = nreal; h.nseed = (int32_t)seed;
        h.om = s.om; h.oml = s.oml; h.hubble = s.hubble;
        h.nparticles = npart;
        h.extras[99] = s.box;
        if (mgg_pm_write(".", moment, &h, px.data(), py.data(), pz.data(), pvx.data(), pvy.data(), pvz.data()) != MGG_OK)
            std::fprintf(stderr, "WriteDataPM: %s\n", mgg_pm_last_error());
    };
    // ReadDataPM(-1) (PMP2main.f90:114): start from PMcrd.DAT when the run directory
    // has one (a restart or ICs from the Fortran tools), else make ICs on the device
    mgg_pm_header h0{};
    if (mgg_pm_read_header(".", -1, &h0) == MGG_OK && h0.nparticles == npart) {
        CHECK(mgg_pm_read(".", -1, &h0, px.data(), py.data(), pz.data(), pvx.data(), pvy.data(), pvz.data(), npart));
        CHECK(mgg_upload_particles(ctx, px.data(), py.data(), pz.data(), pvx.data(), pvy.data(), pvz.data(), npart));
        AEXPN = h0.aexpn;
        ASTEP = h0.astep;
        ISTEP = h0.istep;
        std::printf(" Read PMcrd.DAT: a=%8.4f step=%7d\n", AEXPN, ISTEP);
    } else {
        mgg_ic_params ic{seed, s.sigma8, s.hubble > 0 ? s.hubble : 0.6774, 0.9667, AEXPN, ASTEP};
        CHECK(mgg_make_ics(ctx, &ic));
    }
    std::printf(" Start running:  Nparticles: %lld  Ngrid= %d\n", (long long)s.nrow * s.nrow * s.nrow, s.ngrid);
    std::vector<double> t_prev(MGG_T_NBUCKETS, 0.0), t_now(MGG_T_NBUCKETS, 0.0);
    const int nb = s.ngrid / 2;
    std::vector<double> k(nb), nm(nb), pk(nb), kl(nb), nl(nb), pl(nb);
    double last_ekin = 0.0;
    for (int i = 1; i <= nsteps; ++i) {
        CHECK(mgg_set_time(ctx, AEXPN, ASTEP));
        CHECK(mgg_density(ctx));
        if (s.mg_flag == 1) {
            mgg_mg_report rep{};
            CHECK(mgg_scalar_field(ctx, i, &rep));
            for (int c = 0; c < rep.cycles && c < 64; ++c)
                std::printf("The residual is equal to %20.12f after %5d V-cycles.\n", rep.residual[c], c + 1);
        }
        CHECK(mgg_potential(ctx));
        float FactV = 1.0f;
        if (ASTEP < step_factor / 1.25f * AEXPN && AEXPN < 0.300f) {
            ASTEP = 1.5f * ASTEP;
            FactV = 1.2f;
        }
        if (s.mg_flag == 1) CHECK(mgg_potential_mg(ctx));
        CHECK(mgg_set_time(ctx, AEXPN, ASTEP));
        double enkin = 0.0;
        CHECK(mgg_move(ctx, FactV, &enkin));
        // ADDTIME (PMP2main.f90:256-283)
        ISTEP += 1;
        AEXPN = AEXPN + ASTEP;
        std::printf("Step = %4d A=%8.5f Ekin=%12.4E\n", ISTEP, AEXPN, enkin);
        if (s.ncheckpoint > 0 && ISTEP % s.ncheckpoint == 0) write_pm(-1, enkin);   // checkpoint (62-66)
        if (ISTEP < (int)nlist.size() && nlist[ISTEP] == 1 && s.isave == 1) write_pm(ISTEP, enkin);   // (68-71)
        last_ekin = enkin;
        if (ISTEP < (int)nlist.size() && nlist[ISTEP] == 1 && s.ipower) {
            CHECK(mgg_set_time(ctx, AEXPN, ASTEP));
            CHECK(mgg_power(ctx, 1, nb, k.data(), nm.data(), pk.data(), kl.data(), nl.data(), pl.data()));
            char name[128];
            std::snprintf(name, sizeof(name), "PowerDM.R.%04d.%04d.dat", ISTEP, nreal);
            if (FILE* f = std::fopen(name, "w")) {
                std::fprintf(f, "%s\n", s.header.c_str());
                std::fprintf(f, " Aexpn =%8.5f Step=%4d Redshift= %8.3f Ngrid= %4d kNyq= %8.2f\n", AEXPN, ISTEP,
                             1.0f / AEXPN - 1.0f, s.ngrid, 2.0f * 3.1415926f / s.box * s.ngrid / 2.0f);
                std::fprintf(f, "   bin  k/Mpch     N          Preal\n");
                for (int b = 0; b < nb; ++b)
                    std::fprintf(f, "%6d%9.5f%11.4E%13.5E\n", b + 1, k[b], nm[b], pk[b]);
                std::fclose(f);
            }
        }
        CHECK(mgg_timing(ctx, t_now.data()));
        if (FILE* f = std::fopen("timing.log", "a")) {
            if (ISTEP == 1) {
                std::fprintf(f, " Ngrid    = %11d Npart    = %11lld Nthreads = %11d\n", s.ngrid,
                             (long long)s.nrow * s.nrow * s.nrow, 1);
                std::fprintf(f, "  Step   Tot/min      Force       Move       Density      IO        Bias       BDM"
                                "        Analysis     MG\n");
            }
            std::fprintf(f, "%5d", ISTEP);
            for (int b = 0; b <= 8; ++b) std::fprintf(f, "%13.4f", (t_now[b] - t_prev[b]) / 60000.0);
            std::fprintf(f, "\n");
            std::fclose(f);
        }
        t_prev = t_now;
        if (AEXPN >= 1.0f - ASTEP / 2.0f) break;
    }
    // final snapshot (PMP2main.f90:83-86)
    if (s.isave >= 1 && !(ISTEP < (int)nlist.size() && nlist[ISTEP] == 1)) write_pm(ISTEP, last_ekin);
    mgg_destroy(ctx);
    return 0;
}
