// Host-side background cosmology of the k-mouflage and coupled-scalar-field
// models: the table BackgroundEvolution(i, 1:6) of extradof_ini_background and
// the shooting solve for the potential/kinetic parameter lambda of
// Fix_Parameter_lambda (PMP2mod_MGbackground.f90:37-185, 200-731).
//
// The reference integrates the two-variable ODE in N = ln a with DVERK (a
// Verner 6(5) Runge-Kutta, PMP2MG_subroutines.f90:4-762) at atol 2e-13; this
// restatement uses classical 4th-order Runge-Kutta with 2 sub-steps per table
// interval (dN = |N_start| / 10^5 / 2 ~ 7e-5; the local error ~dN^5 is far
// below that tolerance on this smooth system).  The table rows, their N spacing, the initial values
// (1e-30 / 1e-10 / 1e-6) and the columns are the reference's.
#include "mgg_internal.cuh"
#include <cmath>

namespace mgg {

namespace {

constexpr int kNumPoints = 100000;
constexpr int kNumPointsEx = kNumPoints + 20;
constexpr double kZst = 1000000.0;
constexpr double kG = 6.6738e-11, kSigmaB = 5.6704e-8, kMpc = 3.085678e22, kCol = 2.99792458e8, kTcmb = 2.7255,
                 kNnu = 3.046;

struct Bg {
    int model;
    double Om, hubble;
    int kmf_n;
    double kmf_K0, kmf_beta;
    int csf_coupling, csf_potential;
    double csf_alpha, csf_beta;
    double lambda;
    double grhog, grhornomass, grhom, grhobc;

    void init(const mgg_config& c, double h) {
        model = c.mg_model;
        Om = (double)c.om;
        hubble = (double)(float)h;   // Real*4 hubble of Module Tools
        kmf_n = c.kmf_n;
        kmf_K0 = c.kmf_k0;
        kmf_beta = c.kmf_beta;
        csf_coupling = c.csf_coupling;
        csf_potential = c.csf_potential;
        csf_alpha = c.csf_alpha;
        csf_beta = c.csf_beta;
        const double kappa = 8.0 * acos(-1.0) * kG;
        grhog = kappa / (kCol * kCol) * 4.0 * kSigmaB / (kCol * kCol * kCol) * pow(kTcmb, 4) * kMpc * kMpc;
        const double grhor = (7.0 / 8.0) * pow(4.0 / 11.0, 4.0 / 3.0) * grhog;
        grhornomass = kNnu * grhor;
        grhom = 3.0 * (100.0 * hubble) * (100.0 * hubble) / (kCol * kCol) * 1000.0 * 1000.0;
        grhobc = grhom * Om;
    }
    // Cofpsi (PMP2mod_MGbackground.f90:200-247): exponential coupling for k-mouflage
    double C(double psi, int deriv) const {
        const int type = model == 4 ? 1 : csf_coupling;
        const double b = model == 4 ? kmf_beta : csf_beta;
        if (type == 0) return deriv == 0 ? 1.0 : 0.0;
        if (type == 1) return deriv == 0 ? exp(b * psi) : (deriv == 1 ? b * exp(b * psi) : b * b * exp(b * psi));
        return deriv == 0 ? 1.0 + b * psi * psi : (deriv == 1 ? 2.0 * b * psi : 2.0 * b);
    }
    // Vofpsi (249-286): inverse power law for the coupled scalar field
    double V(double psi, int deriv) const {
        if (csf_potential != 1) return deriv == 0 ? 1.0 - Om : 0.0;
        const double a = csf_alpha;
        if (deriv == 0) return lambda / pow(psi, a);
        if (deriv == 1) return -lambda * a / pow(psi, 1.0 + a);
        return lambda * a * (1.0 + a) / pow(psi, 2.0 + a);
    }
    // (H/H0)^2, H'/H0^2 and sigma (k-mouflage) at N for state y (290-460)
    void hubble_terms(double N, const double* y, double& HoH02, double& HpoH02, double& sig) const {
        HoH02 = (grhog + grhornomass) * exp(-2.0 * N) / grhom;
        HoH02 = HoH02 + C(y[0], 0) * grhobc * exp(-N) / grhom;
        HpoH02 = (grhog + grhornomass) * 2.0 / grhom * exp(-2.0 * N);
        HpoH02 = HpoH02 + C(y[0], 0) * grhobc * exp(-N) / grhom;
        HpoH02 = -HpoH02 / 2.0;
        sig = 0.0;
        if (model == 4) {
            HoH02 = HoH02 + lambda * lambda * exp(2.0 * N) / 3.0;
            double AA = ((double)kmf_n - 0.5) * kmf_K0 * pow(0.5 / (lambda * lambda), kmf_n - 1) *
                        exp(-2.0 * (kmf_n - 1.0) * N) * pow(y[1], 2 * kmf_n) / 3.0;
            const double BB = -1.0 + y[1] * y[1] / 6.0;
            AA = AA > 0.0 ? fmax(AA, 1.0e-20) : fmin(AA, -1.0e-20);
            if (kmf_n == 2) {
                HoH02 = (-BB - sqrt(BB * BB - 4.0 * AA * HoH02)) / (2.0 * AA);
            } else {
                const double S0 = -3.0 * AA * BB, S1 = 27.0 * AA * AA * HoH02;
                if (S1 * S1 >= 4.0 * S0 * S0 * S0) {
                    const double ex = sqrt(1.0 - 4.0 * S0 * S0 * S0 / (S1 * S1));
                    const double Gama = pow(S1 / 2.0 * (1.0 + ex), 1.0 / 3.0);
                    HoH02 = -(Gama + S0 / Gama) / (3.0 * AA);
                } else {
                    const double ex = acos(S1 / 2.0 / sqrt(S0 * S0 * S0));
                    HoH02 = -2.0 * sqrt(S0) * cos(ex / 3.0 - 2.0 * acos(0.5)) / (3.0 * AA);
                }
            }
            sig = 0.5 * HoH02 * y[1] * y[1] * exp(-2.0 * N) / (lambda * lambda);
            const double KK = -1.0 + sig + kmf_K0 * pow(sig, kmf_n);
            const double K_s = 1.0 + kmf_n * kmf_K0 * pow(sig, kmf_n - 1);
            HpoH02 = HpoH02 - K_s * HoH02 * y[1] * y[1] / 6.0 - exp(2.0 * N) * lambda * lambda * KK / 3.0;
        } else {
            HoH02 = HoH02 + V(y[0], 0) * exp(2.0 * N);
            HoH02 = HoH02 / (1.0 - y[1] * y[1] / 6.0);
            HpoH02 = HpoH02 + V(y[0], 0) * exp(2.0 * N);
            HpoH02 = HpoH02 - HoH02 * y[1] * y[1] / 3.0;
        }
    }
    void rhs(double N, const double* y, double* yp) const {
        double HoH02, HpoH02, sig;
        hubble_terms(N, y, HoH02, HpoH02, sig);
        yp[0] = y[1];
        if (model == 4) {
            const double HpoH2 = HpoH02 / HoH02;
            const double sn1 = pow(sig, kmf_n - 1);
            double y2 = 2.0 * (1.0 + (double)kmf_n * (2.0 - (double)kmf_n) * kmf_K0 * sn1) * y[1] +
                        (1.0 + (double)kmf_n * (2.0 * (double)kmf_n - 1.0) * kmf_K0 * sn1) * HpoH2 * y[1] +
                        3.0 * C(y[0], 1) * (grhobc / grhom) * exp(-N) / HoH02;
            yp[1] = -y2 / (1.0 + kmf_n * (2.0 * kmf_n - 1.0) * kmf_K0 * sn1);
        } else {
            yp[1] = -(y[1] * (HpoH02 + 2.0 * HoH02) + 3.0 * V(y[0], 1) * exp(2.0 * N) +
                      3.0 * (grhobc / grhom) * C(y[0], 1) * exp(-N)) /
                    HoH02;
        }
    }
    void step(double& N, double* y, double N1) const {
        const int sub = 2;
        const double h = (N1 - N) / sub;
        for (int s = 0; s < sub; ++s) {
            double k1[2], k2[2], k3[2], k4[2], t[2];
            rhs(N, y, k1);
            t[0] = y[0] + 0.5 * h * k1[0]; t[1] = y[1] + 0.5 * h * k1[1];
            rhs(N + 0.5 * h, t, k2);
            t[0] = y[0] + 0.5 * h * k2[0]; t[1] = y[1] + 0.5 * h * k2[1];
            rhs(N + 0.5 * h, t, k3);
            t[0] = y[0] + h * k3[0]; t[1] = y[1] + h * k3[1];
            rhs(N + h, t, k4);
            y[0] += h / 6.0 * (k1[0] + 2.0 * k2[0] + 2.0 * k3[0] + k4[0]);
            y[1] += h / 6.0 * (k1[1] + 2.0 * k2[1] + 2.0 * k3[1] + k4[1]);
            N += h;
        }
        N = N1;
    }
    void initial(double* y) const {
        if (model == 4) {
            const double v = kmf_K0 < 0.0 ? 1.0e-10 : 1.0e-30;
            y[0] = v;
            y[1] = v;
        } else {
            y[0] = 1.0e-6;
            y[1] = 1.0e-6;
        }
    }
    // H/H0 at a = 1 after integrating from N_start (Fix_Parameter_lambda, 62-105)
    double h_today() const {
        const double Nstart = -log(1.0 + kZst);
        double y[2], N = Nstart;
        initial(y);
        for (int i = 1; i <= kNumPoints; ++i) step(N, y, Nstart + i * fabs(Nstart) / kNumPoints);
        double HoH02, HpoH02, sig;
        hubble_terms(0.0, y, HoH02, HpoH02, sig);
        return sqrt(HoH02);
    }
};

}  // namespace

int background_table(mgg_config& c, double hubble, double* table, int capacity, int* rows, double* lambda_out) {
    if (c.mg_model != 4 && c.mg_model != 5) throw Error{MGG_ERR_ARG, "background: only k-mouflage and csf need it"};
    if (c.mg_model == 4 && c.kmf_n != 2 && c.kmf_n != 3)
        throw Error{MGG_ERR_UNSUPPORTED, "background: k-mouflage n must be 2 or 3 (as in the reference)"};
    if (capacity < kNumPointsEx) throw Error{MGG_ERR_ARG, "background: table needs 100020 rows"};
    Bg b;
    b.init(c, hubble);
    // shooting for lambda (Fix_Parameter_lambda, 48-148): step, halve and reverse
    double lambda = 1.0, steplen = 0.1, flag = 1.0;
    int it = 0;
    for (;;) {
        b.lambda = lambda;
        const double H = b.h_today();
        if (!std::isfinite(H)) throw Error{MGG_ERR_NUMERIC, "background: H/H0 is not finite"};
        if (fabs(H - 1.0) < 1.0e-6) break;
        if ((H - 1.0) * flag < 0.0) steplen = steplen;
        else steplen = -0.5 * steplen;
        flag = -(H - 1.0) / fabs(H - 1.0);
        lambda = lambda + steplen;
        if (++it > 400) throw Error{MGG_ERR_NUMERIC, "background: lambda search did not converge"};
    }
    if (c.mg_model == 4) c.kmf_lambda = lambda;
    else c.csf_lambda = lambda;
    if (lambda_out) *lambda_out = lambda;
    // the table (extradof_ini_background, 469-731)
    const double Nstart = -log(1.0 + kZst);
    double y[2], N = Nstart;
    b.initial(y);
    for (int i = 1; i <= kNumPointsEx; ++i) {
        const double Ni = Nstart + (double)(i - 1) * fabs(Nstart) / (double)kNumPoints;
        if (i > 1) b.step(N, y, Ni);
        double HoH02, HpoH02, sig, yp[2];
        b.hubble_terms(Ni, y, HoH02, HpoH02, sig);
        b.rhs(Ni, y, yp);
        double* r = table + (size_t)(i - 1) * 6;
        r[0] = exp(Ni);
        r[1] = y[0];
        r[2] = y[1];
        r[3] = yp[1];
        r[4] = sqrt(HoH02);
        r[5] = c.mg_model == 4 ? sig : HpoH02;
    }
    *rows = kNumPointsEx;
    return MGG_OK;
}

}  // namespace mgg
