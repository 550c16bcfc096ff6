// Host-side set-up of the engine: parameters, input files, LJ types, the
// k-vector list, the beta tables and the tails.  These run once per system
// (initmc) and are restated from the reference's host routines, cited per
// function; their operation order is kept so that the tables are bit-equal to
// what the reference computes.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "yamc_internal.h"

namespace yamc {

static thread_local std::string g_err;
void set_error(const std::string &msg) { g_err = msg; }
std::string last_error() { return g_err; }

// gfortran turns x**n (integer n) into multiplications.
static double powi(double x, int n) {
    double r = 1.0;
    bool have = false;
    double b = x;
    while (n > 0) {
        if (n & 1) { r = have ? r * b : b; have = true; }
        n >>= 1;
        if (n) b *= b;
    }
    return r;
}

// ---------------------------------------------------------------- parameters

// parameters.f90:18-72
static void params_defaults(yamc_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->sr = 4.0; p->sk = 4.0; p->alphaL = 0.0; p->temp = 298.15; p->external_permutivity = 50.0;
    p->BoxLength = 0.0; p->density = 33.33; p->dr_a = 0.4; p->d_angle_degree = 40.0;
    p->xlambda_c = 0.5; p->xlambda_f = 0.5; p->random_seed = 0; p->pressure = 0.0;
    p->pressure_step_multiplier = 0.0; p->max_volume_scaling = 1.05; p->max_cycle = 1000000;
    p->n_store_traj_interval = 100.0; p->n_store_energy_interval = 100.0;
    p->input_nbytes_xyz = p->input_nbytes_ang = p->output_nbytes_xyz = p->output_nbytes_ang = 2;
    p->precision = YAMC_FP64;
}

// read_parameter (parameters.f90:102-148)
static void apply_parameter(yamc_params *p, const std::string &nam, const std::string &val) {
    struct D { const char *k; double yamc_params::*f; };
    static const D dk[] = {
        {"sr", &yamc_params::sr}, {"sk", &yamc_params::sk}, {"alphaL", &yamc_params::alphaL},
        {"temp", &yamc_params::temp}, {"external_permutivity", &yamc_params::external_permutivity},
        {"BoxLength", &yamc_params::BoxLength}, {"density", &yamc_params::density},
        {"dr_a", &yamc_params::dr_a}, {"d_angle_degree", &yamc_params::d_angle_degree},
        {"xlambda_c", &yamc_params::xlambda_c}, {"xlambda_f", &yamc_params::xlambda_f},
        {"pressure_step_multiplier", &yamc_params::pressure_step_multiplier},
        {"max_volume_scaling", &yamc_params::max_volume_scaling},
        {"n_store_traj_interval", &yamc_params::n_store_traj_interval},
        {"n_store_energy_interval", &yamc_params::n_store_energy_interval},
        {"pressure", &yamc_params::pressure}};
    struct I { const char *k; int32_t yamc_params::*f; };
    static const I ik[] = {
        {"input_nbytes_xyz", &yamc_params::input_nbytes_xyz}, {"input_nbytes_ang", &yamc_params::input_nbytes_ang},
        {"output_nbytes_xyz", &yamc_params::output_nbytes_xyz}, {"output_nbytes_ang", &yamc_params::output_nbytes_ang},
        {"max_cycle", &yamc_params::max_cycle}, {"random_seed", &yamc_params::random_seed}};
    for (const D &d : dk) if (nam == d.k) p->*(d.f) = std::strtod(val.c_str(), nullptr);
    for (const I &i : ik) if (nam == i.k) p->*(i.f) = (int32_t)std::strtol(val.c_str(), nullptr, 10);
    if (nam == "precision") p->precision = (val == "mixed" || val == "1") ? YAMC_MIXED : YAMC_FP64;
}

static std::vector<std::string> tokens(const std::string &line) {
    std::vector<std::string> out;
    std::string cur;
    for (char c : line) {
        if (c == ' ' || c == '\t' || c == ',' || c == '\n' || c == '\r') {
            if (!cur.empty()) { out.push_back(cur); cur.clear(); }
        } else {
            cur.push_back(c);
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}

// Parameters_read_string (parameters.f90:209-263): "nam1=val1,nam2=val2"
static int params_read_string(yamc_params *p, const char *extra) {
    std::string s(extra ? extra : "");
    size_t pos = 0;
    while (pos < s.size()) {
        size_t comma = s.find(',', pos);
        std::string item = s.substr(pos, comma == std::string::npos ? std::string::npos : comma - pos);
        pos = comma == std::string::npos ? s.size() : comma + 1;
        if (item.find_first_not_of(' ') == std::string::npos) continue;
        size_t eq = item.find('=');
        if (eq == std::string::npos) { set_error("parameter string: expected '=' in '" + item + "'"); return YAMC_EPARAMETER; }
        auto nt = tokens(item.substr(0, eq)), vt = tokens(item.substr(eq + 1));
        if (nt.empty() || vt.empty()) { set_error("parameter string: empty name or value"); return YAMC_EPARAMETER; }
        apply_parameter(p, nt[0], vt[0]);
    }
    return YAMC_OK;
}

}  // namespace yamc

using namespace yamc;

extern "C" int yamc_params_recalc(yamc_params *p, double box_length) {
    // Parameters_recalc (parameters.f90:355-413)
    if (!p) return YAMC_EPARAMETER;
    const double boltz = 1.38065e-23, elec = 1.602176e-19, epsi0 = 8.854187e-12, kcal_mol = 6.9477e-21;
    if (!(box_length > 0.0)) { set_error("BoxLength must be positive"); return YAMC_EPARAMETER; }
    p->BoxLength = box_length;
    double alpha = p->alphaL;
    if (alpha < 1e-9) alpha = 2.0 * p->sr;  // rmax = L/2 by default
    p->alpha = alpha;
    p->alphaL = alpha;
    p->rmax = p->sr / alpha;
    p->kmax = (int32_t)std::lround(p->sk * alpha / kPi);
    // the reference build folds the constant ratios: its parameters.out holds
    // (boltz/kcal_mol)*temp and 2*xclb*(pi/(2*eps+1)) to the last bit
    p->kT_kcal_mol = (boltz / kcal_mol) * p->temp;
    p->dbjr_a = elec * elec / (4.0 * kPi * epsi0 * boltz * p->temp) / 1.0e-10;
    p->dbjr = p->dbjr_a / p->BoxLength;
    p->xclb = p->dbjr;
    p->dr = p->dr_a / p->BoxLength;
    p->d_angle = p->d_angle_degree * kPi / 180.0;
    p->alpha_over_sqrt_pi = alpha / std::sqrt(kPi);
    p->two_alpha_over_sqrt_pi = 2.0 * p->alpha_over_sqrt_pi;
    p->kext = 2.0 * p->xclb * (kPi / (2.0 * p->external_permutivity + 1.0));
    p->minus_two_kext = -2.0 * p->kext;
    p->rmax2 = p->rmax * p->rmax;
    p->log_max_volume_scaling = std::log(p->max_volume_scaling);
    p->pressure_angstr_kT = p->pressure / (boltz * p->temp) * 1.0e-30;
    return YAMC_OK;
}

extern "C" int yamc_params_init(yamc_params *p, int32_t nmol) {
    // Parameters_init (parameters.f90:323-352), BoxLength_from_density (:307-321)
    if (!p) return YAMC_EPARAMETER;
    if (std::fabs(p->BoxLength) < 1e-9) {
        if (std::fabs(p->density) < 1e-9) { set_error("both BoxLength and density are zero"); return YAMC_EPARAMETER; }
        double volume = nmol / p->density;
        p->BoxLength = std::pow(volume, 1.0 / 3.0) * 10.0;
    }
    return yamc_params_recalc(p, p->BoxLength);
}

extern "C" int yamc_params_read(const char *path, const char *extra, yamc_params *p) {
    // Parameters_read (parameters.f90:266-305): '=' is a blank, name and value are
    // the first two list-directed tokens, a name starting with '#' is a comment.
    if (!p) return YAMC_EPARAMETER;
    params_defaults(p);
    if (path && *path) {
        FILE *f = std::fopen(path, "r");
        if (!f) { set_error(std::string("cannot open ") + path); return YAMC_EIO; }
        char buf[4096];
        while (std::fgets(buf, sizeof buf, f)) {
            std::string line(buf);
            std::replace(line.begin(), line.end(), '=', ' ');
            auto t = tokens(line);
            if (t.empty() || t[0][0] == '#' || t.size() < 2) continue;
            apply_parameter(p, t[0], t[1]);
        }
        std::fclose(f);
    }
    if (extra && *extra) return params_read_string(p, extra);
    return YAMC_OK;
}

namespace yamc {

// ---------------------------------------------------------------- Functions.f90

// erfc_Luc (Functions.f90:116-142): Taylor series below 0.455, Abramowitz &
// Stegun 7.1.26 up to 3, asymptotic series above.
double erfc_luc(double x, double x2, double ee2) {
    const double P = 0.3275911, A1 = 0.254829592, A2 = -0.284496736, A3 = 1.421413741,
                 A4 = -1.453152027, A5 = 1.061405429, pi05 = 1.7724538509055;
    if (x < 0.455) return 1.0 - 2.0 / pi05 * x * (1.0 - x2 * (1.0 / 3.0 - x2 * (0.1 - x2 * (1.0 / 42.0 - x2 / 216.0))));
    if (x > 3.0) return (1.0 - 0.5 * (1.0 - 1.5 / x2) / x2) / (pi05 * x) * ee2;
    double t = 1.0 / (1.0 + P * x);
    return t * (A1 + t * (A2 + t * (A3 + t * (A4 + t * A5)))) * ee2;
}

// erf_Luc (Functions.f90:145-171)
double erf_luc(double x, double x2, double ee2) {
    const double P = 0.3275911, A1 = 0.254829592, A2 = -0.284496736, A3 = 1.421413741,
                 A4 = -1.453152027, A5 = 1.061405429, pi05 = 1.7724538509055;
    if (x < 0.455) return 2.0 / pi05 * x * (1.0 - x2 * (1.0 / 3.0 - x2 * (0.1 - x2 * (1.0 / 42.0 - x2 / 216.0))));
    if (x > 3.0) return 1.0 - (1.0 - 0.5 * (1.0 - 1.5 / x2) / x2) / (pi05 * x) * ee2;
    double t = 1.0 / (1.0 + P * x);
    return 1.0 - t * (A1 + t * (A2 + t * (A3 + t * (A4 + t * A5)))) * ee2;
}

// erfc_Luc_bet6_bet12 (Functions.f90:26-111): closed forms for b <= 0.5,
// asymptotic forms for b >= 8, trapezoid integration in between.
void erfc_luc_bet6_bet12(double x, double x2, double e2, double *erfk, double *bet6, double *bet12) {
    const double pi = 4.0 * std::atan(1.0);
    const double pi12 = std::sqrt(pi);
    const double pi15 = std::pow(pi, 1.5);
    if (x <= 0.5) {
        double ek = erfc_luc(x, x2, e2);
        *erfk = ek;
        *bet6 = pi15 / 3.0 * powi(x, 3) * (pi12 * ek + (0.5 / x2 - 1.0) / x * e2);
        double poly = ((((1.0 / x2 - 2.0 / 7.0) / x2 + 4.0 / 35.0) / x2 - 8.0 / 105.0) / x2 + 16.0 / 105.0);
        *bet12 = pi15 / 1080.0 * powi(x, 9) * (-16.0 * pi12 / 105.0 * ek + poly / x * e2);
        return;
    }
    if (x >= 8.0) {
        *erfk = e2 / pi12 / x * (1.0 - 0.5 / x2 * (1.0 - 1.5 / x2 * (1.0 - 2.5 / x2)));
        *bet6 = pi15 * e2 / 4.0 / powi(x, 2) * (1.0 - 2.5 / x2 * (1.0 - 3.5 / x2 * (1.0 - 4.5 / x2)));
        *bet12 = pi15 * e2 / 240.0 / powi(x, 2) * (1.0 - 5.5 / x2 * (1.0 - 6.5 / x2 * (1.0 - 7.5 / x2)));
        return;
    }
    const double xmax = 8.0;
    double dx = 1.0e-3;
    const int n = (int)((xmax - x) / dx + 2);
    dx = (xmax - x) / (n - 1);
    double s0 = dx * e2 / 2.0 - dx * dx / 12.0 * 2.0 * x * e2;
    double s6 = dx * e2 / powi(x, 4) / 2.0 - dx * dx / 12.0 * (2.0 / powi(x, 3) + 4.0 / powi(x, 5)) * e2;
    double s12 = dx * e2 / powi(x, 10) / 2.0 - dx * dx / 12.0 * (2.0 / powi(x, 9) + 10.0 / powi(x, 11)) * e2;
    double y = x, e = e2;
    for (int i = 2; i <= n; ++i) {
        y = x + (double)(i - 1) * dx;
        e = std::exp(-(y * y));
        s0 = s0 + dx * e;
        s6 = s6 + dx * e / powi(y, 4);
        s12 = s12 + dx * e / powi(y, 10);
    }
    const double y2 = y * y;
    s0 = s0 - dx * e / 2.0 + dx * dx / 12.0 * 2.0 * y * e;
    s0 = s0 + e / 2.0 / y * (1.0 - 0.5 / y2 * (1.0 - 1.5 / y2 * (1.0 - 2.5 / y2)));
    *erfk = 2.0 / pi12 * s0;
    s6 = s6 - dx * e / powi(y, 4) / 2.0 + dx * dx / 12.0 * (2.0 / powi(y, 3) + 4.0 / powi(y, 5)) * e;
    s6 = s6 + e / 2.0 / powi(y, 5) * (1.0 - 2.5 / y2 * (1.0 - 3.5 / y2 * (1.0 - 4.5 / y2)));
    *bet6 = pi15 * powi(x, 3) / 2.0 * s6;
    s12 = s12 - dx * e / powi(y, 10) / 2.0 + dx * dx / 12.0 * (2.0 / powi(y, 9) + 10.0 / powi(y, 11)) * e;
    s12 = s12 + e / 2.0 / powi(y, 11) * (1.0 - 5.5 / y2 * (1.0 - 6.5 / y2 * (1.0 - 7.5 / y2)));
    *bet12 = pi15 * powi(x, 9) / 120.0 * s12;
}

// FourierGrid_calcNalloc (FourierGrid.f90:37-78)
int grid_count(int kmax) {
    const double km2 = (double)(kmax * kmax);
    int n = 0;
    for (int kx = 0; kx <= kmax; ++kx) {
        const int kymax = (int)std::sqrt(km2 - (double)(kx * kx));
        for (int ky = 0; ky <= kymax; ++ky) {
            const int kzmax = (int)std::sqrt(km2 - (double)(kx * kx) - (double)(ky * ky));
            for (int kz = 0; kz <= kzmax; ++kz)
                if ((double)(kx * kx) + (double)(ky * ky) + (double)(kz * kz) >= 0.1) ++n;
        }
    }
    return n;
}

// ---------------------------------------------------------------- box-dependent tables

// LJTypes_fill_LJ_tab (LJTypes.f90:273-308) with LJTypes_fill_LJ_tab_index (:202-232):
// Lorentz-Berthelot tables from the type list (type_sigma in box units, type_eps in kT)
void fill_lj_tables(HostSystem &H) {
    const int nt = H.nt, n2 = std::max(1, nt * nt);
    H.lj6.assign(n2, 0); H.lj12.assign(n2, 0); H.four_eps.assign(n2, 0); H.sigma6.assign(n2, 0); H.sigma2.assign(n2, 0);
    auto fill = [&](int i, int j, double s12, double e12) {
        const double s2 = s12 * s12, s6 = s2 * s2 * s2;
        for (int pass = 0; pass < (i == j ? 1 : 2); ++pass) {
            const int o = pass == 0 ? (i - 1) * nt + (j - 1) : (j - 1) * nt + (i - 1);
            H.lj6[o] = 4 * e12 * s6;
            H.lj12[o] = H.lj6[o] * s6;
            H.sigma2[o] = s2; H.sigma6[o] = s6; H.four_eps[o] = 4 * e12;
        }
    };
    const std::vector<double> &ts = H.type_sigma, &te = H.type_eps;
    for (int i = 1; i <= nt; ++i) {
        fill(i, i, ts[i - 1], te[i - 1]);
        for (int j = i + 1; j <= nt; ++j) fill(i, j, (ts[i - 1] + ts[j - 1]) / 2, std::sqrt(te[i - 1] * te[j - 1]));
    }
}

// EwaldSumKSpace_initBetaLJ (EwaldSumKSpace.f90:352-386), one row per t1 <= t2, per signed entry
void fill_beta_lj(HostSystem &H) {
    const int nt = H.nt;
    H.ebetalj.assign((size_t)std::max(1, H.npair) * H.S, 0.0);
    for (int t1 = 1; t1 <= nt; ++t1)
        for (int t2 = t1; t2 <= nt; ++t2) {
            const int o = (t1 - 1) * nt + (t2 - 1), pidx = H.pair_index[o];
            for (int e = 0; e < H.S; ++e) {
                const int k = H.ekk[e];
                H.ebetalj[(size_t)pidx * H.S + e] = H.lj12[o] * H.beta12[k] - H.lj6[o] * H.beta6[k];
            }
        }
}

// ewald_sum_coulomb_tail / ewald_sum_lj_tails (EwaldSumTails.f90:18-127); molecule counts
// are read by LJ type (EwaldSumTails.f90:88)
void compute_tails(HostSystem &H) {
    const yamc_params &p = H.p;
    const int N = H.N, nt = H.nt;
    const double alpha = p.alpha;
    double sq = 0;
    for (int i = 0; i < N; ++i) sq = sq + H.q[i] * H.q[i];
    H.U_tail_coul = -(p.xclb * p.alpha_over_sqrt_pi * sq);
    const double a3 = powi(alpha, 3), a6 = a3 * a3, a9 = a3 * a6, a12 = a6 * a6;
    const double pisp = std::pow(kPi, 1.5);
    double sij6 = 0, sij12 = 0, sj6 = 0, sj12 = 0;
    for (int t1 = 1; t1 <= nt; ++t1)
        for (int t2 = t1; t2 <= nt; ++t2) {
            const int o = (t1 - 1) * nt + (t2 - 1);
            const int n1n2 = H.mol_numbers[t1 - 1] * H.mol_numbers[t2 - 1];
            double l6 = H.lj6[o] * n1n2, l12 = H.lj12[o] * n1n2;
            if (t1 != t2) { l6 = l6 + l6; l12 = l12 + l12; }
            sij6 = sij6 + l6; sij12 = sij12 + l12;
        }
    for (int t = 1; t <= nt; ++t) {
        const int o = (t - 1) * nt + (t - 1);
        sj6 = sj6 + H.lj6[o] * H.mol_numbers[t - 1];
        sj12 = sj12 + H.lj12[o] * H.mol_numbers[t - 1];
    }
    H.U_tail_lj6 = pisp * a3 / 6.0 * sij6 - a6 / 12.0 * sj6;
    H.U_tail_lj12 = pisp * a9 / 1080.0 * sij12 - a12 / 1440.0 * sj12;

}

// ---------------------------------------------------------------- system set-up

int prepare_host_system(const yamc_system *sys, const yamc_params *pin, HostSystem *hs) {
    if (!sys || !pin || !hs) return YAMC_EPARAMETER;
    HostSystem &H = *hs;
    H.p = *pin;
    const yamc_params &p = H.p;
    if (!(p.BoxLength > 0) || !(p.alpha > 0) || p.kmax < 1) {
        set_error("parameters not initialised (call yamc_params_init/recalc)");
        return YAMC_EINIT;
    }
    const int N = sys->natom, M = sys->nmol;
    if (N <= 0 || M <= 0 || !sys->x || !sys->y || !sys->z || !sys->charge || !sys->sigma || !sys->epsilon ||
        !sys->hard_core_angstr || !sys->mass || !sys->first_atom || !sys->last_atom) {
        set_error("incomplete yamc_system");
        return YAMC_EPARAMETER;
    }
    for (int i = 0; i < N; ++i) {
        const double v[8] = {sys->x[i], sys->y[i], sys->z[i], sys->charge[i], sys->sigma[i], sys->epsilon[i],
                             sys->hard_core_angstr[i], sys->mass[i]};
        for (double x : v)
            if (!std::isfinite(x)) {
                set_error("non-finite input of atom " + std::to_string(i + 1));
                return YAMC_ENAN;
            }
    }
    H.N = N; H.M = M;
    H.x.assign(sys->x, sys->x + N); H.y.assign(sys->y, sys->y + N); H.z.assign(sys->z, sys->z + N);
    H.q.assign(sys->charge, sys->charge + N); H.sigma.assign(sys->sigma, sys->sigma + N);
    H.eps.assign(sys->epsilon, sys->epsilon + N); H.hc.assign(sys->hard_core_angstr, sys->hard_core_angstr + N);
    H.mass.assign(sys->mass, sys->mass + N);
    H.dhs.resize(N);
    for (int i = 0; i < N; ++i) H.dhs[i] = H.hc[i] / p.BoxLength;  // d_HS (EwaldSumRealSpace.f90:378)
    H.first.resize(M); H.natoms.resize(M); H.molnum.assign(N, -1);
    H.max_mol_atoms = 0;
    for (int m = 0; m < M; ++m) {
        const int f = sys->first_atom[m] - 1, l = sys->last_atom[m] - 1;
        if (f < 0 || l < f || l >= N) { set_error("bad molecule atom range"); return YAMC_EPARAMETER; }
        if (l - f + 1 > kMaxMolAtoms) { set_error("molecules above 4 atoms are not supported on the device"); return YAMC_ELIMITS; }
        H.first[m] = f; H.natoms[m] = l - f + 1;
        H.max_mol_atoms = std::max(H.max_mol_atoms, l - f + 1);
        for (int a = f; a <= l; ++a) H.molnum[a] = m;
        double tm = 0;
        for (int a = f; a <= l; ++a) tm += H.mass[a];
        if (!(tm > 0)) { set_error("molecule with zero total mass"); return YAMC_EPARAMETER; }
    }
    for (int i = 0; i < N; ++i)
        if (H.molnum[i] < 0) { set_error("atom outside every molecule"); return YAMC_EPARAMETER; }

    // runs of consecutive molecules whose atoms carry identical static data (species)
    auto same_mol = [&](int a, int b) {
        if (H.natoms[a] != H.natoms[b]) return false;
        for (int k = 0; k < H.natoms[a]; ++k) {
            const int i = H.first[a] + k, j = H.first[b] + k;
            if (H.q[i] != H.q[j] || H.sigma[i] != H.sigma[j] || H.eps[i] != H.eps[j] || H.hc[i] != H.hc[j] ||
                H.mass[i] != H.mass[j])
                return false;
        }
        return true;
    };
    H.spec.clear();
    for (int m = 0; m < M; ++m) {
        const bool contiguous = m > 0 && H.first[m] == H.first[m - 1] + H.natoms[m - 1];
        if (m > 0 && contiguous && same_mol(m, H.spec[H.spec.size() - 4])) { H.spec[H.spec.size() - 3] += 1; continue; }
        H.spec.push_back(m); H.spec.push_back(1); H.spec.push_back(H.natoms[m]); H.spec.push_back(H.first[m]);
    }

    // LJTypes_fill (LJTypes.f90:134-200): distinct (sigma, epsilon) pairs in order
    // of first appearance, sigma below 1e-8 (single-precision literal) has no LJ.
    std::vector<double> ts, te;
    for (int i = 0; i < N; ++i) {
        if (H.sigma[i] < (double)1e-8f) continue;
        bool found = false;
        for (size_t t = 0; t < ts.size(); ++t)
            if (std::fabs(H.sigma[i] - ts[t]) < 1e-8 && std::fabs(H.eps[i] - te[t]) < 1e-8) { found = true; break; }
        if (!found) {
            if ((int)ts.size() >= kMaxLJTypes) { set_error("more than 20 LJ types"); return YAMC_ELIMITS; }
            ts.push_back(H.sigma[i]); te.push_back(H.eps[i]);
        }
    }
    const int nt = (int)ts.size();
    H.nt = nt;
    H.type_sigma = ts; H.type_eps = te;
    H.type_by_index.assign(N, 0);
    for (int i = 0; i < N; ++i)
        for (int t = 0; t < nt; ++t)
            if (std::fabs(H.sigma[i] - ts[t]) < 1e-8 && std::fabs(H.eps[i] - te[t]) < 1e-8) { H.type_by_index[i] = t + 1; break; }
    fill_lj_tables(H);
    const int n2 = std::max(1, nt * nt);
    H.pair_index.assign(n2, 0);
    H.npair = nt * (nt + 1) / 2;
    for (int t1 = 1, pidx = 0; t1 <= nt; ++t1)
        for (int t2 = t1; t2 <= nt; ++t2, ++pidx) {
            H.pair_index[(t1 - 1) * nt + (t2 - 1)] = pidx;
            H.pair_index[(t2 - 1) * nt + (t1 - 1)] = pidx;
        }

    // FourierGrid_init (FourierGrid.f90:118-189)
    H.kmax = p.kmax;
    const double km2 = (double)(p.kmax * p.kmax);
    for (int kx = 0; kx <= p.kmax; ++kx) {
        const double xkx2 = (double)(kx * kx);
        const int kymax = (int)std::sqrt(km2 - xkx2);
        for (int ky = 0; ky <= kymax; ++ky) {
            const double xky2 = (double)(ky * ky);
            const int kzmax = (int)std::sqrt(km2 - xkx2 - xky2);
            for (int kz = 0; kz <= kzmax; ++kz) {
                if (xkx2 + xky2 + (double)(kz * kz) < 0.1) continue;
                H.kx.push_back(kx); H.ky.push_back(ky); H.kz.push_back(kz);
            }
        }
    }
    H.nk = (int)H.kx.size();
    // EwaldSumKSpace_initBeta (EwaldSumKSpace.f90:263-350)
    H.beta.resize(H.nk); H.beta6.resize(H.nk); H.beta12.resize(H.nk);
    const double alpha = p.alpha;
    const double poa = kPi / alpha, poa2 = poa * poa;
    for (int k = 0; k < H.nk; ++k) {
        const double xk2 = (double)(H.kx[k] * H.kx[k]) + (double)(H.ky[k] * H.ky[k]) + (double)(H.kz[k] * H.kz[k]);
        const double b2 = poa2 * xk2;
        const double e = std::exp(-b2);
        H.beta[k] = p.xclb * e / xk2 / kTwoPi;
        double erfcb, B6, B12;
        erfc_luc_bet6_bet12(poa * std::sqrt(xk2), b2, e, &erfcb, &B6, &B12);
        H.beta6[k] = powi(alpha, 3) * B6;
        H.beta12[k] = powi(alpha, 9) * B12;
        if (H.kx[k] > 0) { H.beta[k] *= 2.0; H.beta6[k] *= 2.0; H.beta12[k] *= 2.0; }
    }
    // signed list: (+,+,+) always, (+,-,+) if ky>0, (+,+,-) if kz>0, (+,-,-) if both
    // (the zero-padded sign arrays of SumSinCosKR.f90:396-427, compacted)
    for (int k = 0; k < H.nk; ++k) {
        const int sy_max = H.ky[k] > 0 ? 2 : 1, sz_max = H.kz[k] > 0 ? 2 : 1;
        for (int a = 0; a < sy_max; ++a)
            for (int b = 0; b < sz_max; ++b) {
                H.ekx.push_back(H.kx[k]);
                H.eky.push_back(a ? -H.ky[k] : H.ky[k]);
                H.ekz.push_back(b ? -H.kz[k] : H.kz[k]);
                H.ekk.push_back(k);
            }
    }
    H.S = (int)H.ekk.size();
    H.ebeta.resize(H.S);
    for (int e = 0; e < H.S; ++e) H.ebeta[e] = H.beta[H.ekk[e]];
    fill_beta_lj(H);

    // EwaldSumTails (EwaldSumTails.f90:18-127); molecule counts are read by LJ type
    H.mol_numbers.assign(sys->mol_numbers, sys->mol_numbers + std::max(0, sys->n_species));
    if (nt > (int)H.mol_numbers.size()) {
        set_error("the LJ tails need mol_numbers for every LJ type (EwaldSumTails.f90:88)");
        return YAMC_EPARAMETER;
    }
    compute_tails(H);

    // BiasedRandom_init (BiasedRandom.f90:44-79) on the move weights (init_freq)
    std::vector<double> w(M, 1.0);
    if (sys->move_weights) w.assign(sys->move_weights, sys->move_weights + M);
    double S = 0;
    for (int i = 0; i < M; ++i) S = S + w[i];
    std::vector<double> prob(M);
    for (int i = 0; i < M; ++i) prob[i] = (S == 0) ? 1.0 / M : w[i] / S;
    H.freq_beg.resize(M); H.freq_end.resize(M);
    H.smv = S;
    H.freq_beg[0] = 0.0; H.freq_end[0] = prob[0];
    for (int i = 1; i < M; ++i) { H.freq_beg[i] = H.freq_end[i - 1]; H.freq_end[i] = H.freq_beg[i] + prob[i]; }
    if (S > 0)
        for (int i = 0; i < M; ++i) if (w[i] == 0) H.freq_end[i] = -1.0;
    H.freq_monotone = 1;
    for (int i = 1; i < M; ++i) if (!(H.freq_end[i] >= H.freq_end[i - 1]) || H.freq_end[i] < 0) H.freq_monotone = 0;
    if (H.freq_end[0] < 0) H.freq_monotone = 0;
    return YAMC_OK;
}

}  // namespace yamc
