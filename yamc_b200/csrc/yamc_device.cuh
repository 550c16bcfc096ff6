// Device-side building blocks of the engine: the pair kernel of the real-space
// Ewald sum, the k-space phase factors, the random stream consumer and the
// move proposal / Metropolis test.  The proposal and acceptance code is
// __host__ __device__ so the host-driven per-move API and the device-resident
// chain draw identical proposals from the same stream.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace yamc {

constexpr int kMaxA = 4;  // atoms per molecule handled on the device
constexpr int kMaxDevTypes = 8;  // LJ types the device tables hold (the kernels take 1..4)

// ------------------------------------------------------------------ system view
struct DevSys {
    int N, M, S, nt, kmax, npair, freq_monotone, n_species;
    double rmax2, alpha, xclb, taosp, kext, m2k, dr, d_angle, xlf, xlc, psm, n_store_energy_interval;
    double rpre;           // max(cutoff, largest hard-core diameter), box units: the pair filter's reach
    double dhs_t[kMaxDevTypes + 1];  // hard-core diameter / L by LJ type (dhs_typed: one value per type)
    int dhs_typed;
    double xprob;          // probability of an exchange step (the chain stops before one; 0 = none)
    long long refresh_every;  // mixed form: FP64 recomputation of rho(k) every this many accepted moves (0 = never)
    double4 *atom;         // x, y, z (box units), q
    const int2 *meta;      // 0-based molecule, LJ type (0 = none)
    const double *dhs;     // hard-core diameter / BoxLength
    const double *mass;    // per atom
    const int2 *mol;       // first atom (0-based), atoms in molecule
    const int4 *kvec;      // kx, signed ky, signed kz, half-space index
    const int *kpack;      // the same k in one word, kx | (ky + 128) << 8 | (kz + 128) << 16 (streamed sweeps)
    const double *ebeta;   // Coulomb beta per signed entry (2x for kx>0 folded in)
    const double *ebetalj; // npair x S
    const float *ebeta_f, *ebetalj_f;  // FP32 copies of ebeta and ebetalj (the mixed form's k-space reads)
    const int *pair_index; // nt*nt -> pair row
    const double *lj_sig6, *lj_feps;  // nt*nt tables (offset (t1-1)*nt + t2-1)
    double2 *rho;          // (1+nt) x S: Coulomb then one row per LJ type
    float2 *rho_f;         // the mixed form's FP32 copy of rho, read by its streamed sweeps: written from rho
                           // before every chain launch (k_stage_order), kept with rho by the chain's commits
    double2 *scratch;      // 2 x (1+nt) x S: the moved molecule's old phase sums, then the rho deltas (FP32 pairs in the mixed form)
    const double *freq_beg, *freq_end;
    double *scal;          // engine scalars, see Scal
    long long *cnt;        // run_mc counters, see Cnt
    int nspec;             // runs of identical consecutive molecules (molecule species)
    const int4 *spec;      // first molecule, count, atoms per molecule, first atom (0-based)
    // the chain kernel's spatial staging: slot[j] = the shared-memory slot of atom j in its CTA
    // (j % G), atom_of[r * nown_max + s] = the atom in slot s of CTA r (written at launch start)
    int *slot, *atom_of;
    int *check;            // bounds-checked builds: source line of the first index found out of bounds (0 = none)
};

// Bounds-checked builds (-DYAMC_CHECKED, libyamc_b200_checked.so): YAMC_IX(i, n) checks every
// index the chain kernel computes into its atom, staging, k-entry, scratch, pair-queue, near-atom
// and table arrays.  An index outside [0, n) records the source line in *D.check (the first one
// wins) and is replaced by 0, so the access stays inside the array: no trap, no fault; the host
// returns YAMC_EBOUNDS after the launch.  In normal builds YAMC_IX(i, n) is i.
__device__ __forceinline__ long long checked_ix(long long i, long long n, int line, int *check) {
    if (i >= 0 && i < n) return i;
    if (check) atomicCAS(check, 0, line);
    return 0;
}
#ifdef YAMC_CHECKED
#define YAMC_IX(i, n) ::yamc::checked_ix((long long)(i), (long long)(n), __LINE__, D.check)
#else
#define YAMC_IX(i, n) (i)
#endif

// engine scalars (double)
enum Scal {
    SC_UU_EW = 0, SC_UU_LJ6, SC_UU_LJ12, SC_EK_C, SC_EK_LJ, SC_MU_X, SC_MU_Y, SC_MU_Z,
    SC_TAIL_C, SC_TAIL_LJ6, SC_TAIL_LJ12, SC_UU_EW_INTRA, SC_UU_LJ6_INTRA, SC_UU_LJ12_INTRA,
    SC_N_MV_STEPS, SC_N_MV_ACC, SC_N_VOL_STEPS, SC_COUNT
};
// run_mc counters (int64)
enum Cnt { CN_ICYCLE = 0, CN_MOVE_IN_CYCLE, CN_ACC_SINCE_REFRESH, CN_REFRESHES, CN_COUNT };

// ------------------------------------------------------------------ arithmetic helpers
// 1/y rounded to nearest (the same value as the IEEE division 1/y) and 1/sqrt(y) (within an
// ulp).  The pair kernel multiplies by these instead of dividing: a floating-point division is a
// long instruction sequence, and the pair term has a dozen of them.  Replacing x / c by
// x * (1/c) changes a result by at most an ulp or two, far inside the 1e-10 parity bound.
template <class R>
__host__ __device__ inline R rcp(R y) {
#ifdef __CUDA_ARCH__
    if constexpr (sizeof(R) == 8) return __drcp_rn(y);
    else return __frcp_rn(y);
#else
    return R(1) / y;
#endif
}
template <class R>
__host__ __device__ inline R rsq(R y) {
#ifdef __CUDA_ARCH__
    if constexpr (sizeof(R) == 8) return rsqrt(y);
    else return rsqrtf(y);
#else
    return R(1) / std::sqrt(y);
#endif
}

// ------------------------------------------------------------------ Functions.f90
// erfc_Luc / erf_Luc (Functions.f90:116-171): Taylor series below 0.455,
// Abramowitz & Stegun 7.1.26 up to 3, asymptotic series above (divisions by
// multiplications with reciprocals, see rcp above).
template <class R>
__host__ __device__ inline R d_erfc_luc(R x, R x2, R ee2) {
    const R P = R(0.3275911), A1 = R(0.254829592), A2 = R(-0.284496736), A3 = R(1.421413741),
            A4 = R(-1.453152027), A5 = R(1.061405429), pi05 = R(1.7724538509055);
    if (x < R(0.455)) return R(1) - R(2) / pi05 * x * (R(1) - x2 * (R(1) / R(3) - x2 * (R(0.1) - x2 * (R(1) / R(42) - x2 * (R(1) / R(216))))));
    if (x > R(3)) {
        const R i2 = rcp(x2);
        return (R(1) - R(0.5) * (R(1) - R(1.5) * i2) * i2) * rcp(pi05 * x) * ee2;
    }
    const R t = rcp(R(1) + P * x);
    return t * (A1 + t * (A2 + t * (A3 + t * (A4 + t * A5)))) * ee2;
}
template <class R>
__host__ __device__ inline R d_erf_luc(R x, R x2, R ee2) {
    const R P = R(0.3275911), A1 = R(0.254829592), A2 = R(-0.284496736), A3 = R(1.421413741),
            A4 = R(-1.453152027), A5 = R(1.061405429), pi05 = R(1.7724538509055);
    if (x < R(0.455)) return R(2) / pi05 * x * (R(1) - x2 * (R(1) / R(3) - x2 * (R(0.1) - x2 * (R(1) / R(42) - x2 * (R(1) / R(216))))));
    if (x > R(3)) {
        const R i2 = rcp(x2);
        return R(1) - (R(1) - R(0.5) * (R(1) - R(1.5) * i2) * i2) * rcp(pi05 * x) * ee2;
    }
    const R t = rcp(R(1) + P * x);
    return R(1) - t * (A1 + t * (A2 + t * (A3 + t * (A4 + t * A5)))) * ee2;
}

// d erfc_Luc(x) / dx of the piecewise function above, piece by piece: the adjoint of the
// energy as implemented (the reference's own forces use the exact erfc derivative instead,
// RealSumLocal.f90:104).  erf_Luc = 1 - erfc_Luc on every piece, so -erf_Luc has the same
// derivative.
template <class R>
__host__ __device__ inline R d_erfc_luc_deriv(R x, R x2, R ee2) {
    const R P = R(0.3275911), A1 = R(0.254829592), A2 = R(-0.284496736), A3 = R(1.421413741),
            A4 = R(-1.453152027), A5 = R(1.061405429), pi05 = R(1.7724538509055);
    if (x < R(0.455))  // 1 - (2/sqrt(pi)) (x - x^3/3 + x^5/10 - x^7/42 + x^9/216)
        return -(R(2) / pi05) * (R(1) - x2 * (R(1) - x2 * (R(0.5) - x2 * (R(1) / R(6) - x2 * (R(1) / R(24))))));
    if (x > R(3)) {    // (x^-1 - 0.5 x^-3 + 0.75 x^-5) e^{-x^2} / sqrt(pi)
        const R i1 = rcp(x), i2 = i1 * i1;
        const R h = i1 * (R(1) - i2 * (R(0.5) - R(0.75) * i2));
        const R dh = -i2 * (R(1) - i2 * (R(1.5) - R(3.75) * i2));
        return (dh - R(2) * x * h) * ee2 * (R(1) / pi05);
    }
    const R t = rcp(R(1) + P * x);  // t A(t) e^{-x^2}, dt/dx = -P t^2
    const R A = A1 + t * (A2 + t * (A3 + t * (A4 + t * A5)));
    const R dA = A2 + t * (R(2) * A3 + t * (R(3) * A4 + t * (R(4) * A5)));
    return ((-P * t * t) * (A + t * dA) - R(2) * x * t * A) * ee2;
}

// Radial force factor of the implemented pair energy (F_i += FR (r_i - r_j)): the Coulomb part
// differentiates qq f(alpha r)/r with f = erfc_Luc (or -erf_Luc inside a molecule), the LJ part
// is the exact derivative of the dispersion-Ewald terms (the same as the reference's).
template <class R>
__host__ __device__ inline R pair_force_adjoint(R r2, R qq_xclb, bool lj, R sigma6, R four_eps, R alpha, bool same_mol) {
    const R ir = rsq(r2);
    const R r = r2 * ir;
    const R ir2 = ir * ir;
    const R a = alpha * r;
    const R a2 = a * a;
    const R e2 = exp(-a2);
    const R f = same_mol ? -d_erf_luc<R>(a, a2, e2) : d_erfc_luc<R>(a, a2, e2);
    const R df = d_erfc_luc_deriv<R>(a, a2, e2);
    R FR = qq_xclb * (f * ir - alpha * df) * ir2;
    if (lj) {
        const R so6 = sigma6 * (ir2 * ir2 * ir2);
        const R C6 = R(1) + a2 * (R(1) + a2 * R(0.5));
        const R a6 = a2 * a2 * a2;
        const R C12 = C6 + a6 * (R(1) + a2 * (R(1) + a2 * (R(1) / R(5))) * R(0.25)) * (R(1) / R(6));
        FR = FR + four_eps * R(6) * so6 * e2 * (R(2) * so6 * (C12 + a6 * a6 * (R(1) / R(720))) - (C6 + a6 * (R(1) / R(6)))) * ir2;
    }
    return FR;
}

// shi_sans_exp_f (Functions.f90:225-289): Shi(x) exp(-x), force-bias acceptance
__host__ __device__ inline double d_shi_sans_exp(double x) {
    const double dx0 = 0.2;
    double shi_f, x1;
    if (x <= 1.0) {
        const double x2 = x * x;
        double fac = 1.0, xn = x;
        shi_f = x;
        for (int i = 1; i <= 4; ++i) {
            const double di = 2.0 * i;
            xn = xn * x2;
            fac = fac * di * (di + 1.0);
            shi_f = shi_f + xn / (di + 1.0) / fac;
        }
        return exp(-x) * shi_f;
    }
    if (x > 20.0) {
        double som = 1.0, term = 1.0;
        for (int i = 1; i <= 6; ++i) { term = term * i / x; som = som + term; }
        return 1.0 / 2.0 / x * som;
    }
    if (x < 5.0) { x1 = 1.0; shi_f = 1.057250875; }
    else if (x < 10.0) { x1 = 5.0; shi_f = 20.093211826; }
    else if (x < 15.0) { x1 = 10.0; shi_f = 1246.11449; }
    else { x1 = 15.0; shi_f = 117477.926; }
    const int n = (int)((x - x1) / dx0 + 2);
    const double dx = (x - x1) / (n - 1);
    shi_f = shi_f + dx * sinh(x1) / x1 / 2.0 + dx * dx / 12.0 * (cosh(x1) / x1 - sinh(x1) / (x1 * x1));
    double t = x1, s = 0.0;
    for (int i = 2; i <= n; ++i) {
        t = x1 + (double)(i - 1) * dx;
        s = sinh(t);
        shi_f = shi_f + dx * s / t;
    }
    shi_f = shi_f - dx * s / t / 2.0 - dx * dx / 12.0 * (cosh(t) / t - s / (t * t));
    return exp(-x) * shi_f;
}

// ------------------------------------------------------------------ pair term
// RealSumLocal (RealSumLocal.f90:63-168): one pair of the real-space sum.
// ew = xclb qi qj erfc_Luc(a)/r (or -erf_Luc for an intra-molecular pair),
// lj6/lj12 the dispersion-Ewald LJ terms, FR the radial force factor
// (F_i += FR * (r_i - r_j)).
template <class R>
struct PairTerm { R ew, lj6, lj12, FR; };

template <class R, bool WANT_FR>
__host__ __device__ inline PairTerm<R> pair_term(R r2, R qq_xclb, bool lj, R sigma6, R four_eps, R alpha,
                                                 R taosp, bool same_mol) {
    PairTerm<R> t;
    const R ir = rsq(r2);       // 1/r
    const R r = r2 * ir;
    const R ir2 = ir * ir;      // 1/r^2
    const R a = alpha * r;
    const R a2 = a * a;
    const R e2 = exp(-a2);
    const R erfc_a = same_mol ? -d_erf_luc<R>(a, a2, e2) : d_erfc_luc<R>(a, a2, e2);
    t.ew = qq_xclb * erfc_a * ir;
    if (WANT_FR) t.FR = qq_xclb * (erfc_a * ir + taosp * e2) * ir2;
    else t.FR = R(0);
    t.lj6 = R(0); t.lj12 = R(0);
    if (lj) {
        const R so6 = sigma6 * (ir2 * ir2 * ir2);
        const R C6 = R(1) + a2 * (R(1) + a2 * R(0.5));
        const R a6 = a2 * a2 * a2;
        const R C12 = C6 + a6 * (R(1) + a2 * (R(1) + a2 * (R(1) / R(5))) * R(0.25)) * (R(1) / R(6));
        t.lj6 = four_eps * so6 * e2 * C6;
        t.lj12 = four_eps * (so6 * so6) * e2 * C12;
        if (WANT_FR)
            t.FR = t.FR + four_eps * R(6) * so6 * e2 *
                              (R(2) * so6 * (C12 + a6 * a6 * (R(1) / R(720))) - (C6 + a6 * (R(1) / R(6)))) * ir2;
    }
    return t;
}

// The mixed form's pair term: the one transcendental, exp(-alpha^2 r^2), in FP32 (its argument
// formed in FP64, so the FP32 rounding of alpha^2 r^2 costs at most an ulp of the argument);
// 1/r, the erfc_Luc polynomials and the products in FP64.  Rounding each pair term to FP32, or
// the A&S polynomial in FP32, would put the per-move dE error above 1e-4 kT.
template <bool WANT_FR>
__device__ inline PairTerm<double> pair_term_mx(double r2, double qq_xclb, bool lj, double sigma6, double four_eps,
                                                double alpha, double taosp, bool same_mol) {
    PairTerm<double> t;
    const double ir = rsq(r2);
    const double r = r2 * ir;
    const double ir2 = ir * ir;
    const double a = alpha * r;
    const double a2 = a * a;
    const double e2 = (double)expf(-(float)a2);
    const double erfc_a = same_mol ? -d_erf_luc<double>(a, a2, e2) : d_erfc_luc<double>(a, a2, e2);
    t.ew = qq_xclb * erfc_a * ir;
    t.FR = WANT_FR ? qq_xclb * (erfc_a * ir + taosp * e2) * ir2 : 0.0;
    t.lj6 = 0.0; t.lj12 = 0.0;
    if (lj) {
        const double so6 = sigma6 * (ir2 * ir2 * ir2);
        const double C6 = 1.0 + a2 * (1.0 + a2 * 0.5);
        const double a6 = a2 * a2 * a2;
        const double C12 = C6 + a6 * (1.0 + a2 * (1.0 + a2 * (1.0 / 5.0)) * 0.25) * (1.0 / 6.0);
        t.lj6 = four_eps * so6 * e2 * C6;
        t.lj12 = four_eps * (so6 * so6) * e2 * C12;
        if (WANT_FR)
            t.FR = t.FR + four_eps * 6.0 * so6 * e2 * (2.0 * so6 * (C12 + a6 * a6 * (1.0 / 720.0)) - (C6 + a6 * (1.0 / 6.0))) * ir2;
    }
    return t;
}

// minimum image by one conditional wrap per axis (EwaldSumRealSpace.f90:394-401)
template <class R>
__host__ __device__ inline R min_image(R d) {
    if (d > R(0.5)) d = d - R(1);
    if (d < R(-0.5)) d = d + R(1);
    return d;
}

// ------------------------------------------------------------------ k-space phase
// q * (cos, sin)(2 pi (x kx + y ky + z kz)) for a signed entry from per-axis
// tables T[m] = (cos 2 pi m u, sin 2 pi m u), with SinCosKR_fill's arithmetic
// (SumSinCosKR.f90:362-448): q cos(X)cos(Y) -/+ q sin(X)sin(Y), then the z factor.
template <class R, class T2>
__host__ __device__ inline void entry_phase(const T2 *tx, const T2 *ty, const T2 *tz, int kx, int ky, int kz, R q,
                                            R &c, R &s) {
    const R cx = tx[kx].x, sx = tx[kx].y;
    const int aky = ky < 0 ? -ky : ky, akz = kz < 0 ? -kz : kz;
    const R cy = ty[aky].x, sy = ky < 0 ? -ty[aky].y : ty[aky].y;
    const R cz = tz[akz].x, sz = kz < 0 ? -tz[akz].y : tz[akz].y;
    const R qcc = q * cx * cy, qss = q * sx * sy, qsc = q * sx * cy, qcs = q * cx * sy;
    const R qc = qcc - qss, qs = qsc + qcs;
    const R c1 = qc * cz, s1 = qs * sz, s2 = qs * cz, c2 = qc * sz;
    c = c1 - s1;
    s = s2 + c2;
}

// ------------------------------------------------------------------ random stream
// rand() of random.f90:65-93: successive REAL(4) random_number values, values
// outside [1e-14, 1-1e-14] are drawn again.  The buffer holds the raw stream.
struct RngReader {
    const float *buf;  // holds stream positions [off, n)
    long long off;
    long long n;       // end of the stream available
    long long cur;     // next position to read
    int out;           // set once the stream ran out
    // optional copies of stream windows [b0, b0+n0) and [b1, b1+n1) (shared memory on the device)
    const float *w0 = nullptr;
    long long b0 = 0;
    int n0 = 0;
    const float *w1 = nullptr;
    long long b1 = 0;
    int n1 = 0;
    __host__ __device__ inline float raw() {
        if (cur >= n) { out = 1; return 0.5f; }
        const long long i = cur++;
        if (w0 && i >= b0 && i < b0 + n0) return w0[i - b0];
        if (w1 && i >= b1 && i < b1 + n1) return w1[i - b1];
        return buf[i - off];
    }
    __host__ __device__ inline double next() {
        const double eps = 1e-14;
        float v = 0.0f;
        while ((double)v < eps || (double)v > 1.0 - eps) {
            v = raw();
            if (out) return 0.5;
        }
        return (double)v;
    }
};

// BiasedRandom_choose (BiasedRandom.f90:81-109): first i with beg(i) < r < end(i),
// else 1.  The intervals are contiguous (beg(i) = end(i-1)) and increasing when
// every weight is positive, so a binary search gives the same answer.
__host__ __device__ inline int choose_molecule(double r, const double *beg, const double *end, int M, int monotone) {
    if (!monotone) {
        for (int i = 0; i < M; ++i)
            if (r > beg[i] && r < end[i]) return i + 1;
        return 1;
    }
    int lo = 0, hi = M - 1;  // smallest i with end[i] > r
    if (!(end[hi] > r)) return 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (end[mid] > r) hi = mid; else lo = mid + 1;
    }
    return (r > beg[lo]) ? lo + 1 : 1;
}

// Same answer with one round trip for flat weights: interval i holds (i, i+1)/M up to the
// rounding of the running sums, so start at floor(r M) and step to the interval whose exact
// boundaries bracket r; a value on a boundary belongs to no interval (answer 1), as in the
// reference's strict comparisons.
__host__ __device__ inline int choose_molecule_guess(double r, const double *beg, const double *end, int M, int monotone) {
    if (!monotone) return choose_molecule(r, beg, end, M, 0);
    int g = (int)(r * M);
    if (g > M - 1) g = M - 1;
    if (g < 0) g = 0;
    for (int step = 0; step < 6; ++step) {
        const double b = beg[g], e = end[g];
        if (r > b && r < e) return g + 1;
        if (r == b || r == e) return 1;
        if (r > e) { if (g == M - 1) return 1; ++g; }
        else { if (g == 0) return 1; --g; }
    }
    return choose_molecule(r, beg, end, M, monotone);
}

// ------------------------------------------------------------------ MonteCarloMove.f90
struct MoveState {
    double fxo, fyo, fzo, fo, cxo, cyo, czo, co, umaxold, vmaxold, cold, qold;
    double vx, vy, vz, deltx, delty, deltz, angle;
    double fxn, fyn, fzn, fn, cxn, cyn, czn, cn, umaxnew, vmaxnew, cnew, qnew;
    double cphi, sphi, ct, st, ca, sa;  // rotation (TRotation)
};

__host__ __device__ inline void cross(double x1, double y1, double z1, double x2, double y2, double z2, double &xp,
                                      double &yp, double &zp) {
    xp = y1 * z2 - z1 * y2;   // prod_vect (geometry.f90:65-101)
    yp = z1 * x2 - x1 * z2;
    zp = x1 * y2 - y1 * x2;
}

// MonteCarloMove_init_old (MonteCarloMove.f90:34-54)
__host__ __device__ inline void mcm_init_old(MoveState &m, const double f[3], const double t[3]) {
    m.fxo = f[0]; m.fyo = f[1]; m.fzo = f[2]; m.fo = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    m.cxo = t[0]; m.cyo = t[1]; m.czo = t[2]; m.co = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
}

// MonteCarloMove_init_new (MonteCarloMove.f90:56-106)
__host__ __device__ inline void mcm_init_new(MoveState &m, const double f[3], const double t[3], double xlf, double xlc,
                                             double dr, double d_angle) {
    m.fxn = f[0]; m.fyn = f[1]; m.fzn = f[2]; m.fn = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
    m.cxn = t[0]; m.cyn = t[1]; m.czn = t[2]; m.cn = sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]);
    double umax = xlf * m.fn * dr;
    if (umax > 1e-2) {
        const double e = exp(-2.0 * umax);
        const double t2 = (umax * (1.0 + e) - (1.0 - e)) / 2.0;
        m.cnew = 3.0 * t2 / (umax * umax * umax);
    } else { umax = 0.0; m.cnew = 1.0; }
    m.umaxnew = umax;
    double vmax = xlc * m.cn * d_angle;
    if (vmax > 1e-2) m.qnew = d_shi_sans_exp(vmax) / vmax;
    else { vmax = 0.0; m.qnew = 1.0; }
    m.vmaxnew = vmax;
}

// MonteCarloMove_chooseDisplacement (MonteCarloMove.f90:109-266): a ball of
// radius dr, or the force-biased distribution exp(lambda F.dr) when biased.
__host__ __device__ inline void mcm_choose_displacement(MoveState &m, RngReader &rng, double xlf, double dr) {
    double umax = xlf * m.fo * dr;
    if (umax > 1e-2) {
        double e = exp(-2.0 * umax);
        const double t = (umax * (1.0 + e) - (1.0 - e)) / 2.0;
        m.cold = 3.0 * t / (umax * umax * umax);
        double xksi = 0.0;
        while (xksi < 1e-10) { xksi = rng.next(); if (rng.out) return; }
        const double z = umax + log(xksi * t);
        double u;
        if (z <= log(4.0)) { const double s = exp(z); u = pow(3.0 * s, 1.0 / 3.0) - s / 10.0; }
        else u = z - log(z / 2.0);
        // Newton on h(u) = u + ln(u ch u - sh u) = z, 10 iterations, the last one only for e at the
        // final u.  Once an update leaves u unchanged every later iteration repeats the same
        // arithmetic on the same u, so the loop stops there with the same u and e bit for bit.
        for (int k = 1; k <= 10; ++k) {
            e = exp(-2.0 * u);
            const double ch = (1.0 + e) / 2.0;
            double sh = (1.0 - e) / 2.0;
            if (u < 1e-5) sh = u - u * u;
            double g = u * ch - sh;
            if (u < 1e-3) g = u * u * u / 3.0;
            const double h = u + log(g);
            const double h1 = u * sh / g;
            if (k < 10) {
                const double un = u + (z - h) / h1;
                if (un == u) break;
                u = un;
            }
        }
        const double deltar = u / (xlf * m.fo);
        xksi = 1.0;
        while (xksi > (1.0 - 1e-10) || xksi < 1e-10) { xksi = rng.next(); if (rng.out) return; }
        double xc = 1.0 + log(xksi + (1.0 - xksi) * e) / u;
        if (u < 1e-7) xc = 1.0 - 2.0 * (1.0 - xksi);
        if (xc > 1.0 - 1e-14) xc = 1.0 - 1e-14;
        if (xc < -1.0 + 1e-14) xc = -1.0 + 1e-14;
        const double xs = sqrt(1.0 - xc * xc);
        double w = -1.0, wx = 0, wy = 0, wz = 0;
        while (w <= 1e-10) {
            double v2 = 2.0, vx = 0, vy = 0, vz = 0;
            while (v2 > 1.0) {
                vx = 2.0 * rng.next() - 1.0; vy = 2.0 * rng.next() - 1.0; vz = 2.0 * rng.next() - 1.0;
                if (rng.out) return;
                v2 = vx * vx + vy * vy + vz * vz;
            }
            cross(vx, vy, vz, m.fxo, m.fyo, m.fzo, wx, wy, wz);
            w = sqrt(wx * wx + wy * wy + wz * wz);
        }
        m.deltx = deltar * (xc * m.fxo / m.fo + xs * wx / w);
        m.delty = deltar * (xc * m.fyo / m.fo + xs * wy / w);
        m.deltz = deltar * (xc * m.fzo / m.fo + xs * wz / w);
    } else {
        double v2 = 2.0, vx = 0, vy = 0, vz = 0;
        while (v2 > 1.0) {
            vx = 2.0 * rng.next() - 1.0; vy = 2.0 * rng.next() - 1.0; vz = 2.0 * rng.next() - 1.0;
            if (rng.out) return;
            v2 = vx * vx + vy * vy + vz * vz;
        }
        m.deltx = dr * vx; m.delty = dr * vy; m.deltz = dr * vz;
        umax = 0.0; m.cold = 1.0;
    }
    m.umaxold = umax;
}

// The random numbers MonteCarloMove_chooseDisplacement draws, without its arithmetic: its
// rejection loops alone (the force direction decides the w test), so the rotation, which draws
// next, can start on another thread while the displacement itself is computed.  Draws exactly
// what mcm_choose_displacement draws, in the same order.
__host__ __device__ inline void mcm_skip_displacement(const MoveState &m, RngReader &rng, double xlf, double dr) {
    const double umax = xlf * m.fo * dr;
    double v2, vx, vy, vz;
    if (umax > 1e-2) {
        double xksi = 0.0;
        while (xksi < 1e-10) { xksi = rng.next(); if (rng.out) return; }
        xksi = 1.0;
        while (xksi > (1.0 - 1e-10) || xksi < 1e-10) { xksi = rng.next(); if (rng.out) return; }
        double w = -1.0, wx, wy, wz;
        while (w <= 1e-10) {
            v2 = 2.0;
            while (v2 > 1.0) {
                vx = 2.0 * rng.next() - 1.0; vy = 2.0 * rng.next() - 1.0; vz = 2.0 * rng.next() - 1.0;
                if (rng.out) return;
                v2 = vx * vx + vy * vy + vz * vz;
            }
            cross(vx, vy, vz, m.fxo, m.fyo, m.fzo, wx, wy, wz);
            w = sqrt(wx * wx + wy * wy + wz * wz);
        }
    } else {
        v2 = 2.0;
        while (v2 > 1.0) {
            vx = 2.0 * rng.next() - 1.0; vy = 2.0 * rng.next() - 1.0; vz = 2.0 * rng.next() - 1.0;
            if (rng.out) return;
            v2 = vx * vx + vy * vy + vz * vz;
        }
    }
}

// the fields MonteCarloMove_chooseRotation sets
__host__ __device__ inline void copy_rotation(MoveState &d, const MoveState &s) {
    d.qold = s.qold; d.vx = s.vx; d.vy = s.vy; d.vz = s.vz; d.angle = s.angle; d.vmaxold = s.vmaxold;
    d.ca = s.ca; d.sa = s.sa; d.ct = s.ct; d.st = s.st; d.cphi = s.cphi; d.sphi = s.sphi;
}

// MonteCarloMove_chooseRotation (MonteCarloMove.f90:269-444)
__host__ __device__ inline void mcm_choose_rotation(MoveState &m, RngReader &rng, double xlc, double d_angle) {
    double vmax = xlc * m.co * d_angle, vx, vy, vz, angle;
    if (vmax > 1e-2) {
        const double emax = exp(-2.0 * vmax);
        const double shmax = (1.0 - emax) / 2.0;
        double xksi = 1.0, proba = 0.0, v = 0.0, e = 0.0;
        while (xksi >= proba) {
            v = 0.0;
            while (fabs(v) < 1e-10) {
                xksi = rng.next();
                if (rng.out) return;
                const double xs = xksi * shmax;
                v = vmax + log(xs + sqrt(xs * xs + emax));
                if (xs * xs < 1e-14 * emax) v = xs / sqrt(emax);
            }
            e = exp(-2.0 * v);
            proba = (1.0 - e) / v / (1.0 + e);
            if (v < 1e-5) proba = (2.0 * v - 2.0 * v * v) / v / (1.0 + e);
            xksi = rng.next();
            if (rng.out) return;
        }
        const double cosx = v / vmax;
        m.qold = d_shi_sans_exp(vmax) / vmax;
        xksi = 1.0;
        while (xksi > (1.0 - 1e-10)) { xksi = rng.next(); if (rng.out) return; }
        angle = d_angle * (1.0 + log(xksi + (1.0 - xksi) * e) / v);
        if (v < 1e-7) angle = d_angle * (1.0 - 2.0 * (1.0 - xksi));
        double w = -1.0, wx = 0, wy = 0, wz = 0;
        vx = vy = vz = 0;
        while (w <= 1e-10) {
            double v2 = 2.0;
            while (v2 > 1.0 || v2 < 1e-10) {
                vx = 2.0 * rng.next() - 1.0; vy = 2.0 * rng.next() - 1.0; vz = 2.0 * rng.next() - 1.0;
                if (rng.out) return;
                v2 = vx * vx + vy * vy + vz * vz;
            }
            cross(vx, vy, vz, m.cxo, m.cyo, m.czo, wx, wy, wz);
            w = sqrt(wx * wx + wy * wy + wz * wz);
        }
        const double sinx = sqrt(1.0 - cosx * cosx);
        vx = m.cxo / m.co * cosx + wx / w * sinx;
        vy = m.cyo / m.co * cosx + wy / w * sinx;
        vz = m.czo / m.co * cosx + wz / w * sinx;
    } else {
        double v2 = 2.0;
        vx = vy = vz = 0;
        while (v2 > 1.0 || v2 < 1e-10) {
            vx = 2.0 * rng.next() - 1.0; vy = 2.0 * rng.next() - 1.0; vz = 2.0 * rng.next() - 1.0;
            if (rng.out) return;
            v2 = vx * vx + vy * vy + vz * vz;
        }
        const double v = sqrt(v2);
        vx = vx / v; vy = vy / v; vz = vz / v;
        angle = d_angle * (2.0 * rng.next() - 1.0);
        if (rng.out) return;
        vmax = 0.0; m.qold = 1.0;
    }
    m.ca = cos(angle); m.sa = sin(angle);
    m.ct = vz; m.st = sqrt(1.0 - m.ct * m.ct);
    m.cphi = 0.0; m.sphi = 0.0;
    if (m.st > 0.0) { m.cphi = vx / m.st; m.sphi = vy / m.st; }
    m.vx = vx; m.vy = vy; m.vz = vz; m.vmaxold = vmax; m.angle = angle;
}

// MonteCarloMove_accept_or_decline (MonteCarloMove.f90:447-570); one draw
__host__ __device__ inline int mcm_accept(const MoveState &m, double dutot, double xlf, double xlc, RngReader &rng) {
    const double exposu = -dutot;
    const double exposf = -xlf * ((m.fxo + m.fxn) * m.deltx + (m.fyo + m.fyn) * m.delty + (m.fzo + m.fzn) * m.deltz);
    const double exposfcorr = m.umaxold - m.umaxnew;
    const double exposc = -xlc * m.angle * ((m.cxo + m.cxn) * m.vx + (m.cyo + m.cyn) * m.vy + (m.czo + m.czn) * m.vz);
    const double exposccorr = m.vmaxold - m.vmaxnew;
    const double factor = m.cold * m.qold / (m.cnew * m.qnew) * exp(exposu + exposf + exposfcorr + exposc + exposccorr);
    const double xksi = rng.next();
    return xksi > factor ? 0 : 1;
}

// movemc Step 5 (MC.f90:1031-1067): new atom positions from the proposal.
// Centre of mass of the old atoms, wrapped new centre (ANINT), rotation of the
// atoms about the centre with fill_rot_matrix/rotate_vect (geometry.f90:103-168).
// (generic over where the positions come from and go to: pos(i, d) is coordinate d of old atom i,
// put(i, x, y, z) stores new atom i; the arithmetic is the same for every caller)
template <class Pos, class Put>
__host__ __device__ inline void place_molecule_f(const MoveState &m, int na, Pos pos, const double *mass, Put put) {
    double sx = 0, sy = 0, sz = 0, tm = 0;
#pragma unroll
    for (int i = 0; i < kMaxA; ++i)
        if (i < na) { sx = sx + mass[i] * pos(i, 0); sy = sy + mass[i] * pos(i, 1); sz = sz + mass[i] * pos(i, 2); tm = tm + mass[i]; }
    const double xc = sx / tm, yc = sy / tm, zc = sz / tm;
    const double xcn = xc + m.deltx - round(xc + m.deltx);
    const double ycn = yc + m.delty - round(yc + m.delty);
    const double zcn = zc + m.deltz - round(zc + m.deltz);
    if (na > 1) {
        const double cphi = m.cphi, sphi = m.sphi, st = m.st, ct = m.ct, ca = m.ca, sa = m.sa, ca1 = 1 - ca;
        const double rxx = (cphi * cphi * (st * st) * ca1 + ca);
        const double rxy = (sphi * cphi * (st * st) * ca1 - ct * sa);
        const double rxz = st * (ct * ca1 * cphi + sa * sphi);
        const double ryx = (cphi * sphi * (st * st) * ca1 + ct * sa);
        const double ryy = (sphi * sphi * (st * st) * ca1 + ca);
        const double ryz = st * (ct * ca1 * sphi - sa * cphi);
        const double rzx = st * (ct * ca1 * cphi - sa * sphi);
        const double rzy = st * (ct * ca1 * sphi + sa * cphi);
        const double rzz = (st * st * ca + ct * ct);
#pragma unroll
        for (int i = 0; i < kMaxA; ++i)
            if (i < na) {
                const double xr = pos(i, 0) - xc, yr = pos(i, 1) - yc, zr = pos(i, 2) - zc;
                put(i, (rxx * xr + rxy * yr + rxz * zr) + xcn, (ryx * xr + ryy * yr + ryz * zr) + ycn,
                    (rzx * xr + rzy * yr + rzz * zr) + zcn);
            }
    } else {
        put(0, xcn, ycn, zcn);
    }
}
__host__ __device__ inline void place_molecule(const MoveState &m, int na, const double *xo, const double *yo,
                                               const double *zo, const double *mass, double *xn, double *yn,
                                               double *zn) {
    place_molecule_f(m, na, [&](int i, int d) { return d == 0 ? xo[i] : (d == 1 ? yo[i] : zo[i]); }, mass,
                     [&](int i, double x, double y, double z) { xn[i] = x; yn[i] = y; zn[i] = z; });
}

// molecular force and torque about the centre of mass (MC.f90:1002-1025)
// (generic: pos(i, d) and frc(i, d) are coordinate d of atom i's position and force)
template <class Pos, class Frc>
__host__ __device__ inline void mol_force_torque_f(int na, Pos pos, const double *mass, Frc frc, double F[3], double T[3]) {
    double sx = 0, sy = 0, sz = 0, tm = 0;
#pragma unroll
    for (int i = 0; i < kMaxA; ++i)
        if (i < na) { sx = sx + mass[i] * pos(i, 0); sy = sy + mass[i] * pos(i, 1); sz = sz + mass[i] * pos(i, 2); tm = tm + mass[i]; }
    const double xc = sx / tm, yc = sy / tm, zc = sz / tm;
    F[0] = F[1] = F[2] = 0; T[0] = T[1] = T[2] = 0;
#pragma unroll
    for (int i = 0; i < kMaxA; ++i)
        if (i < na) { F[0] = F[0] + frc(i, 0); F[1] = F[1] + frc(i, 1); F[2] = F[2] + frc(i, 2); }
#pragma unroll
    for (int i = 0; i < kMaxA; ++i)
        if (i < na) {
            double tx, ty, tz;
            cross(pos(i, 0) - xc, pos(i, 1) - yc, pos(i, 2) - zc, frc(i, 0), frc(i, 1), frc(i, 2), tx, ty, tz);
            T[0] = T[0] + tx; T[1] = T[1] + ty; T[2] = T[2] + tz;
        }
}
__host__ __device__ inline void mol_force_torque(int na, const double *x, const double *y, const double *z,
                                                 const double *mass, const double *fx, const double *fy,
                                                 const double *fz, double F[3], double T[3]) {
    mol_force_torque_f(na, [&](int i, int d) { return d == 0 ? x[i] : (d == 1 ? y[i] : z[i]); }, mass,
                       [&](int i, int d) { return d == 0 ? fx[i] : (d == 1 ? fy[i] : fz[i]); }, F, T);
}

}  // namespace yamc
