// Internal declarations shared by the host set-up (yamc_host.cpp) and the
// device engine (yamc_engine.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/yamc.h"

namespace yamc {

constexpr double kPi = 3.14159265358979323846;        // constants.f90:5
constexpr double kTwoPi = 2.0 * 3.14159265358979323846;
constexpr double kFourPi = 4.0 * 3.14159265358979323846;
constexpr int kMaxLJTypes = 20;                          // LJTypes.f90:20
constexpr int kMaxMolAtoms = 4;                          // atoms per molecule handled on the device

void set_error(const std::string &msg);
std::string last_error();

// Everything the device needs, prepared on the host from a yamc_system +
// yamc_params, with the reference's host-side precompute restated:
// LJTypes_fill, FourierGrid_init, EwaldSumKSpace_initBeta[LJ], EwaldSumTails,
// BiasedRandom_init.
struct HostSystem {
    yamc_params p{};
    int N = 0, M = 0, nt = 0, nk = 0, S = 0, kmax = 0, npair = 0;
    std::vector<double> x, y, z, q, sigma, eps, hc, mass, dhs;  // per atom
    std::vector<int> molnum;          // 0-based molecule of each atom
    std::vector<int> type_by_index;   // 0 = no LJ, 1..nt
    std::vector<int> first, natoms;   // per molecule, 0-based first atom
    std::vector<double> type_sigma, type_eps;                  // per LJ type (box units, kT)
    std::vector<double> lj6, lj12, four_eps, sigma6, sigma2;  // nt*nt, offset (t1-1)*nt + t2-1
    std::vector<int> kx, ky, kz;      // half-space list (FourierGrid_init order)
    std::vector<double> beta, beta6, beta12;  // per half-space k, the (1+sgn(kx)) factor folded in
    // signed-k list: one entry per valid sign combination (+x, sy*y, sz*z)
    std::vector<int> ekx, eky, ekz, ekk;      // signed components and the half-space index
    std::vector<double> ebeta;                // beta per entry
    std::vector<double> ebetalj;              // npair x S, pair p over t1 <= t2
    std::vector<int> pair_index;              // nt*nt -> p
    double U_tail_coul = 0, U_tail_lj6 = 0, U_tail_lj12 = 0;
    std::vector<double> freq_beg, freq_end;   // BiasedRandom intervals
    int freq_monotone = 1;                    // intervals increasing (binary search valid)
    double smv = 0;                           // SUM of the move weights (init_freq's Smv)
    // exchange moves (init_freq with exchange weights): xchange_freq intervals and the
    // probability Sxch / (Smv + Sxch) of an exchange step; 0 = no exchange steps
    std::vector<double> xfreq_beg, xfreq_end;
    double xchange_probability = 0;
    std::vector<int32_t> mol_numbers;
    int max_mol_atoms = 0;
    // runs of identical consecutive molecules: first molecule, count, atoms each, first atom
    std::vector<int> spec;  // 4 ints per run
};

int prepare_host_system(const yamc_system *sys, const yamc_params *p, HostSystem *hs);
// the tables that depend on the box length: LJ tables from type_sigma/type_eps, beta_LJ per
// signed entry from them and beta6/beta12, the tails (used again by the volume move)
void fill_lj_tables(HostSystem &H);
void fill_beta_lj(HostSystem &H);
void compute_tails(HostSystem &H);

// Functions.f90 restated (host)
double erfc_luc(double x, double x2, double ee2);
double erf_luc(double x, double x2, double ee2);
void erfc_luc_bet6_bet12(double x, double x2, double e2, double *erfk, double *bet6, double *bet12);
double shi_sans_exp(double x);
int grid_count(int kmax);

}  // namespace yamc
