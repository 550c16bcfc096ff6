// B200 engine for YAMC's per-trial-move energy evaluation (movemc, MC.f90:831-1322).
//
// Kernels (sm_100a):
//   k_realspace_full  all-pairs real-space sum (EwaldSumRealSpace_calc, full)      -- init / full recompute
//   k_rho_full        structure factors rho(k) of all atoms (RhoSquared_addAtoms)  -- init / full recompute
//   k_kspace_energy   k-space Coulomb + dispersion energy of rho(k)               -- init / full recompute
//   k_chain<NT,EPT>   persistent Markov chain: one thread-block cluster per chain; every move runs
//                     proposal -> fused real-space + k-space pass -> cluster reduction -> Metropolis
//                     -> commit on the device, consuming the host-made random stream by cursor.
//                     The same kernel serves the per-move C ABI (one pass per launch).
//
// Layout in HBM (per system): atoms as double4 (x, y, z, q) + int2 (molecule, LJ type) + double
// hard-core diameter; the k-set as a compact list of S signed entries (+kx, +-ky, +-kz) with their
// beta and beta_LJ rows; rho(k) as double2 (C, S) per structure (Coulomb, then each LJ type) and
// entry, coalesced along the entry index.  During a chain every thread keeps its own entries' rho
// in registers and every CTA stages its share of the atoms in shared memory; HBM is touched only
// for the random stream, the moved molecule and the logs.
#include <cooperative_groups.h>
#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "yamc_device.cuh"
#include "yamc_internal.h"

namespace cg = cooperative_groups;

namespace yamc {

// ------------------------------------------------------------------------------------------
// full sums
// ------------------------------------------------------------------------------------------
constexpr int kFullTile = 256;
constexpr int kFullParts = 8;  // ew, lj6, lj12, ew_intra, lj6_intra, lj12_intra, overlap, spare

template <int BS>
__device__ inline void block_sum(double *vals, int nv, double *sh) {
    // deterministic block reduction of nv values: warp xor tree, then warps in order
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int v = 0; v < nv; ++v) {
        double x = vals[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sh[warp * nv + v] = x;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double s = 0;
        for (int w = 0; w < BS / 32; ++w) s += sh[w * nv + threadIdx.x];
        sh[(BS / 32) * nv + threadIdx.x] = s;
    }
    __syncthreads();
    for (int v = 0; v < nv; ++v) vals[v] = sh[(BS / 32) * nv + v];
    __syncthreads();
}

// EwaldSumRealSpace_calc on the full sum (EwaldSumRealSpace.f90:233-500, j0 = i+1):
// one thread per atom i runs over all j (tiles staged in shared memory), so per-atom
// uu(i) and F(i) accumulate in increasing j order like the reference; the energy
// totals count each pair once (j > i), intra-molecular pairs with -erf_Luc.
__global__ void __launch_bounds__(kFullTile) k_realspace_full(DevSys D, double *uu, double *fx, double *fy, double *fz,
                                                             double *part) {
    __shared__ double4 tp[kFullTile];
    __shared__ int2 tm[kFullTile];
    __shared__ double td[kFullTile];
    __shared__ double red[(kFullTile / 32 + 1) * kFullParts];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < D.N;
    double4 pi = make_double4(0, 0, 0, 0);
    int2 mi = make_int2(-1, 0);
    double di = 0;
    if (valid) { pi = D.atom[i]; mi = D.meta[i]; di = D.dhs[i]; }
    double u = 0, gx = 0, gy = 0, gz = 0;
    double acc[kFullParts] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int nt = D.nt;
    for (int t0 = 0; t0 < D.N; t0 += kFullTile) {
        const int j = t0 + threadIdx.x;
        if (j < D.N) { tp[threadIdx.x] = D.atom[j]; tm[threadIdx.x] = D.meta[j]; td[threadIdx.x] = D.dhs[j]; }
        __syncthreads();
        const int nj = min(kFullTile, D.N - t0);
        if (valid) {
            for (int jj = 0; jj < nj; ++jj) {
                const int jg = t0 + jj;
                if (jg == i) continue;
                const double4 pj = tp[jj];
                const int2 mj = tm[jj];
                const bool same = mi.x == mj.x;
                const double dx = min_image(pi.x - pj.x), dy = min_image(pi.y - pj.y), dz = min_image(pi.z - pj.z);
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (!same && mi.y > 0 && mj.y > 0) {
                    const double d12 = (di + td[jj]) / 2;
                    if (r2 < d12 * d12) acc[6] = 1.0;
                }
                if (r2 >= D.rmax2) continue;
                const bool lj = mi.y > 0 && mj.y > 0;
                const int off = lj ? (mi.y - 1) * nt + (mj.y - 1) : 0;
                const PairTerm<double> t = pair_term<double, true>(r2, D.xclb * pi.w * pj.w, lj, lj ? D.lj_sig6[off] : 0.0,
                                                                    lj ? D.lj_feps[off] : 0.0, D.alpha, D.taosp, same);
                if (jg > i) {
                    acc[0] += t.ew; acc[1] += t.lj6; acc[2] += t.lj12;
                    if (same) { acc[3] += t.ew; acc[4] += t.lj6; acc[5] += t.lj12; }
                }
                if (!same) {
                    u = u + (t.ew + t.lj12 - t.lj6);
                    gx = gx + dx * t.FR; gy = gy + dy * t.FR; gz = gz + dz * t.FR;
                }
            }
        }
        __syncthreads();
    }
    if (valid) { uu[i] = u; fx[i] = gx; fy[i] = gy; fz[i] = gz; }
    block_sum<kFullTile>(acc, kFullParts, red);
    if (threadIdx.x < kFullParts) part[blockIdx.x * kFullParts + threadIdx.x] = acc[threadIdx.x];
}

// RhoSquared_addAtoms (RhoSquared.f90:188-243): for each signed entry the sum over all atoms,
// in atom order, of the charge-weighted phase (Coulomb) and of the unit phase per LJ type,
// the LJ phase being the Coulomb one times 1/q like RhoSquared_addAtom (RhoSquared.f90:173-176).
constexpr int kRhoBlock = 128;
constexpr int kRhoChunk = 32;

template <int NT>
__global__ void __launch_bounds__(kRhoBlock) k_rho_full(DevSys D, double2 *rho) {
    extern __shared__ double2 stab[];  // [kRhoChunk][3][kmax+1]
    __shared__ double sq[kRhoChunk];
    __shared__ int st[kRhoChunk];
    const int KM = D.kmax + 1;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = e < D.S;
    int4 kv = make_int4(0, 0, 0, 0);
    if (valid) kv = D.kvec[e];
    double cC = 0, sC = 0;
    double cL[NT > 0 ? NT : 1], sL[NT > 0 ? NT : 1];
#pragma unroll
    for (int t = 0; t < NT; ++t) { cL[t] = 0; sL[t] = 0; }
    for (int a0 = 0; a0 < D.N; a0 += kRhoChunk) {
        const int na = min(kRhoChunk, D.N - a0);
        for (int idx = threadIdx.x; idx < na * 3 * KM; idx += blockDim.x) {
            const int a = idx / (3 * KM), r = idx % (3 * KM), d = r / KM, m = r % KM;
            const double4 p = D.atom[a0 + a];
            const double u = d == 0 ? p.x : (d == 1 ? p.y : p.z);
            double s, c;
            sincospi(2.0 * (double)m * u, &s, &c);
            if (m == 0) { s = 0.0; c = 1.0; }
            stab[(a * 3 + d) * KM + m] = make_double2(c, s);
        }
        if (threadIdx.x < na) { sq[threadIdx.x] = D.atom[a0 + threadIdx.x].w; st[threadIdx.x] = D.meta[a0 + threadIdx.x].y; }
        __syncthreads();
        if (valid) {
            for (int a = 0; a < na; ++a) {
                const double2 *T = stab + (size_t)a * 3 * KM;
                const double q = sq[a];
                const int t = st[a];
                double c = 0, s = 0;
                if (q != 0.0) {
                    entry_phase<double, double2>(T, T + KM, T + 2 * KM, kv.x, kv.y, kv.z, q, c, s);
                    cC = cC + c; sC = sC + s;
                }
                if (t > 0) {
                    double cl, sl;
                    if (q != 0.0) { const double iq = 1.0 / q; cl = c * iq; sl = s * iq; }
                    else entry_phase<double, double2>(T, T + KM, T + 2 * KM, kv.x, kv.y, kv.z, 1.0, cl, sl);
#pragma unroll
                    for (int tt = 0; tt < NT; ++tt)
                        if (tt == t - 1) { cL[tt] = cL[tt] + cl; sL[tt] = sL[tt] + sl; }
                }
            }
        }
        __syncthreads();
    }
    if (valid) {
        rho[e] = make_double2(cC, sC);
#pragma unroll
        for (int t = 0; t < NT; ++t) rho[(size_t)(1 + t) * D.S + e] = make_double2(cL[t], sL[t]);
    }
}

// EwaldSumKSpace_calc_coulomb_energy / _calc_LJ_energy (EwaldSumKSpace.f90:389-526) per entry,
// reduced per block (host adds the blocks in order).
template <int NT>
__global__ void __launch_bounds__(256) k_kspace_energy(DevSys D, const double2 *rho, double *part) {
    __shared__ double red[(256 / 32 + 1) * 2];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[2] = {0, 0};
    if (e < D.S) {
        const double2 c = rho[e];
        acc[0] = D.ebeta[e] * (c.x * c.x + c.y * c.y);
        double2 r[NT > 0 ? NT : 1];
#pragma unroll
        for (int t = 0; t < NT; ++t) r[t] = rho[(size_t)(1 + t) * D.S + e];
#pragma unroll
        for (int t1 = 0; t1 < NT; ++t1)
#pragma unroll
            for (int t2 = t1; t2 < NT; ++t2) {
                const int p = D.pair_index[t1 * NT + t2];
                double l = D.ebetalj[(size_t)p * D.S + e] * (r[t1].x * r[t2].x + r[t1].y * r[t2].y);
                if (t1 != t2) l = l + l;
                acc[1] += l;
            }
    }
    block_sum<256>(acc, 2, red);
    if (threadIdx.x < 2) part[blockIdx.x * 2 + threadIdx.x] = acc[threadIdx.x];
}

// ------------------------------------------------------------------------------------------
// the chain kernel
// ------------------------------------------------------------------------------------------
// One thread-block cluster runs one Markov chain.  Warp 0 of every CTA is the control warp:
// its lane 0 draws the random numbers, proposes moves and takes the Metropolis decision
// (redundantly in every CTA, on identical data, so the CTAs agree without talking).  The
// other warps are workers: they run the fused real-space + k-space pass of the current move
// over the CTA's atoms and k-vector entries.  For unbiased moves the control warp prepares
// the next move while the workers run the current pass: the next move starts either where the
// current one ends after a hard-core overlap (no acceptance draw) or one draw later, and when
// the next molecule is the one being moved its old positions depend on the decision, so lanes
// 0-2 prepare the (at most) three candidates and the decision picks one.
enum ChainMode { MODE_RUN = 0, MODE_OLD = 1, MODE_EVAL = 2 };

// per-replica run control, in device memory
struct RunSlot {
    const float *rng;       // stream positions [rng_off, n_rng)
    long long rng_off;
    long long n_rng;
    long long cursor;       // in: start cursor; out: cursor after the last completed move
    long long n_moves;      // moves requested
    long long moves_done;   // out
    yamc_move_record *log;  // optional, n_moves records
    double *rows;           // optional energy rows (9 doubles)
    int max_rows, n_rows;
    int status, accepted;
};

struct ChainArgs {
    const DevSys *sys;  // [R]
    RunSlot *run;       // [R]
    int G;              // CTAs per chain (cluster size)
    int mode;
    int nown_max;       // atoms staged per CTA (interleaved ownership: atom j lives in CTA j % G)
    int qcap;           // pair queue capacity per CTA
    // per-move API (R == 1): imol (1-based) and proposed positions in, results out
    const double *api_in;  // [0] imol, [1 + 3a + c] coordinate c of atom a
    double *api_out;       // the reduction vector of the pass (RV_* layout)
    double2 *scratch;      // [2][(1+nt) S]: molecule old sums, rho deltas
    long long *prof;       // optional per-phase cycle counters (PH_* layout), CTA 0
};

// phases timed when ChainArgs::prof is set (control lane 0 or worker thread 32 of CTA 0)
enum Phase { PH_CHOOSE = 0, PH_SPECULATE, PH_PROPOSE, PH_TABLES, PH_KSPACE, PH_FILTER, PH_PAIRS, PH_REDUCE,
             PH_CLUSTER, PH_DECIDE, PH_COMMIT, PH_COUNT };

// reduction vector of one pass
constexpr int RV_EW = 0, RV_LJ6 = 1, RV_LJ12 = 2, RV_DUC = 3, RV_DUL = 4, RV_OVL = 5, RV_F = 6;
constexpr int kNV = 6 + 3 * kMaxA;

enum PassKind { PASS_OLD = 0, PASS_NEW = 1, PASS_BOTH = 2 };

struct Slot { double x, y, z, q, iq, dhs; int type, pad; };
constexpr int kMaxSpecies = 8;
constexpr int kCPT = 4;   // atoms each worker thread tests per filter round
constexpr int kWin = 256; // random-stream window held in shared memory
constexpr int kCtl = 32;  // threads of the control warp
constexpr int kChainMaxThreads = 256;  // one CTA per SM, up to 255 registers per thread
constexpr int kChainMaxThreadsWide = 512;  // streamed k entries, 16 warps, up to 128 registers per thread

// a prepared move: the molecule, its atoms at the old and proposed positions, the proposal
struct Cand {
    int valid, imol, first, na;
    long long cur_start;  // stream position at the start of the move
    long long cur_prop;   // stream position after the proposal
    double mu_old[3];     // dipole of the molecule at the old positions
    Slot slot[2 * kMaxA]; // [0, na): proposed positions, [na, 2na): old positions
    double mass[kMaxA];
    MoveState mv;
};

struct ChainShared {
    Cand cand[4];         // the move being evaluated (cand[icur]) and up to three prepared next moves
    int icur;             // buffer of the move being evaluated
    int spec[3];          // buffers of the candidates: after an overlap / after a draw / accepted same molecule
    int abort, accepted, overlap, last_mol, spec_ok;
    long long cursor;     // stream position after the last completed move
    long long icycle, mic;
    double eold[3], fold[3 * kMaxA];
    double sc[SC_COUNT];
    double lx[kMaxA], ly[kMaxA], lz[kMaxA];  // last accepted move (staged copies may lag in other CTAs)
    int qcount;
    int wcount[64];       // per-warp pair counts and their exclusive prefix
    double tot[kNV];
    double du[4];
    int flags;
    // molecule species (runs of identical consecutive molecules): first molecule, count, atoms, first atom
    int nspec;
    int sp_m0[kMaxSpecies], sp_cnt[kMaxSpecies], sp_na[kMaxSpecies], sp_a0[kMaxSpecies];
    Slot sp_atom[kMaxSpecies][kMaxA];
    double sp_mass[kMaxSpecies][kMaxA];
    // two windows of the random stream
    long long wbase[2];
    int wn[2];
    int wnext;
};

__device__ __forceinline__ void worker_sync(int nwork) {
    asm volatile("bar.sync 1, %0;" ::"r"(nwork) : "memory");
}

template <int I>
struct IntC { static constexpr int value = I; };

// calls f(IntC<I>) for I in [B, E): loop indices known at compile time
template <int B, int E, class F>
__device__ __forceinline__ void static_for(F &&f) {
    if constexpr (B < E) {
        f(IntC<B>{});
        static_for<B + 1, E>(f);
    }
}

template <int NT>
struct NPair { static constexpr int value = NT * (NT + 1) / 2; };

// row of the packed upper triangle t1 <= t2 (the host's pair_index enumeration)
template <int NT>
__host__ __device__ constexpr int pair_idx(int a, int b) {
    return a <= b ? a * NT - a * (a - 1) / 2 + (b - a) : b * NT - b * (b - 1) / 2 + (a - b);
}

template <int NT, int EPT>
struct EntryRegs {
    int e[EPT];
    int kx[EPT], ky[EPT], kz[EPT];
    double beta[EPT];
    double bl[EPT][NPair<NT>::value];  // beta_LJ of every type pair for this entry
    double2 rho[EPT][1 + NT];
    double2 mold[EPT][1 + NT];
    double2 dl[EPT][1 + NT];
};

// EPT <= 0: the streamed layout (EPT == -1: the same with 512-thread CTAs) -- no entry lives in
// registers; each worker loops over its
// entries and reads k, beta, beta_LJ and rho from memory (L2-resident) every pass.  The
// register block of one (never touched) entry only keeps the code uniform.
template <int NT, int EPT>
using RegsOf = EntryRegs<NT, (EPT > 0 ? EPT : 1)>;

// Phase tables of slots [s0, s1) of move m: T[slot][axis][k] = (cos, sin)(2 pi k u), by the workers
__device__ __forceinline__ void build_tables(double2 *tab, const Cand &m, int s0, int s1, int KM, int wtid, int nwork) {
    const int n = (s1 - s0) * 3 * KM;
    for (int idx = wtid; idx < n; idx += nwork) {
        const int sl = s0 + idx / (3 * KM), r = idx % (3 * KM), d = r / KM, k = r % KM;
        const double u = d == 0 ? m.slot[sl].x : (d == 1 ? m.slot[sl].y : m.slot[sl].z);
        double s, c;
        sincospi(2.0 * (double)k * u, &s, &c);
        if (k == 0) { s = 0.0; c = 1.0; }
        tab[(sl * 3 + d) * KM + k] = make_double2(c, s);
    }
}

// Molecule phase sums of one entry over slots [s0, s0+na) -- RhoSquared_addAtom per atom:
// Coulomb phase q (cos, sin), LJ phase = Coulomb phase * (1/q) (the unit phase when q == 0),
// accumulated per LJ type in atom order.  ph/phl keep the per-atom phases for the forces.
template <int NT>
__device__ __forceinline__ void mol_phase_sum(const double2 *tab, const Cand &m, int s0, int na, int KM, int kx, int ky,
                                              int kz, double2 (&out)[1 + NT], double2 (&ph)[kMaxA], double2 (&phl)[kMaxA]) {
#pragma unroll
    for (int t = 0; t <= NT; ++t) out[t] = make_double2(0.0, 0.0);
#pragma unroll
    for (int a = 0; a < kMaxA; ++a) {
        ph[a] = make_double2(0.0, 0.0);
        phl[a] = make_double2(0.0, 0.0);
        if (a < na) {
            const Slot &sl = m.slot[s0 + a];
            const double2 *T = tab + (size_t)(s0 + a) * 3 * KM;
            double c = 0, s = 0;
            if (sl.q != 0.0) {
                entry_phase<double, double2>(T, T + KM, T + 2 * KM, kx, ky, kz, sl.q, c, s);
                out[0].x = out[0].x + c; out[0].y = out[0].y + s;
            }
            ph[a] = make_double2(c, s);
            if (sl.type > 0) {
                double cl, sl2;
                if (sl.q != 0.0) { cl = c * sl.iq; sl2 = s * sl.iq; }
                else entry_phase<double, double2>(T, T + KM, T + 2 * KM, kx, ky, kz, 1.0, cl, sl2);
#pragma unroll
                for (int t = 0; t < NT; ++t)
                    if (t == sl.type - 1) { out[1 + t].x = out[1 + t].x + cl; out[1 + t].y = out[1 + t].y + sl2; }
                phl[a] = make_double2(cl, sl2);
            }
        }
    }
}

// k-space force on the molecule's atoms from one entry: 4 pi beta (C sin - S cos) k per atom,
// Coulomb with the q-weighted phase, plus the dispersion terms of the atom's LJ type against
// every type's structure factor (ForceKSpace.f90:59-302).
template <int NT>
__device__ __forceinline__ void entry_forces(const Cand &m, int s0, int na, int kx, int ky, int kz, double beta,
                                             const double (&bl)[NPair<NT>::value], const double2 (&C)[1 + NT],
                                             const double2 (&ph)[kMaxA], const double2 (&phl)[kMaxA], double (&acc)[kNV]) {
    const double fourpi = kFourPi;
#pragma unroll
    for (int a = 0; a < kMaxA; ++a) {
        if (a < na) {
            const int ta = m.slot[s0 + a].type;
            double w = fourpi * ((C[0].x * ph[a].y - C[0].y * ph[a].x) * beta);
            if (ta > 0) {
#pragma unroll
                for (int t = 0; t < NT; ++t) {
                    double b = 0.0;
#pragma unroll
                    for (int u = 0; u < NT; ++u)
                        if (u == ta - 1) b = bl[pair_idx<NT>(u, t)];
                    w += fourpi * ((C[1 + t].x * phl[a].y - C[1 + t].y * phl[a].x) * b);
                }
            }
            acc[RV_F + 3 * a] += w * kx;
            acc[RV_F + 3 * a + 1] += w * ky;
            acc[RV_F + 3 * a + 2] += w * kz;
        }
    }
}

// One signed entry of a pass: the molecule's phase sums at the old positions (into mold) and/or
// the new ones, the delta (into dl), dU_k Coulomb + LJ against rho, and the k-space forces.
template <int NT, int KIND, bool FORCES>
__device__ __forceinline__ void kspace_entry(const double2 *tab, const Cand &m, int na, int KM, int kx, int ky, int kz,
                                             double beta, const double (&bl)[NPair<NT>::value],
                                             const double2 (&rho)[1 + NT], double2 (&mold)[1 + NT],
                                             double2 (&dl)[1 + NT], double (&acc)[kNV]) {
    double2 ph[kMaxA], phl[kMaxA];
    if constexpr (KIND != PASS_NEW) mol_phase_sum<NT>(tab, m, na, na, KM, kx, ky, kz, mold, ph, phl);
    if constexpr (KIND == PASS_OLD) {
        if constexpr (FORCES) entry_forces<NT>(m, na, na, kx, ky, kz, beta, bl, rho, ph, phl, acc);
    } else {
        double2 mnew[1 + NT];
        mol_phase_sum<NT>(tab, m, 0, na, KM, kx, ky, kz, mnew, ph, phl);
#pragma unroll
        for (int t = 0; t <= NT; ++t) dl[t] = make_double2(mnew[t].x - mold[t].x, mnew[t].y - mold[t].y);
        {   // EwaldSumKSpace_calc_dU_coulomb (EwaldSumKSpace.f90:528-620)
            const double2 C = rho[0], d = dl[0];
            acc[RV_DUC] += (((C.x + C.x) + d.x) * d.x + ((C.y + C.y) + d.y) * d.y) * beta;
        }
        // EwaldSumKSpace_calc_dU_LJ (EwaldSumKSpace.f90:623-753): t1 over all types, t2 over the
        // molecule's types (a type absent from the molecule has a zero delta and adds nothing)
#pragma unroll
        for (int t1 = 0; t1 < NT; ++t1) {
            const double2 C1 = rho[1 + t1], D1 = dl[1 + t1];
            const double tc = (C1.x + C1.x) + D1.x, ts = (C1.y + C1.y) + D1.y;
#pragma unroll
            for (int t2 = 0; t2 < NT; ++t2) {
                const double2 D2 = dl[1 + t2];
                if (D2.x == 0.0 && D2.y == 0.0) continue;
                acc[RV_DUL] += (tc * D2.x + ts * D2.y) * bl[pair_idx<NT>(t1, t2)];
            }
        }
        if constexpr (KIND == PASS_NEW && FORCES) {  // against total_new = rho + delta (MC.f90:1136-1163)
            double2 Cn[1 + NT];
#pragma unroll
            for (int t = 0; t <= NT; ++t) Cn[t] = make_double2(rho[t].x + dl[t].x, rho[t].y + dl[t].y);
            entry_forces<NT>(m, 0, na, kx, ky, kz, beta, bl, Cn, ph, phl, acc);
        }
    }
}

// The workers' part of one pass over the molecule's slots: k-space over their entries, real
// space over the CTA's atoms (pairs inside the cutoff laid out in the queue by a prefix sum
// over threads -- a deterministic order -- then evaluated item i by worker i % nwork), and a
// per-warp reduction into red[worker warp][value].  Worker-only barriers (bar 1).
template <int NT, int EPT, int KIND, bool FORCES>
__device__ __forceinline__ void worker_pass(const DevSys &D, ChainShared &sh, RegsOf<NT, EPT> &R, double2 *tab,
                                            const double4 *atom_s, const double *dhs_s, const int2 *meta_s, int *queue,
                                            int *nearbuf,
                                            double *red, const double *lj_s, int nown, int qcap, int e0, int estep,
                                            long long *prof) {
    constexpr int NVMAX = FORCES ? kNV : RV_F;
    const Cand &m = sh.cand[sh.icur];
    const int na = m.na;
    const int KM = D.kmax + 1;
    const int nt = D.nt;
    const int imol0 = m.imol - 1;
    const int nwork = blockDim.x - kCtl;
    const int wtid = threadIdx.x - kCtl;
    const int lane = threadIdx.x & 31;
    const int wwarp = wtid >> 5, nww = nwork >> 5;
    const int s_lo = (KIND == PASS_OLD) ? na : 0;  // active slots [s_lo, s_hi)
    const int s_hi = (KIND == PASS_NEW) ? na : 2 * na;
    const bool pf = prof && wtid == 0;
    long long t_mark = pf ? clock64() : 0;
#define YAMC_WPH(ph) do { if (pf) { const long long t_now = clock64(); prof[ph] += t_now - t_mark; t_mark = t_now; } } while (0)

    build_tables(tab, m, s_lo, s_hi, KM, wtid, nwork);
    worker_sync(nwork);
    YAMC_WPH(PH_TABLES);

    double acc[FORCES ? kNV : kNV];
#pragma unroll
    for (int v = 0; v < kNV; ++v) acc[v] = 0.0;

    if constexpr (EPT > 0) {
        static_for<0, EPT>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            if (R.e[k] < 0) return;
            kspace_entry<NT, KIND, FORCES>(tab, m, na, KM, R.kx[k], R.ky[k], R.kz[k], R.beta[k], R.bl[k], R.rho[k],
                                           R.mold[k], R.dl[k], acc);
        });
    } else {
        // streamed layout: entries e0, e0 + estep, ... read from memory, the next entry's loads in
        // flight while the current one computes; the old sums and the deltas go to the chain's
        // scratch for the next pass and the commit
        const int S = D.S;
        double2 *mold_g = D.scratch;
        double2 *dl_g = D.scratch + (size_t)(1 + NT) * S;
        int4 kv_n = make_int4(0, 0, 0, 0);
        double beta_n = 0.0, bl_n[NPair<NT>::value];
        double2 rho_n[1 + NT], mold_n[1 + NT];
        auto fetch = [&](int e) {
            kv_n = D.kvec[e];
            beta_n = D.ebeta[e];
#pragma unroll
            for (int p = 0; p < NPair<NT>::value; ++p) bl_n[p] = D.ebetalj[(size_t)p * S + e];
#pragma unroll
            for (int t = 0; t <= NT; ++t) {
                rho_n[t] = D.rho[(size_t)t * S + e];
                mold_n[t] = (KIND == PASS_NEW) ? mold_g[(size_t)t * S + e] : make_double2(0, 0);
            }
        };
        if (e0 < S) fetch(e0);
        for (int e = e0; e < S; e += estep) {
            const int kx = kv_n.x, ky = kv_n.y, kz = kv_n.z;
            const double beta = beta_n;
            double bl[NPair<NT>::value];
            double2 rho[1 + NT], mold[1 + NT], dl[1 + NT];
#pragma unroll
            for (int p = 0; p < NPair<NT>::value; ++p) bl[p] = bl_n[p];
#pragma unroll
            for (int t = 0; t <= NT; ++t) { rho[t] = rho_n[t]; mold[t] = mold_n[t]; }
            if (e + estep < S) fetch(e + estep);
            kspace_entry<NT, KIND, FORCES>(tab, m, na, KM, kx, ky, kz, beta, bl, rho, mold, dl, acc);
#pragma unroll
            for (int t = 0; t <= NT; ++t) {
                if (KIND == PASS_OLD) mold_g[(size_t)t * S + e] = mold[t];
                else dl_g[(size_t)t * S + e] = dl[t];
            }
        }
    }
    YAMC_WPH(PH_KSPACE);

    // bounding spheres of the molecule at its new (slot 0) and old (slot na) positions: an atom
    // farther than rpre + radius from a centre is outside the cutoff and every hard core of all
    // that position's slots (triangle inequality on the periodic box), so its slot tests are skipped
    double rp2;
    {
        double rad2 = 0.0;
        for (int a = 1; a < na; ++a) {
            const double dx = m.slot[a].x - m.slot[0].x, dy = m.slot[a].y - m.slot[0].y, dz = m.slot[a].z - m.slot[0].z;
            rad2 = fmax(rad2, dx * dx + dy * dy + dz * dz);
            const double ex = m.slot[na + a].x - m.slot[na].x, ey = m.slot[na + a].y - m.slot[na].y,
                         ez = m.slot[na + a].z - m.slot[na].z;
            rad2 = fmax(rad2, ex * ex + ey * ey + ez * ez);
        }
        const double rp = (D.rpre + sqrt(rad2)) * (1.0 + 1e-9);
        rp2 = rp * rp;
    }
    const double cnx = m.slot[0].x, cny = m.slot[0].y, cnz = m.slot[0].z;
    const double cox = m.slot[na].x, coy = m.slot[na].y, coz = m.slot[na].z;

    const int round_atoms = nwork * kCPT;
    int *nb = nearbuf + wwarp * 32 * kCPT;  // this warp's near atoms of the round
    for (int c0 = 0; c0 < nown; c0 += round_atoms) {
        // near atoms of the warp's 32 x kCPT candidates, compacted in (c, lane) order
        int nnear = 0;
#pragma unroll
        for (int c = 0; c < kCPT; ++c) {
            const int jl = c0 + c * nwork + wtid;
            bool near = false;
            if (jl < nown && meta_s[jl].x != imol0) {
                const double4 pj = atom_s[jl];
                if (KIND != PASS_OLD) {
                    const double dx = min_image(cnx - pj.x), dy = min_image(cny - pj.y), dz = min_image(cnz - pj.z);
                    near = dx * dx + dy * dy + dz * dz < rp2;
                }
                if (KIND != PASS_NEW) {
                    const double dx = min_image(cox - pj.x), dy = min_image(coy - pj.y), dz = min_image(coz - pj.z);
                    near = near || dx * dx + dy * dy + dz * dz < rp2;
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, near);
            if (near) nb[nnear + __popc(bal & ((1u << lane) - 1u))] = jl;
            nnear += __popc(bal);
        }
        __syncwarp();
        // slot tests of the near atoms, densely: lane takes entries lane, lane + 32, ...
        unsigned masks = 0;  // kCPT slot masks of 8 bits
        int count = 0;
#pragma unroll
        for (int c = 0; c < kCPT; ++c) {
            const int k = c * 32 + lane;
            if (k < nnear) {
                const int jl = nb[k];
                const double4 pj = atom_s[jl];
                const int tj = meta_s[jl].y;
                const double dj = dhs_s[jl];
                unsigned msk = 0;
                for (int s = s_lo; s < s_hi; ++s) {
                    const Slot &sl = m.slot[s];
                    const double dx = min_image(sl.x - pj.x), dy = min_image(sl.y - pj.y), dz = min_image(sl.z - pj.z);
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    if (KIND != PASS_OLD && s < na && sl.type > 0 && tj > 0) {  // hard core (EwaldSumRealSpace.f90:409)
                        const double d12 = (sl.dhs + dj) / 2;
                        if (r2 < d12 * d12) acc[RV_OVL] = 1.0;
                    }
                    if (r2 < D.rmax2) msk |= 1u << s;
                }
                masks |= msk << (8 * c);
                count += __popc(msk);
            }
        }
        int incl = count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) sh.wcount[wwarp] = incl;
        worker_sync(nwork);
        if (wwarp == 0) {
            const int v = lane < nww ? sh.wcount[lane] : 0;
            int x = v;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane < nww) sh.wcount[32 + lane] = x - v;
            if (lane == 31) sh.qcount = x;
        }
        worker_sync(nwork);
        int pos = sh.wcount[32 + wwarp] + incl - count;
#pragma unroll
        for (int c = 0; c < kCPT; ++c) {
            unsigned msk = (masks >> (8 * c)) & 0xffu;
            const int jl = msk ? nb[c * 32 + lane] : 0;
            while (msk) {
                const int s = __ffs(msk) - 1;
                msk &= msk - 1;
                queue[pos++] = (jl << 3) | s;
            }
        }
        worker_sync(nwork);
        YAMC_WPH(PH_FILTER);
        const int nq = sh.qcount;
        for (int qi = wtid; qi < nq; qi += nwork) {
            const int item = queue[qi];
            const int jl = item >> 3, s = item & 7;
            const Slot &sl = m.slot[s];
            const double4 pj = atom_s[jl];
            const int tj = meta_s[jl].y;
            const double dx = min_image(sl.x - pj.x), dy = min_image(sl.y - pj.y), dz = min_image(sl.z - pj.z);
            const double r2 = dx * dx + dy * dy + dz * dz;
            const bool lj = sl.type > 0 && tj > 0;
            const int off = lj ? (sl.type - 1) * nt + (tj - 1) : 0;
            const double qq = D.xclb * sl.q * pj.w;
            const double s6 = lj ? lj_s[off] : 0.0, fe = lj ? lj_s[nt * nt + off] : 0.0;
            const bool isnew = s < na;
            const double sign = (KIND == PASS_BOTH && !isnew) ? -1.0 : 1.0;
            if constexpr (FORCES) {
                const PairTerm<double> t = pair_term<double, true>(r2, qq, lj, s6, fe, D.alpha, D.taosp, false);
                acc[RV_EW] += sign * t.ew; acc[RV_LJ6] += sign * t.lj6; acc[RV_LJ12] += sign * t.lj12;
                const int a = isnew ? s : s - na;
#pragma unroll
                for (int aa = 0; aa < kMaxA; ++aa)
                    if (aa == a) { acc[RV_F + 3 * aa] += dx * t.FR; acc[RV_F + 3 * aa + 1] += dy * t.FR; acc[RV_F + 3 * aa + 2] += dz * t.FR; }
            } else {
                const PairTerm<double> t = pair_term<double, false>(r2, qq, lj, s6, fe, D.alpha, D.taosp, false);
                acc[RV_EW] += sign * t.ew; acc[RV_LJ6] += sign * t.lj6; acc[RV_LJ12] += sign * t.lj12;
            }
        }
        worker_sync(nwork);
        YAMC_WPH(PH_PAIRS);
    }

    // per-warp reduction (xor tree) into red[worker warp][value]
    const int nv = FORCES ? (RV_F + 3 * na) : RV_F;
#pragma unroll
    for (int v = 0; v < NVMAX; ++v) {
        if (v < nv) {
            double x = acc[v];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double y = __shfl_xor_sync(0xffffffffu, x, o);
                x = (v == RV_OVL) ? fmax(x, y) : x + y;
            }
            if (lane == 0) red[wwarp * kNV + v] = x;
        }
    }
#undef YAMC_WPH
}

// Control warp, after the workers' per-warp partials: trees over the worker warps, then over the
// cluster's CTAs in a fixed order, so every CTA holds bit-identical totals in sh.tot.  Called by
// all threads (the cluster barrier needs everyone).
__device__ __forceinline__ void reduce_pass(ChainShared &sh, const double *red, double *xch, int nv, int G, int rank,
                                            int xpar, cg::cluster_group &cluster) {
    const int lane = threadIdx.x & 31;
    const int nww = (blockDim.x - kCtl) >> 5;
    if (threadIdx.x < kCtl) {
        for (int v = 0; v < nv; ++v) {
            double x = lane < nww ? red[lane * kNV + v] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double y = __shfl_xor_sync(0xffffffffu, x, o);
                x = (v == RV_OVL) ? fmax(x, y) : x + y;
            }
            if (G > 1) {
                if (lane < G) {
                    double *dst = cluster.map_shared_rank(xch, lane);
                    dst[(xpar * G + rank) * kNV + v] = x;
                }
            } else if (lane == 0) {
                sh.tot[v] = x;
            }
        }
    }
    if (G > 1) {
        cluster.sync();
        if (threadIdx.x < kCtl) {
            for (int v = 0; v < nv; ++v) {
                double x = lane < G ? xch[(xpar * G + lane) * kNV + v] : 0.0;
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double y = __shfl_xor_sync(0xffffffffu, x, o);
                    x = (v == RV_OVL) ? fmax(x, y) : x + y;
                }
                if (lane == 0) sh.tot[v] = x;
            }
        }
    }
}

// Control lane work: molecule choice (run_mc draws) and the static atom data of the chosen
// molecule at its current positions.  `moving` is the molecule of the move in flight (0-based,
// -1 if none) whose positions come from `moving_pos` (its old or its proposed positions).
struct ChooseCtx {
    const DevSys *D;
    const RunSlot *run;
    const float *w0, *w1;
    const double4 *atom_s;
    int G;
};

__device__ inline RngReader make_reader(const ChooseCtx &X, const ChainShared &sh, long long cur) {
    return RngReader{X.run->rng, X.run->rng_off, X.run->n_rng, cur, 0, X.w0, sh.wbase[0], sh.wn[0],
                     X.w1, sh.wbase[1], sh.wn[1]};
}

__device__ inline void stage_molecule(const ChooseCtx &X, ChainShared &sh, Cand &C, int imol, int moving,
                                      const Slot *moving_pos, cg::cluster_group &cluster) {
    const DevSys &D = *X.D;
    int sp = -1;
    for (int q = 0; q < sh.nspec; ++q)
        if (imol - 1 >= sh.sp_m0[q] && imol - 1 < sh.sp_m0[q] + sh.sp_cnt[q]) { sp = q; break; }
    int first, nam;
    if (sp >= 0) { nam = sh.sp_na[sp]; first = sh.sp_a0[sp] + (imol - 1 - sh.sp_m0[sp]) * nam; }
    else { const int2 mr = D.mol[imol - 1]; first = mr.x; nam = mr.y; }
    C.imol = imol; C.first = first; C.na = nam;
    double mx = 0, my = 0, mz = 0;
    for (int a = 0; a < nam; ++a) {
        const int j = first + a;
        Slot s;
        if (sp >= 0) { s = sh.sp_atom[sp][a]; C.mass[a] = sh.sp_mass[sp][a]; }
        else {
            const double q = D.atom[j].w;
            s.q = q; s.iq = q != 0.0 ? 1.0 / q : 0.0; s.dhs = D.dhs[j]; s.type = D.meta[j].y; s.pad = 0;
            C.mass[a] = D.mass[j];
        }
        if (imol - 1 == moving) { s.x = moving_pos[a].x; s.y = moving_pos[a].y; s.z = moving_pos[a].z; }
        else if (imol - 1 == sh.last_mol) { s.x = sh.lx[a]; s.y = sh.ly[a]; s.z = sh.lz[a]; }
        else {
            const double4 *src = (X.G > 1) ? cluster.map_shared_rank(X.atom_s, j % X.G) : X.atom_s;
            const double4 p = src[j / X.G];
            s.x = p.x; s.y = p.y; s.z = p.z;
        }
        C.slot[nam + a] = s;  // old positions
        C.slot[a] = s;        // proposed positions, replaced by propose()
        // dipole of the molecule at the old positions (EwaldSumExternal_calc_mu)
        mx = mx + s.q * s.x; my = my + s.q * s.y; mz = mz + s.q * s.z;
    }
    C.mu_old[0] = mx; C.mu_old[1] = my; C.mu_old[2] = mz;
}

// run_mc's draws before movemc: the per-cycle pressure draw, the exchange draw, the molecule
// draw (runmc.f90:206, 232, 258).  Returns the 1-based molecule, or 0 when the stream ran out.
__device__ inline int draw_molecule(const DevSys &D, RngReader &rng, bool cycle_start) {
    if (cycle_start) (void)rng.next();
    (void)rng.next();
    const double r = rng.next();
    if (rng.out) return 0;
    return choose_molecule_guess(r, D.freq_beg, D.freq_end, D.M, D.freq_monotone);
}

// movemc Step 5 (MC.f90:1031-1067) for a staged molecule; F/T are the old molecular force and
// torque (zero for unbiased moves)
__device__ inline void propose(const DevSys &D, Cand &C, RngReader &rng, const double F[3], const double T[3]) {
    const int na = C.na;
    MoveState &m = C.mv;
    mcm_init_old(m, F, T);
    mcm_choose_displacement(m, rng, D.xlf, D.dr);
    if (!rng.out) mcm_choose_rotation(m, rng, D.xlc, D.d_angle);
    double xo[kMaxA], yo[kMaxA], zo[kMaxA], xn[kMaxA], yn[kMaxA], zn[kMaxA];
#pragma unroll
    for (int a = 0; a < kMaxA; ++a) {
        const Slot &o = C.slot[a < na ? na + a : na];
        xo[a] = o.x; yo[a] = o.y; zo[a] = o.z;
    }
    place_molecule(m, na, xo, yo, zo, C.mass, xn, yn, zn);
#pragma unroll
    for (int a = 0; a < kMaxA; ++a)
        if (a < na) { C.slot[a].x = xn[a]; C.slot[a].y = yn[a]; C.slot[a].z = zn[a]; }
}

// SPLIT = false: unbiased device-resident chain only (one fused pass per move, speculation);
// SPLIT = true: force-biased moves and the per-move API (old pass + new pass with forces).
template <int NT, int EPT, bool SPLIT>
__global__ void __launch_bounds__(EPT < 0 ? kChainMaxThreadsWide : kChainMaxThreads, 1) k_chain(ChainArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ChainShared sh;
    __shared__ float rwin[2][kWin];

    cg::cluster_group cluster = cg::this_cluster();
    const int G = A.G;
    const int rank = G > 1 ? (int)cluster.block_rank() : 0;
    const int rep = blockIdx.x / G;
    const DevSys D = A.sys[rep];
    RunSlot *run = A.run + rep;
    const int B = blockDim.x;
    const int tid = threadIdx.x;
    const int KM = D.kmax + 1;
    const int S = D.S;
    const int nt = D.nt;
    const int nwork = B - kCtl;
    const int wtid = tid - kCtl;
    const bool ctl = tid < kCtl;
    const int lane = tid & 31;

    // shared memory carve-up (chain_smem_bytes on the host computes the same sizes)
    double2 *tab = reinterpret_cast<double2 *>(smem_raw);                     // [2 kMaxA][3][KM]
    double4 *atom_s = reinterpret_cast<double4 *>(tab + 2 * kMaxA * 3 * KM);  // [nown_max]
    double *dhs_s = reinterpret_cast<double *>(atom_s + A.nown_max);          // [nown_max]
    int2 *meta_s = reinterpret_cast<int2 *>(dhs_s + A.nown_max);              // [nown_max]
    int *queue = reinterpret_cast<int *>(meta_s + A.nown_max);                // [qcap]
    int *nearbuf = queue + ((A.qcap + 1) & ~1);                               // [B/32][32 kCPT]
    double *red = reinterpret_cast<double *>(nearbuf + B * kCPT);             // [B/32][kNV]
    double *xch = red + (B / 32) * kNV;                                       // [2][G][kNV]
    double *lj_s = xch + 2 * G * kNV;                                         // [2][nt*nt]

    // atoms of this CTA: j = rank + G * local (interleaved, so every CTA holds a spatial mix)
    const int nown = (D.N - rank + G - 1) / G;
    for (int i = tid; i < nown; i += B) {
        const int j = rank + G * i;
        atom_s[i] = D.atom[j]; dhs_s[i] = D.dhs[j]; meta_s[i] = D.meta[j];
    }
    for (int i = tid; i < nt * nt; i += B) { lj_s[i] = D.lj_sig6[i]; lj_s[nt * nt + i] = D.lj_feps[i]; }

    // the workers' k-vector entries; rho stays in registers for the whole launch
    RegsOf<NT, EPT> R;
    const int gwork = G * nwork;
    const int e0 = rank * nwork + wtid;  // this worker's entries: e0 + k * gwork
#pragma unroll
    for (int k = 0; k < EPT; ++k) {
        const int e = ctl ? S : rank * nwork + wtid + k * gwork;
        R.e[k] = e < S ? e : -1;
        R.kx[k] = R.ky[k] = R.kz[k] = 0;
        R.beta[k] = 0;
        if (e < S) {
            const int4 kv = D.kvec[e];
            R.kx[k] = kv.x; R.ky[k] = kv.y; R.kz[k] = kv.z;
            R.beta[k] = D.ebeta[e];
        }
#pragma unroll
        for (int p = 0; p < NPair<NT>::value; ++p) R.bl[k][p] = e < S ? D.ebetalj[(size_t)p * S + e] : 0.0;
#pragma unroll
        for (int t = 0; t <= NT; ++t) {
            R.rho[k][t] = e < S ? D.rho[(size_t)t * S + e] : make_double2(0, 0);
            R.mold[k][t] = (A.mode == MODE_EVAL && e < S) ? A.scratch[(size_t)t * S + e] : make_double2(0, 0);
            R.dl[k][t] = make_double2(0, 0);
        }
    }
    const long long n_rng = run->n_rng;
    if (tid == 0) {
        for (int c = 0; c < SC_COUNT; ++c) sh.sc[c] = D.scal[c];
        sh.icycle = D.cnt[CN_ICYCLE];
        sh.mic = D.cnt[CN_MOVE_IN_CYCLE];
        sh.cursor = run->cursor;
        sh.last_mol = -1;
        sh.abort = 0;
        sh.qcount = 0;
        sh.wnext = 0;
        sh.icur = 0;
        sh.spec_ok = 0;
        // static atom data of each molecule species, taken from its first molecule
        sh.nspec = D.nspec <= kMaxSpecies ? D.nspec : 0;
        for (int sp = 0; sp < sh.nspec; ++sp) {
            const int4 c = D.spec[sp];
            sh.sp_m0[sp] = c.x; sh.sp_cnt[sp] = c.y; sh.sp_na[sp] = c.z; sh.sp_a0[sp] = c.w;
            for (int a = 0; a < c.z; ++a) {
                const int j = c.w + a;
                Slot t;
                t.x = t.y = t.z = 0.0;
                t.q = D.atom[j].w; t.iq = t.q != 0.0 ? 1.0 / t.q : 0.0;
                t.dhs = D.dhs[j]; t.type = D.meta[j].y; t.pad = 0;
                sh.sp_atom[sp][a] = t;
                sh.sp_mass[sp][a] = D.mass[j];
            }
        }
    }
    // first random window at the start cursor
    if (ctl && A.mode == MODE_RUN) {
        const long long base = run->cursor;
        const long long avail = n_rng - base;
        const int nw = (int)(avail < (long long)kWin ? (avail > 0 ? avail : 0) : kWin);
        for (int i = lane; i < nw; i += 32) rwin[0][i] = run->rng[base + i - run->rng_off];
        if (lane == 0) { sh.wbase[0] = base; sh.wn[0] = nw; sh.wbase[1] = -1; sh.wn[1] = 0; sh.wnext = 1; }
    }
    __syncthreads();
    const bool biased = SPLIT && (D.xlf > 0.0 || D.xlc > 0.0);
    const bool speculate = !SPLIT;
    const ChooseCtx X{&D, run, rwin[0], rwin[1], atom_s, G};

    long long moves_done = 0;
    int n_acc = 0, rows = 0;
    int xpar = 0;  // parity of the cluster exchange buffer, flipped after every pass
    const long long n_moves = (A.mode == MODE_RUN) ? run->n_moves : 1;
    long long *prof = (A.prof && rank == 0) ? A.prof : nullptr;
    const bool pc = prof && tid == 0;
    long long t_mark = 0;
#define YAMC_PH(ph) do { if (pc) { const long long t_now = clock64(); prof[ph] += t_now - t_mark; t_mark = t_now; } } while (0)

    // ---------------------------------------------------------------- the first move of the launch
    bool have_next = false;  // sh.cur already prepared by the previous iteration's speculation
    for (long long it = 0; it < n_moves; ++it) {
        if (pc) t_mark = clock64();
        if (!have_next) {
            // choose the molecule and stage its atoms (no move in flight)
            if (tid == 0) {
                Cand &C = sh.cand[sh.icur];
                C.cur_start = sh.cursor;
                int imol;
                if (A.mode == MODE_RUN) {
                    RngReader rng = make_reader(X, sh, sh.cursor);
                    imol = draw_molecule(D, rng, sh.mic == 0);
                    C.valid = imol > 0;
                    C.cur_prop = rng.cur;
                    if (!imol) imol = 1;
                } else {
                    imol = (int)A.api_in[0];
                    C.valid = 1;
                    C.cur_prop = sh.cursor;
                }
                stage_molecule(X, sh, C, imol, -1, nullptr, cluster);
                sh.abort = C.valid ? 0 : 1;
            }
            __syncthreads();
            if (sh.abort) break;
            YAMC_PH(PH_CHOOSE);
            const int na0 = sh.cand[sh.icur].na;
            // old forces for force-biased moves and the per-move API (movemc Steps 3-4)
            if constexpr (SPLIT) if ((biased && A.mode == MODE_RUN) || A.mode == MODE_OLD) {
                if (!ctl) worker_pass<NT, EPT, PASS_OLD, true>(D, sh, R, tab, atom_s, dhs_s, meta_s, queue, nearbuf, red, lj_s, nown, A.qcap, e0, gwork, prof);
                __syncthreads();
                reduce_pass(sh, red, xch, RV_F + 3 * na0, G, rank, xpar, cluster);
                xpar ^= 1;
                __syncthreads();
                if (tid == 0) {
                    sh.eold[0] = sh.tot[RV_EW]; sh.eold[1] = sh.tot[RV_LJ6]; sh.eold[2] = sh.tot[RV_LJ12];
                    for (int a = 0; a < na0; ++a) {  // external-field force -2 kext q mu (MC.f90:988-997)
                        const double q = sh.cand[sh.icur].slot[na0 + a].q;
                        sh.fold[3 * a] = sh.tot[RV_F + 3 * a] + D.m2k * q * sh.sc[SC_MU_X];
                        sh.fold[3 * a + 1] = sh.tot[RV_F + 3 * a + 1] + D.m2k * q * sh.sc[SC_MU_Y];
                        sh.fold[3 * a + 2] = sh.tot[RV_F + 3 * a + 2] + D.m2k * q * sh.sc[SC_MU_Z];
                    }
                }
                if (A.mode == MODE_OLD) {
#pragma unroll
                    for (int k = 0; k < EPT; ++k)
                        if (R.e[k] >= 0) {
#pragma unroll
                            for (int t = 0; t <= NT; ++t) A.scratch[(size_t)t * S + R.e[k]] = R.mold[k][t];
                        }
                    __syncthreads();
                    if (tid == 0 && rank == 0) {
                        for (int c = 0; c < 3; ++c) A.api_out[c] = sh.eold[c];
                        for (int c = 0; c < 3 * na0; ++c) A.api_out[RV_F + c] = sh.fold[c];
                    }
                    moves_done = 1;
                    break;
                }
            }
            // the proposal (movemc Step 5)
            if (tid == 0) {
                Cand &C = sh.cand[sh.icur];
                if (A.mode == MODE_RUN) {
                    RngReader rng = make_reader(X, sh, C.cur_prop);
                    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
                    if (biased) {
                        double xo[kMaxA], yo[kMaxA], zo[kMaxA], fx[kMaxA], fy[kMaxA], fz[kMaxA];
                        for (int a = 0; a < na0; ++a) {
                            xo[a] = C.slot[na0 + a].x; yo[a] = C.slot[na0 + a].y; zo[a] = C.slot[na0 + a].z;
                            fx[a] = sh.fold[3 * a]; fy[a] = sh.fold[3 * a + 1]; fz[a] = sh.fold[3 * a + 2];
                        }
                        mol_force_torque(na0, xo, yo, zo, C.mass, fx, fy, fz, F, T);
                    }
                    propose(D, C, rng, F, T);
                    C.cur_prop = rng.cur;
                    if (rng.out) { C.valid = 0; sh.abort = 1; }
                } else {  // MODE_EVAL: positions from the host
                    for (int a = 0; a < na0; ++a) {
                        C.slot[a].x = A.api_in[1 + 3 * a]; C.slot[a].y = A.api_in[2 + 3 * a]; C.slot[a].z = A.api_in[3 + 3 * a];
                    }
                }
            }
            __syncthreads();
            if (sh.abort) break;
            YAMC_PH(PH_PROPOSE);
        }
        const int na = sh.cand[sh.icur].na;
        const bool split = SPLIT;

        // ------------------------------------------------ the pass over the new positions
        if (!ctl) {
            if constexpr (SPLIT) worker_pass<NT, EPT, PASS_NEW, true>(D, sh, R, tab, atom_s, dhs_s, meta_s, queue, nearbuf, red, lj_s, nown, A.qcap, e0, gwork, prof);
            else worker_pass<NT, EPT, PASS_BOTH, false>(D, sh, R, tab, atom_s, dhs_s, meta_s, queue, nearbuf, red, lj_s, nown, A.qcap, e0, gwork, prof);
        } else if (speculate && it + 1 < n_moves) {
            // prepare the next move's candidates while the workers run: lane 0 after an overlap
            // (no acceptance draw), lanes 1-2 after the acceptance draw, lane 2 with the molecule
            // in flight at its proposed positions (used only if it is chosen again and accepted)
            const Cand &M = sh.cand[sh.icur];
            const long long c1 = M.cur_prop;
            const bool next_cycle = (sh.mic + 1 == D.M);
            // the window of the stream the candidates read: make sure it covers c1 onwards
            {
                const int b = sh.wnext;
                const bool covered0 = sh.wbase[0] >= 0 && c1 >= sh.wbase[0] && c1 + kWin / 2 <= sh.wbase[0] + sh.wn[0];
                const bool covered1 = sh.wbase[1] >= 0 && c1 >= sh.wbase[1] && c1 + kWin / 2 <= sh.wbase[1] + sh.wn[1];
                if (!covered0 && !covered1) {
                    const long long avail = n_rng - c1;
                    const int nw = (int)(avail < (long long)kWin ? (avail > 0 ? avail : 0) : kWin);
                    __syncwarp();
                    for (int i = lane; i < nw; i += 32) rwin[b][i] = run->rng[c1 + i - run->rng_off];
                    __syncwarp();
                    if (lane == 0) { sh.wbase[b] = c1; sh.wn[b] = nw; sh.wnext = b ^ 1; }
                    __syncwarp();
                }
            }
            if (lane < 3) {
                const int buf = (sh.icur + 1 + lane) & 3;
                if (lane == 0) { sh.spec[0] = (sh.icur + 1) & 3; sh.spec[1] = (sh.icur + 2) & 3; sh.spec[2] = (sh.icur + 3) & 3; }
                Cand &C = sh.cand[buf];
                RngReader rng = make_reader(X, sh, c1);
                if (lane > 0) (void)rng.next();  // the acceptance draw (MonteCarloMove.f90:553)
                C.cur_start = rng.cur;
                const int imol = rng.out ? 0 : draw_molecule(D, rng, next_cycle);
                C.valid = imol > 0;
                const Slot *moving = (lane == 2) ? &M.slot[0] : &M.slot[M.na];
                stage_molecule(X, sh, C, imol > 0 ? imol : 1, M.imol - 1, moving, cluster);
                const double Z[3] = {0, 0, 0};
                if (C.valid) propose(D, C, rng, Z, Z);
                C.cur_prop = rng.cur;
                if (rng.out) C.valid = 0;
            }
            if (pc) { const long long t_now = clock64(); prof[PH_SPECULATE] += t_now - t_mark; t_mark = t_now; }
        }
        __syncthreads();
        reduce_pass(sh, red, xch, split ? RV_F + 3 * na : RV_F, G, rank, xpar, cluster);
        xpar ^= 1;
        YAMC_PH(PH_REDUCE);

        if (A.mode == MODE_EVAL) {
#pragma unroll
            for (int k = 0; k < EPT; ++k)
                if (R.e[k] >= 0) {
#pragma unroll
                    for (int t = 0; t <= NT; ++t) A.scratch[(size_t)(1 + nt + t) * S + R.e[k]] = R.dl[k][t];
                }
            __syncthreads();
            if (tid == 0 && rank == 0)
                for (int v = 0; v < RV_F + 3 * na; ++v) A.api_out[v] = sh.tot[v];
            moves_done = 1;
            break;
        }

        // ------------------------------------------------ Metropolis (Steps 7-13) and commit (Step 14)
        if (tid == 0) {
            const Cand &M = sh.cand[sh.icur];
            const bool overlap = sh.tot[RV_OVL] > 0.0;
            int flags = overlap ? 2 : 0;
            double du_real = 0, du_kc = 0, du_kl = 0, du_ext = 0, dmx = 0, dmy = 0, dmz = 0;
            double dew = 0, dlj6 = 0, dlj12 = 0;
            int acc = 0;
            long long cur_after = M.cur_prop;
            bool out = false;
            if (!overlap) {
                RngReader rng = make_reader(X, sh, M.cur_prop);
                if (biased) {
                    dew = sh.tot[RV_EW] - sh.eold[0]; dlj6 = sh.tot[RV_LJ6] - sh.eold[1]; dlj12 = sh.tot[RV_LJ12] - sh.eold[2];
                    du_real = (sh.tot[RV_EW] + sh.tot[RV_LJ12] - sh.tot[RV_LJ6]) - (sh.eold[0] + sh.eold[2] - sh.eold[1]);
                } else {
                    dew = sh.tot[RV_EW]; dlj6 = sh.tot[RV_LJ6]; dlj12 = sh.tot[RV_LJ12];
                    du_real = dew + dlj12 - dlj6;
                }
                du_kc = sh.tot[RV_DUC];
                du_kl = sh.tot[RV_DUL];
                double mx = 0, my = 0, mz = 0;
                for (int a = 0; a < na; ++a) { mx = mx + M.slot[a].q * M.slot[a].x; my = my + M.slot[a].q * M.slot[a].y; mz = mz + M.slot[a].q * M.slot[a].z; }
                dmx = mx - M.mu_old[0]; dmy = my - M.mu_old[1]; dmz = mz - M.mu_old[2];
                const double mux = sh.sc[SC_MU_X], muy = sh.sc[SC_MU_Y], muz = sh.sc[SC_MU_Z];
                // EwaldSumExternal_calc_dU (EwaldSumExternal.f90:68-82)
                du_ext = D.kext * ((2 * mux + dmx) * dmx + (2 * muy + dmy) * dmy + (2 * muz + dmz) * dmz);
                double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
                if (biased) {
                    double fx[kMaxA], fy[kMaxA], fz[kMaxA], x[kMaxA], y[kMaxA], z[kMaxA];
                    for (int a = 0; a < na; ++a) {
                        const double q = M.slot[a].q;
                        fx[a] = sh.tot[RV_F + 3 * a] + D.m2k * q * (mux + dmx);
                        fy[a] = sh.tot[RV_F + 3 * a + 1] + D.m2k * q * (muy + dmy);
                        fz[a] = sh.tot[RV_F + 3 * a + 2] + D.m2k * q * (muz + dmz);
                        x[a] = M.slot[a].x; y[a] = M.slot[a].y; z[a] = M.slot[a].z;
                    }
                    mol_force_torque(na, x, y, z, M.mass, fx, fy, fz, F, T);
                }
                const double du_total = du_real + (du_kc + du_kl) + du_ext;
                MoveState mv = M.mv;
                mcm_init_new(mv, F, T, D.xlf, D.xlc, D.dr, D.d_angle);
                acc = mcm_accept(mv, du_total, D.xlf, D.xlc, rng);
                out = rng.out != 0;
                cur_after = rng.cur;
                flags |= acc;
            }
            sh.accepted = 0;
            if (out) {
                sh.abort = 1;  // the interrupted move restarts from its first draw (sh.cursor unchanged)
            } else {
                sh.accepted = acc;
                if (acc) {
                    sh.sc[SC_UU_EW] += dew; sh.sc[SC_UU_LJ6] += dlj6; sh.sc[SC_UU_LJ12] += dlj12;
                    sh.sc[SC_EK_C] += du_kc; sh.sc[SC_EK_LJ] += du_kl;
                    sh.sc[SC_MU_X] += dmx; sh.sc[SC_MU_Y] += dmy; sh.sc[SC_MU_Z] += dmz;
                    sh.sc[SC_N_MV_ACC] += 1.0;
                    sh.last_mol = M.imol - 1;
                    for (int a = 0; a < na; ++a) { sh.lx[a] = M.slot[a].x; sh.ly[a] = M.slot[a].y; sh.lz[a] = M.slot[a].z; }
                    // this CTA's staged copy of the moved atoms; every reader of the old copy (this
                    // move's pass, the candidates prepared during it, in any CTA) has passed the barriers
                    for (int a = 0; a < na; ++a) {
                        const int j = M.first + a;
                        if (j % G == rank) {
                            double4 p = atom_s[j / G];
                            p.x = M.slot[a].x; p.y = M.slot[a].y; p.z = M.slot[a].z;
                            atom_s[j / G] = p;
                        }
                    }
                    ++n_acc;
                }
                sh.sc[SC_N_MV_STEPS] += 1.0;
                sh.cursor = cur_after;
                if (rank == 0) {
                    if (acc)
                        for (int a = 0; a < na; ++a) {
                            double4 p = D.atom[M.first + a];
                            p.x = M.slot[a].x; p.y = M.slot[a].y; p.z = M.slot[a].z;
                            D.atom[M.first + a] = p;
                        }
                    if (run->log) {
                        yamc_move_record rec;
                        rec.imol = M.imol; rec.flags = flags; rec.cursor = cur_after;
                        rec.du_real = du_real; rec.du_k_coul = du_kc; rec.du_k_lj = du_kl; rec.du_ext = du_ext;
                        run->log[it] = rec;
                    }
                }
                // cycle bookkeeping and energy.dat rows (runmc.f90:230-279)
                sh.mic += 1;
                if (sh.mic == D.M) {
                    sh.mic = 0;
                    const double fr = sh.sc[SC_N_MV_STEPS] / D.M + sh.sc[SC_N_VOL_STEPS];
                    if (fmod(fr, D.n_store_energy_interval) < 1e-10 && rank == 0 && run->rows && rows < run->max_rows) {
                        const double *sc = sh.sc;
                        const double uext = D.kext * (sc[SC_MU_X] * sc[SC_MU_X] + sc[SC_MU_Y] * sc[SC_MU_Y] + sc[SC_MU_Z] * sc[SC_MU_Z]);
                        const double utew = sc[SC_UU_EW] + sc[SC_EK_C] + sc[SC_TAIL_C] + uext;
                        const double utlj = sc[SC_UU_LJ12] - sc[SC_UU_LJ6] + sc[SC_EK_LJ] + sc[SC_TAIL_LJ12] - sc[SC_TAIL_LJ6];
                        double *row = run->rows + 9 * (size_t)rows;
                        row[0] = (double)sh.icycle; row[1] = utew + utlj; row[2] = utew; row[3] = utlj;
                        row[4] = sc[SC_UU_EW]; row[5] = sc[SC_UU_LJ6]; row[6] = sc[SC_UU_LJ12];
                        row[7] = sc[SC_EK_C]; row[8] = sc[SC_EK_LJ];
                        ++rows;
                    }
                    sh.icycle += 1;
                }
                // the next move: the prepared candidate that matches what happened
                sh.spec_ok = 0;
                if (speculate && it + 1 < n_moves) {
                    const int sel = overlap ? 0 : ((acc && sh.cand[sh.spec[2]].imol == M.imol) ? 2 : 1);
                    const int buf = sh.spec[sel];
                    const Cand &C = sh.cand[buf];
                    if (C.valid && C.cur_start == sh.cursor) {
                        sh.icur = buf;
                        sh.spec_ok = 1;
                    }
                }
            }
        }
        __syncthreads();
        YAMC_PH(PH_DECIDE);
        if (sh.abort) break;
        if (sh.accepted) {
            // commit: rho += delta (MC.f90:1245), in registers or in memory by the entry's owner
#pragma unroll
            for (int k = 0; k < EPT; ++k)
#pragma unroll
                for (int t = 0; t <= NT; ++t) { R.rho[k][t].x += R.dl[k][t].x; R.rho[k][t].y += R.dl[k][t].y; }
            if constexpr (EPT <= 0) {
                if (!ctl) {
                    const double2 *dl_g = D.scratch + (size_t)(1 + NT) * S;
                    for (int e = e0; e < S; e += gwork)
#pragma unroll
                        for (int t = 0; t <= NT; ++t) {
                            double2 r = D.rho[(size_t)t * S + e];
                            const double2 d = dl_g[(size_t)t * S + e];
                            r.x += d.x; r.y += d.y;
                            D.rho[(size_t)t * S + e] = r;
                        }
                }
            }
        }
        ++moves_done;
        have_next = sh.spec_ok != 0;
        __syncthreads();
        YAMC_PH(PH_COMMIT);
    }
#undef YAMC_PH

    if (A.mode == MODE_RUN) {  // write back the register and shared state
#pragma unroll
        for (int k = 0; k < EPT; ++k)
            if (R.e[k] >= 0) {
#pragma unroll
                for (int t = 0; t <= NT; ++t) D.rho[(size_t)t * S + R.e[k]] = R.rho[k][t];
            }
        if (tid == 0 && rank == 0) {
            for (int c = 0; c < SC_COUNT; ++c) D.scal[c] = sh.sc[c];
            D.cnt[CN_ICYCLE] = sh.icycle;
            D.cnt[CN_MOVE_IN_CYCLE] = sh.mic;
            run->cursor = sh.cursor;
            run->moves_done = moves_done;
            run->n_rows = rows;
            run->accepted = n_acc;
            run->status = sh.abort ? YAMC_ERNG_EXHAUSTED : YAMC_OK;
        }
    } else if (tid == 0 && rank == 0) {
        run->moves_done = moves_done;
        run->status = YAMC_OK;
    }
    if (G > 1) cluster.sync();  // no CTA leaves while another may still address its shared memory
}

// ------------------------------------------------------------------------------------------
// adjoint: forces = -dE/dr of the implemented total energy
// ------------------------------------------------------------------------------------------
// Real space: one thread per atom i over all j (tiles in shared memory, increasing j), every
// pair inside the cutoff, intra-molecular pairs with the -erf_Luc energy; F_i += FR (r_i - r_j).
__global__ void __launch_bounds__(kFullTile) k_forces_real(DevSys D, double *fx, double *fy, double *fz) {
    __shared__ double4 tp[kFullTile];
    __shared__ int2 tm[kFullTile];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < D.N;
    double4 pi = make_double4(0, 0, 0, 0);
    int2 mi = make_int2(-1, 0);
    if (valid) { pi = D.atom[i]; mi = D.meta[i]; }
    double gx = 0, gy = 0, gz = 0;
    const int nt = D.nt;
    for (int t0 = 0; t0 < D.N; t0 += kFullTile) {
        const int j = t0 + threadIdx.x;
        if (j < D.N) { tp[threadIdx.x] = D.atom[j]; tm[threadIdx.x] = D.meta[j]; }
        __syncthreads();
        const int nj = min(kFullTile, D.N - t0);
        if (valid) {
            for (int jj = 0; jj < nj; ++jj) {
                if (t0 + jj == i) continue;
                const double4 pj = tp[jj];
                const int2 mj = tm[jj];
                const double dx = min_image(pi.x - pj.x), dy = min_image(pi.y - pj.y), dz = min_image(pi.z - pj.z);
                const double r2 = dx * dx + dy * dy + dz * dz;
                if (r2 >= D.rmax2) continue;
                const bool lj = mi.y > 0 && mj.y > 0;
                const int off = lj ? (mi.y - 1) * nt + (mj.y - 1) : 0;
                const double FR = pair_force_adjoint<double>(r2, D.xclb * pi.w * pj.w, lj, lj ? D.lj_sig6[off] : 0.0,
                                                             lj ? D.lj_feps[off] : 0.0, D.alpha, mi.x == mj.x);
                gx = gx + dx * FR; gy = gy + dy * FR; gz = gz + dz * FR;
            }
        }
        __syncthreads();
    }
    if (valid) { fx[i] = gx; fy[i] = gy; fz[i] = gz; }
}

// k space (ForceKSpace_coulomb / _LJ, ForceKSpace.f90:59-302, over the signed entries): one
// warp per atom, the lanes over the entries; sin/cos(k r) come from the atom's per-axis tables,
// recomputed here instead of stored per atom and k.  Adds to fx/fy/fz.
constexpr int kForceAtoms = 8;  // atoms (warps) per block

template <int NT>
__global__ void __launch_bounds__(32 * kForceAtoms) k_forces_kspace(DevSys D, double *fx, double *fy, double *fz) {
    extern __shared__ double2 ftab[];  // [kForceAtoms][3][KM]
    const int KM = D.kmax + 1;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i = blockIdx.x * kForceAtoms + w;
    if (i >= D.N) return;
    const double4 p = D.atom[i];
    const int ta = D.meta[i].y;
    double2 *T = ftab + (size_t)w * 3 * KM;
    for (int idx = lane; idx < 3 * KM; idx += 32) {
        const int d = idx / KM, m = idx % KM;
        const double u = d == 0 ? p.x : (d == 1 ? p.y : p.z);
        double sn, cs;
        sincospi(2.0 * (double)m * u, &sn, &cs);
        if (m == 0) { sn = 0.0; cs = 1.0; }
        T[idx] = make_double2(cs, sn);
    }
    __syncwarp();
    const double q = p.w, iq = q != 0.0 ? 1.0 / q : 0.0;
    const int S = D.S;
    double gx = 0, gy = 0, gz = 0;
    for (int e = lane; e < S; e += 32) {
        const int4 kv = D.kvec[e];
        double c = 0, sn = 0;
        double wgt = 0;
        if (q != 0.0) {
            entry_phase<double, double2>(T, T + KM, T + 2 * KM, kv.x, kv.y, kv.z, q, c, sn);
            const double2 C = D.rho[e];
            wgt = D.ebeta[e] * (C.x * sn - C.y * c);
        }
        if (ta > 0) {
            double cl, sl;
            if (q != 0.0) { cl = c * iq; sl = sn * iq; }
            else entry_phase<double, double2>(T, T + KM, T + 2 * KM, kv.x, kv.y, kv.z, 1.0, cl, sl);
#pragma unroll
            for (int t = 0; t < NT; ++t) {
                int pr = 0;
#pragma unroll
                for (int u = 0; u < NT; ++u)
                    if (u == ta - 1) pr = pair_idx<NT>(u, t);
                const double2 Ct = D.rho[(size_t)(1 + t) * S + e];
                wgt += D.ebetalj[(size_t)pr * S + e] * (Ct.x * sl - Ct.y * cl);
            }
        }
        const double f = kFourPi * wgt;
        gx = gx + f * kv.x; gy = gy + f * kv.y; gz = gz + f * kv.z;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gx += __shfl_xor_sync(0xffffffffu, gx, o);
        gy += __shfl_xor_sync(0xffffffffu, gy, o);
        gz += __shfl_xor_sync(0xffffffffu, gz, o);
    }
    if (lane == 0) { fx[i] += gx; fy[i] += gy; fz[i] += gz; }
}

// per-move API commit: rho += delta (Step 14, MC.f90:1245)
__global__ void k_commit_rho(double2 *rho, const double2 *delta, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { double2 r = rho[i]; const double2 d = delta[i]; r.x += d.x; r.y += d.y; rho[i] = r; }
}

}  // namespace yamc

// ==========================================================================================
// host side: context, launches and the C ABI
// ==========================================================================================
using namespace yamc;

namespace {

#define CUDA_TRY(expr)                                                                        \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess) {                                                              \
            set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));                    \
            return YAMC_ECUDA;                                                                \
        }                                                                                     \
    } while (0)

template <class T>
int dalloc(T **p, size_t n) {
    *p = nullptr;
    if (n == 0) n = 1;
    CUDA_TRY(cudaMalloc((void **)p, n * sizeof(T)));
    return YAMC_OK;
}

template <class T>
int upload(T *d, const T *h, size_t n, cudaStream_t s) {
    if (n) CUDA_TRY(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return YAMC_OK;
}

struct LaunchCfg {
    int G = 0, B = 0, EPT = 0;
    int nown_max = 0, qcap = 0;
    size_t smem = 0;
};

size_t chain_smem_bytes(int G, int B, int kmax, int nt, int nown_max, int qcap) {
    const int KM = kmax + 1;
    size_t b = sizeof(double2) * 2 * kMaxA * 3 * KM;
    b += (sizeof(double4) + sizeof(double) + sizeof(int2)) * (size_t)nown_max;
    b += sizeof(int) * (size_t)((qcap + 1) & ~1);
    b += sizeof(int) * (size_t)B * kCPT;
    b += sizeof(double) * (size_t)(B / 32) * kNV;
    b += sizeof(double) * (size_t)2 * G * kNV;
    b += sizeof(double) * (size_t)2 * nt * nt;
    return b;
}

}  // namespace

struct yamc_ctx {
    HostSystem H;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    float last_ms = 0.f;
    // device state
    double4 *atom = nullptr;
    int2 *meta = nullptr, *mol = nullptr;
    double *dhs = nullptr, *mass = nullptr, *ebeta = nullptr, *ebetalj = nullptr, *lj_sig6 = nullptr, *lj_feps = nullptr;
    int4 *kvec = nullptr;
    int *pair_index = nullptr;
    double2 *rho = nullptr, *scratch = nullptr;
    double *freq_beg = nullptr, *freq_end = nullptr, *scal = nullptr;
    long long *cnt = nullptr;
    int4 *spec = nullptr;
    double *uu = nullptr, *fx = nullptr, *fy = nullptr, *fz = nullptr, *part = nullptr;
    DevSys hsys{};
    DevSys *d_sys = nullptr;
    RunSlot *d_run = nullptr;
    double *api_in = nullptr, *api_out = nullptr;
    float *d_rng = nullptr;
    size_t rng_cap = 0;
    yamc_move_record *d_log = nullptr;
    size_t log_cap = 0;
    double *d_rows = nullptr;
    int rows_cap = 0;
    // host mirrors
    double sc[SC_COUNT] = {};
    long long cnt_h[CN_COUNT] = {};
    bool pos_valid = true;  // H.x/y/z mirror the device positions
    LaunchCfg cfg;
    int force_G = 0, force_B = 0, force_layout = YAMC_KSPACE_AUTO;
    // per-move API state
    int api_imol = 0, api_stage = 0;
    double api_eold[3] = {}, api_fold[3 * kMaxA] = {};
    double api_new[kNV] = {};
    double api_xn[kMaxA] = {}, api_yn[kMaxA] = {}, api_zn[kMaxA] = {};
    double api_dmu[3] = {};
    long long *d_prof = nullptr;
    bool prof_on = false;
    double *d_gx = nullptr, *d_gy = nullptr, *d_gz = nullptr;  // adjoint forces
};

namespace {

// The first (G, B) that fits every system of hosts: each worker thread holds at most 2 signed
// entries, the CTA's atoms and the pair queue fit in shared memory.  G (1..16 CTAs per cluster)
// from large to small when large_first (the shortest move for a lone chain), else from small to
// large; B from 256 to 128 threads; force_G / force_B pin either (0 = free).
int pick_launch_for(const std::vector<const HostSystem *> &hosts, int device, int force_G, int force_B, int layout,
                    LaunchCfg *out, bool large_first = true) {
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    const size_t smem_max = prop.sharedMemPerBlockOptin - sizeof(ChainShared) - 1024;
    int Smax = 0, Nmax = 0, Nmin = 1 << 30, kmax = 0, nt = 0;
    for (const HostSystem *h : hosts) {
        Smax = std::max(Smax, h->S); Nmax = std::max(Nmax, h->N); Nmin = std::min(Nmin, h->N);
        kmax = std::max(kmax, h->kmax); nt = std::max(nt, h->nt);
    }
    const int Bs[] = {kChainMaxThreads, kChainMaxThreadsWide, 128};  // unforced: 256 only
    for (int gi = 0; gi < 16; ++gi) {
        const int G = large_first ? 16 - gi : 1 + gi;
        if (force_G && G != force_G) continue;
        if (G > Nmin) continue;  // every CTA owns at least one atom
        for (int bi = 0; bi < 3; ++bi) {
            const int B = Bs[bi];
            if (force_B ? B != force_B : B != kChainMaxThreads) continue;
            const int nwork = B - kCtl;  // warp 0 is the control warp
            int EPT = (Smax + G * nwork - 1) / (G * nwork);
            // entries in registers (at most 2 per worker) or streamed from memory (EPT 0; EPT -1
            // for 512-thread CTAs, which only the streamed layout runs)
            if (layout == YAMC_KSPACE_STREAMED || (layout == YAMC_KSPACE_AUTO && EPT > 2)) EPT = 0;
            if (B > kChainMaxThreads) {
                if (layout == YAMC_KSPACE_REGISTERS) continue;
                EPT = -1;
            }
            if (EPT > 2) continue;
            const int nown_max = (Nmax + G - 1) / G;
            const int qcap = std::min(nown_max, nwork * kCPT) * 2 * kMaxA;  // one filter round of pairs
            const size_t sm = chain_smem_bytes(G, B, kmax, nt, nown_max, qcap);
            if (sm > smem_max) continue;
            out->G = G; out->B = B; out->EPT = EPT; out->nown_max = nown_max; out->qcap = qcap; out->smem = sm;
            return YAMC_OK;
        }
    }
    set_error("no launch configuration fits this system (k-set or atoms too large for one cluster)");
    return YAMC_ELIMITS;
}

int pick_launch(yamc_ctx *c, LaunchCfg *out) {
    return pick_launch_for({&c->H}, c->device, c->force_G, c->force_B, c->force_layout, out);
}

// nrep chains of one launch shape: nrep clusters of L.G CTAs, chain r on cluster r
template <int NT, int EPT, bool SPLIT>
int launch_chain_t(const LaunchCfg &L, cudaStream_t stream, int nrep, const ChainArgs &args) {
    auto kfn = k_chain<NT, EPT, SPLIT>;
    CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
    if (L.G > 8) CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(L.G * nrep, 1, 1);
    cfg.blockDim = dim3(L.B, 1, 1);
    cfg.dynamicSmemBytes = L.smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = L.G;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUDA_TRY(cudaLaunchKernelEx(&cfg, kfn, args));
    return YAMC_OK;
}

// clusters of shape L that can be resident at once (0 if the shape does not launch)
template <int NT, int EPT, bool SPLIT>
int max_clusters_t(const LaunchCfg &L, int *out) {
    auto kfn = k_chain<NT, EPT, SPLIT>;
    CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem));
    if (L.G > 8) CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(L.G, 1, 1);
    cfg.blockDim = dim3(L.B, 1, 1);
    cfg.dynamicSmemBytes = L.smem;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = L.G;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    CUDA_TRY(cudaOccupancyMaxActiveClusters(out, kfn, &cfg));
    return YAMC_OK;
}

// kernel instance for (LJ types, entries per thread, split old pass); WHAT(NT, EPT, SPLIT) is
// a call of a template above
#ifdef YAMC_ONE_VARIANT  // development builds: a single instantiation compiles in seconds
#define YAMC_CHAIN_VARIANTS(X) X(3, -1) X(3, 0) X(3, 1) X(3, 2)
#else
#define YAMC_CHAIN_VARIANTS(X) \
    X(1, -1) X(1, 0) X(1, 1) X(1, 2) X(2, -1) X(2, 0) X(2, 1) X(2, 2) \
    X(3, -1) X(3, 0) X(3, 1) X(3, 2) X(4, -1) X(4, 0) X(4, 1) X(4, 2)
#endif

int launch_chain_cfg(const LaunchCfg &L, int nt, bool split, cudaStream_t stream, int nrep, const ChainArgs &args) {
#define YAMC_CASE(NT_, EPT_)                                                                                  \
    if (nt == NT_ && L.EPT == EPT_)                                                                            \
        return split ? launch_chain_t<NT_, EPT_, true>(L, stream, nrep, args)                                  \
                     : launch_chain_t<NT_, EPT_, false>(L, stream, nrep, args);
    YAMC_CHAIN_VARIANTS(YAMC_CASE)
#undef YAMC_CASE
    set_error("LJ type count outside 1..4 or k-set too large for the chain kernel");
    return YAMC_ELIMITS;
}

int max_clusters_cfg(const LaunchCfg &L, int nt, bool split, int *out) {
#define YAMC_CASE(NT_, EPT_)                                                                                  \
    if (nt == NT_ && L.EPT == EPT_) return split ? max_clusters_t<NT_, EPT_, true>(L, out) : max_clusters_t<NT_, EPT_, false>(L, out);
    YAMC_CHAIN_VARIANTS(YAMC_CASE)
#undef YAMC_CASE
    set_error("LJ type count outside 1..4 or k-set too large for the chain kernel");
    return YAMC_ELIMITS;
}

bool split_variant(const HostSystem &H, int mode) {
    return mode != MODE_RUN || H.p.xlambda_f > 0.0 || H.p.xlambda_c > 0.0;
}

int launch_chain(yamc_ctx *c, const ChainArgs &args) {
    return launch_chain_cfg(c->cfg, c->H.nt, split_variant(c->H, args.mode), c->stream, 1, args);
}

template <int NT>
int launch_rho_full(yamc_ctx *c) {
    const int KM = c->H.kmax + 1;
    const size_t sm = sizeof(double2) * kRhoChunk * 3 * KM;
    CUDA_TRY(cudaFuncSetAttribute(k_rho_full<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_rho_full<NT><<<(c->H.S + kRhoBlock - 1) / kRhoBlock, kRhoBlock, sm, c->stream>>>(c->hsys, c->rho);
    CUDA_TRY(cudaGetLastError());
    return YAMC_OK;
}

template <int NT>
int launch_kspace_energy(yamc_ctx *c, int nb) {
    k_kspace_energy<NT><<<nb, 256, 0, c->stream>>>(c->hsys, c->rho, c->part);
    CUDA_TRY(cudaGetLastError());
    return YAMC_OK;
}

int sync_positions(yamc_ctx *c) {
    if (c->pos_valid) return YAMC_OK;
    std::vector<double4> a(c->H.N);
    CUDA_TRY(cudaMemcpyAsync(a.data(), c->atom, sizeof(double4) * c->H.N, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int i = 0; i < c->H.N; ++i) { c->H.x[i] = a[i].x; c->H.y[i] = a[i].y; c->H.z[i] = a[i].z; }
    c->pos_valid = true;
    return YAMC_OK;
}

int pull_state(yamc_ctx *c) {
    CUDA_TRY(cudaMemcpyAsync(c->sc, c->scal, sizeof(double) * SC_COUNT, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->cnt_h, c->cnt, sizeof(long long) * CN_COUNT, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return YAMC_OK;
}

int push_state(yamc_ctx *c) {
    CUDA_TRY(cudaMemcpyAsync(c->scal, c->sc, sizeof(double) * SC_COUNT, cudaMemcpyHostToDevice, c->stream));
    CUDA_TRY(cudaMemcpyAsync(c->cnt, c->cnt_h, sizeof(long long) * CN_COUNT, cudaMemcpyHostToDevice, c->stream));
    return YAMC_OK;
}

// mc_calc_total_sums (MC.f90:477-585) on the device
int full_sums(yamc_ctx *c) {
    HostSystem &H = c->H;
    int r = sync_positions(c);
    if (r) return r;
    const int nbr = (H.N + kFullTile - 1) / kFullTile;
    k_realspace_full<<<nbr, kFullTile, 0, c->stream>>>(c->hsys, c->uu, c->fx, c->fy, c->fz, c->part);
    CUDA_TRY(cudaGetLastError());
    std::vector<double> pr((size_t)nbr * kFullParts);
    CUDA_TRY(cudaMemcpyAsync(pr.data(), c->part, sizeof(double) * pr.size(), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    double tot[kFullParts] = {};
    for (int b = 0; b < nbr; ++b)
        for (int v = 0; v < kFullParts; ++v) tot[v] = (v == 6) ? std::max(tot[v], pr[b * kFullParts + v]) : tot[v] + pr[b * kFullParts + v];
    if (tot[6] > 0) { set_error("hard-core overlap in the configuration"); return YAMC_EOVERLAP_INIT; }
    switch (H.nt) {
        case 1: r = launch_rho_full<1>(c); break;
        case 2: r = launch_rho_full<2>(c); break;
        case 3: r = launch_rho_full<3>(c); break;
        case 4: r = launch_rho_full<4>(c); break;
        default: set_error("LJ type count outside 1..4"); return YAMC_ELIMITS;
    }
    if (r) return r;
    const int nbk = (H.S + 255) / 256;
    switch (H.nt) {
        case 1: r = launch_kspace_energy<1>(c, nbk); break;
        case 2: r = launch_kspace_energy<2>(c, nbk); break;
        case 3: r = launch_kspace_energy<3>(c, nbk); break;
        default: r = launch_kspace_energy<4>(c, nbk); break;
    }
    if (r) return r;
    std::vector<double> pk((size_t)nbk * 2);
    CUDA_TRY(cudaMemcpyAsync(pk.data(), c->part, sizeof(double) * pk.size(), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    double ekc = 0, ekl = 0;
    for (int b = 0; b < nbk; ++b) { ekc += pk[2 * b]; ekl += pk[2 * b + 1]; }
    // EwaldSumExternal_calc_mu over all atoms, in atom order (EwaldSumExternal.f90:34-52)
    double mx = 0, my = 0, mz = 0;
    for (int i = 0; i < H.N; ++i) { mx = mx + H.q[i] * H.x[i]; my = my + H.q[i] * H.y[i]; mz = mz + H.q[i] * H.z[i]; }
    c->sc[SC_UU_EW] = tot[0]; c->sc[SC_UU_LJ6] = tot[1]; c->sc[SC_UU_LJ12] = tot[2];
    c->sc[SC_UU_EW_INTRA] = tot[3]; c->sc[SC_UU_LJ6_INTRA] = tot[4]; c->sc[SC_UU_LJ12_INTRA] = tot[5];
    c->sc[SC_EK_C] = ekc; c->sc[SC_EK_LJ] = ekl;
    c->sc[SC_MU_X] = mx; c->sc[SC_MU_Y] = my; c->sc[SC_MU_Z] = mz;
    c->sc[SC_TAIL_C] = H.U_tail_coul; c->sc[SC_TAIL_LJ6] = H.U_tail_lj6; c->sc[SC_TAIL_LJ12] = H.U_tail_lj12;
    return push_state(c);
}

// mc_total_energy (MC.f90:681-698) from the engine scalars
void energies_from(const double *sc, double kext, double e[8]) {
    const double uext = kext * (sc[SC_MU_X] * sc[SC_MU_X] + sc[SC_MU_Y] * sc[SC_MU_Y] + sc[SC_MU_Z] * sc[SC_MU_Z]);
    const double utew = sc[SC_UU_EW] + sc[SC_EK_C] + sc[SC_TAIL_C] + uext;
    const double utlj = sc[SC_UU_LJ12] - sc[SC_UU_LJ6] + sc[SC_EK_LJ] + sc[SC_TAIL_LJ12] - sc[SC_TAIL_LJ6];
    e[0] = utew + utlj; e[1] = utew; e[2] = utlj;
    e[3] = sc[SC_UU_EW]; e[4] = sc[SC_UU_LJ6]; e[5] = sc[SC_UU_LJ12]; e[6] = sc[SC_EK_C]; e[7] = sc[SC_EK_LJ];
}

int ensure_cfg(yamc_ctx *c) {
    if (c->cfg.G) return YAMC_OK;
    return pick_launch(c, &c->cfg);
}

template <int NT>
int launch_forces_kspace(yamc_ctx *c) {
    const size_t sm = sizeof(double2) * kForceAtoms * 3 * (c->H.kmax + 1);
    CUDA_TRY(cudaFuncSetAttribute(k_forces_kspace<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_forces_kspace<NT><<<(c->H.N + kForceAtoms - 1) / kForceAtoms, 32 * kForceAtoms, sm, c->stream>>>(c->hsys, c->d_gx,
                                                                                                      c->d_gy, c->d_gz);
    CUDA_TRY(cudaGetLastError());
    return YAMC_OK;
}

ChainArgs base_args(yamc_ctx *c, int mode) {
    ChainArgs a{};
    a.sys = c->d_sys; a.run = c->d_run; a.G = c->cfg.G; a.mode = mode;
    a.nown_max = c->cfg.nown_max; a.qcap = c->cfg.qcap;
    a.api_in = c->api_in; a.api_out = c->api_out; a.scratch = c->scratch;
    a.prof = c->prof_on ? c->d_prof : nullptr;
    return a;
}

}  // namespace

// A batch: independent replicas (each a yamc_ctx with its own system and device state),
// grouped by kernel variant (LJ type count, split old pass); each group is one cluster launch,
// the groups run concurrently on their own streams, and the whole step is one CUDA graph.
namespace {
struct BatchGroup {
    std::vector<int> idx;       // replicas of the group
    int nt = 0;
    bool split = false;
    LaunchCfg cfg;
    int max_clusters = 0;       // resident at once for cfg
    DevSys *d_sys = nullptr;    // [n]
    RunSlot *d_run = nullptr;   // [n]
    RunSlot *h_run = nullptr;   // [n], pinned
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
};
}  // namespace

struct yamc_batch {
    int device = 0;
    std::vector<yamc_ctx *> reps;
    std::vector<BatchGroup> groups;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, fork = nullptr;
    cudaGraphExec_t graph = nullptr;
    float last_ms = 0.f;
    int force_G = 0, force_B = 0, force_layout = YAMC_KSPACE_AUTO;
    float *d_rng = nullptr;
    size_t rng_cap = 0;
    yamc_move_record *d_log = nullptr;
    size_t log_cap = 0;
};

namespace {

void batch_drop_graph(yamc_batch *b) {
    if (b->graph) cudaGraphExecDestroy(b->graph);
    b->graph = nullptr;
}

// launch shape of every group for the current force_G / force_B
int batch_configure(yamc_batch *b) {
    batch_drop_graph(b);
    for (BatchGroup &g : b->groups) {
        std::vector<const HostSystem *> hs;
        for (int i : g.idx) hs.push_back(&b->reps[i]->H);
        int r = pick_launch_for(hs, b->device, b->force_G, b->force_B, b->force_layout, &g.cfg);
        if (r) return r;
        if ((r = max_clusters_cfg(g.cfg, g.nt, g.split, &g.max_clusters))) return r;
    }
    return YAMC_OK;
}

// one batch step as a graph: run slots up, every group's launch (concurrently), run slots down
int batch_build_graph(yamc_batch *b) {
    if (b->graph) return YAMC_OK;
    cudaGraph_t graph = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeRelaxed));
    int r = YAMC_OK;
    for (BatchGroup &g : b->groups) {
        if (cudaMemcpyAsync(g.d_run, g.h_run, sizeof(RunSlot) * g.idx.size(), cudaMemcpyHostToDevice, b->stream) != cudaSuccess) {
            r = YAMC_ECUDA; break;
        }
    }
    if (!r && cudaEventRecord(b->fork, b->stream) != cudaSuccess) r = YAMC_ECUDA;
    for (size_t k = 0; !r && k < b->groups.size(); ++k) {
        BatchGroup &g = b->groups[k];
        if (cudaStreamWaitEvent(g.stream, b->fork, 0) != cudaSuccess) { r = YAMC_ECUDA; break; }
        ChainArgs a{};
        a.sys = g.d_sys; a.run = g.d_run; a.G = g.cfg.G; a.mode = MODE_RUN;
        a.nown_max = g.cfg.nown_max; a.qcap = g.cfg.qcap;
        if ((r = launch_chain_cfg(g.cfg, g.nt, g.split, g.stream, (int)g.idx.size(), a))) break;
        if (cudaEventRecord(g.done, g.stream) != cudaSuccess || cudaStreamWaitEvent(b->stream, g.done, 0) != cudaSuccess)
            r = YAMC_ECUDA;
    }
    for (size_t k = 0; !r && k < b->groups.size(); ++k) {
        BatchGroup &g = b->groups[k];
        if (cudaMemcpyAsync(g.h_run, g.d_run, sizeof(RunSlot) * g.idx.size(), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess)
            r = YAMC_ECUDA;
    }
    const cudaError_t ee = cudaStreamEndCapture(b->stream, &graph);
    if (r) {
        if (graph) cudaGraphDestroy(graph);
        if (r == YAMC_ECUDA) set_error("capturing the batch step failed");
        return r;
    }
    CUDA_TRY(ee);
    const cudaError_t ei = cudaGraphInstantiate(&b->graph, graph, 0);
    cudaGraphDestroy(graph);
    CUDA_TRY(ei);
    return YAMC_OK;
}

// one step of every replica: replica i's stream holds positions [rng_off[i], n_rng[i]) at rng[i]
int batch_step(yamc_batch *b, const float *const *rng, const int64_t *rng_off, const int64_t *n_rng,
               int64_t *cursors, int64_t n_moves, int64_t *moves_done, int32_t *status, yamc_move_record *d_log) {
    int r = batch_build_graph(b);
    if (r) return r;
    for (BatchGroup &g : b->groups)
        for (size_t k = 0; k < g.idx.size(); ++k) {
            const int i = g.idx[k];
            RunSlot &rs = g.h_run[k];
            rs = RunSlot{};
            rs.rng = rng[i]; rs.rng_off = rng_off[i]; rs.n_rng = n_rng[i];
            rs.cursor = cursors[i]; rs.n_moves = n_moves;
            rs.log = d_log ? d_log + (size_t)i * n_moves : nullptr;
        }
    CUDA_TRY(cudaEventRecord(b->ev0, b->stream));
    CUDA_TRY(cudaGraphLaunch(b->graph, b->stream));
    CUDA_TRY(cudaEventRecord(b->ev1, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
    int worst = YAMC_OK;
    for (BatchGroup &g : b->groups)
        for (size_t k = 0; k < g.idx.size(); ++k) {
            const int i = g.idx[k];
            const RunSlot &rs = g.h_run[k];
            cursors[i] = rs.cursor;
            if (moves_done) moves_done[i] = rs.moves_done;
            if (status) status[i] = rs.status;
            b->reps[i]->pos_valid = false;
            if (rs.status != YAMC_OK && (worst == YAMC_OK || worst == YAMC_ERNG_EXHAUSTED)) worst = rs.status;
        }
    return worst;
}

// device copies of the chain state of every replica (positions, rho, scalars, counters)
struct BatchBackup {
    std::vector<double4 *> atom;
    std::vector<double2 *> rho;
    std::vector<double *> scal;
    std::vector<long long *> cnt;
    ~BatchBackup() {
        for (auto p : atom) if (p) cudaFree(p);
        for (auto p : rho) if (p) cudaFree(p);
        for (auto p : scal) if (p) cudaFree(p);
        for (auto p : cnt) if (p) cudaFree(p);
    }
};

int batch_copy_state(yamc_batch *b, BatchBackup &k, bool save) {
    const size_t R = b->reps.size();
    if (save) { k.atom.assign(R, nullptr); k.rho.assign(R, nullptr); k.scal.assign(R, nullptr); k.cnt.assign(R, nullptr); }
    for (size_t i = 0; i < R; ++i) {
        yamc_ctx *c = b->reps[i];
        const size_t nr = (size_t)(1 + c->H.nt) * c->H.S;
        int r;
        if (save && ((r = dalloc(&k.atom[i], c->H.N)) || (r = dalloc(&k.rho[i], nr)) || (r = dalloc(&k.scal[i], SC_COUNT)) ||
                     (r = dalloc(&k.cnt[i], CN_COUNT))))
            return r;
        const cudaMemcpyKind kd = cudaMemcpyDeviceToDevice;
        if (save) {
            CUDA_TRY(cudaMemcpyAsync(k.atom[i], c->atom, sizeof(double4) * c->H.N, kd, b->stream));
            CUDA_TRY(cudaMemcpyAsync(k.rho[i], c->rho, sizeof(double2) * nr, kd, b->stream));
            CUDA_TRY(cudaMemcpyAsync(k.scal[i], c->scal, sizeof(double) * SC_COUNT, kd, b->stream));
            CUDA_TRY(cudaMemcpyAsync(k.cnt[i], c->cnt, sizeof(long long) * CN_COUNT, kd, b->stream));
        } else {
            CUDA_TRY(cudaMemcpyAsync(c->atom, k.atom[i], sizeof(double4) * c->H.N, kd, b->stream));
            CUDA_TRY(cudaMemcpyAsync(c->rho, k.rho[i], sizeof(double2) * nr, kd, b->stream));
            CUDA_TRY(cudaMemcpyAsync(c->scal, k.scal[i], sizeof(double) * SC_COUNT, kd, b->stream));
            CUDA_TRY(cudaMemcpyAsync(c->cnt, k.cnt[i], sizeof(long long) * CN_COUNT, kd, b->stream));
        }
    }
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return YAMC_OK;
}

}  // namespace

extern "C" {

const char *yamc_error_string(int s) {
    switch (s) {
        case YAMC_OK: return "ok";
        case YAMC_EIO: return "I/O error";
        case YAMC_ELIMITS: return "limits exceeded";
        case YAMC_EPARAMETER: return "bad parameter";
        case YAMC_EINIT: return "not initialised";
        case YAMC_EWRONG_FUNCTION: return "wrong function for this state";
        case YAMC_ECUDA: return "CUDA error";
        case YAMC_ETIMEOUT: return "device wait timed out";
        case YAMC_ERNG_EXHAUSTED: return "random stream exhausted";
        case YAMC_ENAN: return "non-finite value";
        case YAMC_EOVERLAP_INIT: return "hard-core overlap in the initial configuration";
        default: return "unknown status";
    }
}

int yamc_destroy(yamc_ctx *c);

static int create_impl(yamc_ctx *c, const yamc_system *sys, const yamc_params *p, int32_t device) {
    int r = prepare_host_system(sys, p, &c->H);
    if (r) return r;
    HostSystem &H = c->H;
    if (H.nt < 1 || H.nt > 4) { set_error("the device kernels support 1..4 LJ types"); return YAMC_ELIMITS; }
    c->device = device;
    CUDA_TRY(cudaSetDevice(device));
    CUDA_TRY(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreate(&c->ev0));
    CUDA_TRY(cudaEventCreate(&c->ev1));
    const int N = H.N, M = H.M, S = H.S, nt = H.nt;
    if ((r = dalloc(&c->atom, N)) || (r = dalloc(&c->meta, N)) || (r = dalloc(&c->dhs, N)) || (r = dalloc(&c->mass, N)) ||
        (r = dalloc(&c->mol, M)) || (r = dalloc(&c->kvec, S)) || (r = dalloc(&c->ebeta, S)) ||
        (r = dalloc(&c->ebetalj, (size_t)H.npair * S)) || (r = dalloc(&c->pair_index, nt * nt)) ||
        (r = dalloc(&c->lj_sig6, nt * nt)) || (r = dalloc(&c->lj_feps, nt * nt)) || (r = dalloc(&c->rho, (size_t)(1 + nt) * S)) ||
        (r = dalloc(&c->scratch, (size_t)2 * (1 + nt) * S)) || (r = dalloc(&c->freq_beg, M)) || (r = dalloc(&c->freq_end, M)) ||
        (r = dalloc(&c->scal, SC_COUNT)) || (r = dalloc(&c->cnt, CN_COUNT)) || (r = dalloc(&c->uu, N)) ||
        (r = dalloc(&c->fx, N)) || (r = dalloc(&c->fy, N)) || (r = dalloc(&c->fz, N)) ||
        (r = dalloc(&c->part, (size_t)std::max((N + kFullTile - 1) / kFullTile * kFullParts, (S + 255) / 256 * 2))) ||
        (r = dalloc(&c->d_sys, 1)) || (r = dalloc(&c->d_run, 1)) || (r = dalloc(&c->api_in, 1 + 3 * kMaxA)) ||
        (r = dalloc(&c->api_out, kNV)) || (r = dalloc(&c->spec, H.spec.size() / 4)))
        return r;
    std::vector<double4> a(N);
    std::vector<int2> m(N);
    for (int i = 0; i < N; ++i) { a[i] = make_double4(H.x[i], H.y[i], H.z[i], H.q[i]); m[i] = make_int2(H.molnum[i], H.type_by_index[i]); }
    std::vector<int2> mo(M);
    for (int i = 0; i < M; ++i) mo[i] = make_int2(H.first[i], H.natoms[i]);
    std::vector<int4> kv(S);
    for (int e = 0; e < S; ++e) kv[e] = make_int4(H.ekx[e], H.eky[e], H.ekz[e], H.ekk[e]);
    std::vector<int> pidx(nt * nt);
    for (int i = 0; i < nt * nt; ++i) pidx[i] = H.pair_index[i];
    if ((r = upload(c->atom, a.data(), N, c->stream)) || (r = upload(c->meta, m.data(), N, c->stream)) ||
        (r = upload(c->dhs, H.dhs.data(), N, c->stream)) || (r = upload(c->mass, H.mass.data(), N, c->stream)) ||
        (r = upload(c->mol, mo.data(), M, c->stream)) || (r = upload(c->kvec, kv.data(), S, c->stream)) ||
        (r = upload(c->ebeta, H.ebeta.data(), S, c->stream)) || (r = upload(c->ebetalj, H.ebetalj.data(), (size_t)H.npair * S, c->stream)) ||
        (r = upload(c->pair_index, pidx.data(), nt * nt, c->stream)) || (r = upload(c->lj_sig6, H.sigma6.data(), nt * nt, c->stream)) ||
        (r = upload(c->lj_feps, H.four_eps.data(), nt * nt, c->stream)) || (r = upload(c->freq_beg, H.freq_beg.data(), M, c->stream)) ||
        (r = upload(c->freq_end, H.freq_end.data(), M, c->stream)) ||
        (r = upload(c->spec, reinterpret_cast<const int4 *>(H.spec.data()), H.spec.size() / 4, c->stream)))
        return r;
    DevSys &D = c->hsys;
    D.N = N; D.M = M; D.S = S; D.nt = nt; D.kmax = H.kmax; D.npair = H.npair; D.freq_monotone = H.freq_monotone;
    D.n_species = (int)H.mol_numbers.size();
    const yamc_params &P = H.p;
    D.rmax2 = P.rmax2; D.alpha = P.alpha; D.xclb = P.xclb; D.taosp = P.two_alpha_over_sqrt_pi; D.kext = P.kext;
    D.m2k = P.minus_two_kext; D.dr = P.dr; D.d_angle = P.d_angle; D.xlf = P.xlambda_f; D.xlc = P.xlambda_c;
    D.psm = P.pressure_step_multiplier; D.n_store_energy_interval = P.n_store_energy_interval;
    D.rpre = std::sqrt(P.rmax2);
    for (int i = 0; i < N; ++i) D.rpre = std::max(D.rpre, H.dhs[i]);
    D.atom = c->atom; D.meta = c->meta; D.dhs = c->dhs; D.mass = c->mass; D.mol = c->mol; D.kvec = c->kvec;
    D.ebeta = c->ebeta; D.ebetalj = c->ebetalj; D.pair_index = c->pair_index; D.lj_sig6 = c->lj_sig6; D.lj_feps = c->lj_feps;
    D.rho = c->rho; D.scratch = c->scratch; D.freq_beg = c->freq_beg; D.freq_end = c->freq_end; D.scal = c->scal; D.cnt = c->cnt;
    D.nspec = (int)(H.spec.size() / 4); D.spec = c->spec;
    if ((r = upload(c->d_sys, &D, 1, c->stream))) return r;
    c->cnt_h[CN_ICYCLE] = 1;
    c->cnt_h[CN_MOVE_IN_CYCLE] = 0;
    if ((r = full_sums(c))) return r;  // initmc
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return YAMC_OK;
}

int yamc_create(const yamc_system *sys, const yamc_params *p, int32_t device, yamc_ctx **out) {
    if (!out) return YAMC_EPARAMETER;
    *out = nullptr;
    yamc_ctx *c = new yamc_ctx();
    const int r = create_impl(c, sys, p, device);
    if (r) { yamc_destroy(c); return r; }
    *out = c;
    return YAMC_OK;
}

int yamc_destroy(yamc_ctx *c) {
    if (!c) return YAMC_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    void *ptrs[] = {c->atom, c->meta, c->mol, c->dhs, c->mass, c->ebeta, c->ebetalj, c->lj_sig6, c->lj_feps, c->kvec,
                    c->pair_index, c->rho, c->scratch, c->freq_beg, c->freq_end, c->scal, c->cnt, c->uu, c->fx, c->fy,
                    c->fz, c->part, c->d_sys, c->d_run, c->api_in, c->api_out, c->d_rng, c->d_log, c->d_rows,
                    c->d_prof, c->spec, c->d_gx, c->d_gy, c->d_gz};
    for (void *p : ptrs) if (p) cudaFree(p);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return YAMC_OK;
}

int yamc_sizes(yamc_ctx *c, int32_t out[5]) {
    if (!c || !out) return YAMC_EPARAMETER;
    out[0] = c->H.N; out[1] = c->H.M; out[2] = c->H.nk; out[3] = c->H.S; out[4] = c->H.nt;
    return YAMC_OK;
}

int yamc_energies(yamc_ctx *c, double e[8]) {
    if (!c || !e) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    int r = pull_state(c);
    if (r) return r;
    energies_from(c->sc, c->H.p.kext, e);
    return YAMC_OK;
}

int yamc_full_sums(yamc_ctx *c, double e[8]) {
    if (!c) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    int r = pull_state(c);
    if (r) return r;
    if ((r = full_sums(c))) return r;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (e) energies_from(c->sc, c->H.p.kext, e);
    return YAMC_OK;
}

int yamc_get_positions(yamc_ctx *c, double *x, double *y, double *z) {
    if (!c) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    int r = sync_positions(c);
    if (r) return r;
    for (int i = 0; i < c->H.N; ++i) {
        if (x) x[i] = c->H.x[i];
        if (y) y[i] = c->H.y[i];
        if (z) z[i] = c->H.z[i];
    }
    return YAMC_OK;
}

int yamc_set_launch(yamc_ctx *c, int32_t cluster_blocks, int32_t threads) {
    if (!c) return YAMC_EPARAMETER;
    if (cluster_blocks < 0 || cluster_blocks > 16 || threads < 0 || threads > kChainMaxThreadsWide || (threads % 32) ||
        (threads > 0 && threads < 64))
        return YAMC_EPARAMETER;
    const int oG = c->force_G, oB = c->force_B;
    c->force_G = cluster_blocks;
    c->force_B = threads;
    LaunchCfg L;
    const int r = pick_launch(c, &L);
    if (r) { c->force_G = oG; c->force_B = oB; return r; }  // a refused shape changes nothing
    c->cfg = L;
    return YAMC_OK;
}

int yamc_set_kspace_layout(yamc_ctx *c, int32_t layout) {
    if (!c || layout < YAMC_KSPACE_AUTO || layout > YAMC_KSPACE_STREAMED) return YAMC_EPARAMETER;
    const int oL = c->force_layout;
    c->force_layout = layout;
    LaunchCfg L;
    const int r = pick_launch(c, &L);
    if (r) { c->force_layout = oL; return r; }
    c->cfg = L;
    return YAMC_OK;
}

int yamc_get_launch(yamc_ctx *c, int32_t out[4]) {
    if (!c || !out) return YAMC_EPARAMETER;
    int r = ensure_cfg(c);
    if (r) return r;
    out[0] = c->cfg.G; out[1] = c->cfg.B; out[2] = std::max(c->cfg.EPT, 0); out[3] = (int32_t)c->cfg.smem;
    return YAMC_OK;
}

int yamc_last_kernel_ms(yamc_ctx *c, double *ms) {
    if (!c || !ms) return YAMC_EPARAMETER;
    *ms = c->last_ms;
    return YAMC_OK;
}

static int run_chain_impl(yamc_ctx *c, const float *d_rng, long long rng_off, long long n_rng, int64_t *cursor,
                          int64_t n_moves, int64_t *moves_done, yamc_move_record *d_log, double *d_rows, int max_rows,
                          int32_t *n_rows) {
    int r = ensure_cfg(c);
    if (r) return r;
    RunSlot rs{};
    rs.rng = d_rng; rs.rng_off = rng_off; rs.n_rng = n_rng; rs.cursor = *cursor; rs.n_moves = n_moves;
    rs.log = d_log; rs.rows = d_rows; rs.max_rows = max_rows;
    if ((r = upload(c->d_run, &rs, 1, c->stream))) return r;
    ChainArgs a = base_args(c, MODE_RUN);
    CUDA_TRY(cudaEventRecord(c->ev0, c->stream));
    if ((r = launch_chain(c, a))) return r;
    CUDA_TRY(cudaEventRecord(c->ev1, c->stream));
    RunSlot back{};
    CUDA_TRY(cudaMemcpyAsync(&back, c->d_run, sizeof(RunSlot), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    cudaEventElapsedTime(&c->last_ms, c->ev0, c->ev1);
    c->pos_valid = false;
    *cursor = back.cursor;
    if (moves_done) *moves_done = back.moves_done;
    if (n_rows) *n_rows = back.n_rows;
    return back.status;
}

int yamc_run_chain_device(yamc_ctx *c, const float *d_rng, int64_t n_rng, int64_t *cursor, int64_t n_moves,
                          int64_t *moves_done, yamc_move_record *d_log, double *d_rows, int32_t max_rows, int32_t *n_rows) {
    if (!c || !d_rng || !cursor || n_moves < 0) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    return run_chain_impl(c, d_rng, 0, n_rng, cursor, n_moves, moves_done, d_log, d_rows, max_rows, n_rows);
}

int yamc_run_chain(yamc_ctx *c, const float *rng, int64_t n_rng, int64_t *cursor, int64_t n_moves, int64_t *moves_done,
                   yamc_move_record *log, double *rows, int32_t max_rows, int32_t *n_rows) {
    if (!c || !rng || !cursor || n_moves < 0 || *cursor < 0 || *cursor > n_rng) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    const size_t nr = (size_t)(n_rng - *cursor);
    if (nr > c->rng_cap) {
        if (c->d_rng) cudaFree(c->d_rng);
        c->d_rng = nullptr;
        c->rng_cap = 0;
        int r = dalloc(&c->d_rng, nr);
        if (r) return r;
        c->rng_cap = nr;
    }
    CUDA_TRY(cudaMemcpyAsync(c->d_rng, rng + *cursor, nr * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    if (log && (size_t)n_moves > c->log_cap) {
        if (c->d_log) cudaFree(c->d_log);
        c->d_log = nullptr;
        c->log_cap = 0;
        int r = dalloc(&c->d_log, (size_t)n_moves);
        if (r) return r;
        c->log_cap = (size_t)n_moves;
    }
    if (rows && max_rows > c->rows_cap) {
        if (c->d_rows) cudaFree(c->d_rows);
        c->d_rows = nullptr;
        c->rows_cap = 0;
        int r = dalloc(&c->d_rows, (size_t)9 * max_rows);
        if (r) return r;
        c->rows_cap = max_rows;
    }
    int64_t done = 0;
    int32_t nrow = 0;
    const int st = run_chain_impl(c, c->d_rng, *cursor, n_rng, cursor, n_moves, &done, log ? c->d_log : nullptr,
                                  rows ? c->d_rows : nullptr, rows ? max_rows : 0, &nrow);
    if (st != YAMC_OK && st != YAMC_ERNG_EXHAUSTED) return st;
    if (log && done) CUDA_TRY(cudaMemcpy(log, c->d_log, sizeof(yamc_move_record) * done, cudaMemcpyDeviceToHost));
    if (rows && nrow) CUDA_TRY(cudaMemcpy(rows, c->d_rows, sizeof(double) * 9 * nrow, cudaMemcpyDeviceToHost));
    if (moves_done) *moves_done = done;
    if (n_rows) *n_rows = nrow;
    return st;
}

// ---------------------------------------------------------------- per-move drop-in

int yamc_move_old(yamc_ctx *c, int32_t imol, double f[3], double tau[3]) {
    if (!c || imol < 1 || imol > c->H.M) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    int r = ensure_cfg(c);
    if (r) return r;
    if ((r = sync_positions(c)) || (r = pull_state(c))) return r;
    double in[1 + 3 * kMaxA] = {};
    in[0] = imol;
    if ((r = upload(c->api_in, in, 1 + 3 * kMaxA, c->stream))) return r;
    RunSlot rs{};
    if ((r = upload(c->d_run, &rs, 1, c->stream))) return r;
    if ((r = launch_chain(c, base_args(c, MODE_OLD)))) return r;
    double out[kNV];
    CUDA_TRY(cudaMemcpyAsync(out, c->api_out, sizeof(out), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    const HostSystem &H = c->H;
    const int f0 = H.first[imol - 1], na = H.natoms[imol - 1];
    for (int k = 0; k < 3; ++k) c->api_eold[k] = out[k];
    for (int k = 0; k < 3 * na; ++k) c->api_fold[k] = out[RV_F + k];
    double fx[kMaxA], fy[kMaxA], fz[kMaxA];
    for (int a = 0; a < na; ++a) { fx[a] = out[RV_F + 3 * a]; fy[a] = out[RV_F + 3 * a + 1]; fz[a] = out[RV_F + 3 * a + 2]; }
    double F[3], T[3];
    mol_force_torque(na, &H.x[f0], &H.y[f0], &H.z[f0], &H.mass[f0], fx, fy, fz, F, T);
    if (f) { f[0] = F[0]; f[1] = F[1]; f[2] = F[2]; }
    if (tau) { tau[0] = T[0]; tau[1] = T[1]; tau[2] = T[2]; }
    c->api_imol = imol;
    c->api_stage = 1;
    return YAMC_OK;
}

int yamc_move_eval(yamc_ctx *c, int32_t imol, const double *xn, const double *yn, const double *zn, double du[4],
                   int32_t *overlap, double f[3], double tau[3]) {
    if (!c || !xn || !yn || !zn) return YAMC_EPARAMETER;
    if (c->api_stage != 1 || imol != c->api_imol) { set_error("yamc_move_eval must follow yamc_move_old for the same molecule"); return YAMC_EWRONG_FUNCTION; }
    CUDA_TRY(cudaSetDevice(c->device));
    const HostSystem &H = c->H;
    const int f0 = H.first[imol - 1], na = H.natoms[imol - 1];
    double in[1 + 3 * kMaxA] = {};
    in[0] = imol;
    for (int a = 0; a < na; ++a) { in[1 + 3 * a] = xn[a]; in[2 + 3 * a] = yn[a]; in[3 + 3 * a] = zn[a]; }
    int r = upload(c->api_in, in, 1 + 3 * kMaxA, c->stream);
    if (r) return r;
    if ((r = launch_chain(c, base_args(c, MODE_EVAL)))) return r;
    double out[kNV];
    CUDA_TRY(cudaMemcpyAsync(out, c->api_out, sizeof(out), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int v = 0; v < kNV; ++v) c->api_new[v] = out[v];
    for (int a = 0; a < na; ++a) { c->api_xn[a] = xn[a]; c->api_yn[a] = yn[a]; c->api_zn[a] = zn[a]; }
    const int ovl = out[RV_OVL] > 0.0;
    if (overlap) *overlap = ovl;
    // Steps 7, 10-11, 11A
    const double enew = out[RV_EW] + out[RV_LJ12] - out[RV_LJ6];
    const double eold = c->api_eold[0] + c->api_eold[2] - c->api_eold[1];
    double mo[3] = {0, 0, 0}, mn[3] = {0, 0, 0};
    for (int a = 0; a < na; ++a) {
        const double q = H.q[f0 + a];
        mo[0] = mo[0] + q * H.x[f0 + a]; mo[1] = mo[1] + q * H.y[f0 + a]; mo[2] = mo[2] + q * H.z[f0 + a];
        mn[0] = mn[0] + q * xn[a]; mn[1] = mn[1] + q * yn[a]; mn[2] = mn[2] + q * zn[a];
    }
    const double *mu = &c->sc[SC_MU_X];
    for (int k = 0; k < 3; ++k) c->api_dmu[k] = mn[k] - mo[k];
    const double *dm = c->api_dmu;
    const double du_ext = H.p.kext * ((2 * mu[0] + dm[0]) * dm[0] + (2 * mu[1] + dm[1]) * dm[1] + (2 * mu[2] + dm[2]) * dm[2]);
    if (du) { du[0] = ovl ? 0.0 : enew - eold; du[1] = ovl ? 0.0 : out[RV_DUC]; du[2] = ovl ? 0.0 : out[RV_DUL]; du[3] = ovl ? 0.0 : du_ext; }
    double fx[kMaxA], fy[kMaxA], fz[kMaxA];
    for (int a = 0; a < na; ++a) {
        const double q = H.q[f0 + a];
        fx[a] = out[RV_F + 3 * a] + H.p.minus_two_kext * q * (mu[0] + dm[0]);
        fy[a] = out[RV_F + 3 * a + 1] + H.p.minus_two_kext * q * (mu[1] + dm[1]);
        fz[a] = out[RV_F + 3 * a + 2] + H.p.minus_two_kext * q * (mu[2] + dm[2]);
    }
    double F[3], T[3];
    mol_force_torque(na, xn, yn, zn, &H.mass[f0], fx, fy, fz, F, T);
    if (f) { f[0] = F[0]; f[1] = F[1]; f[2] = F[2]; }
    if (tau) { tau[0] = T[0]; tau[1] = T[1]; tau[2] = T[2]; }
    c->api_stage = ovl ? 0 : 2;
    return YAMC_OK;
}

int yamc_move_commit(yamc_ctx *c, int32_t accepted) {
    if (!c) return YAMC_EPARAMETER;
    if (!accepted) { c->api_stage = 0; return YAMC_OK; }
    if (c->api_stage != 2) { set_error("yamc_move_commit(accepted) must follow a successful yamc_move_eval"); return YAMC_EWRONG_FUNCTION; }
    CUDA_TRY(cudaSetDevice(c->device));
    HostSystem &H = c->H;
    const int imol = c->api_imol, f0 = H.first[imol - 1], na = H.natoms[imol - 1];
    const int n = (1 + H.nt) * H.S;
    k_commit_rho<<<(n + 255) / 256, 256, 0, c->stream>>>(c->rho, c->scratch + n, n);
    CUDA_TRY(cudaGetLastError());
    std::vector<double4> a(na);
    for (int i = 0; i < na; ++i) {
        H.x[f0 + i] = c->api_xn[i]; H.y[f0 + i] = c->api_yn[i]; H.z[f0 + i] = c->api_zn[i];
        a[i] = make_double4(H.x[f0 + i], H.y[f0 + i], H.z[f0 + i], H.q[f0 + i]);
    }
    int r = upload(c->atom + f0, a.data(), na, c->stream);
    if (r) return r;
    c->sc[SC_UU_EW] += c->api_new[RV_EW] - c->api_eold[0];
    c->sc[SC_UU_LJ6] += c->api_new[RV_LJ6] - c->api_eold[1];
    c->sc[SC_UU_LJ12] += c->api_new[RV_LJ12] - c->api_eold[2];
    c->sc[SC_EK_C] += c->api_new[RV_DUC];
    c->sc[SC_EK_LJ] += c->api_new[RV_DUL];
    c->sc[SC_MU_X] += c->api_dmu[0]; c->sc[SC_MU_Y] += c->api_dmu[1]; c->sc[SC_MU_Z] += c->api_dmu[2];
    if ((r = push_state(c))) return r;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->api_stage = 0;
    return YAMC_OK;
}

// ---------------------------------------------------------------- batched replicas

int yamc_batch_destroy(yamc_batch *b) {
    if (!b) return YAMC_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graph(b);
    for (BatchGroup &g : b->groups) {
        if (g.stream) cudaStreamSynchronize(g.stream);
        if (g.d_sys) cudaFree(g.d_sys);
        if (g.d_run) cudaFree(g.d_run);
        if (g.h_run) cudaFreeHost(g.h_run);
        if (g.done) cudaEventDestroy(g.done);
        if (g.stream) cudaStreamDestroy(g.stream);
    }
    for (yamc_ctx *c : b->reps) yamc_destroy(c);
    if (b->d_rng) cudaFree(b->d_rng);
    if (b->d_log) cudaFree(b->d_log);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return YAMC_OK;
}

static int batch_create_impl(yamc_batch *b, int32_t n, const yamc_system *systems, const yamc_params *params) {
    CUDA_TRY(cudaSetDevice(b->device));
    CUDA_TRY(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
    CUDA_TRY(cudaEventCreate(&b->ev0));
    CUDA_TRY(cudaEventCreate(&b->ev1));
    CUDA_TRY(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    for (int i = 0; i < n; ++i) {
        yamc_ctx *c = nullptr;
        const int r = yamc_create(&systems[i], &params[i], b->device, &c);
        if (r) {
            set_error("replica " + std::to_string(i) + ": " + last_error());
            return r;
        }
        b->reps.push_back(c);
    }
    for (int i = 0; i < n; ++i) {
        const HostSystem &H = b->reps[i]->H;
        const bool split = split_variant(H, MODE_RUN);
        size_t k = 0;
        while (k < b->groups.size() && !(b->groups[k].nt == H.nt && b->groups[k].split == split)) ++k;
        if (k == b->groups.size()) {
            b->groups.emplace_back();
            b->groups.back().nt = H.nt;
            b->groups.back().split = split;
        }
        b->groups[k].idx.push_back(i);
    }
    for (BatchGroup &g : b->groups) {
        const size_t m = g.idx.size();
        int r;
        if ((r = dalloc(&g.d_sys, m)) || (r = dalloc(&g.d_run, m))) return r;
        CUDA_TRY(cudaMallocHost((void **)&g.h_run, sizeof(RunSlot) * m));
        CUDA_TRY(cudaStreamCreateWithFlags(&g.stream, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
        std::vector<DevSys> hs(m);
        for (size_t k = 0; k < m; ++k) hs[k] = b->reps[g.idx[k]]->hsys;
        if ((r = upload(g.d_sys, hs.data(), m, b->stream))) return r;
    }
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    return batch_configure(b);
}

int yamc_batch_create(int32_t n, const yamc_system *systems, const yamc_params *params, int32_t device, yamc_batch **out) {
    if (!out || n < 1 || !systems || !params) return YAMC_EPARAMETER;
    *out = nullptr;
    yamc_batch *b = new yamc_batch();
    b->device = device;
    const int r = batch_create_impl(b, n, systems, params);
    if (r) { yamc_batch_destroy(b); return r; }
    *out = b;
    return YAMC_OK;
}

int yamc_batch_replica(yamc_batch *b, int32_t i, yamc_ctx **ctx) {
    if (!b || !ctx || i < 0 || i >= (int)b->reps.size()) return YAMC_EPARAMETER;
    *ctx = b->reps[i];
    return YAMC_OK;
}

int yamc_batch_run_device(yamc_batch *b, const float *const *d_rng, const int64_t *n_rng, int64_t *cursors,
                          int64_t n_moves, int64_t *moves_done, int32_t *status, yamc_move_record *d_log) {
    if (!b || !d_rng || !n_rng || !cursors || n_moves < 0) return YAMC_EPARAMETER;
    const size_t R = b->reps.size();
    std::vector<int64_t> off(R, 0);
    for (size_t i = 0; i < R; ++i)
        if (!d_rng[i] || n_rng[i] < 0 || cursors[i] < 0 || cursors[i] > n_rng[i]) {
            set_error("replica " + std::to_string(i) + ": bad random stream or cursor");
            return YAMC_EPARAMETER;
        }
    CUDA_TRY(cudaSetDevice(b->device));
    return batch_step(b, d_rng, off.data(), n_rng, cursors, n_moves, moves_done, status, d_log);
}

int yamc_batch_run(yamc_batch *b, const float *const *rng, const int64_t *n_rng, int64_t *cursors, int64_t n_moves,
                   int64_t *moves_done, int32_t *status, yamc_move_record *log) {
    if (!b || !rng || !n_rng || !cursors || n_moves < 0) return YAMC_EPARAMETER;
    const size_t R = b->reps.size();
    std::vector<size_t> base(R);
    size_t total = 0;
    for (size_t i = 0; i < R; ++i) {
        if (!rng[i] || n_rng[i] < 0 || cursors[i] < 0 || cursors[i] > n_rng[i]) {
            set_error("replica " + std::to_string(i) + ": bad random stream or cursor");
            return YAMC_EPARAMETER;
        }
        base[i] = total;  // the unread window [cursor, n_rng) of replica i, packed
        total += (size_t)(n_rng[i] - cursors[i]);
    }
    CUDA_TRY(cudaSetDevice(b->device));
    if (total > b->rng_cap || !b->d_rng) {
        if (b->d_rng) cudaFree(b->d_rng);
        b->d_rng = nullptr;
        b->rng_cap = 0;
        int r = dalloc(&b->d_rng, std::max<size_t>(total, 1));
        if (r) return r;
        b->rng_cap = std::max<size_t>(total, 1);
    }
    std::vector<const float *> dptr(R);
    for (size_t i = 0; i < R; ++i) {
        dptr[i] = b->d_rng + base[i];
        if (n_rng[i] > cursors[i])
            CUDA_TRY(cudaMemcpyAsync(b->d_rng + base[i], rng[i] + cursors[i], sizeof(float) * (n_rng[i] - cursors[i]),
                                     cudaMemcpyHostToDevice, b->stream));
    }
    const size_t nlog = log ? R * (size_t)n_moves : 0;
    if (nlog > b->log_cap) {
        if (b->d_log) cudaFree(b->d_log);
        b->d_log = nullptr;
        b->log_cap = 0;
        int r = dalloc(&b->d_log, nlog);
        if (r) return r;
        b->log_cap = nlog;
    }
    std::vector<int64_t> done(R, 0), off(cursors, cursors + R);
    const int st = batch_step(b, dptr.data(), off.data(), n_rng, cursors, n_moves, done.data(), status,
                              log ? b->d_log : nullptr);
    if (st != YAMC_OK && st != YAMC_ERNG_EXHAUSTED) return st;
    if (log) CUDA_TRY(cudaMemcpy(log, b->d_log, sizeof(yamc_move_record) * nlog, cudaMemcpyDeviceToHost));
    if (moves_done) for (size_t i = 0; i < R; ++i) moves_done[i] = done[i];
    return st;
}

int yamc_batch_set_launch(yamc_batch *b, int32_t cluster_blocks, int32_t threads) {
    if (!b) return YAMC_EPARAMETER;
    if (cluster_blocks < 0 || cluster_blocks > 16 || threads < 0 || threads > kChainMaxThreadsWide || (threads % 32) ||
        (threads > 0 && threads < 64))
        return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(b->device));
    const int oG = b->force_G, oB = b->force_B;
    b->force_G = cluster_blocks;
    b->force_B = threads;
    const int r = batch_configure(b);
    if (r) { b->force_G = oG; b->force_B = oB; batch_configure(b); }
    return r;
}

int yamc_batch_set_kspace_layout(yamc_batch *b, int32_t layout) {
    if (!b || layout < YAMC_KSPACE_AUTO || layout > YAMC_KSPACE_STREAMED) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(b->device));
    const int oL = b->force_layout;
    b->force_layout = layout;
    const int r = batch_configure(b);
    if (r) { b->force_layout = oL; batch_configure(b); }
    return r;
}

int yamc_batch_get_launch(yamc_batch *b, int32_t out[5]) {
    if (!b || !out || b->groups.empty()) return YAMC_EPARAMETER;
    const BatchGroup &g = b->groups[0];
    out[0] = g.cfg.G; out[1] = g.cfg.B; out[2] = std::max(g.cfg.EPT, 0); out[3] = (int32_t)g.cfg.smem; out[4] = g.max_clusters;
    return YAMC_OK;
}

int yamc_batch_last_kernel_ms(yamc_batch *b, double *ms) {
    if (!b || !ms) return YAMC_EPARAMETER;
    *ms = b->last_ms;
    return YAMC_OK;
}

int yamc_batch_tune(yamc_batch *b, const float *const *d_rng, const int64_t *n_rng, const int64_t *cursors,
                    int64_t n_moves, double *best_moves_per_s) {
    if (!b || !d_rng || !n_rng || !cursors || n_moves < 1) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(b->device));
    const size_t R = b->reps.size();
    BatchBackup keep;
    int r = batch_copy_state(b, keep, true);
    if (r) return r;
    const int fG = b->force_G, fB = b->force_B, fL = b->force_layout;
    const int Bs[] = {kChainMaxThreadsWide, kChainMaxThreads, 128};
    const int Ls[] = {YAMC_KSPACE_REGISTERS, YAMC_KSPACE_STREAMED};
    double best = -1.0;
    int bestG = 0, bestB = 0, bestL = 0;
    std::vector<int64_t> cur(R), done(R);
    for (int L : Ls)
    for (int G = 1; G <= 16; ++G) {
        for (int B : Bs) {
            if (fL != YAMC_KSPACE_AUTO && L != fL) continue;
            b->force_G = G; b->force_B = B; b->force_layout = L;
            if (batch_configure(b) != YAMC_OK) continue;  // shape does not fit
            bool ok = true;
            for (const BatchGroup &g : b->groups) ok = ok && g.cfg.G == G && g.cfg.B == B && g.max_clusters > 0;
            if (!ok) continue;
            for (size_t i = 0; i < R; ++i) cur[i] = cursors[i];
            r = yamc_batch_run_device(b, d_rng, n_rng, cur.data(), n_moves, done.data(), nullptr, nullptr);
            const int rr = batch_copy_state(b, keep, false);
            if (rr) return rr;
            if (r != YAMC_OK && r != YAMC_ERNG_EXHAUSTED) return r;
            double moves = 0;
            for (size_t i = 0; i < R; ++i) moves += (double)done[i];
            const double rate = b->last_ms > 0 ? moves / (1e-3 * b->last_ms) : 0.0;
            if (rate > best) { best = rate; bestG = G; bestB = B; bestL = L; }
        }
    }
    if (best < 0) {
        b->force_G = fG; b->force_B = fB; b->force_layout = fL;
        batch_configure(b);
        set_error("no launch shape fits every replica of the batch");
        return YAMC_ELIMITS;
    }
    b->force_G = bestG; b->force_B = bestB; b->force_layout = bestL;
    r = batch_configure(b);
    for (yamc_ctx *c : b->reps) c->pos_valid = false;
    if (best_moves_per_s) *best_moves_per_s = best;
    return r;
}

// ---------------------------------------------------------------- adjoint forces

int yamc_forces(yamc_ctx *c, double *fx, double *fy, double *fz, double *mol_f, double *mol_tau) {
    if (!c) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    HostSystem &H = c->H;
    const int N = H.N;
    int r;
    if (!c->d_gx && ((r = dalloc(&c->d_gx, N)) || (r = dalloc(&c->d_gy, N)) || (r = dalloc(&c->d_gz, N)))) return r;
    if ((r = sync_positions(c)) || (r = pull_state(c))) return r;
    k_forces_real<<<(N + kFullTile - 1) / kFullTile, kFullTile, 0, c->stream>>>(c->hsys, c->d_gx, c->d_gy, c->d_gz);
    CUDA_TRY(cudaGetLastError());
    switch (H.nt) {
        case 1: r = launch_forces_kspace<1>(c); break;
        case 2: r = launch_forces_kspace<2>(c); break;
        case 3: r = launch_forces_kspace<3>(c); break;
        default: r = launch_forces_kspace<4>(c); break;
    }
    if (r) return r;
    std::vector<double> gx(N), gy(N), gz(N);
    CUDA_TRY(cudaMemcpyAsync(gx.data(), c->d_gx, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(gy.data(), c->d_gy, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaMemcpyAsync(gz.data(), c->d_gz, sizeof(double) * N, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    // external term: F = -2 kext q mu (EwaldSumExternal.f90:84-102)
    const double mx = c->sc[SC_MU_X], my = c->sc[SC_MU_Y], mz = c->sc[SC_MU_Z], m2k = H.p.minus_two_kext;
    for (int i = 0; i < N; ++i) {
        gx[i] = gx[i] + m2k * H.q[i] * mx; gy[i] = gy[i] + m2k * H.q[i] * my; gz[i] = gz[i] + m2k * H.q[i] * mz;
        if (fx) fx[i] = gx[i];
        if (fy) fy[i] = gy[i];
        if (fz) fz[i] = gz[i];
    }
    if (mol_f || mol_tau) {
        for (int m = 0; m < H.M; ++m) {
            const int a0 = H.first[m], na = H.natoms[m];
            if (na > kMaxA) { set_error("molecule with more than 4 atoms"); return YAMC_ELIMITS; }
            double x[kMaxA], y[kMaxA], z[kMaxA], ms[kMaxA], ax[kMaxA], ay[kMaxA], az[kMaxA], F[3], T[3];
            for (int a = 0; a < na; ++a) {
                x[a] = H.x[a0 + a]; y[a] = H.y[a0 + a]; z[a] = H.z[a0 + a]; ms[a] = H.mass[a0 + a];
                ax[a] = gx[a0 + a]; ay[a] = gy[a0 + a]; az[a] = gz[a0 + a];
            }
            mol_force_torque(na, x, y, z, ms, ax, ay, az, F, T);
            for (int k = 0; k < 3; ++k) {
                if (mol_f) mol_f[3 * m + k] = F[k];
                if (mol_tau) mol_tau[3 * m + k] = T[k];
            }
        }
    }
    return YAMC_OK;
}

int yamc_set_positions(yamc_ctx *c, const double *x, const double *y, const double *z, double e[8]) {
    if (!c || !x || !y || !z) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    HostSystem &H = c->H;
    std::vector<double4> a(H.N);
    for (int i = 0; i < H.N; ++i) {
        H.x[i] = x[i]; H.y[i] = y[i]; H.z[i] = z[i];
        a[i] = make_double4(x[i], y[i], z[i], H.q[i]);
    }
    int r = upload(c->atom, a.data(), H.N, c->stream);
    if (r) return r;
    c->pos_valid = true;
    if ((r = pull_state(c)) || (r = full_sums(c))) return r;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (e) energies_from(c->sc, H.p.kext, e);
    return YAMC_OK;
}

int yamc_phase_cycles(yamc_ctx *c, int32_t mode, int64_t *out, int32_t n) {
    if (!c) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    if (!c->d_prof) {
        int r = dalloc(&c->d_prof, PH_COUNT);
        if (r) return r;
        CUDA_TRY(cudaMemset(c->d_prof, 0, sizeof(long long) * PH_COUNT));
    }
    if (mode == 1) { c->prof_on = true; CUDA_TRY(cudaMemset(c->d_prof, 0, sizeof(long long) * PH_COUNT)); }
    if (mode == 0) c->prof_on = false;
    if (out && n > 0) {
        long long h[PH_COUNT];
        CUDA_TRY(cudaMemcpy(h, c->d_prof, sizeof h, cudaMemcpyDeviceToHost));
        for (int i = 0; i < n && i < PH_COUNT; ++i) out[i] = h[i];
    }
    return YAMC_OK;
}

const char *yamc_last_error_detail(void) {
    static thread_local std::string copy;
    copy = yamc::last_error();
    return copy.c_str();
}

}  // extern "C"
