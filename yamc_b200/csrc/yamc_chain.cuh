// The persistent chain kernel (run_mc + movemc on the device) and its launch helpers.
// Included by the engine (types and declarations) and by one instantiation file per LJ type
// count (yamc_chain_inst.cu, compiled once per count), so the kernel variants compile in parallel.
#pragma once

#include <cooperative_groups.h>
#include <cuda_pipeline.h>
#include <cuda_runtime.h>

#include <string>
#include <type_traits>

#include "yamc_device.cuh"
#include "yamc_internal.h"

#define CUDA_TRY(expr)                                                                        \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess) {                                                              \
            yamc::set_error(std::string(#expr) + ": " + cudaGetErrorString(_e));              \
            return YAMC_ECUDA;                                                                \
        }                                                                                     \
    } while (0)

#ifndef YAMC_WIDE_THREADS
#define YAMC_WIDE_THREADS 384  // threads of the wide streamed variant (up to 170 registers each)
#endif
#ifndef YAMC_KSPACE_UNROLL
#define YAMC_KSPACE_UNROLL 1  // streamed k entries handled per loop iteration
#endif

namespace yamc {

namespace cg = cooperative_groups;

struct LaunchCfg {
    int G = 0, B = 0, EPT = 0;  // EPT: entries per worker in registers; 0 streamed; -1 streamed, wide CTAs
    int nown_max = 0, qcap = 0;
    size_t smem = 0;
};

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
    int nown_max;       // atoms staged per CTA (interleaved ownership: atom j lives in CTA j % G, in slot D.slot[j])
    int qcap;           // pair queue capacity per CTA
    double2 *scratch;      // [2][(1+nt) S]: molecule old sums, rho deltas (scratch_buf: FP32 pairs in the mixed form)
    long long *prof;       // optional per-phase cycle counters (PH_* layout), CTA 0
};

// phases timed when ChainArgs::prof is set (control lane 0 or worker thread 32 of CTA 0)
enum Phase { PH_CHOOSE = 0, PH_SPECULATE, PH_PROPOSE, PH_TABLES, PH_KSPACE, PH_FILTER, PH_PAIRS, PH_REDUCE,
             PH_OLD_PASS, PH_DECIDE, PH_COMMIT, PH_KSPACE_NEXT, PH_COUNT };

// reduction vector of one pass: the moved molecule's energies, k-space energy change, overlap
// flag and per-atom forces
constexpr int RV_EW = 0, RV_LJ6 = 1, RV_LJ12 = 2, RV_DUC = 3, RV_DUL = 4, RV_OVL = 5, RV_F = 6;
constexpr int kNV = 6 + 3 * kMaxA;
constexpr int kNVP = kNV;

enum PassKind { PASS_OLD = 0, PASS_NEW = 1, PASS_BOTH = 2 };

struct Slot { double x, y, z, q, iq, dhs; int type, pad; };
constexpr int kMaxSpecies = 8;
constexpr int kCPT = 8;   // atoms each worker thread tests per filter round
constexpr int kBlk = 32;  // atoms per bounding box of the pair filter (one warp's candidates per round and c)
constexpr int kQueueMax = 4096;  // pair-queue chunk (items); a round's pairs are consumed in chunks
constexpr int kWin = 256; // random-stream window held in shared memory
constexpr int kCtl = 32;  // threads of the control warp
constexpr int kChainMaxThreads = 256;  // one CTA per SM, up to 255 registers per thread
constexpr int kChainMaxThreadsWide = YAMC_WIDE_THREADS;  // streamed k entries, more warps, fewer registers

// ------------------------------------------------------------------ spatial staging
// Each CTA stages its atoms in spatial order (k_stage_order), so kBlk consecutive slots hold
// atoms of a compact region; per block a bounding box (centre and half extent per axis, box
// units, float) lets the pair filter skip blocks that lie outside the query sphere.  The box
// holds every staged position p of the block as p = centre + t + n (n integer, |t| <= half);
// kBoxPad widens the half extents beyond the rounding of centre and extent to float.
constexpr double kBoxPad = 1e-6;

__device__ __forceinline__ double wrap_half(double d) { return d - rint(d); }  // into [-1/2, 1/2]

// the block's box from its staged positions, relative to its first atom
__device__ inline void block_box(const double4 *atom_s, int b, int nown, float4 *box_s) {
    const int s0 = b * kBlk, s1 = min(s0 + kBlk, nown);
    const double4 r = atom_s[s0];
    double lx = 0, ly = 0, lz = 0, hx = 0, hy = 0, hz = 0;
    for (int s = s0 + 1; s < s1; ++s) {
        const double4 p = atom_s[s];
        const double tx = wrap_half(p.x - r.x), ty = wrap_half(p.y - r.y), tz = wrap_half(p.z - r.z);
        lx = fmin(lx, tx); ly = fmin(ly, ty); lz = fmin(lz, tz);
        hx = fmax(hx, tx); hy = fmax(hy, ty); hz = fmax(hz, tz);
    }
    box_s[2 * b] = make_float4((float)(r.x + 0.5 * (lx + hx)), (float)(r.y + 0.5 * (ly + hy)),
                               (float)(r.z + 0.5 * (lz + hz)), 0.f);
    box_s[2 * b + 1] = make_float4(__double2float_ru(0.5 * (hx - lx) + kBoxPad), __double2float_ru(0.5 * (hy - ly) + kBoxPad),
                                   __double2float_ru(0.5 * (hz - lz) + kBoxPad), 0.f);
}

// the block's box grown to hold position (x, y, z) as well (an accepted move's new position)
__device__ inline void box_expand(float4 *box_s, int b, double x, double y, double z) {
    float4 c = box_s[2 * b], h = box_s[2 * b + 1];
    const double p[3] = {x, y, z};
    float *cc[3] = {&c.x, &c.y, &c.z}, *hh[3] = {&h.x, &h.y, &h.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const double t = wrap_half(p[d] - (double)*cc[d]), e = (double)*hh[d];
        if (t > e || t < -e) {
            const double lo = fmin(-e, t), hi = fmax(e, t);
            *cc[d] = (float)((double)*cc[d] + 0.5 * (lo + hi));
            *hh[d] = __double2float_ru(0.5 * (hi - lo) + kBoxPad);
        }
    }
    box_s[2 * b] = c;
    box_s[2 * b + 1] = h;
}

// false only if no position the box holds is within sqrt(r2) of (qx, qy, qz) under any periodic
// image: per axis the nearest image of the box is |wrap(q - centre)| - half away (or 0)
__device__ __forceinline__ bool box_near(const float4 *box_s, int b, double qx, double qy, double qz, double r2) {
    const float4 c = box_s[2 * b], h = box_s[2 * b + 1];
    const double ex = fmax(fabs(wrap_half(qx - (double)c.x)) - (double)h.x, 0.0);
    const double ey = fmax(fabs(wrap_half(qy - (double)c.y)) - (double)h.y, 0.0);
    const double ez = fmax(fabs(wrap_half(qz - (double)c.z)) - (double)h.z, 0.0);
    return ex * ex + ey * ey + ez * ez < r2;
}

// Order of the staged atoms (one block per chain and CTA, before each chain launch): CTA r of a
// chain of G CTAs owns atoms j = r + G i; they are ordered by the Morton index of their cell on
// an nc^3 grid (nc a power of two <= 16, about four owned atoms per cell), stably (by i) within a
// cell.  Writes D.slot[j] (the slot of atom j in its CTA) and D.atom_of[s G + r] (the atom in
// slot s of CTA r), and the FP32 copy of rho that the mixed form's streamed sweeps read (the
// chain's blocks split its entries).  Shared memory: kStageMaxCells + atoms-per-CTA ints.
constexpr int kStageThreads = 256;
constexpr int kStageMaxCells = 4096;

__device__ __forceinline__ unsigned spread3(unsigned v) {  // bits b of v (b < 4) to bits 3 b
    return (v & 1u) | ((v & 2u) << 2) | ((v & 4u) << 4) | ((v & 8u) << 6);
}

__device__ __forceinline__ int cell_axis(double u, int nc) {
    const double w = u - floor(u);
    return min((int)(w * nc), nc - 1);
}

static __global__ void __launch_bounds__(kStageThreads) k_stage_order(const DevSys *sys, int G) {
    extern __shared__ int st_smem[];
    const int rank = blockIdx.x % G;
    const DevSys &D = sys[blockIdx.x / G];
    const int tid = threadIdx.x, lane = tid & 31;
    const int nown = (D.N - rank + G - 1) / G;
    for (int i = rank * kStageThreads + tid, n = (1 + D.nt) * D.S; i < n; i += G * kStageThreads) {
        const double2 r = D.rho[i];
        D.rho_f[i] = make_float2((float)r.x, (float)r.y);
    }
    int nc = 1;
    while (nc < 16 && 4 * (2 * nc) * (2 * nc) * (2 * nc) <= nown) nc *= 2;
    const int ncell = nc * nc * nc;
    int *hist = st_smem, *key = st_smem + kStageMaxCells;
    for (int c = tid; c < ncell; c += kStageThreads) hist[c] = 0;
    __syncthreads();
    for (int i = tid; i < nown; i += kStageThreads) {
        const double4 p = D.atom[rank + G * i];
        const int k = (int)(spread3(cell_axis(p.x, nc)) | (spread3(cell_axis(p.y, nc)) << 1) |
                            (spread3(cell_axis(p.z, nc)) << 2));
        key[i] = k;
        atomicAdd(&hist[k], 1);
    }
    __syncthreads();
    if (tid < 32) {
        // exclusive prefix of the cell counts: each lane a contiguous run of cells
        const int per = (ncell + 31) / 32;
        const int lo = min(lane * per, ncell), hi = min(lo + per, ncell);
        int sum = 0;
        for (int c = lo; c < hi; ++c) sum += hist[c];
        int x = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        int run = x - sum;
        for (int c = lo; c < hi; ++c) { const int h = hist[c]; hist[c] = run; run += h; }
        __syncwarp();
        // stable placement, 32 atoms at a time: atoms of one cell take consecutive slots in i order
        for (int i0 = 0; i0 < nown; i0 += 32) {
            const int i = i0 + lane;
            const int k = i < nown ? key[i] : -1;
            const unsigned peers = __match_any_sync(0xffffffffu, k);
            const int before = __popc(peers & ((1u << lane) - 1u));
            const int pos = i < nown ? hist[k] + before : 0;
            __syncwarp();
            if (i < nown && before == __popc(peers) - 1) hist[k] = pos + 1;
            if (i < nown) key[i] = pos;
            __syncwarp();
        }
    }
    __syncthreads();
    for (int i = tid; i < nown; i += kStageThreads) {
        const int j = rank + G * i, s = key[i];
        D.slot[j] = s;
        D.atom_of[YAMC_IX(s * G + rank, D.N + 16)] = j;
    }
}

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
    // the biased proposal on two warps: the rotation thread's result and stream positions
    MoveState mrot;
    long long disp_end, rot_start, rot_end;
    int disp_out, rot_out;
    double sc[SC_COUNT];
    double lx[kMaxA], ly[kMaxA], lz[kMaxA];  // last accepted move (staged copies may lag in other CTAs)
    int qcount;
    int wcount[64];       // per-warp pair counts and their exclusive prefix
    int wmore[32];        // per worker warp: near blocks left after this filter round
    int qmore;            // some worker warp has near blocks left
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

// why a chain stops before its last move (ChainShared::abort)
constexpr int kAbortStream = 1;     // the random stream ran out (YAMC_ERNG_EXHAUSTED, resumable)
constexpr int kAbortNonFinite = 2;  // a non-finite energy change or bias force (YAMC_ENAN)

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

// Arithmetic of a pass: MX = false is the plain FP64 method; MX = true the mixed form (pair
// terms, erfc_Luc, phases and per-thread sums in FP32; rho(k), the cross-warp and cross-CTA
// sums, the energy bookkeeping and the Metropolis test in FP64).
template <bool MX> struct Prec { using R = double; using R2 = double2; };
template <> struct Prec<true> { using R = float; using R2 = float2; };

__device__ __forceinline__ double2 mk2(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 mk2(float x, float y) { return make_float2(x, y); }
template <class R2> __device__ __forceinline__ R2 cvt2(double2 v);
template <> __device__ __forceinline__ double2 cvt2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 cvt2<float2>(double2 v) { return make_float2((float)v.x, (float)v.y); }
template <class R2> __device__ __forceinline__ R2 cvt2(float2 v);  // (FP32 rho copies: the mixed form only)
template <> __device__ __forceinline__ float2 cvt2<float2>(float2 v) { return v; }
__device__ __forceinline__ double2 to_d2(double2 v) { return v; }
__device__ __forceinline__ double2 to_d2(float2 v) { return make_double2((double)v.x, (double)v.y); }

// Buffer i of a chain's scratch (0: the moved molecule's old phase sums, 1: the rho deltas of the
// pass), in the pass's arithmetic type: FP64 pairs in the plain form, FP32 pairs in the mixed
// form (half the bytes, and loads that need no conversion).
template <bool MX>
__host__ __device__ __forceinline__ typename Prec<MX>::R2 *scratch_buf(double2 *base, int i, int nstruct, int S) {
    return reinterpret_cast<typename Prec<MX>::R2 *>(base) + (size_t)i * nstruct * S;
}

// Per-thread partial sums of a pass: FP64; in the mixed form FP64 for the pair terms (which
// reach tens of kT) and FP32 with two-sum compensation (the running sum and its rounding
// error, added in FP64 when the warp reduces) for the FP32 k-space terms.
template <bool MX, int N = kNVP>
struct Acc {
    double v[N];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = 0.0;
    }
    __device__ __forceinline__ void add(int i, double x) { v[i] += x; }
    __device__ __forceinline__ void add_plain(int i, double x) { v[i] += x; }
    __device__ __forceinline__ void flag(int i) { v[i] = 1.0; }
    __device__ __forceinline__ double get(int i) const { return v[i]; }
};
template <int N>
struct Acc<true, N> {
    double d[N];
    float s[N], c[N];
    __device__ __forceinline__ void zero() {
#pragma unroll
        for (int i = 0; i < N; ++i) { d[i] = 0.0; s[i] = 0.f; c[i] = 0.f; }
    }
    __device__ __forceinline__ void add(int i, double x) { d[i] += x; }
    __device__ __forceinline__ void add(int i, float x) {  // TwoSum (Knuth)
        const float t = s[i] + x;
        const float bp = t - s[i];
        c[i] += (s[i] - (t - bp)) + (x - bp);
        s[i] = t;
    }
    // plain FP32 sum, for the k-space forces: they only bias the proposal (their error is
    // reported beside the dE error), and a few entries per thread keep it near FP32 rounding
    __device__ __forceinline__ void add_plain(int i, float x) { s[i] += x; }
    __device__ __forceinline__ void flag(int i) { d[i] = 1.0; }
    __device__ __forceinline__ double get(int i) const { return d[i] + ((double)s[i] + (double)c[i]); }
    // the FP32 part alone, and its clearing (the k-space sums are reduced before the real space)
    __device__ __forceinline__ double kpart(int i) const { return (double)s[i] + (double)c[i]; }
    __device__ __forceinline__ void clear_kpart(int i) { s[i] = 0.f; c[i] = 0.f; }
};

template <int NT, int EPT, bool MX = false>
struct EntryRegs {
    using R = typename Prec<MX>::R;
    using R2 = typename Prec<MX>::R2;
    int e[EPT];
    int kx[EPT], ky[EPT], kz[EPT];
    R beta[EPT];
    R bl[EPT][NPair<NT>::value];  // beta_LJ of every type pair for this entry
    double2 rho[EPT][1 + NT];     // FP64 in both forms
    R2 mold[EPT][1 + NT];
    R2 dl[EPT][1 + NT];
};

// EPT <= 0: the streamed layout (EPT == -1: the same with wide CTAs) -- no entry lives in
// registers; each worker loops over its entries and reads k, beta, beta_LJ and rho from memory
// (L2-resident) every pass.  The register block of one (never touched) entry only keeps the
// code uniform.
template <int NT, int EPT, bool MX = false>
using RegsOf = EntryRegs<NT, (EPT > 0 ? EPT : 1), MX>;

// The per-move phase tables of the molecule's slots, T[slot][axis][m] = (cos, sin)(2 pi m u),
// and tmask: the LJ types the moving molecule carries.
template <bool MX>
struct PhaseTabs {
    const typename Prec<MX>::R2 *T;
    int KM;
    int tmask;
};

// Phase tables of slots [s0, s1) of move m, by the workers.  The FP32 form reduces 2 k u
// modulo 2 in FP64 before the FP32 sincospi.
template <bool MX>
__device__ __forceinline__ void build_tables(typename Prec<MX>::R2 *tab, const Slot *slots, int s0, int s1, int KM,
                                             int wtid, int nwork) {
    using R = typename Prec<MX>::R;
    const int n = (s1 - s0) * 3 * KM;
    for (int idx = wtid; idx < n; idx += nwork) {
        const int sl = s0 + idx / (3 * KM), r = idx % (3 * KM), d = r / KM, k = r % KM;
        const double u = d == 0 ? slots[sl].x : (d == 1 ? slots[sl].y : slots[sl].z);
        R s, c;
        if constexpr (MX) {
            double t = 2.0 * (double)k * u;
            t = t - 2.0 * rint(0.5 * t);
            sincospif((float)t, &s, &c);
        } else {
            sincospi(2.0 * (double)k * u, &s, &c);
        }
        if (k == 0) { s = R(0); c = R(1); }
        tab[(sl * 3 + d) * KM + k] = mk2(c, s);
    }
}

// Molecule phase sums of one entry over slots [s0, s0+na) -- RhoSquared_addAtom per atom:
// Coulomb phase q (cos, sin), LJ phase = Coulomb phase * (1/q) (the unit phase when q == 0),
// accumulated per LJ type in atom order.  ph/phl keep the per-atom phases for the forces.
template <int NT, bool MX>
__device__ __forceinline__ void mol_phase_sum(const PhaseTabs<MX> &pt, const Slot *slots, int s0, int na, int kx, int ky,
                                              int kz, typename Prec<MX>::R2 (&out)[1 + NT],
                                              typename Prec<MX>::R2 (&ph)[kMaxA], typename Prec<MX>::R2 (&phl)[kMaxA]) {
    using R = typename Prec<MX>::R;
    using R2 = typename Prec<MX>::R2;
    const int KM = pt.KM;
#pragma unroll
    for (int t = 0; t <= NT; ++t) out[t] = mk2(R(0), R(0));
#pragma unroll
    for (int a = 0; a < kMaxA; ++a) {
        ph[a] = mk2(R(0), R(0));
        phl[a] = mk2(R(0), R(0));
        if (a < na) {
            const Slot &sl = slots[s0 + a];
            const R2 *T = pt.T + (size_t)(s0 + a) * 3 * KM;
            const R q = (R)sl.q;
            R c = 0, s = 0;
            if (sl.q != 0.0) {
                entry_phase<R, R2>(T, T + KM, T + 2 * KM, kx, ky, kz, q, c, s);
                out[0].x = out[0].x + c; out[0].y = out[0].y + s;
            }
            ph[a] = mk2(c, s);
            if (sl.type > 0) {
                R cl, sl2;
                if (sl.q != 0.0) { const R iq = (R)sl.iq; cl = c * iq; sl2 = s * iq; }
                else entry_phase<R, R2>(T, T + KM, T + 2 * KM, kx, ky, kz, R(1), cl, sl2);
#pragma unroll
                for (int t = 0; t < NT; ++t)
                    if (t == sl.type - 1) { out[1 + t].x = out[1 + t].x + cl; out[1 + t].y = out[1 + t].y + sl2; }
                phl[a] = mk2(cl, sl2);
            }
        }
    }
}

// k-space force on the molecule's atoms from one entry: 4 pi beta (C sin - S cos) k per atom,
// Coulomb with the q-weighted phase, plus the dispersion terms of the atom's LJ type against
// every type's structure factor (ForceKSpace.f90:59-302).
template <int NT, bool MX, class AccT>
__device__ __forceinline__ void entry_forces(const Slot *slots, int s0, int na, int kx, int ky, int kz,
                                             typename Prec<MX>::R beta,
                                             const typename Prec<MX>::R (&bl)[NPair<NT>::value],
                                             const typename Prec<MX>::R2 (&C)[1 + NT],
                                             const typename Prec<MX>::R2 (&ph)[kMaxA],
                                             const typename Prec<MX>::R2 (&phl)[kMaxA], AccT &acc, int f0 = RV_F) {
    using R = typename Prec<MX>::R;
    const R fourpi = (R)kFourPi;
#pragma unroll
    for (int a = 0; a < kMaxA; ++a) {
        if (a < na) {
            const int ta = slots[s0 + a].type;
            R w = fourpi * ((C[0].x * ph[a].y - C[0].y * ph[a].x) * beta);
            if (ta > 0) {
#pragma unroll
                for (int t = 0; t < NT; ++t) {
                    R b = R(0);
#pragma unroll
                    for (int u = 0; u < NT; ++u)
                        if (u == ta - 1) b = bl[pair_idx<NT>(u, t)];
                    w += fourpi * ((C[1 + t].x * phl[a].y - C[1 + t].y * phl[a].x) * b);
                }
            }
            acc.add_plain(f0 + 3 * a, w * (R)kx);
            acc.add_plain(f0 + 3 * a + 1, w * (R)ky);
            acc.add_plain(f0 + 3 * a + 2, w * (R)kz);
        }
    }
}

// One signed entry of a pass: the molecule's phase sums at the old positions (into mold) and/or
// the new ones, the delta (into dl), dU_k Coulomb + LJ against rho, and the k-space forces.
template <int NT, int KIND, bool FORCES, bool MX, class AccT, class RhoT>
__device__ __forceinline__ void kspace_entry(const PhaseTabs<MX> &pt, const Slot *slots, int na, int kx,
                                             int ky, int kz, typename Prec<MX>::R beta,
                                             const typename Prec<MX>::R (&bl)[NPair<NT>::value],
                                             const RhoT (&rho)[1 + NT], typename Prec<MX>::R2 (&mold)[1 + NT],
                                             typename Prec<MX>::R2 (&dl)[1 + NT], AccT &acc) {
    using R = typename Prec<MX>::R;
    using R2 = typename Prec<MX>::R2;
    R2 ph[kMaxA], phl[kMaxA];
    R2 C[1 + NT];
#pragma unroll
    for (int t = 0; t <= NT; ++t) C[t] = cvt2<R2>(rho[t]);
    if constexpr (KIND != PASS_NEW) mol_phase_sum<NT, MX>(pt, slots, na, na, kx, ky, kz, mold, ph, phl);
    if constexpr (KIND == PASS_OLD) {
        if constexpr (FORCES) entry_forces<NT, MX>(slots, na, na, kx, ky, kz, beta, bl, C, ph, phl, acc);
    } else {
        R2 mnew[1 + NT];
        mol_phase_sum<NT, MX>(pt, slots, 0, na, kx, ky, kz, mnew, ph, phl);
#pragma unroll
        for (int t = 0; t <= NT; ++t) dl[t] = mk2(mnew[t].x - mold[t].x, mnew[t].y - mold[t].y);
        {   // EwaldSumKSpace_calc_dU_coulomb (EwaldSumKSpace.f90:528-620)
            const R2 Cc = C[0], d = dl[0];
            acc.add(RV_DUC, (((Cc.x + Cc.x) + d.x) * d.x + ((Cc.y + Cc.y) + d.y) * d.y) * beta);
        }
        // EwaldSumKSpace_calc_dU_LJ (EwaldSumKSpace.f90:623-753): t1 over all types, t2 over the
        // molecule's types (a type absent from the molecule has a zero delta and adds nothing)
        // (the entry's terms summed in order first, then added to the compensated running sum)
        R dul = R(0);
#pragma unroll
        for (int t1 = 0; t1 < NT; ++t1) {
            const R2 C1 = C[1 + t1], D1 = dl[1 + t1];
            const R tc = (C1.x + C1.x) + D1.x, ts = (C1.y + C1.y) + D1.y;
#pragma unroll
            for (int t2 = 0; t2 < NT; ++t2) {
                if (!((pt.tmask >> t2) & 1)) continue;
                const R2 D2 = dl[1 + t2];
                dul += (tc * D2.x + ts * D2.y) * bl[pair_idx<NT>(t1, t2)];
            }
        }
        acc.add(RV_DUL, dul);
        if constexpr (KIND == PASS_NEW && FORCES) {  // against total_new = rho + delta (MC.f90:1136-1163)
            R2 Cn[1 + NT];
#pragma unroll
            for (int t = 0; t <= NT; ++t) Cn[t] = mk2(C[t].x + dl[t].x, C[t].y + dl[t].y);
            entry_forces<NT, MX>(slots, 0, na, kx, ky, kz, beta, bl, Cn, ph, phl, acc);
        }
    }
}

// The k-space sweep of one pass over the worker's entries (kspace_entry per entry).
// Registers layout: k, beta, beta_LJ and rho stay in registers (R); the old phase sums are R.mold
// (or read from mold_in when given), the delta R.dl.  Streamed layout: every entry is read from
// memory (L2-resident), the next entry's loads in flight while the current one computes; the old
// sums come from mold_in (PASS_NEW, PASS_BOTH's are computed), the delta goes to the chain's
// scratch.  PASS_OLD stores its phase sums to mold_out (registers layout: when mold_store).
template <int NT, int EPT, int KIND, bool FORCES, bool MX, class AccT>
__device__ __forceinline__ void kspace_sweep(const DevSys &D, RegsOf<NT, EPT, MX> &R, const PhaseTabs<MX> &pt,
                                             const Slot *slots, int na, int e0, int estep,
                                             const typename Prec<MX>::R2 *mold_in, typename Prec<MX>::R2 *mold_out,
                                             bool mold_store, AccT &acc) {
    using Rt = typename Prec<MX>::R;
    using R2 = typename Prec<MX>::R2;
    const int S = D.S;
    R2 *dl_g = scratch_buf<MX>(D.scratch, 1, 1 + NT, S);
    if constexpr (EPT > 0) {
        static_for<0, EPT>([&](auto kc) {
            constexpr int k = decltype(kc)::value;
            if (R.e[k] < 0) return;
            if (KIND == PASS_NEW && mold_in) {
#pragma unroll
                for (int t = 0; t <= NT; ++t) R.mold[k][t] = mold_in[(size_t)t * S + R.e[k]];
            }
            kspace_entry<NT, KIND, FORCES, MX>(pt, slots, na, R.kx[k], R.ky[k], R.kz[k], R.beta[k], R.bl[k],
                                               R.rho[k], R.mold[k], R.dl[k], acc);
            if (KIND == PASS_OLD && mold_store) {
#pragma unroll
                for (int t = 0; t <= NT; ++t) mold_out[(size_t)t * S + R.e[k]] = R.mold[k][t];
            }
        });
    } else {
        // U entries per iteration: their independent dependency chains interleave
        constexpr int U = YAMC_KSPACE_UNROLL;
        constexpr bool IN_MOLD = KIND == PASS_NEW;   // read the old sums
        // the mixed form reads FP32 rho (D.rho_f, equal to rho rounded to FP32, which is what its
        // arithmetic takes), FP32 beta tables and FP32 scratch; k comes packed in one word
        using RhoT = std::conditional_t<MX, float2, double2>;
        int kv_n[U];
        Rt beta_n[U], bl_n[U][NPair<NT>::value];
        RhoT rho_n[U][1 + NT];
        R2 mold_n[U][1 + NT];
        // the loads of the next entry stay in flight until the entry is taken up: no value is
        // converted here
        auto fetch = [&](int j, int e) {
            kv_n[j] = D.kpack[YAMC_IX(e, S)];
            if constexpr (MX) {
                beta_n[j] = D.ebeta_f[e];
#pragma unroll
                for (int p = 0; p < NPair<NT>::value; ++p) bl_n[j][p] = D.ebetalj_f[(size_t)p * S + e];
            } else {
                beta_n[j] = D.ebeta[e];
#pragma unroll
                for (int p = 0; p < NPair<NT>::value; ++p) bl_n[j][p] = D.ebetalj[(size_t)p * S + e];
            }
#pragma unroll
            for (int t = 0; t <= NT; ++t) {
                if constexpr (MX) rho_n[j][t] = D.rho_f[(size_t)t * S + e];
                else rho_n[j][t] = D.rho[(size_t)t * S + e];
                mold_n[j][t] = IN_MOLD ? mold_in[(size_t)t * S + e] : mk2(Rt(0), Rt(0));
            }
        };
        const int step = U * estep;
#pragma unroll
        for (int j = 0; j < U; ++j)
            if (e0 + j * estep < S) fetch(j, e0 + j * estep);
        for (int e = e0; e < S; e += step) {
            int kx[U], ky[U], kz[U];
            Rt beta[U], bl[U][NPair<NT>::value];
            RhoT rho[U][1 + NT];
            R2 mold[U][1 + NT], dl[U][1 + NT];
#pragma unroll
            for (int j = 0; j < U; ++j) {
                kx[j] = kv_n[j] & 255; ky[j] = ((kv_n[j] >> 8) & 255) - 128; kz[j] = (kv_n[j] >> 16) - 128;
                beta[j] = beta_n[j];
#pragma unroll
                for (int p = 0; p < NPair<NT>::value; ++p) bl[j][p] = bl_n[j][p];
#pragma unroll
                for (int t = 0; t <= NT; ++t) { rho[j][t] = rho_n[j][t]; mold[j][t] = mold_n[j][t]; }
            }
#pragma unroll
            for (int j = 0; j < U; ++j)
                if (e + step + j * estep < S) fetch(j, e + step + j * estep);
#pragma unroll
            for (int j = 0; j < U; ++j)
                if (e + j * estep < S)
                    kspace_entry<NT, KIND, FORCES, MX>(pt, slots, na, kx[j], ky[j], kz[j], beta[j], bl[j], rho[j],
                                                       mold[j], dl[j], acc);
#pragma unroll
            for (int j = 0; j < U; ++j) {
                const int ej = e + j * estep;
                if (ej >= S) continue;
#pragma unroll
                for (int t = 0; t <= NT; ++t) {
                    if (KIND == PASS_OLD) mold_out[(size_t)t * S + ej] = mold[j][t];
                    else dl_g[(size_t)t * S + ej] = dl[j][t];
                }
            }
        }
    }
}

// The workers' part of one pass over the molecule's slots: k-space over their entries, real
// space over the CTA's atoms (pairs inside the cutoff laid out in the queue by a prefix sum
// over threads -- a deterministic order -- then evaluated item i by worker i % nwork), and a
// per-warp reduction into red[worker warp][value].  Worker-only barriers (bar 1).
template <int NT, int EPT, int KIND, bool FORCES, bool MX>
__device__ __forceinline__ void worker_pass_body(const DevSys &D, ChainShared &sh, RegsOf<NT, EPT, MX> &R, double2 *tab_raw,
                                            const double4 *atom_s, const double *dhs_ts, const double *dhs_g,
                                            int dhs_typed, int grank, int gsize, const int2 *meta_s, const float4 *box_s,
                                            int *blist, int *queue,
                                            int *nearbuf,
                                            double *red, const double *lj_s, int nown, int qcap, int e0, int estep,
                                            long long *prof, typename Prec<MX>::R2 *mold_buf, bool mold_out) {
    constexpr int NVMAX = FORCES ? kNVP : RV_F;
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
    using Rt = typename Prec<MX>::R;
    using R2 = typename Prec<MX>::R2;
    R2 *tab = reinterpret_cast<R2 *>(tab_raw);
    const bool pf = prof && wtid == 0;
    long long t_mark = pf ? clock64() : 0;
#define YAMC_WPH(ph) do { if (pf) { const long long t_now = clock64(); prof[ph] += t_now - t_mark; t_mark = t_now; } } while (0)

    build_tables<MX>(tab, m.slot, s_lo, s_hi, KM, wtid, nwork);
    worker_sync(nwork);
    YAMC_WPH(PH_TABLES);
    int tmask = 0;
    for (int a = 0; a < na; ++a)
        if (m.slot[a].type > 0) tmask |= 1 << (m.slot[a].type - 1);
    const PhaseTabs<MX> pt{tab, KM, tmask};

    Acc<MX> acc;
    acc.zero();
    kspace_sweep<NT, EPT, KIND, FORCES, MX>(D, R, pt, m.slot, na, e0, estep, EPT > 0 ? nullptr : mold_buf, mold_buf,
                                            mold_out, acc);
    // the mixed form's FP32 k-space sums (dU_k, k-space forces) leave the registers here: reduced
    // over the warp into its row now, so the real-space phase holds only its own accumulators;
    // the real-space values are added to the row at the end
    const int nv = FORCES ? (RV_F + 3 * na) : RV_F;
    auto kvalue = [&](int v) { return (KIND != PASS_OLD && (v == RV_DUC || v == RV_DUL)) || (FORCES && v >= RV_F && v < nv); };
    if constexpr (MX) {
#pragma unroll
        for (int v = 0; v < NVMAX; ++v) {
            if (!kvalue(v)) continue;
            double x = acc.kpart(v);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
            if (lane == 0) red[wwarp * kNV + v] = x;
            acc.clear_kpart(v);
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
    // a pass over both positions tests one sphere around the midpoint of the two centres that
    // holds both spheres (the centre may have been wrapped: the shift is taken by minimum image)
    double cbx = cox, cby = coy, cbz = coz, rb2 = rp2;
    if (KIND == PASS_BOTH) {
        const double hx = 0.5 * min_image(cnx - cox), hy = 0.5 * min_image(cny - coy), hz = 0.5 * min_image(cnz - coz);
        cbx = cox + hx; cby = coy + hy; cbz = coz + hz;
        const double rb = (sqrt(rp2) + sqrt(hx * hx + hy * hy + hz * hz)) * (1.0 + 1e-9);
        rb2 = rb * rb;
    }

    // this warp's near blocks: of the blocks wwarp + nww k (kBlk consecutive slots each; the
    // staged atoms are in spatial order), those whose bounding box comes within the query sphere.
    // A block outside it holds no atom that the per-atom test below keeps.
    const int nblk = (nown + kBlk - 1) / kBlk;
    const int wcap = (nblk + nww - 1) / nww;
    int *wl = blist + wwarp * wcap;
    int nnb = 0;
    {
        const double qx = KIND == PASS_BOTH ? cbx : (KIND == PASS_NEW ? cnx : cox);
        const double qy = KIND == PASS_BOTH ? cby : (KIND == PASS_NEW ? cny : coy);
        const double qz = KIND == PASS_BOTH ? cbz : (KIND == PASS_NEW ? cnz : coz);
        const double qr2 = KIND == PASS_BOTH ? rb2 : rp2;
        for (int k0 = 0; k0 < wcap; k0 += 32) {
            const int k = k0 + lane, b = wwarp + nww * k;
            const bool near = k < wcap && b < nblk && box_near(box_s, b, qx, qy, qz, qr2);
            const unsigned bal = __ballot_sync(0xffffffffu, near);
            if (near) wl[YAMC_IX(nnb + __popc(bal & ((1u << lane) - 1u)), wcap)] = b;
            nnb += __popc(bal);
        }
        __syncwarp();
    }
    int *nb = nearbuf + wwarp * 32 * kCPT;  // this warp's near atoms of the round
    for (int r0 = 0;; r0 += kCPT) {
        // near atoms of the warp's next kCPT near blocks, compacted in (block, lane) order
        int nnear = 0;
#pragma unroll
        for (int c = 0; c < kCPT; ++c) {
            const int jl = r0 + c < nnb ? wl[YAMC_IX(r0 + c, wcap)] * kBlk + lane : nown;
            bool near = false;
            if (jl < nown && meta_s[YAMC_IX(jl, nown)].x != imol0) {
                const double4 pj = atom_s[YAMC_IX(jl, nown)];
                if (KIND == PASS_BOTH) {
                    const double dx = min_image(cbx - pj.x), dy = min_image(cby - pj.y), dz = min_image(cbz - pj.z);
                    near = dx * dx + dy * dy + dz * dz < rb2;
                } else if (KIND == PASS_NEW) {
                    const double dx = min_image(cnx - pj.x), dy = min_image(cny - pj.y), dz = min_image(cnz - pj.z);
                    near = dx * dx + dy * dy + dz * dz < rp2;
                } else {
                    const double dx = min_image(cox - pj.x), dy = min_image(coy - pj.y), dz = min_image(coz - pj.z);
                    near = dx * dx + dy * dy + dz * dz < rp2;
                }
            }
            const unsigned bal = __ballot_sync(0xffffffffu, near);
            if (near) nb[YAMC_IX(nnear + __popc(bal & ((1u << lane) - 1u)), 32 * kCPT)] = jl;
            nnear += __popc(bal);
        }
        __syncwarp();
        // slot tests of the near atoms, densely: lane takes entries lane, lane + 32, ...
        unsigned long long masks = 0;  // kCPT slot masks of 8 bits
        int count = 0;
#pragma unroll
        for (int c = 0; c < kCPT; ++c) {
            const int k = c * 32 + lane;
            if (k < nnear) {
                const int jl = nb[YAMC_IX(k, 32 * kCPT)];
                const double4 pj = atom_s[YAMC_IX(jl, nown)];
                const int tj = meta_s[YAMC_IX(jl, nown)].y;
                // hard-core diameter: by LJ type when every atom of a type has the same one
                // (a shared-memory table), else the atom's own (global memory, by the atom in slot jl)
                const double dj = dhs_typed ? dhs_ts[tj] : dhs_g[D.atom_of[YAMC_IX(jl * gsize + grank, D.N + 16)]];
                unsigned msk = 0;
                for (int s = s_lo; s < s_hi; ++s) {
                    const Slot &sl = m.slot[s];
                    const double dx = min_image(sl.x - pj.x), dy = min_image(sl.y - pj.y), dz = min_image(sl.z - pj.z);
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    if (KIND != PASS_OLD && s < na && sl.type > 0 && tj > 0) {  // hard core (EwaldSumRealSpace.f90:409)
                        const double d12 = (sl.dhs + dj) / 2;
                        if (r2 < d12 * d12) acc.flag(RV_OVL);
                    }
                    if (r2 < D.rmax2) msk |= 1u << s;
                }
                masks |= (unsigned long long)msk << (8 * c);
                count += __popc(msk);
            }
        }
        int incl = count;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        if (lane == 31) { sh.wcount[wwarp] = incl; sh.wmore[wwarp] = nnb > r0 + kCPT; }
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
            const bool more = __any_sync(0xffffffffu, lane < nww && sh.wmore[lane] != 0);
            if (lane == 0) sh.qmore = more;
        }
        worker_sync(nwork);
        // another round while some warp has near blocks left (read here: the next round's
        // writes come after its first barrier)
        const bool more_rounds = sh.qmore != 0;
        // the round's pairs in queue order (thread order by the prefix sums), consumed in chunks of
        // qcap: each thread writes its items that fall in the chunk, the workers evaluate them
        const int base = sh.wcount[32 + wwarp] + incl - count;
        const int nq = sh.qcount;
        for (int q0 = 0; q0 < nq; q0 += qcap) {
            if (base < q0 + qcap && base + count > q0) {
                int pos = base;
#pragma unroll
                for (int c = 0; c < kCPT; ++c) {
                    unsigned msk = (unsigned)(masks >> (8 * c)) & 0xffu;
                    const int jl = msk ? nb[c * 32 + lane] : 0;
                    while (msk) {
                        const int s = __ffs(msk) - 1;
                        msk &= msk - 1;
                        if (pos >= q0 && pos < q0 + qcap) queue[YAMC_IX(pos - q0, qcap)] = (jl << 3) | s;
                        ++pos;
                    }
                }
            }
            worker_sync(nwork);
            if (q0 == 0) YAMC_WPH(PH_FILTER);
            const int nc = min(qcap, nq - q0);
            for (int qi = wtid; qi < nc; qi += nwork) {
                const int item = queue[YAMC_IX(qi, qcap)];
                const int jl = item >> 3, s = item & 7;
                const Slot &sl = m.slot[s];
                const double4 pj = atom_s[YAMC_IX(jl, nown)];
                const int tj = meta_s[YAMC_IX(jl, nown)].y;
                const double dx = min_image(sl.x - pj.x), dy = min_image(sl.y - pj.y), dz = min_image(sl.z - pj.z);
                const double r2 = dx * dx + dy * dy + dz * dz;
                const bool lj = sl.type > 0 && tj > 0;
                const int off = lj ? (sl.type - 1) * nt + (tj - 1) : 0;
                const double qq = D.xclb * sl.q * pj.w;
                const double s6 = lj ? lj_s[off] : 0.0, fe = lj ? lj_s[nt * nt + off] : 0.0;
                const bool isnew = s < na;
                const double sign = (KIND == PASS_BOTH && !isnew) ? -1.0 : 1.0;
                const PairTerm<double> t = MX ? pair_term_mx<FORCES>(r2, qq, lj, s6, fe, D.alpha, D.taosp, false)
                                              : pair_term<double, FORCES>(r2, qq, lj, s6, fe, D.alpha, D.taosp, false);
                acc.add(RV_EW, sign * t.ew); acc.add(RV_LJ6, sign * t.lj6); acc.add(RV_LJ12, sign * t.lj12);
                if constexpr (FORCES) {
                    const int a = isnew ? s : s - na;
#pragma unroll
                    for (int aa = 0; aa < kMaxA; ++aa)
                        if (aa == a) {
                            acc.add(RV_F + 3 * aa, dx * t.FR);
                            acc.add(RV_F + 3 * aa + 1, dy * t.FR);
                            acc.add(RV_F + 3 * aa + 2, dz * t.FR);
                        }
                }
            }
            worker_sync(nwork);
        }
        YAMC_WPH(PH_PAIRS);
        if (!more_rounds) break;
    }

    // per-warp reduction (xor tree) into red[worker warp][value] (the mixed form adds its
    // k-space part, already there)
#pragma unroll
    for (int v = 0; v < NVMAX; ++v) {
        if (v < nv) {
            double x = acc.get(v);
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double y = __shfl_xor_sync(0xffffffffu, x, o);
                x = (v == RV_OVL) ? fmax(x, y) : x + y;
            }
            if (lane == 0) red[wwarp * kNV + v] = (MX && kvalue(v)) ? red[wwarp * kNV + v] + x : x;
        }
    }
#undef YAMC_WPH
}

// The passes are called, not inlined, when the k entries are streamed (EPT <= 0): each pass then
// gets the kernel's whole register budget for its own loops instead of sharing it with the
// control code and the other passes (fewer spills); with entries in registers (EPT > 0) they
// are inlined, since the entry registers R must stay registers across the passes.
template <int NT, int EPT, int KIND, bool FORCES, bool MX>
__device__ __noinline__ void worker_pass_call(const DevSys &D, ChainShared &sh, RegsOf<NT, EPT, MX> &R, double2 *tab_raw,
                                              const double4 *atom_s, const double *dhs_ts, const double *dhs_g,
                                              int dhs_typed, int grank, int gsize, const int2 *meta_s, const float4 *box_s,
                                            int *blist, int *queue,
                                              int *nearbuf, double *red, const double *lj_s, int nown, int qcap, int e0,
                                              int estep, long long *prof, typename Prec<MX>::R2 *mold_buf, bool mold_out) {
    worker_pass_body<NT, EPT, KIND, FORCES, MX>(D, sh, R, tab_raw, atom_s, dhs_ts, dhs_g, dhs_typed, grank, gsize, meta_s,
                                                box_s, blist, queue, nearbuf, red, lj_s, nown, qcap, e0, estep, prof, mold_buf, mold_out);
}

template <int NT, int EPT, int KIND, bool FORCES, bool MX>
__device__ __forceinline__ void worker_pass(const DevSys &D, ChainShared &sh, RegsOf<NT, EPT, MX> &R, double2 *tab_raw,
                                            const double4 *atom_s, const double *dhs_ts, const double *dhs_g,
                                            int dhs_typed, int grank, int gsize, const int2 *meta_s, const float4 *box_s,
                                            int *blist, int *queue,
                                            int *nearbuf, double *red, const double *lj_s, int nown, int qcap, int e0,
                                            int estep, long long *prof, typename Prec<MX>::R2 *mold_buf, bool mold_out) {
    if constexpr (EPT > 0)
        worker_pass_body<NT, EPT, KIND, FORCES, MX>(D, sh, R, tab_raw, atom_s, dhs_ts, dhs_g, dhs_typed, grank, gsize,
                                                    meta_s, box_s, blist, queue, nearbuf, red, lj_s, nown, qcap, e0, estep, prof,
                                                    mold_buf, mold_out);
    else
        worker_pass_call<NT, EPT, KIND, FORCES, MX>(D, sh, R, tab_raw, atom_s, dhs_ts, dhs_g, dhs_typed, grank, gsize,
                                                    meta_s, box_s, blist, queue, nearbuf, red, lj_s, nown, qcap, e0, estep, prof,
                                                    mold_buf, mold_out);
}

// Control warp, after the workers' per-warp partials: trees over the worker warps, then over the
// cluster's CTAs in a fixed order, so every CTA holds bit-identical totals in sh.tot.  Called by
// all threads (the cluster barrier needs everyone).  Lane l of the control warp owns values l and
// l + 32 (nv <= 64).
__device__ __forceinline__ void reduce_pass(ChainShared &sh, const double *red, double *xch, int nv, int G, int rank,
                                            int xpar, cg::cluster_group &cluster) {
    // the worker warps' partials in warp order, then (cluster) every CTA's sum in rank order --
    // the same order in every CTA
    const int lane = threadIdx.x & 31;
    const int nww = (blockDim.x - kCtl) >> 5;
    if (threadIdx.x < kCtl) {
        double x[2] = {0.0, 0.0};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int v = lane + 32 * h;
            if (v < nv)
                for (int w = 0; w < nww; ++w) {
                    const double y = red[w * kNV + v];
                    x[h] = (v == RV_OVL) ? fmax(x[h], y) : x[h] + y;
                }
        }
        if (G > 1) {
            // value v of this CTA to every rank's exchange row; lanes cover (v, r) pairs
            for (int idx = 0; idx < nv * G; idx += 32) {
                const int my = idx + lane;
                const int v = my % nv, r = my / nv;
                const double x0 = __shfl_sync(0xffffffffu, x[0], v & 31);
                const double x1 = __shfl_sync(0xffffffffu, x[1], v & 31);
                if (my < nv * G) {
                    double *dst = cluster.map_shared_rank(xch, r);
                    dst[(xpar * G + rank) * kNV + v] = v < 32 ? x0 : x1;
                }
            }
        } else {
#pragma unroll
            for (int h = 0; h < 2; ++h)
                if (lane + 32 * h < nv) sh.tot[lane + 32 * h] = x[h];
        }
    }
    if (G > 1) {
        cluster.sync();
        if (threadIdx.x < kCtl) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int v = lane + 32 * h;
                if (v >= nv) continue;
                double x = 0.0;
                for (int r = 0; r < G; ++r) {
                    const double y = xch[(xpar * G + r) * kNV + v];
                    x = (v == RV_OVL) ? fmax(x, y) : x + y;
                }
                sh.tot[v] = x;
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
    else { const int2 mr = D.mol[YAMC_IX(imol - 1, D.M)]; first = mr.x; nam = mr.y; }
    C.imol = imol; C.first = first; C.na = nam;
    double mx = 0, my = 0, mz = 0;
    int slots[kMaxA];  // staging slots of the molecule's atoms (loaded together)
#pragma unroll
    for (int a = 0; a < kMaxA; ++a) slots[a] = a < nam ? D.slot[YAMC_IX(first + a, D.N)] : 0;
#pragma unroll
    for (int a = 0; a < kMaxA; ++a) {
        if (a >= nam) break;
        const int j = first + a;
        Slot s;
        if (sp >= 0) { s = sh.sp_atom[sp][a]; C.mass[a] = sh.sp_mass[sp][a]; }
        else {
            const int jc = (int)YAMC_IX(j, D.N);
            const double q = D.atom[jc].w;
            s.q = q; s.iq = q != 0.0 ? 1.0 / q : 0.0; s.dhs = D.dhs[jc]; s.type = D.meta[jc].y;
            C.mass[a] = D.mass[jc];
        }
        s.pad = slots[a];  // the commit updates the staged copy in this slot of CTA j % G
        if (imol - 1 == moving) { s.x = moving_pos[a].x; s.y = moving_pos[a].y; s.z = moving_pos[a].z; }
        else if (imol - 1 == sh.last_mol) { s.x = sh.lx[a]; s.y = sh.ly[a]; s.z = sh.lz[a]; }
        else {
            const double4 *src = (X.G > 1) ? cluster.map_shared_rank(X.atom_s, j % X.G) : X.atom_s;
            const double4 p = src[slots[a]];
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
// draw (runmc.f90:206, 232, 258).  Returns the 1-based molecule, or 0 when the stream ran out or
// the draws make this step an exchange step or the cycle a volume cycle (the chain then stops
// before it, like at the end of the stream, and the host runs it).
__device__ inline int draw_molecule(const DevSys &D, RngReader &rng, bool cycle_start) {
    const double pd = cycle_start ? rng.next() : 0.0;
    const double xd = rng.next();
    const double r = rng.next();
    if (rng.out || xd < D.xprob) return 0;
    if (cycle_start && D.psm > 0 && pd * (D.psm + 1) > D.psm) return 0;  // a volume cycle: the host runs it
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
    // old positions from slots [na, 2 na), new ones into [0, na): no overlap
    const Slot *os = C.slot + na;
    Slot *ns = C.slot;
    place_molecule_f(m, na, [&](int i, int d) { return d == 0 ? os[i].x : (d == 1 ? os[i].y : os[i].z); }, C.mass,
                     [&](int i, double x, double y, double z) { ns[i].x = x; ns[i].y = y; ns[i].z = z; });
}

// The mixed form's FP64 recomputation of rho(k) (RhoSquared_addAtoms, RhoSquared.f90:188-243)
// inside the chain, by all threads of every CTA of the cluster: the worker threads recompute the
// entries they own from every atom's FP64 position (D.atom, kept current by rank 0), with the
// atoms' per-axis phase tables built in chunks in the scratch region; then the k-space energies
// (EwaldSumKSpace_calc_coulomb_energy / _calc_LJ_energy, EwaldSumKSpace.f90:389-526) are
// reduced over the cluster into the engine scalars.
template <int NT, int EPT, class Regs>
__device__ __noinline__ void refresh_in_chain(const DevSys &D, Regs &R, double2 *scr, int scr_atoms, int e0, int estep,
                                              int G, int rank, ChainShared &sh, double *red, double *xch, int xpar,
                                              cg::cluster_group &cluster) {
    const int tid = threadIdx.x, B = blockDim.x;
    const bool ctl = tid < kCtl;
    const int lane = tid & 31, wwarp = (tid - kCtl) >> 5;
    const int KM = D.kmax + 1, S = D.S, N = D.N;
    const int CH = scr_atoms < 64 ? scr_atoms : 64;
    double2 *tabs = scr;                                                  // [CH][3][KM]
    double *sq = reinterpret_cast<double *>(tabs + (size_t)CH * 3 * KM);  // [CH]
    int *st = reinterpret_cast<int *>(sq + CH);                           // [CH]
    // the positions rank 0 wrote for accepted moves are visible to every CTA after this barrier
    __threadfence();
    if (G > 1) cluster.sync(); else __syncthreads();
    constexpr int EB = EPT > 0 ? EPT : 4;  // entries per batch
    const int nbatch = EPT > 0 ? 1 : (S + estep * EB - 1) / (estep * EB);
    double ekc = 0.0, ekl = 0.0;
    for (int b = 0; b < nbatch; ++b) {
        int ent[EB];
        int4 kv[EB];
        double2 acc[EB][1 + NT];
#pragma unroll
        for (int j = 0; j < EB; ++j) {
            int e;
            if constexpr (EPT > 0) e = R.e[j];
            else e = e0 + (b * EB + j) * estep;
            ent[j] = (!ctl && e >= 0 && e < S) ? e : -1;
            kv[j] = ent[j] >= 0 ? D.kvec[ent[j]] : make_int4(0, 0, 0, 0);
#pragma unroll
            for (int t = 0; t <= NT; ++t) acc[j][t] = make_double2(0.0, 0.0);
        }
        for (int a0 = 0; a0 < N; a0 += CH) {
            const int na = min(CH, N - a0);
            for (int idx = tid; idx < na * 3 * KM; idx += B) {
                const int a = idx / (3 * KM), r = idx % (3 * KM), d = r / KM, m = r % KM;
                const double4 p = D.atom[a0 + a];
                const double u = d == 0 ? p.x : (d == 1 ? p.y : p.z);
                double sn, cs;
                sincospi(2.0 * (double)m * u, &sn, &cs);
                if (m == 0) { sn = 0.0; cs = 1.0; }
                tabs[(a * 3 + d) * KM + m] = make_double2(cs, sn);
            }
            for (int a = tid; a < na; a += B) { sq[a] = D.atom[a0 + a].w; st[a] = D.meta[a0 + a].y; }
            __syncthreads();
            if (!ctl) {
                for (int a = 0; a < na; ++a) {
                    const double2 *T = tabs + (size_t)a * 3 * KM;
                    const double q = sq[a];
                    const int ty = st[a];
#pragma unroll
                    for (int j = 0; j < EB; ++j) {
                        if (ent[j] < 0) continue;
                        double c = 0, s = 0;
                        if (q != 0.0) {
                            entry_phase<double, double2>(T, T + KM, T + 2 * KM, kv[j].x, kv[j].y, kv[j].z, q, c, s);
                            acc[j][0].x = acc[j][0].x + c; acc[j][0].y = acc[j][0].y + s;
                        }
                        if (ty > 0) {
                            double cl, sl;
                            if (q != 0.0) { const double iq = 1.0 / q; cl = c * iq; sl = s * iq; }
                            else entry_phase<double, double2>(T, T + KM, T + 2 * KM, kv[j].x, kv[j].y, kv[j].z, 1.0, cl, sl);
#pragma unroll
                            for (int t = 0; t < NT; ++t)
                                if (t == ty - 1) { acc[j][1 + t].x = acc[j][1 + t].x + cl; acc[j][1 + t].y = acc[j][1 + t].y + sl; }
                        }
                    }
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < EB; ++j) {
            const int e = ent[j];
            if (e < 0) continue;
#pragma unroll
            for (int t = 0; t <= NT; ++t) {
                if constexpr (EPT > 0) R.rho[j][t] = acc[j][t];
                else {
                    D.rho[(size_t)t * S + e] = acc[j][t];
                    D.rho_f[(size_t)t * S + e] = make_float2((float)acc[j][t].x, (float)acc[j][t].y);
                }
            }
            ekc += D.ebeta[e] * (acc[j][0].x * acc[j][0].x + acc[j][0].y * acc[j][0].y);
#pragma unroll
            for (int t1 = 0; t1 < NT; ++t1)
#pragma unroll
                for (int t2 = t1; t2 < NT; ++t2) {
                    double l = D.ebetalj[(size_t)pair_idx<NT>(t1, t2) * S + e] *
                               (acc[j][1 + t1].x * acc[j][1 + t2].x + acc[j][1 + t1].y * acc[j][1 + t2].y);
                    if (t1 != t2) l = l + l;
                    ekl += l;
                }
        }
    }
    // k-space energies over the cluster (the pass reduction with two values)
    if (!ctl) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ekc += __shfl_xor_sync(0xffffffffu, ekc, o);
            ekl += __shfl_xor_sync(0xffffffffu, ekl, o);
        }
        if (lane == 0)
            for (int v = 0; v <= RV_DUL; ++v) red[wwarp * kNV + v] = v == RV_DUC ? ekc : (v == RV_DUL ? ekl : 0.0);
    }
    __syncthreads();
    reduce_pass(sh, red, xch, RV_DUL + 1, G, rank, xpar, cluster);
    __syncthreads();
    if (tid == 0) { sh.sc[SC_EK_C] = sh.tot[RV_DUC]; sh.sc[SC_EK_LJ] = sh.tot[RV_DUL]; }
    __syncthreads();
}

// SPLIT = false: unbiased device-resident chain only (one fused pass per move, speculation);
// SPLIT = true: force-biased moves (old pass + new pass with forces).
template <int NT, int EPT, bool SPLIT, bool MX>
__global__ void __launch_bounds__(EPT < 0 ? kChainMaxThreadsWide : kChainMaxThreads, 1) k_chain(ChainArgs A) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ ChainShared sh;
    __shared__ float rwin[2][kWin];

    cg::cluster_group cluster = cg::this_cluster();
    const int G = A.G;
    const int rank = G > 1 ? (int)cluster.block_rank() : 0;
    const int rep = blockIdx.x / G;
    // the system's parameters and array pointers in shared memory: every thread reads them from
    // there (a per-thread copy would live in local memory, which the staged atoms leave little L1 for)
    __shared__ DevSys D_s;
    {
        const int *src = reinterpret_cast<const int *>(A.sys + rep);
        int *dst = reinterpret_cast<int *>(&D_s);
        for (int i = threadIdx.x; i < (int)(sizeof(DevSys) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
        __syncthreads();
    }
    const DevSys &D = D_s;
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
    const int nblk_max = (A.nown_max + kBlk - 1) / kBlk;
    double2 *tab = reinterpret_cast<double2 *>(smem_raw);                     // [2 kMaxA][3][KM]
    float4 *box_s = reinterpret_cast<float4 *>(tab + 2 * kMaxA * 3 * KM);     // [nblk_max][2]
    double4 *atom_s = reinterpret_cast<double4 *>(box_s + 2 * nblk_max);      // [nown_max]
    int2 *meta_s = reinterpret_cast<int2 *>(atom_s + A.nown_max);             // [nown_max]
    int *queue = reinterpret_cast<int *>(meta_s + A.nown_max);                // [qcap]
    int *nearbuf = queue + ((A.qcap + 1) & ~1);                               // [B/32][32 kCPT]
    double *red = reinterpret_cast<double *>(nearbuf + B * kCPT);             // [B/32][kNV]
    // the mixed form's rho refresh reuses the pair queue and near buffer as atom phase tables
    double2 *scr = reinterpret_cast<double2 *>((reinterpret_cast<uintptr_t>(queue) + 15) & ~uintptr_t(15));
    const int scr_atoms = (int)(((reinterpret_cast<char *>(red) - reinterpret_cast<char *>(scr))) /
                                (long)(sizeof(double2) * 3 * KM + sizeof(double) + sizeof(int)));
    double *xch = red + (B / 32) * kNV;                                       // [2][G][kNV]
    double *lj_s = xch + 2 * G * kNV;                                         // [2][nt*nt]
    double *dhs_ts = lj_s + 2 * nt * nt;                                      // [nt+1] hard core by LJ type
    int *blist = reinterpret_cast<int *>(dhs_ts + nt + 1);                    // [nblk_max + 32] near blocks

    // atoms of this CTA: j = rank + G * i (interleaved, so every CTA holds a spatial mix), in
    // the spatial order of k_stage_order (slot D.slot[j]), with the bounding box of every kBlk slots
    const int nown = (D.N - rank + G - 1) / G;
    for (int i = tid; i < nown; i += B) {
        const int j = rank + G * i, sl = (int)YAMC_IX(D.slot[j], A.nown_max);
        atom_s[sl] = D.atom[j]; meta_s[sl] = D.meta[j];
    }
    __syncthreads();
    for (int b = tid; b < (nown + kBlk - 1) / kBlk; b += B) block_box(atom_s, b, nown, box_s);
    for (int i = tid; i < nt * nt; i += B) { lj_s[i] = D.lj_sig6[i]; lj_s[nt * nt + i] = D.lj_feps[i]; }
    for (int i = tid; i <= nt; i += B) dhs_ts[i] = D.dhs_t[i];

    // the workers' k-vector entries; rho stays in registers for the whole launch
    using Rt = typename Prec<MX>::R;
    using R2 = typename Prec<MX>::R2;
    RegsOf<NT, EPT, MX> R;
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
            R.beta[k] = (Rt)D.ebeta[e];
        }
#pragma unroll
        for (int p = 0; p < NPair<NT>::value; ++p) R.bl[k][p] = e < S ? (Rt)D.ebetalj[(size_t)p * S + e] : Rt(0);
#pragma unroll
        for (int t = 0; t <= NT; ++t) {
            R.rho[k][t] = e < S ? D.rho[(size_t)t * S + e] : make_double2(0, 0);
            R.mold[k][t] = mk2(Rt(0), Rt(0));
            R.dl[k][t] = mk2(Rt(0), Rt(0));
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
    if (ctl) {
        const long long base = run->cursor;
        const long long avail = n_rng - base;
        const int nw = (int)(avail < (long long)kWin ? (avail > 0 ? avail : 0) : kWin);
        for (int i = lane; i < nw; i += 32) rwin[0][i] = run->rng[YAMC_IX(base + i - run->rng_off, n_rng - run->rng_off)];
        if (lane == 0) { sh.wbase[0] = base; sh.wn[0] = nw; sh.wbase[1] = -1; sh.wn[1] = 0; sh.wnext = 1; }
    }
    __syncthreads();
    const bool biased = SPLIT && (D.xlf > 0.0 || D.xlc > 0.0);
    // the next move is prepared while the workers run the current pass: chosen and proposed for
    // unbiased moves, only chosen for force-biased ones (their proposal needs the old forces)
    const bool choose_only = biased;
    const bool speculate = !SPLIT || choose_only;
    const ChooseCtx X{&D, run, rwin[0], rwin[1], atom_s, G};

    long long moves_done = 0;
    int n_acc = 0, rows = 0;
    // mixed form: accepted moves since the last FP64 recomputation of rho(k), known to every thread
    long long acc_since = D.cnt[CN_ACC_SINCE_REFRESH], refreshes = 0;
    const long long refresh_every = MX ? D.refresh_every : 0;
    int xpar = 0;  // parity of the cluster exchange buffer, flipped after every pass
    const long long n_moves = run->n_moves;
    long long *prof = (A.prof && rank == 0) ? A.prof : nullptr;
    const bool pc = prof && tid == 0;
    long long t_mark = 0;
#define YAMC_PH(ph) do { if (pc) { const long long t_now = clock64(); prof[ph] += t_now - t_mark; t_mark = t_now; } } while (0)

    // ---------------------------------------------------------------- the first move of the launch
    bool have_next = false;  // sh.cur already prepared by the previous iteration's speculation
    for (long long it = 0; it < n_moves; ++it) {
        if (pc) t_mark = clock64();
        R2 *mold_g = scratch_buf<MX>(D.scratch, 0, 1 + NT, S);  // the moved molecule's old phase sums
        if (!have_next) {
            // choose the molecule and stage its atoms (no move in flight)
            if (tid == 0) {
                Cand &C = sh.cand[sh.icur];
                C.cur_start = sh.cursor;
                RngReader rng = make_reader(X, sh, sh.cursor);
                int imol = draw_molecule(D, rng, sh.mic == 0);
                C.valid = imol > 0;
                C.cur_prop = rng.cur;
                if (!imol) imol = 1;
                stage_molecule(X, sh, C, imol, -1, nullptr, cluster);
                sh.abort = C.valid ? 0 : kAbortStream;
            }
            __syncthreads();
            if (sh.abort) break;
            YAMC_PH(PH_CHOOSE);
        }
        if (!have_next || choose_only) {
            const int na0 = sh.cand[sh.icur].na;
            // old forces for force-biased moves (movemc Steps 3-4)
            if constexpr (SPLIT) if (biased) {
                if (!ctl) worker_pass<NT, EPT, PASS_OLD, true, MX>(D, sh, R, tab, atom_s, dhs_ts, D.dhs, D.dhs_typed, rank, G, meta_s, box_s, blist, queue, nearbuf, red, lj_s, nown, A.qcap, e0, gwork, prof, mold_g, false);
                __syncthreads();
                reduce_pass(sh, red, xch, RV_F + 3 * na0, G, rank, xpar, cluster);
                xpar ^= 1;
                __syncthreads();
                YAMC_PH(PH_OLD_PASS);  // the force-biased old pass and its reduction (the control warp's view)
                if (tid == 0) {
                    sh.eold[0] = sh.tot[RV_EW]; sh.eold[1] = sh.tot[RV_LJ6]; sh.eold[2] = sh.tot[RV_LJ12];
                    for (int a = 0; a < na0; ++a) {  // external-field force -2 kext q mu (MC.f90:988-997)
                        const double q = sh.cand[sh.icur].slot[na0 + a].q;
                        sh.fold[3 * a] = sh.tot[RV_F + 3 * a] + D.m2k * q * sh.sc[SC_MU_X];
                        sh.fold[3 * a + 1] = sh.tot[RV_F + 3 * a + 1] + D.m2k * q * sh.sc[SC_MU_Y];
                        sh.fold[3 * a + 2] = sh.tot[RV_F + 3 * a + 2] + D.m2k * q * sh.sc[SC_MU_Z];
                    }
                }
            }
            // the proposal (movemc Step 5)
            if (biased) {
                // on two warps: thread 0 draws the displacement (its Newton iteration is the long
                // serial part) while thread 32 skips the displacement's draws and draws the rotation;
                // both read the old forces thread 0 has just written
                __syncthreads();
                if (tid == 0 || tid == 32) {
                    const Cand &C = sh.cand[sh.icur];
                    double F[3], T[3];
                    // (old positions and forces read where they are, in shared memory)
                    const Slot *os = C.slot + na0;
                    mol_force_torque_f(na0, [&](int i, int d) { return d == 0 ? os[i].x : (d == 1 ? os[i].y : os[i].z); },
                                       C.mass, [&](int i, int d) { return sh.fold[3 * i + d]; }, F, T);
                    RngReader rng = make_reader(X, sh, C.cur_prop);
                    if (tid == 0) {
                        MoveState &m = sh.cand[sh.icur].mv;
                        mcm_init_old(m, F, T);
                        mcm_choose_displacement(m, rng, D.xlf, D.dr);
                        sh.disp_end = rng.cur;
                        sh.disp_out = rng.out;
                    } else {
                        MoveState &mr = sh.mrot;
                        mcm_init_old(mr, F, T);
                        mcm_skip_displacement(mr, rng, D.xlf, D.dr);
                        sh.rot_start = rng.cur;
                        if (!rng.out) mcm_choose_rotation(mr, rng, D.xlc, D.d_angle);
                        sh.rot_end = rng.cur;
                        sh.rot_out = rng.out;
                    }
                }
                __syncthreads();
                if (tid == 0) {
                    Cand &C = sh.cand[sh.icur];
                    MoveState &m = C.mv;
                    bool out = sh.disp_out != 0;
                    long long cur = sh.disp_end;
                    if (!out) {
                        if (sh.rot_start == sh.disp_end) {
                            copy_rotation(m, sh.mrot);
                            cur = sh.rot_end;
                            out = sh.rot_out != 0;
                        } else {  // (the skip always draws what the displacement draws; kept as a guard)
                            RngReader rng = make_reader(X, sh, sh.disp_end);
                            mcm_choose_rotation(m, rng, D.xlc, D.d_angle);
                            cur = rng.cur;
                            out = rng.out != 0;
                        }
                    }
                    if (out) {
                        C.valid = 0;
                        sh.abort = kAbortStream;
                    } else {
                        // old positions from slots [na0, 2 na0), new ones into [0, na0): no overlap
                        const Slot *os = C.slot + na0;
                        Slot *ns = C.slot;
                        place_molecule_f(m, na0, [&](int i, int d) { return d == 0 ? os[i].x : (d == 1 ? os[i].y : os[i].z); },
                                         C.mass, [&](int i, double x, double y, double z) { ns[i].x = x; ns[i].y = y; ns[i].z = z; });
                        C.cur_prop = cur;
                    }
                }
            } else if (tid == 0) {
                Cand &C = sh.cand[sh.icur];
                RngReader rng = make_reader(X, sh, C.cur_prop);
                const double Z[3] = {0, 0, 0};
                propose(D, C, rng, Z, Z);
                C.cur_prop = rng.cur;
                if (rng.out) { C.valid = 0; sh.abort = kAbortStream; }
            }
            __syncthreads();
            if (sh.abort) break;
            YAMC_PH(PH_PROPOSE);
        }
        const int na = sh.cand[sh.icur].na;
        const bool split = SPLIT;

        // ------------------------------------------------ the pass over the new positions
        if (!ctl) {
            if constexpr (SPLIT) worker_pass<NT, EPT, PASS_NEW, true, MX>(D, sh, R, tab, atom_s, dhs_ts, D.dhs, D.dhs_typed, rank, G, meta_s, box_s, blist, queue, nearbuf, red, lj_s, nown, A.qcap, e0, gwork, prof, mold_g, false);
            else worker_pass<NT, EPT, PASS_BOTH, false, MX>(D, sh, R, tab, atom_s, dhs_ts, D.dhs, D.dhs_typed, rank, G, meta_s, box_s, blist, queue, nearbuf, red, lj_s, nown, A.qcap, e0, gwork, prof, mold_g, false);
        } else if (speculate && it + 1 < n_moves) {
            // prepare the next move's candidates while the workers run: lanes 1-2 after the
            // acceptance draw, lane 2 with the molecule in flight at its proposed positions (used
            // only if it is chosen again and accepted)
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
                    for (int i = lane; i < nw; i += 32) rwin[b][i] = run->rng[YAMC_IX(c1 + i - run->rng_off, n_rng - run->rng_off)];
                    __syncwarp();
                    if (lane == 0) { sh.wbase[b] = c1; sh.wn[b] = nw; sh.wnext = b ^ 1; }
                    __syncwarp();
                }
            }
            if (lane == 0) {
                // the candidate after an overlap is not prepared: overlaps are rare, and a third
                // lane on its own random numbers diverges from lanes 1-2 (which draw the same
                // numbers and run in step); an overlap takes the unspeculated path instead
                sh.spec[0] = (sh.icur + 1) & 3; sh.spec[1] = (sh.icur + 2) & 3; sh.spec[2] = (sh.icur + 3) & 3;
                sh.cand[(sh.icur + 1) & 3].valid = 0;
            } else if (lane < 3) {
                const int buf = (sh.icur + 1 + lane) & 3;
                Cand &C = sh.cand[buf];
                RngReader rng = make_reader(X, sh, c1);
                (void)rng.next();  // the acceptance draw (MonteCarloMove.f90:553)
                C.cur_start = rng.cur;
                const int imol = rng.out ? 0 : draw_molecule(D, rng, next_cycle);
                C.valid = imol > 0;
                const Slot *moving = (lane == 2) ? &M.slot[0] : &M.slot[M.na];
                stage_molecule(X, sh, C, imol > 0 ? imol : 1, M.imol - 1, moving, cluster);
                const double Z[3] = {0, 0, 0};
                if (C.valid && !choose_only) propose(D, C, rng, Z, Z);
                C.cur_prop = rng.cur;
                if (rng.out) C.valid = 0;
            }
            if (pc) { const long long t_now = clock64(); prof[PH_SPECULATE] += t_now - t_mark; t_mark = t_now; }
        }
        __syncthreads();
        reduce_pass(sh, red, xch, split ? RV_F + 3 * na : RV_F, G, rank, xpar, cluster);
        xpar ^= 1;
        YAMC_PH(PH_REDUCE);

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
                    // (loops over kMaxA with constant indices: the arrays stay in registers)
                    double fx[kMaxA], fy[kMaxA], fz[kMaxA], x[kMaxA], y[kMaxA], z[kMaxA];
#pragma unroll
                    for (int a = 0; a < kMaxA; ++a) {
                        const int b = a < na ? a : 0;
                        const double q = M.slot[b].q;
                        fx[a] = sh.tot[RV_F + 3 * b] + D.m2k * q * (mux + dmx);
                        fy[a] = sh.tot[RV_F + 3 * b + 1] + D.m2k * q * (muy + dmy);
                        fz[a] = sh.tot[RV_F + 3 * b + 2] + D.m2k * q * (muz + dmz);
                        x[a] = M.slot[b].x; y[a] = M.slot[b].y; z[a] = M.slot[b].z;
                    }
                    mol_force_torque(na, x, y, z, M.mass, fx, fy, fz, F, T);
                }
                const double du_total = du_real + (du_kc + du_kl) + du_ext;
                // a non-finite energy change or bias force (an input the arithmetic cannot take:
                // NaN positions or random numbers, coincident charges) stops the chain before
                // the move is decided, with the state as it was after the last completed move
                bool finite = isfinite(du_total);
                if (biased)
                    for (int c = 0; c < 3; ++c) finite = finite && isfinite(F[c]) && isfinite(T[c]);
                if (!finite) { sh.abort = kAbortNonFinite; sh.accepted = 0; goto decided; }
                if (biased || SPLIT) {
                    // (the bias state in shared memory, where the proposal left it: no copy to spill)
                    MoveState &mv = sh.cand[sh.icur].mv;
                    mcm_init_new(mv, F, T, D.xlf, D.xlc, D.dr, D.d_angle);
                    acc = mcm_accept(mv, du_total, D.xlf, D.xlc, rng);
                } else {
                    // MonteCarloMove_accept_or_decline without bias: every bias term is an exact 0
                    // or 1 (cold = qold = cnew = qnew = 1), so the factor is exp(-dU) bit for bit
                    const double factor = exp(-du_total);
                    acc = rng.next() > factor ? 0 : 1;
                }
                out = rng.out != 0;
                cur_after = rng.cur;
                flags |= acc;
            }
            sh.accepted = 0;
            if (out) {
                sh.abort = kAbortStream;  // the interrupted move restarts from its first draw (sh.cursor unchanged)
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
                            const int sl = (int)YAMC_IX(M.slot[a].pad, nown);  // the atom's staging slot
                            double4 p = atom_s[sl];
                            p.x = M.slot[a].x; p.y = M.slot[a].y; p.z = M.slot[a].z;
                            atom_s[sl] = p;
                            box_expand(box_s, sl / kBlk, p.x, p.y, p.z);
                        }
                    }
                    ++n_acc;
                }
                sh.sc[SC_N_MV_STEPS] += 1.0;
                sh.cursor = cur_after;
                if (rank == 0) {
                    if (acc)
                        for (int a = 0; a < na; ++a) {  // x, y, z of the double4 (q unchanged): no read
                            double *pa = reinterpret_cast<double *>(D.atom + M.first + a);
                            pa[0] = M.slot[a].x; pa[1] = M.slot[a].y; pa[2] = M.slot[a].z;
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
        decided:;
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
                    const R2 *dl_g = scratch_buf<MX>(D.scratch, 1, 1 + NT, S);
                    for (int e = e0; e < S; e += gwork)
#pragma unroll
                        for (int t = 0; t <= NT; ++t) {
                            double2 r = D.rho[(size_t)t * S + e];
                            const double2 d = to_d2(dl_g[(size_t)t * S + e]);
                            r.x += d.x; r.y += d.y;
                            D.rho[(size_t)t * S + e] = r;
                            if constexpr (MX) D.rho_f[(size_t)t * S + e] = make_float2((float)r.x, (float)r.y);
                        }
                }
            }
        }
        ++moves_done;
        have_next = sh.spec_ok != 0;
        __syncthreads();
        YAMC_PH(PH_COMMIT);
        if constexpr (MX) {
            acc_since += sh.accepted;  // the same decisions in every CTA: every thread agrees
            if (refresh_every > 0 && acc_since >= refresh_every) {
                refresh_in_chain<NT, EPT>(D, R, scr, scr_atoms, e0, gwork, G, rank, sh, red, xch, xpar, cluster);
                xpar ^= 1;
                acc_since = 0;
                ++refreshes;
            }
        }
    }
#undef YAMC_PH

    {  // write back the register and shared state
#pragma unroll
        for (int k = 0; k < EPT; ++k)
            if (R.e[k] >= 0) {
#pragma unroll
                for (int t = 0; t <= NT; ++t) D.rho[(size_t)t * S + R.e[k]] = R.rho[k][t];
            }
        if (tid == 0 && rank == 0) {
            for (int c = 0; c < SC_COUNT; ++c) D.scal[c] = sh.sc[c];
            D.cnt[CN_ICYCLE] = sh.icycle;
            D.cnt[CN_ACC_SINCE_REFRESH] = acc_since;
            D.cnt[CN_REFRESHES] += refreshes;
            D.cnt[CN_MOVE_IN_CYCLE] = sh.mic;
            run->cursor = sh.cursor;
            run->moves_done = moves_done;
            run->n_rows = rows;
            run->accepted = n_acc;
            run->status = sh.abort == kAbortNonFinite ? YAMC_ENAN : (sh.abort ? YAMC_ERNG_EXHAUSTED : YAMC_OK);
        }
    }
    if (G > 1) cluster.sync();  // no CTA leaves while another may still address its shared memory
}

// nrep chains of one launch shape: nrep clusters of L.G CTAs, chain r on cluster r
template <int NT, int EPT, bool SPLIT, bool MX>
int launch_chain_t(const LaunchCfg &L, cudaStream_t stream, int nrep, const ChainArgs &args) {
    auto kfn = k_chain<NT, EPT, SPLIT, MX>;
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
template <int NT, int EPT, bool SPLIT, bool MX>
int max_clusters_t(const LaunchCfg &L, int *out) {
    auto kfn = k_chain<NT, EPT, SPLIT, MX>;
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


// the launch entry points of each LJ type count, defined in yamc_chain_inst.cu (compiled once per
// count): every (entries per thread, split, mixed) variant of that count
template <int NT> int launch_chain_nt(const LaunchCfg &L, bool split, bool mx, cudaStream_t s, int nrep, const ChainArgs &a);
template <int NT> int max_clusters_nt(const LaunchCfg &L, bool split, bool mx, int *out);
#define YAMC_DECLARE_NT(N)                                                                                       \
    template <> int launch_chain_nt<N>(const LaunchCfg &, bool, bool, cudaStream_t, int, const ChainArgs &);     \
    template <> int max_clusters_nt<N>(const LaunchCfg &, bool, bool, int *);
YAMC_DECLARE_NT(1)
YAMC_DECLARE_NT(2)
YAMC_DECLARE_NT(3)
YAMC_DECLARE_NT(4)
#undef YAMC_DECLARE_NT

}  // namespace yamc
