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
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "yamc_chain.cuh"
#include "yamc_device.cuh"
#include "yamc_internal.h"


// an NVTX range around each public entry point (header-only NVTX 3: it costs nothing unless a
// profiler that records NVTX ranges is attached)
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};
#define YAMC_RANGE(name) NvtxRange yamc_nvtx_range_(name)

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

// EwaldSumRealSpace_calc on the full sum (EwaldSumRealSpace.f90:233-500, j0 = i+1): the
// energy totals of every pair once.  One block per pair of atom tiles (ti <= tj, the upper
// triangle, listed in tpairs), so the grid grows as (N/256)^2/2 and fills the GPU even for a
// few thousand atoms; the j tile sits in shared memory, each thread owns one atom i and runs
// over it (j > i on the diagonal tile).  Intra-molecular pairs use -erf_Luc and count in the
// intra totals too; LJ-LJ pairs of different molecules closer than their mean hard-core
// diameter set the overlap flag.  One partial per block (part[blk*8 + v]), reduced in block
// order by k_sum_parts.  (The reference's per-atom uu/F of the full sum are not needed: the
// chain kernel evaluates the moved molecule's old energy directly.)
__global__ void __launch_bounds__(kFullTile) k_realspace_full(DevSys D, const int2 *tpairs, double *part) {
    __shared__ double4 tp[kFullTile];
    __shared__ int2 tm[kFullTile];
    __shared__ double td[kFullTile];
    __shared__ double red[(kFullTile / 32 + 1) * kFullParts];
    const int2 tt = tpairs[blockIdx.x];
    const int i = tt.x * kFullTile + threadIdx.x, j0 = tt.y * kFullTile;
    const bool valid = i < D.N;
    double4 pi = make_double4(0, 0, 0, 0);
    int2 mi = make_int2(-1, 0);
    double di = 0;
    if (valid) { pi = D.atom[i]; mi = D.meta[i]; di = D.dhs[i]; }
    double acc[kFullParts] = {0, 0, 0, 0, 0, 0, 0, 0};
    const int nt = D.nt;
    {
        const int j = j0 + threadIdx.x;
        if (j < D.N) { tp[threadIdx.x] = D.atom[j]; tm[threadIdx.x] = D.meta[j]; td[threadIdx.x] = D.dhs[j]; }
    }
    __syncthreads();
    const int nj = min(kFullTile, D.N - j0);
    if (valid) {
        const int jstart = tt.x == tt.y ? threadIdx.x + 1 : 0;  // j > i
        for (int jj = jstart; jj < nj; ++jj) {
            const double4 pj = tp[jj];
            const int2 mj = tm[jj];
            const bool same = mi.x == mj.x;
            const double dx = min_image(pi.x - pj.x), dy = min_image(pi.y - pj.y), dz = min_image(pi.z - pj.z);
            const double r2 = dx * dx + dy * dy + dz * dz;
            const bool lj = mi.y > 0 && mj.y > 0;
            if (!same && lj) {
                const double d12 = (di + td[jj]) / 2;
                if (r2 < d12 * d12) acc[6] = 1.0;
            }
            if (r2 >= D.rmax2) continue;
            const int off = lj ? (mi.y - 1) * nt + (mj.y - 1) : 0;
            const PairTerm<double> t = pair_term<double, false>(r2, D.xclb * pi.w * pj.w, lj, lj ? D.lj_sig6[off] : 0.0,
                                                                 lj ? D.lj_feps[off] : 0.0, D.alpha, D.taosp, same);
            acc[0] += t.ew; acc[1] += t.lj6; acc[2] += t.lj12;
            if (same) { acc[3] += t.ew; acc[4] += t.lj6; acc[5] += t.lj12; }
        }
    }
    block_sum<kFullTile>(acc, kFullParts, red);
    if (threadIdx.x < kFullParts) part[(size_t)blockIdx.x * kFullParts + threadIdx.x] = acc[threadIdx.x];
}

// part[b*nv + v] over b in [0, nb) -> out[v]: thread t adds blocks t, t+256, ... in order, then
// a fixed tree over the threads (deterministic); value vmax is a flag, reduced by max
constexpr int kSumThreads = 256;
__global__ void __launch_bounds__(kSumThreads) k_sum_parts(const double *part, int nb, int nv, int vmax, double *out) {
    __shared__ double sh[kSumThreads];
    for (int v = 0; v < nv; ++v) {
        double x = 0;
        for (int b = threadIdx.x; b < nb; b += kSumThreads) {
            const double y = part[(size_t)b * nv + v];
            x = v == vmax ? fmax(x, y) : x + y;
        }
        sh[threadIdx.x] = x;
        __syncthreads();
        for (int w = kSumThreads / 2; w > 0; w >>= 1) {
            if (threadIdx.x < w) sh[threadIdx.x] = v == vmax ? fmax(sh[threadIdx.x], sh[threadIdx.x + w]) : sh[threadIdx.x] + sh[threadIdx.x + w];
            __syncthreads();
        }
        if (threadIdx.x == 0) out[v] = sh[0];
        __syncthreads();
    }
}

// RhoSquared_addAtoms (RhoSquared.f90:188-243): for each signed entry the sum over atoms, in
// atom order within a slice, of the charge-weighted phase (Coulomb) and of the unit phase per
// LJ type, the LJ phase being the Coulomb one times 1/q like RhoSquared_addAtom
// (RhoSquared.f90:173-176).  Grid: entry blocks x atom slices (blockIdx.y), so a few thousand
// entries still fill the GPU; slice s writes its partial sums to
// part[((1+t) * nslice + s) * S + e], and k_rho_reduce adds the slices in order.
constexpr int kRhoBlock = 512;  // entries per block: the block's atom tables serve 512 entries
constexpr int kRhoChunk = 32;

template <int NT>
__global__ void __launch_bounds__(kRhoBlock) k_rho_full(DevSys D, int slice_atoms, double2 *part) {
    extern __shared__ double2 stab[];  // [kRhoChunk][3][kmax+1]
    __shared__ double sq[kRhoChunk];
    __shared__ int st[kRhoChunk];
    const int KM = D.kmax + 1;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = e < D.S;
    const int abeg = blockIdx.y * slice_atoms, aend = min(D.N, abeg + slice_atoms);
    int4 kv = make_int4(0, 0, 0, 0);
    if (valid) kv = D.kvec[e];
    double cC = 0, sC = 0;
    double cL[NT > 0 ? NT : 1], sL[NT > 0 ? NT : 1];
#pragma unroll
    for (int t = 0; t < NT; ++t) { cL[t] = 0; sL[t] = 0; }
    for (int a0 = abeg; a0 < aend; a0 += kRhoChunk) {
        const int na = min(kRhoChunk, aend - a0);
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
                    for (int tt = 0; tt < NT; ++tt) {  // selects, not an indexed store: the sums stay in registers
                        const bool hit = tt == t - 1;
                        cL[tt] = hit ? cL[tt] + cl : cL[tt];
                        sL[tt] = hit ? sL[tt] + sl : sL[tt];
                    }
                }
            }
        }
        __syncthreads();
    }
    if (valid) {
        const size_t ns = gridDim.y, s0 = blockIdx.y;
        part[s0 * D.S + e] = make_double2(cC, sC);
#pragma unroll
        for (int t = 0; t < NT; ++t) part[((1 + t) * ns + s0) * D.S + e] = make_double2(cL[t], sL[t]);
    }
}

// rho[(t)*S + e] = sum over slices s in order of part[(t*nslice + s)*S + e], t over 1+nt rows
__global__ void k_rho_reduce(const double2 *part, int nslice, int S, int nrow, double2 *rho) {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= nrow * S) return;
    const int t = idx / S, e = idx % S;
    double c = 0, s = 0;
    for (int k = 0; k < nslice; ++k) {
        const double2 v = part[((size_t)t * nslice + k) * S + e];
        c = c + v.x; s = s + v.y;
    }
    rho[idx] = make_double2(c, s);
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
// adjoint: forces = -dE/dr of the implemented total energy
// ------------------------------------------------------------------------------------------
// Real space: one thread per atom i over the j tiles of one slice (blockIdx.y; tiles in shared
// memory, increasing j), every pair inside the cutoff, intra-molecular pairs with the -erf_Luc
// energy; F_i += FR (r_i - r_j).  Slices let a few thousand atoms fill the GPU: slice s writes
// its partial forces to pf[(c * nslice + s) * N + i] (c = x, y, z), k_forces_reduce adds them.
__global__ void __launch_bounds__(kFullTile) k_forces_real(DevSys D, int slice_tiles, double *pf) {
    __shared__ double4 tp[kFullTile];
    __shared__ int2 tm[kFullTile];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < D.N;
    double4 pi = make_double4(0, 0, 0, 0);
    int2 mi = make_int2(-1, 0);
    if (valid) { pi = D.atom[i]; mi = D.meta[i]; }
    double gx = 0, gy = 0, gz = 0;
    const int nt = D.nt;
    const int jbeg = blockIdx.y * slice_tiles * kFullTile, jend = min(D.N, jbeg + slice_tiles * kFullTile);
    for (int t0 = jbeg; t0 < jend; t0 += kFullTile) {
        const int j = t0 + threadIdx.x;
        if (j < jend) { tp[threadIdx.x] = D.atom[j]; tm[threadIdx.x] = D.meta[j]; }
        __syncthreads();
        const int nj = min(kFullTile, jend - t0);
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
    if (valid) {
        const size_t ns = gridDim.y, s0 = blockIdx.y, N = D.N;
        pf[(0 * ns + s0) * N + i] = gx; pf[(1 * ns + s0) * N + i] = gy; pf[(2 * ns + s0) * N + i] = gz;
    }
}

// f{x,y,z}[i] = sum over slices in order of pf[(c * nslice + s) * N + i]
__global__ void k_forces_reduce(const double *pf, int nslice, int N, double *fx, double *fy, double *fz) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double g[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        double x = 0;
        for (int k = 0; k < nslice; ++k) x = x + pf[((size_t)c * nslice + k) * N + i];
        g[c] = x;
    }
    fx[i] = g[0]; fy[i] = g[1]; fz[i] = g[2];
}

// k space (ForceKSpace_coulomb / _LJ, ForceKSpace.f90:59-302, over the signed entries): one
// warp per kForceAPW atoms, the lanes over the entries, so each entry's k, rho and beta rows are
// loaded once for kForceAPW atoms; sin/cos(k r) come from the atoms' per-axis tables,
// recomputed here instead of stored per atom and k.  Adds to fx/fy/fz.
constexpr int kForceWarps = 8;  // warps per block
constexpr int kForceAPW = 4;    // atoms per warp

template <int NT>
__global__ void __launch_bounds__(32 * kForceWarps, 2) k_forces_kspace(DevSys D, double *fx, double *fy, double *fz) {
    extern __shared__ double2 ftab[];  // [kForceWarps][kForceAPW][3][KM]
    const int KM = D.kmax + 1;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = (blockIdx.x * kForceWarps + w) * kForceAPW;
    if (i0 >= D.N) return;
    const int na = min(kForceAPW, D.N - i0);
    double2 *T = ftab + (size_t)w * kForceAPW * 3 * KM;
    double q[kForceAPW], iq[kForceAPW];
    int ta[kForceAPW];
#pragma unroll
    for (int a = 0; a < kForceAPW; ++a) {
        q[a] = 0; iq[a] = 0; ta[a] = 0;
        if (a < na) {
            const double4 p = D.atom[i0 + a];
            q[a] = p.w; iq[a] = p.w != 0.0 ? 1.0 / p.w : 0.0; ta[a] = D.meta[i0 + a].y;
        }
    }
    for (int idx = lane; idx < na * 3 * KM; idx += 32) {
        const int a = idx / (3 * KM), r = idx % (3 * KM), d = r / KM, m = r % KM;
        const double4 p = D.atom[i0 + a];
        const double u = d == 0 ? p.x : (d == 1 ? p.y : p.z);
        double sn, cs;
        sincospi(2.0 * (double)m * u, &sn, &cs);
        if (m == 0) { sn = 0.0; cs = 1.0; }
        T[idx] = make_double2(cs, sn);
    }
    __syncwarp();
    const int S = D.S;
    double gx[kForceAPW], gy[kForceAPW], gz[kForceAPW];
#pragma unroll
    for (int a = 0; a < kForceAPW; ++a) { gx[a] = 0; gy[a] = 0; gz[a] = 0; }
    for (int e = lane; e < S; e += 32) {
        const int4 kv = D.kvec[e];
        const double2 C = D.rho[e];
        const double be = D.ebeta[e];
        double2 Ct[NT > 0 ? NT : 1];
#pragma unroll
        for (int t = 0; t < NT; ++t) Ct[t] = D.rho[(size_t)(1 + t) * S + e];
        double bl[NT * (NT + 1) / 2 > 0 ? NT * (NT + 1) / 2 : 1];
#pragma unroll
        for (int pr = 0; pr < NT * (NT + 1) / 2; ++pr) bl[pr] = D.ebetalj[(size_t)pr * S + e];
#pragma unroll
        for (int a = 0; a < kForceAPW; ++a) {
            if (a >= na) break;
            const double2 *Ta = T + (size_t)a * 3 * KM;
            double c = 0, sn = 0, wgt = 0;
            if (q[a] != 0.0) {
                entry_phase<double, double2>(Ta, Ta + KM, Ta + 2 * KM, kv.x, kv.y, kv.z, q[a], c, sn);
                wgt = be * (C.x * sn - C.y * c);
            }
            if (ta[a] > 0) {
                double cl, sl;
                if (q[a] != 0.0) { cl = c * iq[a]; sl = sn * iq[a]; }
                else entry_phase<double, double2>(Ta, Ta + KM, Ta + 2 * KM, kv.x, kv.y, kv.z, 1.0, cl, sl);
#pragma unroll
                for (int t = 0; t < NT; ++t) {
                    const int row = pair_idx<NT>(ta[a] - 1, t);
                    double b = bl[0];  // selects, not an indexed load: bl stays in registers
#pragma unroll
                    for (int pr = 1; pr < NT * (NT + 1) / 2; ++pr) b = row == pr ? bl[pr] : b;
                    wgt += b * (Ct[t].x * sl - Ct[t].y * cl);
                }
            }
            const double f = kFourPi * wgt;
            gx[a] = gx[a] + f * kv.x; gy[a] = gy[a] + f * kv.y; gz[a] = gz[a] + f * kv.z;
        }
    }
#pragma unroll
    for (int a = 0; a < kForceAPW; ++a) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            gx[a] += __shfl_xor_sync(0xffffffffu, gx[a], o);
            gy[a] += __shfl_xor_sync(0xffffffffu, gy[a], o);
            gz[a] += __shfl_xor_sync(0xffffffffu, gz[a], o);
        }
        if (lane == 0 && a < na) { fx[i0 + a] += gx[a]; fy[i0 + a] += gy[a]; fz[i0 + a] += gz[a]; }
    }
}

// ------------------------------------------------------------------------------------------
// exchange move (mc_xchange, MC.f90:1325-1954): two molecules swap centres of mass
// ------------------------------------------------------------------------------------------
// The two molecules' atoms (molecule 1 first), at the old and the swapped positions.
struct XchgIn {
    int m1, m2, n1, n2;                 // 0-based molecules, their atom counts
    double4 o[2 * kMaxA], n[2 * kMaxA]; // x, y, z (box units), q
    int type[2 * kMaxA];                // LJ type (0 = none)
    double dhs[2 * kMaxA];              // hard-core diameter / L
};
constexpr int kXParts = 16;  // (old 1, new 1, old 2, new 2) x (ew, lj6, lj12), then the overlap flag at 12

// Real space of both molecules, old and new, against every atom outside them (the 1-2 pairs are
// added on the host): one thread per atom j, block partials for k_sum_parts.  Overlap: an LJ site
// of either molecule, at its new position, inside the mean hard-core diameter of an LJ site j
// (EwaldSumRealSpace.f90:409-433).
__global__ void __launch_bounds__(256) k_xchg_real(DevSys D, XchgIn X, double *part) {
    __shared__ double red[(256 / 32 + 1) * kXParts];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[kXParts];
#pragma unroll
    for (int v = 0; v < kXParts; ++v) acc[v] = 0;
    if (j < D.N) {
        const int2 mj = D.meta[j];
        if (mj.x != X.m1 && mj.x != X.m2) {
            const double4 pj = D.atom[j];
            const double dj = D.dhs[j];
            const int na = X.n1 + X.n2;
            for (int a = 0; a < na; ++a) {
                const int set0 = a < X.n1 ? 0 : 2;
                const int ta = X.type[a];
                const bool lj = ta > 0 && mj.y > 0;
                const int off = lj ? (ta - 1) * D.nt + (mj.y - 1) : 0;
                for (int w = 0; w < 2; ++w) {
                    const double4 pa = w ? X.n[a] : X.o[a];
                    const double dx = min_image(pa.x - pj.x), dy = min_image(pa.y - pj.y), dz = min_image(pa.z - pj.z);
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    if (w == 1 && lj) {
                        const double d12 = (X.dhs[a] + dj) / 2;
                        if (r2 < d12 * d12) acc[12] = 1.0;
                    }
                    if (r2 >= D.rmax2) continue;
                    const PairTerm<double> t = pair_term<double, false>(r2, D.xclb * pa.w * pj.w, lj, lj ? D.lj_sig6[off] : 0.0,
                                                                         lj ? D.lj_feps[off] : 0.0, D.alpha, D.taosp, false);
                    const int s = (set0 + w) * 3;
                    acc[s] += t.ew; acc[s + 1] += t.lj6; acc[s + 2] += t.lj12;
                }
            }
        }
    }
    block_sum<256>(acc, kXParts, red);
    if (threadIdx.x < kXParts) part[(size_t)blockIdx.x * kXParts + threadIdx.x] = acc[threadIdx.x];
}

// k space: per signed entry the structure factors of both molecules at the new positions minus
// the old ones (RhoSquared_addAtom per atom, molecule 1 then 2, MC.f90:1467-1490, 1652-1672),
// written to delta (rows: Coulomb, then LJ types) for the commit, and the entry's terms of
// EwaldSumKSpace_calc_dU_coulomb / _LJ (EwaldSumKSpace.f90:528-753) against the resident rho.
template <int NT>
__global__ void __launch_bounds__(256) k_xchg_kspace(DevSys D, XchgIn X, double2 *delta, double *part) {
    extern __shared__ double2 xt[];  // [atom][old/new][3][KM]
    __shared__ double red[(256 / 32 + 1) * 2];
    const int KM = D.kmax + 1, na = X.n1 + X.n2;
    for (int idx = threadIdx.x; idx < na * 2 * 3 * KM; idx += blockDim.x) {
        const int a = idx / (6 * KM), r = idx % (6 * KM), w = r / (3 * KM), r3 = r % (3 * KM), d = r3 / KM, m = r3 % KM;
        const double4 p = w ? X.n[a] : X.o[a];
        const double u = d == 0 ? p.x : (d == 1 ? p.y : p.z);
        double sn, cs;
        sincospi(2.0 * (double)m * u, &sn, &cs);
        if (m == 0) { sn = 0.0; cs = 1.0; }
        xt[idx] = make_double2(cs, sn);
    }
    __syncthreads();
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double acc[2] = {0, 0};
    if (e < D.S) {
        const int4 kv = D.kvec[e];
        double2 sum[2][1 + NT];
        int tmask = 0;
#pragma unroll
        for (int w = 0; w < 2; ++w)
#pragma unroll
            for (int t = 0; t <= NT; ++t) sum[w][t] = make_double2(0, 0);
#pragma unroll
        for (int w = 0; w < 2; ++w) {
            for (int a = 0; a < na; ++a) {
                const double2 *T = xt + (size_t)(a * 2 + w) * 3 * KM;
                const double q = X.o[a].w;
                const int ta = X.type[a];
                double c = 0, sn = 0;
                if (q != 0.0) {
                    entry_phase<double, double2>(T, T + KM, T + 2 * KM, kv.x, kv.y, kv.z, q, c, sn);
                    sum[w][0].x = sum[w][0].x + c; sum[w][0].y = sum[w][0].y + sn;
                }
                if (ta > 0) {
                    double cl, sl;
                    if (q != 0.0) { const double iq = 1.0 / q; cl = c * iq; sl = sn * iq; }
                    else entry_phase<double, double2>(T, T + KM, T + 2 * KM, kv.x, kv.y, kv.z, 1.0, cl, sl);
#pragma unroll
                    for (int t = 0; t < NT; ++t) {
                        const bool hit = t == ta - 1;
                        sum[w][1 + t].x = hit ? sum[w][1 + t].x + cl : sum[w][1 + t].x;
                        sum[w][1 + t].y = hit ? sum[w][1 + t].y + sl : sum[w][1 + t].y;
                    }
                    tmask |= 1 << (ta - 1);
                }
            }
        }
        double2 dl[1 + NT], C[1 + NT];
#pragma unroll
        for (int t = 0; t <= NT; ++t) {
            dl[t] = make_double2(sum[1][t].x - sum[0][t].x, sum[1][t].y - sum[0][t].y);
            C[t] = D.rho[(size_t)t * D.S + e];
            delta[(size_t)t * D.S + e] = dl[t];
        }
        acc[0] = (((C[0].x + C[0].x) + dl[0].x) * dl[0].x + ((C[0].y + C[0].y) + dl[0].y) * dl[0].y) * D.ebeta[e];
#pragma unroll
        for (int t1 = 0; t1 < NT; ++t1) {
            const double tc = (C[1 + t1].x + C[1 + t1].x) + dl[1 + t1].x, ts = (C[1 + t1].y + C[1 + t1].y) + dl[1 + t1].y;
#pragma unroll
            for (int t2 = 0; t2 < NT; ++t2) {
                if (!((tmask >> t2) & 1)) continue;
                acc[1] += (tc * dl[1 + t2].x + ts * dl[1 + t2].y) * D.ebetalj[(size_t)pair_idx<NT>(t1, t2) * D.S + e];
            }
        }
    }
    block_sum<256>(acc, 2, red);
    if (threadIdx.x < 2) part[(size_t)blockIdx.x * 2 + threadIdx.x] = acc[threadIdx.x];
}

// ------------------------------------------------------------------------------------------
// radial distribution functions of molecule centres (mcrdf2, count_distances, mcrdf2.f90:110-333)
// ------------------------------------------------------------------------------------------
// centre of mass of every molecule (center_of_mass, geometry.f90:170-201) from the device positions
__global__ void k_mol_centres(DevSys D, double *cx, double *cy, double *cz) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= D.M) return;
    const int2 mo = D.mol[m];
    double sx = 0, sy = 0, sz = 0, tm = 0;
    for (int a = mo.x; a < mo.x + mo.y; ++a) {
        const double4 p = D.atom[a];
        const double w = D.mass[a];
        sx = __dadd_rn(sx, __dmul_rn(w, p.x)); sy = __dadd_rn(sy, __dmul_rn(w, p.y));
        sz = __dadd_rn(sz, __dmul_rn(w, p.z)); tm = __dadd_rn(tm, w);
    }
    cx[m] = sx / tm; cy[m] = sy / tm; cz[m] = sz / tm;
}

// One frame: every ordered pair (i, j) of centres, grid-stride over i*M + j, each block counting
// into shared-memory histograms (hist[(t1*ntypes + t2)*nbin + b], t1 <= t2, then the per-pair
// totals) that it adds to the device totals at the end.  The distance arithmetic is written with
// explicitly rounded operations (no contraction), so the bins match the oracle's exactly.
__global__ void __launch_bounds__(256) k_rdf_count(const double *cx, const double *cy, const double *cz, const int *type,
                                                   int M, int ntypes, int nbin, double L, double dr, double rmax2,
                                                   int nbox, unsigned long long *hist) {
    extern __shared__ unsigned int hs[];
    const int npair = ntypes * ntypes, nh = npair * nbin + npair;
    for (int k = threadIdx.x; k < nh; k += blockDim.x) hs[k] = 0;
    __syncthreads();
    const long long total = (long long)M * M;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < total; p += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(p / M), j = (int)(p % M);
        const double x1 = cx[i], y1 = cy[i], z1 = cz[i];
        double x2 = cx[j], y2 = cy[j], z2 = cz[j];
        if (__dsub_rn(x1, x2) > 0.5) x2 = __dadd_rn(x2, 1.0);
        if (__dsub_rn(x1, x2) < -0.5) x2 = __dsub_rn(x2, 1.0);
        if (__dsub_rn(y1, y2) > 0.5) y2 = __dadd_rn(y2, 1.0);
        if (__dsub_rn(y1, y2) < -0.5) y2 = __dsub_rn(y2, 1.0);
        if (__dsub_rn(z1, z2) > 0.5) z2 = __dadd_rn(z2, 1.0);
        if (__dsub_rn(z1, z2) < -0.5) z2 = __dsub_rn(z2, 1.0);
        const int ti = type[i] - 1, tj = type[j] - 1;
        const int off = ti < tj ? ti * ntypes + tj : tj * ntypes + ti;
        for (int nx = -nbox; nx <= nbox; ++nx)
            for (int ny = -nbox; ny <= nbox; ++ny)
                for (int nz = -nbox; nz <= nbox; ++nz) {
                    if (i == j && nx == 0 && ny == 0 && nz == 0) continue;
                    const double dx = __dmul_rn(__dadd_rn(__dsub_rn(x1, x2), (double)nx), L);
                    const double dy = __dmul_rn(__dadd_rn(__dsub_rn(y1, y2), (double)ny), L);
                    const double dz = __dmul_rn(__dadd_rn(__dsub_rn(z1, z2), (double)nz), L);
                    const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                    if (r2 > __dsub_rn(rmax2, 1e-10)) continue;
                    const int b = (int)__ddiv_rn(__dsqrt_rn(r2), dr);
                    atomicAdd(&hs[npair * nbin + off], 1u);
                    if (b < nbin) atomicAdd(&hs[off * nbin + b], 1u);
                }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < nh; k += blockDim.x)
        if (hs[k]) atomicAdd(&hist[k], (unsigned long long)hs[k]);
}

// the exchange step's commit: rho += delta (MC.f90:1245 for the two molecules)
__global__ void k_commit_rho(double2 *rho, const double2 *delta, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) { double2 r = rho[i]; const double2 d = delta[i]; r.x += d.x; r.y += d.y; rho[i] = r; }
}

// ------------------------------------------------------------------------------------------
// the per-move drop-in (yamc_move_old / yamc_move_eval): one grid-wide pass per call
// ------------------------------------------------------------------------------------------
// The molecule (1-based) and, for an evaluation, its proposed atom positions (box units).
struct MoveIn {
    int imol;
    double x[kMaxA], y[kMaxA], z[kMaxA];
    long long seq;  // the call's sequence number, written as the completion word when the results are out
};

constexpr int kMoveThreads = 256;

// One pass of a single move over the whole system, spread over the GPU (the persistent chain
// kernel stages every atom and k entry of the system in one cluster first, which a single move
// does not repay).  Every block stages the molecule's slots -- the proposed positions (EVAL) at
// [0, na), the current ones at [na, 2 na), as the chain's candidates -- and builds their phase
// tables, then each thread takes one slice of the signed k entries (kspace_entry, the chain
// pass's arithmetic: the old phase sums to scratch buffer 0 (OLD), or the deltas against them to
// buffer 1, dU_k and the k-space forces (EVAL)) and one slice of the atoms (the molecule's pairs
// inside the cutoff with their forces; EVAL: the hard-core overlap test).  Block sums in a fixed
// tree; the last block to finish adds the blocks in block order and writes the reduction vector
// (RV_* layout; OLD: the old energies and forces with the external field -2 kext q mu added, as
// the chain's old pass hands them on).  Deterministic run to run.
template <int NT, bool MX, bool EVAL>
__global__ void __launch_bounds__(kMoveThreads) k_move_pass(DevSys D, MoveIn in, double *part, unsigned *counter,
                                                            double *out) {
    using R = typename Prec<MX>::R;
    using R2 = typename Prec<MX>::R2;
    constexpr int KIND = EVAL ? PASS_NEW : PASS_OLD;
    extern __shared__ __align__(16) unsigned char move_smem[];
    __shared__ Slot sl[2 * kMaxA];
    __shared__ double red[(kMoveThreads / 32 + 1) * kNV];
    __shared__ int na_s, last;
    const int tid = threadIdx.x;
    const int KM = D.kmax + 1, S = D.S, nt = D.nt;
    const int imol0 = in.imol - 1;
    if (tid == 0) {
        const int2 mr = D.mol[imol0];
        na_s = mr.y;
        for (int a = 0; a < mr.y; ++a) {
            const int j = mr.x + a;
            const double4 p = D.atom[j];
            Slot o;
            o.x = p.x; o.y = p.y; o.z = p.z; o.q = p.w; o.iq = p.w != 0.0 ? 1.0 / p.w : 0.0;
            o.dhs = D.dhs[j]; o.type = D.meta[j].y; o.pad = 0;
            sl[mr.y + a] = o;
            if (EVAL) { o.x = in.x[a]; o.y = in.y[a]; o.z = in.z[a]; }
            sl[a] = o;
        }
    }
    __syncthreads();
    const int na = na_s;
    const int s_lo = EVAL ? 0 : na, s_hi = EVAL ? na : 2 * na;
    R2 *tab = reinterpret_cast<R2 *>(move_smem);
    build_tables<MX>(tab, sl, s_lo, s_hi, KM, tid, kMoveThreads);
    int tmask = 0;
    for (int a = 0; a < na; ++a)
        if (sl[a].type > 0) tmask |= 1 << (sl[a].type - 1);
    __syncthreads();
    const PhaseTabs<MX> pt{tab, KM, tmask};
    Acc<MX> acc;
    acc.zero();
    const int gt = blockIdx.x * kMoveThreads + tid, gs = gridDim.x * kMoveThreads;
    // k space: the chain pass's arithmetic, one entry at a time
    R2 *mold_g = scratch_buf<MX>(D.scratch, 0, 1 + NT, S), *dl_g = scratch_buf<MX>(D.scratch, 1, 1 + NT, S);
    for (int e = gt; e < S; e += gs) {
        const int4 kv = D.kvec[e];
        R beta, bl[NPair<NT>::value];
        if constexpr (MX) {
            beta = D.ebeta_f[e];
#pragma unroll
            for (int p = 0; p < NPair<NT>::value; ++p) bl[p] = D.ebetalj_f[(size_t)p * S + e];
        } else {
            beta = D.ebeta[e];
#pragma unroll
            for (int p = 0; p < NPair<NT>::value; ++p) bl[p] = D.ebetalj[(size_t)p * S + e];
        }
        double2 rho[1 + NT];
        R2 mold[1 + NT], dl[1 + NT];
#pragma unroll
        for (int t = 0; t <= NT; ++t) {
            rho[t] = D.rho[(size_t)t * S + e];
            mold[t] = EVAL ? mold_g[(size_t)t * S + e] : mk2(R(0), R(0));
        }
        kspace_entry<NT, KIND, true, MX>(pt, sl, na, kv.x, kv.y, kv.z, beta, bl, rho, mold, dl, acc);
#pragma unroll
        for (int t = 0; t <= NT; ++t) {
            if (EVAL) dl_g[(size_t)t * S + e] = dl[t];
            else mold_g[(size_t)t * S + e] = mold[t];
        }
    }
    // real space: the molecule's pairs with every other atom
    for (int j = gt; j < D.N; j += gs) {
        const int2 mt = D.meta[j];
        if (mt.x == imol0) continue;
        const double4 pj = D.atom[j];
        const double dj = D.dhs[j];
        const int tj = mt.y;
#pragma unroll
        for (int a = 0; a < kMaxA; ++a) {
            if (a >= na) continue;
            const Slot &ss = sl[s_lo + a];
            const double dx = min_image(ss.x - pj.x), dy = min_image(ss.y - pj.y), dz = min_image(ss.z - pj.z);
            const double r2 = dx * dx + dy * dy + dz * dz;
            const bool lj = ss.type > 0 && tj > 0;
            if (EVAL && lj) {  // hard core (EwaldSumRealSpace.f90:409)
                const double d12 = (ss.dhs + dj) / 2;
                if (r2 < d12 * d12) acc.flag(RV_OVL);
            }
            if (r2 >= D.rmax2) continue;
            const int off = lj ? (ss.type - 1) * nt + (tj - 1) : 0;
            const double qq = D.xclb * ss.q * pj.w;
            const double s6 = lj ? D.lj_sig6[off] : 0.0, fe = lj ? D.lj_feps[off] : 0.0;
            const PairTerm<double> t = MX ? pair_term_mx<true>(r2, qq, lj, s6, fe, D.alpha, D.taosp, false)
                                          : pair_term<double, true>(r2, qq, lj, s6, fe, D.alpha, D.taosp, false);
            acc.add(RV_EW, t.ew); acc.add(RV_LJ6, t.lj6); acc.add(RV_LJ12, t.lj12);
            acc.add(RV_F + 3 * a, dx * t.FR); acc.add(RV_F + 3 * a + 1, dy * t.FR); acc.add(RV_F + 3 * a + 2, dz * t.FR);
        }
    }
    double v[kNV];
#pragma unroll
    for (int i = 0; i < kNV; ++i) v[i] = acc.get(i);
    block_sum<kMoveThreads>(v, kNV, red);  // (the overlap flags add up: a positive total is an overlap)
    if (tid < kNV) part[(size_t)blockIdx.x * kNV + tid] = v[tid];
    __threadfence();
    __syncthreads();
    if (tid == 0) last = atomicAdd(counter, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    if (tid < kNV) {
        const volatile double *pv = part;
        double x = 0.0;
        for (int b = 0; b < (int)gridDim.x; ++b) x += pv[(size_t)b * kNV + tid];
        if (tid == RV_OVL) x = x > 0.0 ? 1.0 : 0.0;
        if (!EVAL && tid >= RV_F && tid < RV_F + 3 * na) {  // the external field at the old dipole (MC.f90:988-997)
            const int a = (tid - RV_F) / 3, c = (tid - RV_F) % 3;
            x = x + D.m2k * sl[na + a].q * D.scal[SC_MU_X + c];
        }
        out[tid] = x;
    }
    // the engine scalars and counters beside them (the host's copies of the state the next calls use)
    if (tid >= 64 && tid < 64 + SC_COUNT) out[kNV + tid - 64] = D.scal[tid - 64];
    if (tid >= 96 && tid < 96 + CN_COUNT) reinterpret_cast<long long *>(out + kNV + SC_COUNT)[tid - 96] = D.cnt[tid - 96];
    if (tid == 0) *counter = 0u;
    // then the completion word (after CN_COUNT counters): every result is visible to the host first
    __threadfence_system();
    __syncthreads();
    if (tid == 0) reinterpret_cast<volatile long long *>(out + kNV + SC_COUNT)[CN_COUNT] = in.seq;
}

// The step-14 commit of an accepted per-move step in one launch: rho += the pass's deltas
// (FP32 deltas in the mixed form), the moved atoms' positions and the engine scalars and
// counters from the host (kernel arguments, nothing staged in host memory).
struct MoveCommit {
    int first, na;
    double x[kMaxA], y[kMaxA], z[kMaxA];
    double sc[SC_COUNT];
    long long cnt[CN_COUNT];
};
template <class D2>
__global__ void k_commit_move(double2 *rho, const D2 *delta, int n, DevSys D, MoveCommit mc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        double2 r = rho[i];
        const D2 d = delta[i];
        r.x += (double)d.x;
        r.y += (double)d.y;
        rho[i] = r;
    }
    if (blockIdx.x == 0) {
        const int t = threadIdx.x;
        if (t < mc.na) {  // x, y, z of the double4 (q unchanged)
            double *pa = reinterpret_cast<double *>(D.atom + mc.first + t);
            pa[0] = mc.x[t]; pa[1] = mc.y[t]; pa[2] = mc.z[t];
        }
        if (t >= 32 && t < 32 + SC_COUNT) D.scal[t - 32] = mc.sc[t - 32];
        if (t >= 64 && t < 64 + CN_COUNT) D.cnt[t - 64] = mc.cnt[t - 64];
    }
}

}  // namespace yamc

// ==========================================================================================
// host side: context, launches and the C ABI
// ==========================================================================================
using namespace yamc;

namespace {

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

size_t chain_smem_bytes(int G, int B, int kmax, int nt, int nown_max, int qcap) {
    const int KM = kmax + 1;
    const size_t nblk_max = (size_t)(nown_max + kBlk - 1) / kBlk;
    size_t b = sizeof(double2) * 2 * kMaxA * 3 * KM;
    b += sizeof(float4) * 2 * nblk_max;
    b += (sizeof(double4) + sizeof(int2)) * (size_t)nown_max;
    b += sizeof(int) * (size_t)((qcap + 1) & ~1);
    b += sizeof(int) * (size_t)B * kCPT;
    b += sizeof(double) * (size_t)(B / 32) * kNV;
    b += sizeof(double) * (size_t)2 * G * kNV;
    b += sizeof(double) * ((size_t)2 * nt * nt + nt + 1);
    b += sizeof(int) * (nblk_max + 32);
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
    float *ebeta_f = nullptr, *ebetalj_f = nullptr;  // FP32 copies of ebeta / ebetalj for the mixed form
    std::vector<float> h_ebeta_f, h_ebetalj_f;       // their host sources (kept: the uploads are asynchronous)
    int4 *kvec = nullptr;
    int *kpack = nullptr;      // kvec packed in one word (the chain kernel's streamed sweeps)
    int *d_check = nullptr;    // bounds-checked builds: the first out-of-bounds source line (DevSys::check)
    float2 *rho_f = nullptr;   // FP32 copy of rho (the mixed form's streamed sweeps)
    int *pair_index = nullptr;
    double2 *rho = nullptr, *scratch = nullptr;
    double *freq_beg = nullptr, *freq_end = nullptr, *scal = nullptr;
    long long *cnt = nullptr;
    int4 *spec = nullptr;
    int *slot = nullptr, *atom_of = nullptr;  // the chain kernel's staging order (k_stage_order)
    double *part = nullptr, *sums = nullptr;  // block partials of the full sums, their totals
    int2 *tpairs = nullptr;                    // atom-tile pairs of the real-space full sum
    int ntpairs = 0;
    double2 *rho_part = nullptr;               // per-slice rho(k) sums of the full recompute
    int rho_slices = 1, rho_slice_atoms = 0;
    int nsm = 148;                             // SMs of the device
    DevSys hsys{};
    DevSys *d_sys = nullptr;
    RunSlot *d_run = nullptr;
    // the per-move pass's outputs: its reduction vector, then the engine scalars and counters, in
    // mapped pinned host memory the kernel writes directly (h_out on the host, d_hout on the device):
    // kNV pass values, SC_COUNT scalars, CN_COUNT counters, then the per-move passes' completion word
    double *h_out = nullptr, *d_hout = nullptr;
    long long move_seq = 0;  // sequence number of the last per-move pass
    // the per-move pass (k_move_pass): block partials and the finished-block counter
    double *d_mpart = nullptr;
    unsigned *d_mcount = nullptr;
    int mblocks = 0;
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
    double *d_fpart = nullptr;                                  // their per-slice real-space parts
    // NPT volume move: rho(k) as it was before the step, accepted volume steps
    double2 *rho_save = nullptr;
    double n_vol_accepted = 0;
    bool in_batch = false;  // a batch replica: the batch's graph runs it (NVT, no exchange steps)
    int vol_stage = 0;  // 1 between yamc_volume_eval and yamc_volume_commit
    // exchange step between yamc_xchange_eval and yamc_xchange_commit (1 evaluated, 2 overlap)
    int xch_stage = 0;
    struct XchgPending {
        int m1 = 0, m2 = 0;
        double x[2 * kMaxA] = {}, y[2 * kMaxA] = {}, z[2 * kMaxA] = {};  // swapped positions, molecule 1 first
        double d_ew = 0, d_lj6 = 0, d_lj12 = 0, du_kc = 0, du_kl = 0, dmu[3] = {};
    } xch;
    struct VolSaved {
        yamc_params p{};
        std::vector<double> x, y, z, sigma, type_sigma, beta, ebetalj, lj6, lj12, four_eps, sigma6, sigma2, dhs;
        double sc[SC_COUNT] = {};
        double tail_c = 0, tail6 = 0, tail12 = 0;
        double old_L = 0, new_L = 0, xclb_old = 0, xclb_new = 0, U_old = 0;
    } vol;
    // mixed form: FP64 recomputation of rho(k) every refresh_every accepted moves (in the chain kernel)
    long long refresh_every = 10000;
};

namespace {

// The first (G, B) that fits every system of hosts: each worker thread holds at most 2 signed
// entries, the CTA's atoms and the pair queue fit in shared memory.  G (1..16 CTAs per cluster)
// from large to small when large_first (the shortest move for a lone chain), else from small to
// large; B from 256 to 128 threads; force_G / force_B pin either (0 = free).
int pick_launch_for(const std::vector<const HostSystem *> &hosts, int device, int force_G, int force_B, int layout,
                    bool mx, LaunchCfg *out, bool large_first = true) {
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    // the kernel's static shared memory (ChainShared and the two random-stream windows) comes first
    const size_t smem_max = prop.sharedMemPerBlockOptin - sizeof(ChainShared) - sizeof(float) * 2 * kWin - 256;
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
            // for the wide CTAs, which only the streamed layout runs)
            if (layout == YAMC_KSPACE_STREAMED || (layout == YAMC_KSPACE_AUTO && EPT > 2)) EPT = 0;
            if (B > kChainMaxThreads) {
                if (layout == YAMC_KSPACE_REGISTERS) continue;
                EPT = -1;
            }
            if (EPT > 2) continue;
            const int nown_max = (Nmax + G - 1) / G;
            const int qcap = std::min(kQueueMax, std::min(nown_max, nwork * kCPT) * 2 * kMaxA);  // pair-queue chunk
            const size_t sm = chain_smem_bytes(G, B, kmax, nt, nown_max, qcap);
            if (sm > smem_max) continue;
            out->G = G; out->B = B; out->EPT = EPT; out->nown_max = nown_max; out->qcap = qcap; out->smem = sm;
            return YAMC_OK;
        }
    }
    set_error("no launch configuration fits this system (k-set or atoms too large for one cluster)");
    return YAMC_ELIMITS;
}

bool is_mixed(const yamc_ctx *c) { return c->H.p.precision == YAMC_MIXED; }

// one k_move_pass launch (OLD: the molecule's current positions; EVAL: in's proposed ones) into
// c->api_out on the context's stream
template <int NT, bool MX>
int launch_move_pass_t(yamc_ctx *c, const MoveIn &in, bool eval, size_t smem) {
    auto kfn = eval ? k_move_pass<NT, MX, true> : k_move_pass<NT, MX, false>;
    if (smem > 48 * 1024) CUDA_TRY(cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kfn<<<c->mblocks, kMoveThreads, smem, c->stream>>>(c->hsys, in, c->d_mpart, c->d_mcount, c->d_hout);
    CUDA_TRY(cudaGetLastError());
    return YAMC_OK;
}

// the per-move passes' completion word in mapped host memory
volatile long long &move_pass_done(yamc_ctx *c) {
    return reinterpret_cast<volatile long long *>(c->h_out + kNV + SC_COUNT)[CN_COUNT];
}

// Waits for the per-move pass with sequence number seq: the kernel writes its results into mapped
// host memory and then the completion word, so the host spins on that word (for up to 200 ms)
// rather than synchronising the stream, which saves the synchronisation's wake-up latency.  A
// pass that has not finished by then, or has failed, is reported by the stream synchronisation
// that follows.  Later work goes to the same stream, so it stays ordered after the pass.
int wait_move_pass(yamc_ctx *c, long long seq) {
    const auto t0 = std::chrono::steady_clock::now();
    for (long long n = 1; move_pass_done(c) != seq; ++n)
        if (n % 1024 == 0 && std::chrono::steady_clock::now() - t0 > std::chrono::milliseconds(200)) break;
    if (move_pass_done(c) == seq) return YAMC_OK;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (move_pass_done(c) != seq) { set_error("a per-move pass ended without its results"); return YAMC_ECUDA; }
    return YAMC_OK;
}

int launch_move_pass(yamc_ctx *c, MoveIn &in, bool eval) {
    const HostSystem &H = c->H;
    in.seq = ++c->move_seq;
    if (!c->d_mpart) {
        // one thread per atom and per signed entry, at most two blocks per SM
        const int need = std::max((H.N + kMoveThreads - 1) / kMoveThreads, (H.S + kMoveThreads - 1) / kMoveThreads);
        c->mblocks = std::max(1, std::min(need, 2 * c->nsm));
        int r;
        if ((r = dalloc(&c->d_mpart, (size_t)c->mblocks * kNV)) || (r = dalloc(&c->d_mcount, 1))) return r;
        CUDA_TRY(cudaMemsetAsync(c->d_mcount, 0, sizeof(unsigned), c->stream));
    }
    const size_t smem = sizeof(double2) * 2 * kMaxA * 3 * (size_t)(H.kmax + 1);
    const bool mx = is_mixed(c);
    switch (H.nt) {
        case 1: return mx ? launch_move_pass_t<1, true>(c, in, eval, smem) : launch_move_pass_t<1, false>(c, in, eval, smem);
        case 2: return mx ? launch_move_pass_t<2, true>(c, in, eval, smem) : launch_move_pass_t<2, false>(c, in, eval, smem);
        case 3: return mx ? launch_move_pass_t<3, true>(c, in, eval, smem) : launch_move_pass_t<3, false>(c, in, eval, smem);
        case 4: return launch_move_pass_t<4, false>(c, in, eval, smem);
        default: set_error("LJ type count outside 1..4"); return YAMC_ELIMITS;
    }
}


int pick_launch(yamc_ctx *c, LaunchCfg *out) {
    return pick_launch_for({&c->H}, c->device, c->force_G, c->force_B, c->force_layout, is_mixed(c), out);
}

// the spatial staging order of every CTA of nrep chains (k_stage_order), ahead of their launch
int launch_stage_order(const LaunchCfg &L, cudaStream_t stream, int nrep, const DevSys *d_sys) {
    const size_t smem = sizeof(int) * ((size_t)kStageMaxCells + L.nown_max);
    if (smem > 48 * 1024)
        CUDA_TRY(cudaFuncSetAttribute(k_stage_order, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_stage_order<<<L.G * nrep, kStageThreads, smem, stream>>>(d_sys, L.G);
    CUDA_TRY(cudaGetLastError());
    return YAMC_OK;
}

// nrep chains: the staging order, then the chain kernel (two launches)
int launch_chain_cfg(const LaunchCfg &L, int nt, bool split, bool mx, cudaStream_t stream, int nrep,
                     const ChainArgs &args) {
    if (const int r = launch_stage_order(L, stream, nrep, args.sys)) return r;
    switch (nt) {
        case 1: return launch_chain_nt<1>(L, split, mx, stream, nrep, args);
        case 2: return launch_chain_nt<2>(L, split, mx, stream, nrep, args);
        case 3: return launch_chain_nt<3>(L, split, mx, stream, nrep, args);
        case 4: return launch_chain_nt<4>(L, split, mx, stream, nrep, args);
    }
    set_error("LJ type count outside 1..4");
    return YAMC_ELIMITS;
}

int max_clusters_cfg(const LaunchCfg &L, int nt, bool split, bool mx, int *out) {
    switch (nt) {
        case 1: return max_clusters_nt<1>(L, split, mx, out);
        case 2: return max_clusters_nt<2>(L, split, mx, out);
        case 3: return max_clusters_nt<3>(L, split, mx, out);
        case 4: return max_clusters_nt<4>(L, split, mx, out);
    }
    set_error("LJ type count outside 1..4");
    return YAMC_ELIMITS;
}

// the chain kernel with separate old and new passes: force-biased moves
bool split_variant(const HostSystem &H) { return H.p.xlambda_f > 0.0 || H.p.xlambda_c > 0.0; }

int launch_chain(yamc_ctx *c, const ChainArgs &args) {
    return launch_chain_cfg(c->cfg, c->H.nt, split_variant(c->H), c->H.p.precision == YAMC_MIXED, c->stream, 1,
                            args);
}

template <int NT>
int launch_rho_full(yamc_ctx *c) {
    const int KM = c->H.kmax + 1;
    const size_t sm = sizeof(double2) * kRhoChunk * 3 * KM;
    CUDA_TRY(cudaFuncSetAttribute(k_rho_full<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const dim3 grid((c->H.S + kRhoBlock - 1) / kRhoBlock, c->rho_slices);
    k_rho_full<NT><<<grid, kRhoBlock, sm, c->stream>>>(c->hsys, c->rho_slice_atoms, c->rho_part);
    CUDA_TRY(cudaGetLastError());
    const int n = (1 + NT) * c->H.S;
    k_rho_reduce<<<(n + 255) / 256, 256, 0, c->stream>>>(c->rho_part, c->rho_slices, c->H.S, 1 + NT, c->rho);
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

// mc_calc_total_sums (MC.f90:477-585) on the device.  A hard-core overlap is an error
// (YAMC_EOVERLAP_INIT) unless overlap is given, which then receives it (the volume move's
// case: the sums are still completed, as the reference completes them).
int full_sums(yamc_ctx *c, int *overlap = nullptr) {
    HostSystem &H = c->H;
    int r = sync_positions(c);
    if (r) return r;
    k_realspace_full<<<c->ntpairs, kFullTile, 0, c->stream>>>(c->hsys, c->tpairs, c->part);
    CUDA_TRY(cudaGetLastError());
    k_sum_parts<<<1, kSumThreads, 0, c->stream>>>(c->part, c->ntpairs, kFullParts, 6, c->sums);
    CUDA_TRY(cudaGetLastError());
    double tot[kFullParts] = {};
    CUDA_TRY(cudaMemcpyAsync(tot, c->sums, sizeof(tot), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    for (int v = 0; v < 6; ++v)
        if (!std::isfinite(tot[v])) { set_error("non-finite real-space sum"); return YAMC_ENAN; }
    if (overlap) *overlap = tot[6] > 0;
    else if (tot[6] > 0) { set_error("hard-core overlap in the configuration"); return YAMC_EOVERLAP_INIT; }
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
    k_sum_parts<<<1, kSumThreads, 0, c->stream>>>(c->part, nbk, 2, -1, c->sums + kFullParts);
    CUDA_TRY(cudaGetLastError());
    double ek[2];
    CUDA_TRY(cudaMemcpyAsync(ek, c->sums + kFullParts, sizeof(ek), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    const double ekc = ek[0], ekl = ek[1];
    if (!std::isfinite(ekc) || !std::isfinite(ekl)) { set_error("non-finite k-space sum"); return YAMC_ENAN; }
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
    const size_t sm = sizeof(double2) * kForceWarps * kForceAPW * 3 * (c->H.kmax + 1);
    const int per_block = kForceWarps * kForceAPW;
    CUDA_TRY(cudaFuncSetAttribute(k_forces_kspace<NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_forces_kspace<NT><<<(c->H.N + per_block - 1) / per_block, 32 * kForceWarps, sm, c->stream>>>(c->hsys, c->d_gx,
                                                                                                      c->d_gy, c->d_gz);
    CUDA_TRY(cudaGetLastError());
    return YAMC_OK;
}

// hard-core diameter / L by LJ type, when every LJ atom of a type has the same one (the chain
// kernel then keeps the table in shared memory instead of a per-atom array)
void fill_dhs_types(const HostSystem &H, DevSys &D) {
    D.dhs_typed = 1;
    for (int t = 0; t <= kMaxDevTypes; ++t) D.dhs_t[t] = -1.0;
    for (int i = 0; i < H.N; ++i) {
        const int t = H.type_by_index[i];
        if (t <= 0) continue;
        if (t > kMaxDevTypes) { D.dhs_typed = 0; continue; }
        if (D.dhs_t[t] < 0) D.dhs_t[t] = H.dhs[i];
        else if (D.dhs_t[t] != H.dhs[i]) D.dhs_typed = 0;
    }
    D.dhs_t[0] = 0.0;
    for (int t = 1; t <= kMaxDevTypes; ++t) if (D.dhs_t[t] < 0) D.dhs_t[t] = 0.0;
}

ChainArgs base_args(yamc_ctx *c) {
    ChainArgs a{};
    a.sys = c->d_sys; a.run = c->d_run; a.G = c->cfg.G;
    a.nown_max = c->cfg.nown_max; a.qcap = c->cfg.qcap;
    a.scratch = c->scratch;
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
    bool mx = false;            // mixed precision
    int size_class = 0;         // replicas of similar atom counts share a launch shape
    int fG = 0, fB = 0, fL = YAMC_KSPACE_AUTO;  // the group's tuned shape (0 / AUTO: the batch's)
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
    int last_launches = 0;  // kernels launched by the last run (staging order + chain, per group)
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
        const int G = g.fG ? g.fG : b->force_G, B = g.fB ? g.fB : b->force_B;
        const int L = g.fL != YAMC_KSPACE_AUTO ? g.fL : b->force_layout;
        // a batch prefers the smallest cluster that fits: more chains resident at once
        int r = pick_launch_for(hs, b->device, G, B, L, g.mx, &g.cfg, false);
        if (r) return r;
        if ((r = max_clusters_cfg(g.cfg, g.nt, g.split, g.mx, &g.max_clusters))) return r;
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
        a.sys = g.d_sys; a.run = g.d_run; a.G = g.cfg.G;
        a.nown_max = g.cfg.nown_max; a.qcap = g.cfg.qcap;
        if ((r = launch_chain_cfg(g.cfg, g.nt, g.split, g.mx, g.stream, (int)g.idx.size(), a))) break;
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
// Bounds-checked builds: the index check word of a context after its kernels ran (YAMC_EBOUNDS
// with the source line when an index was out of bounds; the word is cleared).  Normal builds
// compile the checks out and return `status`.
static int bounds_status(yamc_ctx *c, int status) {
#ifdef YAMC_CHECKED
    int line = 0;
    CUDA_TRY(cudaMemcpyAsync(&line, c->d_check, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    if (line) {
        CUDA_TRY(cudaMemsetAsync(c->d_check, 0, sizeof(int), c->stream));
        set_error("index out of bounds in the chain kernel at yamc_chain.cuh line " + std::to_string(line));
        return YAMC_EBOUNDS;
    }
#else
    (void)c;
#endif
    return status;
}

int batch_step(yamc_batch *b, const float *const *rng, const int64_t *rng_off, const int64_t *n_rng,
               int64_t *cursors, int64_t n_moves, int64_t *moves_done, int32_t *status, yamc_move_record *d_log,
               int only_group = -1) {
    int r = batch_build_graph(b);
    if (r) return r;
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        BatchGroup &g = b->groups[gi];
        const bool on = only_group < 0 || (int)gi == only_group;  // a group left out runs no moves
        // the replicas' DevSys again (their refresh settings may have changed since the batch began)
        std::vector<DevSys> hs(g.idx.size());
        for (size_t k = 0; k < g.idx.size(); ++k) hs[k] = b->reps[g.idx[k]]->hsys;
        if ((r = upload(g.d_sys, hs.data(), hs.size(), b->stream))) return r;
        for (size_t k = 0; k < g.idx.size(); ++k) {
            const int i = g.idx[k];
            RunSlot &rs = g.h_run[k];
            rs = RunSlot{};
            rs.rng = rng[i]; rs.rng_off = rng_off[i]; rs.n_rng = n_rng[i];
            rs.cursor = cursors[i]; rs.n_moves = on ? n_moves : 0;
            rs.log = d_log ? d_log + (size_t)i * n_moves : nullptr;
        }
    }
    CUDA_TRY(cudaEventRecord(b->ev0, b->stream));
    CUDA_TRY(cudaGraphLaunch(b->graph, b->stream));
    CUDA_TRY(cudaEventRecord(b->ev1, b->stream));
    CUDA_TRY(cudaStreamSynchronize(b->stream));
    cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
    b->last_launches = 2 * (int)b->groups.size();
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
    for (yamc_ctx *c : b->reps) {
        const int bs = bounds_status(c, YAMC_OK);
        if (bs != YAMC_OK) return bs;
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
        case YAMC_EBOUNDS: return "index out of bounds (bounds-checked build)";
        default: return "unknown status";
    }
}

int yamc_destroy(yamc_ctx *c);

static int upload_beta_f(yamc_ctx *c);

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
        (r = dalloc(&c->mol, M)) || (r = dalloc(&c->kvec, S)) || (r = dalloc(&c->kpack, S)) ||
        (r = dalloc(&c->rho_f, (size_t)(1 + nt) * S)) || (r = dalloc(&c->d_check, 1)) || (r = dalloc(&c->ebeta, S)) ||
        (r = dalloc(&c->ebeta_f, S)) || (r = dalloc(&c->ebetalj_f, (size_t)H.npair * S)) ||
        (r = dalloc(&c->ebetalj, (size_t)H.npair * S)) || (r = dalloc(&c->pair_index, nt * nt)) ||
        (r = dalloc(&c->lj_sig6, nt * nt)) || (r = dalloc(&c->lj_feps, nt * nt)) || (r = dalloc(&c->rho, (size_t)(1 + nt) * S)) ||
        (r = dalloc(&c->scratch, (size_t)2 * (1 + nt) * S)) || (r = dalloc(&c->freq_beg, M)) || (r = dalloc(&c->freq_end, M)) ||
        (r = dalloc(&c->scal, SC_COUNT)) || (r = dalloc(&c->cnt, CN_COUNT)) ||
        (r = dalloc(&c->d_sys, 1)) || (r = dalloc(&c->d_run, 1)) || (r = dalloc(&c->slot, N)) ||
        (r = dalloc(&c->atom_of, (size_t)N + 16)) || (r = dalloc(&c->spec, H.spec.size() / 4)))
        return r;
    CUDA_TRY(cudaHostAlloc(&c->h_out, sizeof(double) * (kNV + SC_COUNT) + sizeof(long long) * (CN_COUNT + 1),
                           cudaHostAllocMapped));
    move_pass_done(c) = 0;
    CUDA_TRY(cudaHostGetDevicePointer(reinterpret_cast<void **>(&c->d_hout), c->h_out, 0));
    // full-sum work split: atom-tile pairs of the real-space sum; atom slices of rho(k) so that
    // entry blocks x slices cover the SMs about twice
    int nsm = 148;
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
    c->nsm = nsm;
    {
        const int T = (N + kFullTile - 1) / kFullTile;
        std::vector<int2> tp;
        tp.reserve((size_t)T * (T + 1) / 2);
        for (int ti = 0; ti < T; ++ti)
            for (int tj = ti; tj < T; ++tj) tp.push_back(make_int2(ti, tj));
        c->ntpairs = (int)tp.size();
        const int eb = (S + kRhoBlock - 1) / kRhoBlock;
        const int chunks = (N + kRhoChunk - 1) / kRhoChunk;
        const int want = std::max(1, std::min(chunks, (2 * nsm + eb - 1) / eb));
        c->rho_slice_atoms = ((chunks + want - 1) / want) * kRhoChunk;
        c->rho_slices = (N + c->rho_slice_atoms - 1) / c->rho_slice_atoms;
        if ((r = dalloc(&c->tpairs, tp.size())) || (r = upload(c->tpairs, tp.data(), tp.size(), c->stream)) ||
            // block partials: the full sums' tile pairs, the k-space energy blocks and the
            // exchange step's atom blocks (kXParts each); the totals of any of them
            (r = dalloc(&c->part, std::max({(size_t)c->ntpairs * kFullParts, (size_t)(S + 255) / 256 * 2,
                                            (size_t)(N + 255) / 256 * kXParts}))) ||
            (r = dalloc(&c->sums, std::max(kFullParts + 2, kXParts))) ||
            (r = dalloc(&c->rho_part, (size_t)(1 + nt) * c->rho_slices * S)))
            return r;
    }
    std::vector<double4> a(N);
    std::vector<int2> m(N);
    for (int i = 0; i < N; ++i) { a[i] = make_double4(H.x[i], H.y[i], H.z[i], H.q[i]); m[i] = make_int2(H.molnum[i], H.type_by_index[i]); }
    std::vector<int2> mo(M);
    for (int i = 0; i < M; ++i) mo[i] = make_int2(H.first[i], H.natoms[i]);
    std::vector<int4> kv(S);
    for (int e = 0; e < S; ++e) kv[e] = make_int4(H.ekx[e], H.eky[e], H.ekz[e], H.ekk[e]);
    if (H.kmax > 127) { set_error("kmax above 127 (the packed k of the chain kernel holds 8 bits per component)"); return YAMC_ELIMITS; }
    std::vector<int> kp(S);
    for (int e = 0; e < S; ++e) kp[e] = H.ekx[e] | ((H.eky[e] + 128) << 8) | ((H.ekz[e] + 128) << 16);
    std::vector<int> pidx(nt * nt);
    for (int i = 0; i < nt * nt; ++i) pidx[i] = H.pair_index[i];
    if ((r = upload(c->atom, a.data(), N, c->stream)) || (r = upload(c->meta, m.data(), N, c->stream)) ||
        (r = upload(c->dhs, H.dhs.data(), N, c->stream)) || (r = upload(c->mass, H.mass.data(), N, c->stream)) ||
        (r = upload(c->mol, mo.data(), M, c->stream)) || (r = upload(c->kvec, kv.data(), S, c->stream)) ||
        (r = upload(c->kpack, kp.data(), S, c->stream)) ||
        (r = upload(c->ebeta, H.ebeta.data(), S, c->stream)) || (r = upload(c->ebetalj, H.ebetalj.data(), (size_t)H.npair * S, c->stream)) ||
        (r = upload_beta_f(c)) || (r = upload(c->pair_index, pidx.data(), nt * nt, c->stream)) || (r = upload(c->lj_sig6, H.sigma6.data(), nt * nt, c->stream)) ||
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
    D.refresh_every = P.precision == YAMC_MIXED ? c->refresh_every : 0;
    D.rpre = std::sqrt(P.rmax2);
    for (int i = 0; i < N; ++i) D.rpre = std::max(D.rpre, H.dhs[i]);
    fill_dhs_types(H, D);
    D.xprob = 0.0;
    D.atom = c->atom; D.meta = c->meta; D.dhs = c->dhs; D.mass = c->mass; D.mol = c->mol; D.kvec = c->kvec;
    D.kpack = c->kpack; D.rho_f = c->rho_f; D.check = c->d_check;
    CUDA_TRY(cudaMemsetAsync(c->d_check, 0, sizeof(int), c->stream));
    D.ebeta = c->ebeta; D.ebetalj = c->ebetalj; D.pair_index = c->pair_index; D.lj_sig6 = c->lj_sig6; D.lj_feps = c->lj_feps;
    D.ebeta_f = c->ebeta_f; D.ebetalj_f = c->ebetalj_f;
    D.rho = c->rho; D.scratch = c->scratch; D.freq_beg = c->freq_beg; D.freq_end = c->freq_end; D.scal = c->scal; D.cnt = c->cnt;
    D.nspec = (int)(H.spec.size() / 4); D.spec = c->spec;
    D.slot = c->slot; D.atom_of = c->atom_of;
    if ((r = upload(c->d_sys, &D, 1, c->stream))) return r;
    c->cnt_h[CN_ICYCLE] = 1;
    c->cnt_h[CN_MOVE_IN_CYCLE] = 0;
    if ((r = full_sums(c))) return r;  // initmc
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return YAMC_OK;
}

int yamc_create(const yamc_system *sys, const yamc_params *p, int32_t device, yamc_ctx **out) {
    YAMC_RANGE("yamc_create");
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
    void *ptrs[] = {c->atom, c->meta, c->mol, c->dhs, c->mass, c->ebeta, c->ebetalj, c->ebeta_f, c->ebetalj_f,
                    c->lj_sig6, c->lj_feps, c->kvec, c->kpack, c->rho_f, c->d_check,
                    c->pair_index, c->rho, c->scratch, c->freq_beg, c->freq_end, c->scal, c->cnt, c->part, c->sums,
                    c->tpairs, c->rho_part, c->d_sys, c->d_run, c->d_rng, c->d_log, c->d_rows,
                    c->d_prof, c->spec, c->d_gx, c->d_gy, c->d_gz, c->d_fpart, c->rho_save, c->d_mpart,
                    c->d_mcount, c->slot, c->atom_of};
    for (void *p : ptrs) if (p) cudaFree(p);
    if (c->h_out) cudaFreeHost(c->h_out);
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
    YAMC_RANGE("yamc_full_sums");
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
    ChainArgs a = base_args(c);
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
    return bounds_status(c, back.status);
}

int yamc_set_refresh(yamc_ctx *c, int64_t accepted_moves) {
    if (!c || accepted_moves < 0) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    c->refresh_every = accepted_moves;
    c->hsys.refresh_every = is_mixed(c) ? accepted_moves : 0;
    int r = upload(c->d_sys, &c->hsys, 1, c->stream);
    if (r) return r;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return YAMC_OK;
}

int yamc_refresh_count(yamc_ctx *c, int64_t *count) {
    if (!c || !count) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    int r = pull_state(c);
    if (r) return r;
    *count = c->cnt_h[CN_REFRESHES];
    return YAMC_OK;
}

int yamc_run_chain_device(yamc_ctx *c, const float *d_rng, int64_t n_rng, int64_t *cursor, int64_t n_moves,
                          int64_t *moves_done, yamc_move_record *d_log, double *d_rows, int32_t max_rows, int32_t *n_rows) {
    YAMC_RANGE("yamc_run_chain_device");
    if (!c || !d_rng || !cursor || n_moves < 0) return YAMC_EPARAMETER;
    if (c->H.p.pressure_step_multiplier > 0 || c->H.xchange_probability > 0) {
        set_error("NPT volume cycles or exchange steps are on: they run through yamc_run_mc");
        return YAMC_EWRONG_FUNCTION;
    }
    CUDA_TRY(cudaSetDevice(c->device));
    return run_chain_impl(c, d_rng, 0, n_rng, cursor, n_moves, moves_done, d_log, d_rows, max_rows, n_rows);
}

int yamc_run_chain(yamc_ctx *c, const float *rng, int64_t n_rng, int64_t *cursor, int64_t n_moves, int64_t *moves_done,
                   yamc_move_record *log, double *rows, int32_t max_rows, int32_t *n_rows) {
    YAMC_RANGE("yamc_run_chain");
    if (!c || !rng || !cursor || n_moves < 0 || *cursor < 0 || *cursor > n_rng) return YAMC_EPARAMETER;
    if (c->H.p.pressure_step_multiplier > 0 || c->H.xchange_probability > 0) {
        set_error("NPT volume cycles or exchange steps are on: they run through yamc_run_mc");
        return YAMC_EWRONG_FUNCTION;
    }
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
    if (st != YAMC_OK && st != YAMC_ERNG_EXHAUSTED && st != YAMC_ENAN) return st;
    if (st == YAMC_ENAN) set_error("non-finite energy change or bias force: the chain stopped before that move");
    if (log && done) CUDA_TRY(cudaMemcpy(log, c->d_log, sizeof(yamc_move_record) * done, cudaMemcpyDeviceToHost));
    if (rows && nrow) CUDA_TRY(cudaMemcpy(rows, c->d_rows, sizeof(double) * 9 * nrow, cudaMemcpyDeviceToHost));
    if (moves_done) *moves_done = done;
    if (n_rows) *n_rows = nrow;
    return st;
}

// ---------------------------------------------------------------- NPT volume move

// rand() of random.f90:65-93 on the host: the next value of the stream, values outside
// [1e-14, 1 - 1e-14] drawn again; false when the stream runs out
static bool host_rand(const float *rng, int64_t n_rng, int64_t *cursor, double *out) {
    float v = 0.0f;
    while ((double)v < 1e-14 || (double)v > 1.0 - 1e-14) {
        if (*cursor >= n_rng) return false;
        v = rng[(*cursor)++];
    }
    *out = (double)v;
    return true;
}

// the device data that depend on the box length, from the host copy: positions, hard-core
// diameters / L, beta and beta_LJ per signed entry, the LJ tables and the scalar parameters
// the mixed form's FP32 copies of the beta tables, from H.ebeta / H.ebetalj as they stand
static int upload_beta_f(yamc_ctx *c) {
    const HostSystem &H = c->H;
    c->h_ebeta_f.assign(H.ebeta.begin(), H.ebeta.end());
    c->h_ebetalj_f.assign(H.ebetalj.begin(), H.ebetalj.end());
    int r;
    if ((r = upload(c->ebeta_f, c->h_ebeta_f.data(), c->h_ebeta_f.size(), c->stream)) ||
        (r = upload(c->ebetalj_f, c->h_ebetalj_f.data(), c->h_ebetalj_f.size(), c->stream)))
        return r;
    return YAMC_OK;
}

static int upload_box(yamc_ctx *c) {
    HostSystem &H = c->H;
    const int N = H.N, S = H.S, nt = H.nt;
    std::vector<double4> a(N);
    for (int i = 0; i < N; ++i) a[i] = make_double4(H.x[i], H.y[i], H.z[i], H.q[i]);
    for (int e = 0; e < S; ++e) H.ebeta[e] = H.beta[H.ekk[e]];
    int r;
    if ((r = upload(c->atom, a.data(), N, c->stream)) || (r = upload(c->dhs, H.dhs.data(), N, c->stream)) ||
        (r = upload(c->ebeta, H.ebeta.data(), S, c->stream)) ||
        (r = upload(c->ebetalj, H.ebetalj.data(), (size_t)H.npair * S, c->stream)) || (r = upload_beta_f(c)) ||
        (r = upload(c->lj_sig6, H.sigma6.data(), nt * nt, c->stream)) ||
        (r = upload(c->lj_feps, H.four_eps.data(), nt * nt, c->stream)))
        return r;
    DevSys &D = c->hsys;
    const yamc_params &P = H.p;
    D.rmax2 = P.rmax2; D.alpha = P.alpha; D.xclb = P.xclb; D.taosp = P.two_alpha_over_sqrt_pi; D.kext = P.kext;
    D.m2k = P.minus_two_kext; D.dr = P.dr; D.d_angle = P.d_angle;
    D.rpre = std::sqrt(P.rmax2);
    for (int i = 0; i < N; ++i) D.rpre = std::max(D.rpre, H.dhs[i]);
    fill_dhs_types(H, D);
    if ((r = upload(c->d_sys, &D, 1, c->stream))) return r;
    c->pos_valid = true;
    return YAMC_OK;
}

// scale_box (scale_box.f90:6-62) on the host copy: each molecule's centre of mass
// (center_of_mass, geometry.f90:170-201) keeps its box coordinates, its atoms' offsets scale
// by L_old / L_new (bond lengths in Angstrom stay), one-atom molecules stay; sigma scales too
static void scale_box_host(HostSystem &H, double new_L) {
    const double c = H.p.BoxLength / new_L;
    for (int m = 0; m < H.M; ++m) {
        const int f = H.first[m], n = H.natoms[m];
        if (n == 1) continue;
        double sx = 0, sy = 0, sz = 0, tm = 0;
        for (int a = f; a < f + n; ++a) {
            sx = sx + H.mass[a] * H.x[a]; sy = sy + H.mass[a] * H.y[a]; sz = sz + H.mass[a] * H.z[a];
            tm = tm + H.mass[a];
        }
        const double xc = sx / tm, yc = sy / tm, zc = sz / tm;
        for (int a = f; a < f + n; ++a) {
            H.x[a] = (H.x[a] - xc) * c + xc;
            H.y[a] = (H.y[a] - yc) * c + yc;
            H.z[a] = (H.z[a] - zc) * c + zc;
        }
    }
    for (int i = 0; i < H.N; ++i) H.sigma[i] = H.sigma[i] * c;
}

// mcvol up to the acceptance test (MC.f90:735-799): save the state (mc_save_state), scale
// the box, Parameters_recalc, LJTypes_scale_sigma, EwaldSumKSpace_initBetaLJ and the full
// sums with beta scaled by xclb_new / xclb_old (mc_calc_total_sums with scale_beta; alpha*L
// is fixed, so beta6/beta12 and the k-set do not change)
static int volume_eval(yamc_ctx *c, double new_L, double *du, int *overlap) {
    HostSystem &H = c->H;
    auto &v = c->vol;
    int r;
    if ((r = sync_positions(c)) || (r = pull_state(c))) return r;
    double e[8];
    energies_from(c->sc, H.p.kext, e);
    v.U_old = e[0];
    v.p = H.p; v.x = H.x; v.y = H.y; v.z = H.z; v.sigma = H.sigma; v.type_sigma = H.type_sigma; v.beta = H.beta;
    v.ebetalj = H.ebetalj; v.lj6 = H.lj6; v.lj12 = H.lj12; v.four_eps = H.four_eps; v.sigma6 = H.sigma6;
    v.sigma2 = H.sigma2; v.dhs = H.dhs;
    std::copy(c->sc, c->sc + SC_COUNT, v.sc);
    v.tail_c = H.U_tail_coul; v.tail6 = H.U_tail_lj6; v.tail12 = H.U_tail_lj12;
    const size_t nrho = (size_t)(1 + H.nt) * H.S;
    if (!c->rho_save && (r = dalloc(&c->rho_save, nrho))) return r;
    CUDA_TRY(cudaMemcpyAsync(c->rho_save, c->rho, sizeof(double2) * nrho, cudaMemcpyDeviceToDevice, c->stream));
    v.old_L = H.p.BoxLength; v.new_L = new_L;
    scale_box_host(H, new_L);
    v.xclb_old = H.p.xclb;
    if ((r = yamc_params_recalc(&H.p, new_L))) return r;
    v.xclb_new = H.p.xclb;
    for (double &t : H.type_sigma) t = t * (v.old_L / new_L);
    fill_lj_tables(H);
    fill_beta_lj(H);
    const double scale_beta = v.xclb_new / v.xclb_old;  // positive: the recompute branch of EwaldSumKSpace_init is never taken
    for (double &b : H.beta) b = b * scale_beta;
    for (int i = 0; i < H.N; ++i) H.dhs[i] = H.hc[i] / new_L;
    compute_tails(H);
    if ((r = upload_box(c))) return r;
    int ov = 0;
    if ((r = full_sums(c, &ov))) return r;
    energies_from(c->sc, H.p.kext, e);
    *du = ov ? 0.0 : e[0] - v.U_old;
    *overlap = ov;
    c->vol_stage = 1;
    return YAMC_OK;
}

// the end of mcvol (MC.f90:801-823): an accepted step keeps the new box; a rejected one
// takes mc_restore_state and puts the parameters, LJ tables and beta back as the reference
// does (sigma scaled by L_new / L_old, beta by xclb_old / xclb_new, both to rounding).
// exact != 0 instead restores every table bit for bit (a step abandoned because the random
// stream ran out, which the reference never meets).
static int volume_commit(yamc_ctx *c, bool accepted, bool exact) {
    HostSystem &H = c->H;
    auto &v = c->vol;
    c->vol_stage = 0;
    if (accepted) {
        CUDA_TRY(cudaStreamSynchronize(c->stream));
        return YAMC_OK;
    }
    H.x = v.x; H.y = v.y; H.z = v.z; H.sigma = v.sigma;
    std::copy(v.sc, v.sc + SC_COUNT, c->sc);
    H.U_tail_coul = v.tail_c; H.U_tail_lj6 = v.tail6; H.U_tail_lj12 = v.tail12;
    if (exact) {
        H.p = v.p; H.type_sigma = v.type_sigma; H.beta = v.beta; H.ebetalj = v.ebetalj; H.lj6 = v.lj6;
        H.lj12 = v.lj12; H.four_eps = v.four_eps; H.sigma6 = v.sigma6; H.sigma2 = v.sigma2;
    } else {
        int r = yamc_params_recalc(&H.p, v.old_L);
        if (r) return r;
        for (double &t : H.type_sigma) t = t * (v.new_L / v.old_L);
        fill_lj_tables(H);
        fill_beta_lj(H);
        for (double &b : H.beta) b = b * v.xclb_old / v.xclb_new;
    }
    H.dhs = v.dhs;
    const size_t nrho = (size_t)(1 + H.nt) * H.S;
    CUDA_TRY(cudaMemcpyAsync(c->rho, c->rho_save, sizeof(double2) * nrho, cudaMemcpyDeviceToDevice, c->stream));
    int r;
    if ((r = upload_box(c)) || (r = push_state(c))) return r;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return YAMC_OK;
}

// one whole mcvol (MC.f90:701-825) with its draws from a host stream: lambda, then the
// acceptance draw only when the probability is not above 1 (`(proba > 1) .or. (rand() <
// proba)` with the short-circuit of gfortran's optimised builds); an overlap gives
// proba = -1, so it draws and rejects.  On exhaustion the step is undone and the cursor
// put back to where it was.
static int volume_step(yamc_ctx *c, const float *rng, int64_t n_rng, int64_t *cursor, yamc_volume_record *rec) {
    const int64_t cur0 = *cursor;
    double u;
    if (!host_rand(rng, n_rng, cursor, &u)) {
        *cursor = cur0;
        set_error("random stream exhausted at a volume step");
        return YAMC_ERNG_EXHAUSTED;
    }
    const double old_L = c->H.p.BoxLength, old_V = old_L * old_L * old_L;
    const double lambda = 2 * u - 1.0;
    const double log_new_V = std::log(old_V) + lambda * c->H.p.log_max_volume_scaling;
    const double new_V = std::exp(log_new_V);
    const double new_L = std::pow(new_V, 1.0 / 3.0);
    double du = 0;
    int ov = 0;
    int r = volume_eval(c, new_L, &du, &ov);
    if (r) return r;
    double proba, arg = 0;
    if (!ov) {
        const double dV = new_V - old_V;
        arg = -du - c->H.p.pressure_angstr_kT * dV + (c->H.M + 1) * std::log(new_V / old_V);
        proba = std::exp(arg);
    } else {
        proba = -1.0;
    }
    bool acc = true;
    if (!(proba > 1)) {
        double x;
        if (!host_rand(rng, n_rng, cursor, &x)) {
            if ((r = volume_commit(c, false, true))) return r;
            *cursor = cur0;
            set_error("random stream exhausted inside a volume step (undone)");
            return YAMC_ERNG_EXHAUSTED;
        }
        acc = x < proba;
    }
    if ((r = volume_commit(c, acc, false))) return r;
    rec->flags = (acc ? 1 : 0) | (ov ? 2 : 0);
    rec->pad = 0;
    rec->cursor = *cursor;
    rec->box_old = old_L; rec->box_new = new_L; rec->du = du; rec->arg = arg;
    return YAMC_OK;
}

// ---------------------------------------------------------------- exchange move

// mc_xchange (MC.f90:1325-1954) up to the acceptance test.  The real-space change follows the
// reference: the two molecules' per-atom energies after the swap minus before
// (MC.f90:1451-1452, 1639-1642), each of which holds the 1-2 pair energy, so that pair term
// enters twice; the device sums both molecules (old and new) against every other atom, the host
// adds the 1-2 pairs (at most 16).  k space and the external term are the exact two-molecule
// changes.  du = {dU_real, dU_k_coulomb, dU_k_LJ, dU_ext}.
static int xchange_eval(yamc_ctx *c, int imol1, int imol2, double du[4], int *overlap) {
    HostSystem &H = c->H;
    auto &X = c->xch;
    int r;
    if ((r = sync_positions(c)) || (r = pull_state(c))) return r;
    const int m1 = imol1 - 1, m2 = imol2 - 1;
    const int f1 = H.first[m1], n1 = H.natoms[m1], f2 = H.first[m2], n2 = H.natoms[m2];
    XchgIn in{};
    in.m1 = m1; in.m2 = m2; in.n1 = n1; in.n2 = n2;
    double cm[2][3];
    for (int k = 0; k < 2; ++k) {  // center_of_mass (geometry.f90:170-201)
        const int f = k ? f2 : f1, n = k ? n2 : n1;
        double sx = 0, sy = 0, sz = 0, tm = 0;
        for (int a = f; a < f + n; ++a) {
            sx = sx + H.mass[a] * H.x[a]; sy = sy + H.mass[a] * H.y[a]; sz = sz + H.mass[a] * H.z[a]; tm = tm + H.mass[a];
        }
        cm[k][0] = sx / tm; cm[k][1] = sy / tm; cm[k][2] = sz / tm;
    }
    for (int a = 0; a < n1 + n2; ++a) {
        const int k = a < n1 ? 0 : 1, i = k ? f2 + (a - n1) : f1 + a;
        const double *co = cm[k], *cn = cm[1 - k];
        in.o[a] = make_double4(H.x[i], H.y[i], H.z[i], H.q[i]);
        // xnew = xold - x_center(own) + x_center(other), not wrapped (MC.f90:1516-1524)
        X.x[a] = H.x[i] - co[0] + cn[0]; X.y[a] = H.y[i] - co[1] + cn[1]; X.z[a] = H.z[i] - co[2] + cn[2];
        in.n[a] = make_double4(X.x[a], X.y[a], X.z[a], H.q[i]);
        in.type[a] = H.type_by_index[i];
        in.dhs[a] = H.dhs[i];
    }
    X.m1 = m1; X.m2 = m2;
    const int nb = (H.N + 255) / 256;
    k_xchg_real<<<nb, 256, 0, c->stream>>>(c->hsys, in, c->part);
    CUDA_TRY(cudaGetLastError());
    k_sum_parts<<<1, kSumThreads, 0, c->stream>>>(c->part, nb, kXParts, 12, c->sums);
    CUDA_TRY(cudaGetLastError());
    double rs[kXParts];
    CUDA_TRY(cudaMemcpyAsync(rs, c->sums, sizeof(rs), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    // the 1-2 pairs, old and new, on the host with the device's pair formula
    const yamc_params &P = H.p;
    double u12[2][3] = {};
    bool ov12 = false;
    for (int w = 0; w < 2; ++w)
        for (int a = 0; a < n1; ++a)
            for (int b = n1; b < n1 + n2; ++b) {
                const double4 pa = w ? in.n[a] : in.o[a], pb = w ? in.n[b] : in.o[b];
                const double dx = min_image(pa.x - pb.x), dy = min_image(pa.y - pb.y), dz = min_image(pa.z - pb.z);
                const double r2 = dx * dx + dy * dy + dz * dz;
                const bool lj = in.type[a] > 0 && in.type[b] > 0;
                if (w == 1 && lj) {
                    const double d12 = (in.dhs[a] + in.dhs[b]) / 2;
                    if (r2 < d12 * d12) ov12 = true;
                }
                if (r2 >= P.rmax2) continue;
                const int off = lj ? (in.type[a] - 1) * H.nt + (in.type[b] - 1) : 0;
                const PairTerm<double> t = pair_term<double, false>(r2, P.xclb * pa.w * pb.w, lj, lj ? H.sigma6[off] : 0.0,
                                                                     lj ? H.four_eps[off] : 0.0, P.alpha,
                                                                     P.two_alpha_over_sqrt_pi, false);
                u12[w][0] += t.ew; u12[w][1] += t.lj6; u12[w][2] += t.lj12;
            }
    *overlap = rs[12] > 0 || ov12;
    if (*overlap) {
        du[0] = du[1] = du[2] = du[3] = 0;
        c->xch_stage = 2;
        return YAMC_OK;
    }
    auto E = [&](const double *v) { return v[0] + v[2] - v[1]; };  // ew + lj12 - lj6
    const double Eo1 = E(rs + 0), En1 = E(rs + 3), Eo2 = E(rs + 6), En2 = E(rs + 9);
    const double U12o = E(u12[0]), U12n = E(u12[1]);
    const double E_old = (Eo1 + U12o) + (Eo2 + U12o), E_new = (En1 + U12n) + (En2 + U12n);
    du[0] = E_new - E_old;
    // the bookkeeping change of the totals takes the 1-2 pairs once (MC.f90:1813-1826)
    X.d_ew = (rs[3] + rs[9] + u12[1][0]) - (rs[0] + rs[6] + u12[0][0]);
    X.d_lj6 = (rs[4] + rs[10] + u12[1][1]) - (rs[1] + rs[7] + u12[0][1]);
    X.d_lj12 = (rs[5] + rs[11] + u12[1][2]) - (rs[2] + rs[8] + u12[0][2]);
    // k space
    const size_t sm = sizeof(double2) * (size_t)(n1 + n2) * 2 * 3 * (H.kmax + 1);
    const int nbk = (H.S + 255) / 256;
    switch (H.nt) {
        case 1: CUDA_TRY(cudaFuncSetAttribute(k_xchg_kspace<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                k_xchg_kspace<1><<<nbk, 256, sm, c->stream>>>(c->hsys, in, c->scratch, c->part); break;
        case 2: CUDA_TRY(cudaFuncSetAttribute(k_xchg_kspace<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                k_xchg_kspace<2><<<nbk, 256, sm, c->stream>>>(c->hsys, in, c->scratch, c->part); break;
        case 3: CUDA_TRY(cudaFuncSetAttribute(k_xchg_kspace<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                k_xchg_kspace<3><<<nbk, 256, sm, c->stream>>>(c->hsys, in, c->scratch, c->part); break;
        default: CUDA_TRY(cudaFuncSetAttribute(k_xchg_kspace<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
                 k_xchg_kspace<4><<<nbk, 256, sm, c->stream>>>(c->hsys, in, c->scratch, c->part); break;
    }
    CUDA_TRY(cudaGetLastError());
    k_sum_parts<<<1, kSumThreads, 0, c->stream>>>(c->part, nbk, 2, -1, c->sums);
    CUDA_TRY(cudaGetLastError());
    double ek[2];
    CUDA_TRY(cudaMemcpyAsync(ek, c->sums, sizeof(ek), cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    X.du_kc = ek[0]; X.du_kl = ek[1];
    du[1] = ek[0]; du[2] = ek[1];
    // external term (EwaldSumExternal_calc_dU) with dmu = dmu1 + dmu2
    double dm[2][3] = {};
    for (int k = 0; k < 2; ++k) {
        double mo[3] = {}, mn[3] = {};
        const int a0 = k ? n1 : 0, a1 = k ? n1 + n2 : n1;
        for (int a = a0; a < a1; ++a) {
            const double q = in.o[a].w;
            mo[0] = mo[0] + q * in.o[a].x; mo[1] = mo[1] + q * in.o[a].y; mo[2] = mo[2] + q * in.o[a].z;
            mn[0] = mn[0] + q * X.x[a]; mn[1] = mn[1] + q * X.y[a]; mn[2] = mn[2] + q * X.z[a];
        }
        for (int d = 0; d < 3; ++d) dm[k][d] = mn[d] - mo[d];
    }
    for (int d = 0; d < 3; ++d) X.dmu[d] = dm[0][d] + dm[1][d];
    const double mu[3] = {c->sc[SC_MU_X], c->sc[SC_MU_Y], c->sc[SC_MU_Z]};
    du[3] = P.kext * ((2 * mu[0] + X.dmu[0]) * X.dmu[0] + (2 * mu[1] + X.dmu[1]) * X.dmu[1] + (2 * mu[2] + X.dmu[2]) * X.dmu[2]);
    c->xch_stage = 1;
    return YAMC_OK;
}

// the acceptance branch of mc_xchange (MC.f90:1758-1848): rho += delta, the two molecules at the
// swapped positions, the totals and the dipole updated; a rejection changes nothing
static int xchange_commit(yamc_ctx *c, bool accepted) {
    HostSystem &H = c->H;
    const auto &X = c->xch;
    const int stage = c->xch_stage;
    c->xch_stage = 0;
    if (!accepted || stage != 1) return YAMC_OK;
    const int n = (1 + H.nt) * H.S;
    k_commit_rho<<<(n + 255) / 256, 256, 0, c->stream>>>(c->rho, c->scratch, n);
    CUDA_TRY(cudaGetLastError());
    const int f1 = H.first[X.m1], n1 = H.natoms[X.m1], f2 = H.first[X.m2], n2 = H.natoms[X.m2];
    for (int k = 0; k < 2; ++k) {
        const int f = k ? f2 : f1, na = k ? n2 : n1, a0 = k ? n1 : 0;
        double4 a[kMaxA];
        for (int i = 0; i < na; ++i) {
            H.x[f + i] = X.x[a0 + i]; H.y[f + i] = X.y[a0 + i]; H.z[f + i] = X.z[a0 + i];
            a[i] = make_double4(H.x[f + i], H.y[f + i], H.z[f + i], H.q[f + i]);
        }
        int r = upload(c->atom + f, a, na, c->stream);
        if (r) return r;
    }
    c->sc[SC_UU_EW] = c->sc[SC_UU_EW] + X.d_ew;
    c->sc[SC_UU_LJ6] = c->sc[SC_UU_LJ6] + X.d_lj6;
    c->sc[SC_UU_LJ12] = c->sc[SC_UU_LJ12] + X.d_lj12;
    c->sc[SC_EK_C] = c->sc[SC_EK_C] + X.du_kc;
    c->sc[SC_EK_LJ] = c->sc[SC_EK_LJ] + X.du_kl;
    c->sc[SC_MU_X] = c->sc[SC_MU_X] + X.dmu[0];
    c->sc[SC_MU_Y] = c->sc[SC_MU_Y] + X.dmu[1];
    c->sc[SC_MU_Z] = c->sc[SC_MU_Z] + X.dmu[2];
    int r = push_state(c);
    if (r) return r;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return YAMC_OK;
}

// BiasedRandom_choose (BiasedRandom.f90:81-109): the first interval with beg < rnd < end, else 1
static int host_choose(const std::vector<double> &beg, const std::vector<double> &end, double rnd) {
    for (size_t i = 0; i < beg.size(); ++i)
        if (rnd > beg[i] && rnd < end[i]) return (int)i + 1;
    return 1;
}

int yamc_set_xchange_weights(yamc_ctx *c, const double *w) {
    if (!c || !w) return YAMC_EPARAMETER;
    if (c->in_batch) { set_error("a batch replica runs NVT moves only (volume and exchange steps need a context of its own)"); return YAMC_EWRONG_FUNCTION; }
    HostSystem &H = c->H;
    const int M = H.M;
    double S = 0;
    for (int i = 0; i < M; ++i) {
        if (!(w[i] >= 0)) { set_error("exchange weights must be non-negative"); return YAMC_EPARAMETER; }
        S = S + w[i];
    }
    // BiasedRandom_init (BiasedRandom.f90:44-79) on the exchange weights
    H.xfreq_beg.assign(M, 0.0); H.xfreq_end.assign(M, 0.0);
    std::vector<double> prob(M);
    for (int i = 0; i < M; ++i) prob[i] = (S == 0) ? 1.0 / M : w[i] / S;
    H.xfreq_beg[0] = 0.0; H.xfreq_end[0] = prob[0];
    for (int i = 1; i < M; ++i) { H.xfreq_beg[i] = H.xfreq_end[i - 1]; H.xfreq_end[i] = H.xfreq_beg[i] + prob[i]; }
    if (S > 0)
        for (int i = 0; i < M; ++i) if (w[i] == 0) H.xfreq_end[i] = -1.0;
    int nz = 0;
    for (int i = 0; i < M; ++i) nz += w[i] > 0;
    if (S > 0 && nz < 2) { set_error("exchange steps need at least two molecules with a positive weight"); return YAMC_EPARAMETER; }
    H.xchange_probability = S / (H.smv + S);
    CUDA_TRY(cudaSetDevice(c->device));
    c->hsys.xprob = H.xchange_probability;
    int r = upload(c->d_sys, &c->hsys, 1, c->stream);
    if (r) return r;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    return YAMC_OK;
}

int yamc_xchange_eval(yamc_ctx *c, int32_t imol1, int32_t imol2, double du[4], int32_t *overlap) {
    YAMC_RANGE("yamc_xchange_eval");
    if (!c || !du || !overlap || imol1 < 1 || imol2 < 1 || imol1 > c->H.M || imol2 > c->H.M || imol1 == imol2)
        return YAMC_EPARAMETER;
    if (c->in_batch) { set_error("a batch replica runs NVT moves only (volume and exchange steps need a context of its own)"); return YAMC_EWRONG_FUNCTION; }
    if (c->api_stage || c->vol_stage || c->xch_stage) { set_error("a move, volume or exchange step is pending"); return YAMC_EWRONG_FUNCTION; }
    CUDA_TRY(cudaSetDevice(c->device));
    int ov = 0;
    const int r = xchange_eval(c, imol1, imol2, du, &ov);
    *overlap = ov;
    return r;
}

int yamc_xchange_commit(yamc_ctx *c, int32_t accepted) {
    YAMC_RANGE("yamc_xchange_commit");
    if (!c) return YAMC_EPARAMETER;
    if (!c->xch_stage) { set_error("no exchange step is pending"); return YAMC_EWRONG_FUNCTION; }
    CUDA_TRY(cudaSetDevice(c->device));
    return xchange_commit(c, accepted != 0);
}

// ---------------------------------------------------------------- radial distribution functions

struct yamc_rdf {
    int device = 0, M = 0, ntypes = 0, nbin = 0, grid = 1, n_frame = 0;
    double dr = 0, rmax = 0, sum_inv_vol = 0;
    size_t smem = 0;
    std::vector<int32_t> mol_numbers;
    cudaStream_t stream = nullptr;
    int *type = nullptr;
    double *cx = nullptr, *cy = nullptr, *cz = nullptr;
    unsigned long long *hist = nullptr;  // [ntypes^2][nbin] counts, then [ntypes^2] pair totals
};

static int rdf_frame(yamc_rdf *h, double L) {
    const int nbox = h->rmax < L / 2 ? 0 : (int)((h->rmax - L / 2) / L) + 1;  // mcrdf2.f90:206-210
    k_rdf_count<<<h->grid, 256, h->smem, h->stream>>>(h->cx, h->cy, h->cz, h->type, h->M, h->ntypes, h->nbin, L, h->dr,
                                                      h->rmax * h->rmax, nbox, h->hist);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    h->n_frame += 1;
    h->sum_inv_vol += 1.0 / (L * L * L);
    return YAMC_OK;
}

int yamc_rdf_destroy(yamc_rdf *h) {
    if (!h) return YAMC_OK;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    void *ptrs[] = {h->type, h->cx, h->cy, h->cz, h->hist};
    for (void *p : ptrs) if (p) cudaFree(p);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return YAMC_OK;
}

static int rdf_create_impl(yamc_rdf *h, int32_t nmol, const int32_t *mol_type, int32_t ntypes, const int32_t *mol_numbers,
                           double dr, double rmax, int32_t device) {
    if (nmol < 1 || !mol_type || ntypes < 1 || !mol_numbers || !(dr > 0) || !(rmax > dr)) return YAMC_EPARAMETER;
    for (int i = 0; i < nmol; ++i)
        if (mol_type[i] < 1 || mol_type[i] > ntypes) { set_error("mol_type outside 1..ntypes"); return YAMC_EPARAMETER; }
    h->device = device; h->M = nmol; h->ntypes = ntypes; h->dr = dr; h->rmax = rmax;
    h->nbin = (int)((rmax - 1e-10) / dr) + 2;  // N of count_distances (mcrdf2.f90:140)
    h->mol_numbers.assign(mol_numbers, mol_numbers + ntypes);
    const size_t nh = (size_t)ntypes * ntypes * h->nbin + (size_t)ntypes * ntypes;
    h->smem = sizeof(unsigned int) * nh;
    CUDA_TRY(cudaSetDevice(device));
    cudaDeviceProp prop;
    CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (h->smem > prop.sharedMemPerBlockOptin) { set_error("too many RDF bins x species pairs for one block's histogram"); return YAMC_ELIMITS; }
    CUDA_TRY(cudaFuncSetAttribute(k_rdf_count, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)h->smem));
    const long long pairs = (long long)nmol * nmol;
    h->grid = (int)std::max(1LL, std::min((pairs + 255) / 256, 4LL * prop.multiProcessorCount));
    CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    int r;
    if ((r = dalloc(&h->type, nmol)) || (r = dalloc(&h->cx, nmol)) || (r = dalloc(&h->cy, nmol)) || (r = dalloc(&h->cz, nmol)) ||
        (r = dalloc(&h->hist, nh)) || (r = upload(h->type, mol_type, nmol, h->stream)))
        return r;
    CUDA_TRY(cudaMemsetAsync(h->hist, 0, sizeof(unsigned long long) * nh, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return YAMC_OK;
}

int yamc_rdf_create(int32_t nmol, const int32_t *mol_type, int32_t ntypes, const int32_t *mol_numbers, double dr,
                    double rmax, int32_t device, yamc_rdf **out) {
    if (!out) return YAMC_EPARAMETER;
    *out = nullptr;
    yamc_rdf *h = new yamc_rdf();
    const int r = rdf_create_impl(h, nmol, mol_type, ntypes, mol_numbers, dr, rmax, device);
    if (r) { yamc_rdf_destroy(h); return r; }
    *out = h;
    return YAMC_OK;
}

int yamc_rdf_nbin(yamc_rdf *h, int32_t *nbin) {
    if (!h || !nbin) return YAMC_EPARAMETER;
    *nbin = h->nbin;
    return YAMC_OK;
}

int yamc_rdf_add_frame(yamc_rdf *h, const double *x, const double *y, const double *z, double box_length) {
    if (!h || !x || !y || !z || !(box_length > 0)) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(h->device));
    int r;
    if ((r = upload(h->cx, x, h->M, h->stream)) || (r = upload(h->cy, y, h->M, h->stream)) ||
        (r = upload(h->cz, z, h->M, h->stream)))
        return r;
    return rdf_frame(h, box_length);
}

int yamc_rdf_add_ctx(yamc_rdf *h, yamc_ctx *c) {
    if (!h || !c) return YAMC_EPARAMETER;
    if (c->device != h->device || c->H.M != h->M) { set_error("the context's device or molecule count differs from the RDF's"); return YAMC_EPARAMETER; }
    if (c->api_stage || c->vol_stage || c->xch_stage) { set_error("a move, volume or exchange step is pending"); return YAMC_EWRONG_FUNCTION; }
    CUDA_TRY(cudaSetDevice(h->device));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    k_mol_centres<<<(h->M + 255) / 256, 256, 0, h->stream>>>(c->hsys, h->cx, h->cy, h->cz);
    CUDA_TRY(cudaGetLastError());
    return rdf_frame(h, c->H.p.BoxLength);
}

int yamc_rdf_result(yamc_rdf *h, double *g, double *counts, int32_t *n_frames) {
    if (!h) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(h->device));
    const int nt = h->ntypes, nb = h->nbin, npair = nt * nt;
    std::vector<unsigned long long> hc((size_t)npair * nb + npair);
    CUDA_TRY(cudaMemcpyAsync(hc.data(), h->hist, sizeof(unsigned long long) * hc.size(), cudaMemcpyDeviceToHost, h->stream));
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    if (n_frames) *n_frames = h->n_frame;
    if (counts)
        for (size_t k = 0; k < (size_t)npair * nb; ++k) counts[k] = (double)hc[k];
    if (g) {
        // save_rdfs (mcrdf2.f90:371-440): g = cnt4 / N_frame / <1/V> / N_i / N_j / dV / factor
        const double dr = h->dr, four_pi_dr = kFourPi * dr, small_ball = 4.0 / 3.0 * kPi * dr * dr * dr;
        const double avg_inv_vol = h->n_frame ? h->sum_inv_vol / h->n_frame : 0.0;
        for (int i = 0; i < nt; ++i)
            for (int j = 0; j < nt; ++j) {
                const int off = i * nt + j;
                double r = 0.0;
                for (int k = 0; k < nb; ++k) {
                    double v = 0.0;
                    if (j >= i && h->n_frame > 0 && hc[(size_t)npair * nb + off] > 0) {
                        const double dV = four_pi_dr * (r * r + r * dr) + small_ball;
                        const double factor = i == j ? 1.0 : 2.0;
                        v = (double)hc[(size_t)off * nb + k] / h->n_frame / avg_inv_vol / h->mol_numbers[i] /
                            h->mol_numbers[j] / dV / factor;
                    }
                    g[(size_t)off * nb + k] = v;
                    r = r + dr;
                }
            }
    }
    return YAMC_OK;
}

int yamc_volume_eval(yamc_ctx *c, double new_box_length, double *du, int32_t *overlap) {
    YAMC_RANGE("yamc_volume_eval");
    if (!c || !du || !overlap || !(new_box_length > 0)) return YAMC_EPARAMETER;
    if (c->in_batch) { set_error("a batch replica runs NVT moves only (volume and exchange steps need a context of its own)"); return YAMC_EWRONG_FUNCTION; }
    if (c->api_stage || c->vol_stage || c->xch_stage) { set_error("a move, volume or exchange step is pending"); return YAMC_EWRONG_FUNCTION; }
    CUDA_TRY(cudaSetDevice(c->device));
    int ov = 0;
    const int r = volume_eval(c, new_box_length, du, &ov);
    *overlap = ov;
    return r;
}

int yamc_volume_commit(yamc_ctx *c, int32_t accepted) {
    YAMC_RANGE("yamc_volume_commit");
    if (!c) return YAMC_EPARAMETER;
    if (!c->vol_stage) { set_error("no volume step is pending"); return YAMC_EWRONG_FUNCTION; }
    CUDA_TRY(cudaSetDevice(c->device));
    return volume_commit(c, accepted != 0, false);
}

int yamc_get_params(yamc_ctx *c, yamc_params *p) {
    if (!c || !p) return YAMC_EPARAMETER;
    *p = c->H.p;
    return YAMC_OK;
}

// energy.dat row at the end of a cycle the host ran (runmc.f90:276-279), then the next cycle
static void host_cycle_end(yamc_ctx *c, double *rows, int32_t max_rows, int32_t *nrow) {
    const HostSystem &H = c->H;
    const double fr = c->sc[SC_N_MV_STEPS] / H.M + c->sc[SC_N_VOL_STEPS];
    if (std::fmod(fr, H.p.n_store_energy_interval) < 1e-10 && rows && *nrow < max_rows) {
        double e[8];
        energies_from(c->sc, H.p.kext, e);
        double *row = rows + 9 * (size_t)*nrow;
        row[0] = (double)c->cnt_h[CN_ICYCLE];
        for (int k = 0; k < 8; ++k) row[1 + k] = e[k];
        ++*nrow;
    }
    c->cnt_h[CN_ICYCLE] += 1;
}

int yamc_run_mc(yamc_ctx *c, const float *rng, int64_t n_rng, int64_t *cursor, int64_t n_cycles, int64_t *cycles_done,
                yamc_move_record *log, int64_t max_log, int64_t *n_log, yamc_volume_record *vlog, int64_t max_vlog,
                int64_t *n_vlog, double *rows, int32_t max_rows, int32_t *n_rows) {
    YAMC_RANGE("yamc_run_mc");
    if (!c || !rng || !cursor || n_cycles < 0 || *cursor < 0 || *cursor > n_rng) return YAMC_EPARAMETER;
    if (c->in_batch) { set_error("a batch replica runs NVT moves only (volume and exchange steps need a context of its own)"); return YAMC_EWRONG_FUNCTION; }
    if (c->api_stage || c->vol_stage || c->xch_stage) { set_error("a move, volume or exchange step is pending"); return YAMC_EWRONG_FUNCTION; }
    CUDA_TRY(cudaSetDevice(c->device));
    HostSystem &H = c->H;
    const int64_t base = *cursor;
    const size_t nr = (size_t)(n_rng - base);
    int r;
    if (nr > c->rng_cap) {
        if (c->d_rng) cudaFree(c->d_rng);
        c->d_rng = nullptr;
        c->rng_cap = 0;
        if ((r = dalloc(&c->d_rng, nr))) return r;
        c->rng_cap = nr;
    }
    if (nr) CUDA_TRY(cudaMemcpyAsync(c->d_rng, rng + base, nr * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    // device buffers for a launch's records and rows (a launch runs at most log_cap moves when logging)
    const size_t want_log = (size_t)std::max<int64_t>(H.M, std::min<int64_t>(n_cycles * (int64_t)H.M, 1 << 20));
    if (log && want_log > c->log_cap) {
        if (c->d_log) cudaFree(c->d_log);
        c->d_log = nullptr;
        c->log_cap = 0;
        if ((r = dalloc(&c->d_log, want_log))) return r;
        c->log_cap = want_log;
    }
    if (rows && max_rows > c->rows_cap) {
        if (c->d_rows) cudaFree(c->d_rows);
        c->d_rows = nullptr;
        c->rows_cap = 0;
        if ((r = dalloc(&c->d_rows, (size_t)9 * max_rows))) return r;
        c->rows_cap = max_rows;
    }
    int64_t done = 0, nlog = 0, nvlog = 0;
    int32_t nrow = 0;
    int st = YAMC_OK;
    if ((r = pull_state(c))) return r;
    const double psm = H.p.pressure_step_multiplier, xprob = H.xchange_probability;
    // The chain kernel runs stretches of movemc steps and stops before a volume cycle or an
    // exchange step (and at the end of the stream); the host reads the draws that decide what
    // comes next (runmc.f90:206-259) and runs volume and exchange steps itself.
    while (done < n_cycles) {
        const int64_t c0 = *cursor;
        const bool at_start = c->cnt_h[CN_MOVE_IN_CYCLE] == 0;
        double u = 0, xd = 1.0;
        bool out = at_start && !host_rand(rng, n_rng, cursor, &u);
        if (!out && at_start && psm > 0 && u * (psm + 1) > psm) {
            // a volume cycle (mcvol, MC.f90:701-825)
            yamc_volume_record vr{};
            vr.cycle = c->cnt_h[CN_ICYCLE];
            r = volume_step(c, rng, n_rng, cursor, &vr);
            if (r == YAMC_ERNG_EXHAUSTED) { *cursor = c0; st = r; break; }
            if (r) return r;
            if (vr.flags & 1) c->n_vol_accepted += 1;
            c->sc[SC_N_VOL_STEPS] += 1;
            if (vlog && nvlog < max_vlog) vlog[nvlog++] = vr;
            host_cycle_end(c, rows, max_rows, &nrow);
            if ((r = push_state(c))) return r;
            ++done;
            continue;
        }
        if (!out && xprob > 0) out = !host_rand(rng, n_rng, cursor, &xd);
        if (out) { *cursor = c0; st = YAMC_ERNG_EXHAUSTED; break; }
        if (xprob > 0 && xd < xprob) {
            // an exchange step (mc_xchange, MC.f90:1325-1954): two different molecules from xchange_freq
            double r1 = 0, r2 = 0;
            out = !host_rand(rng, n_rng, cursor, &r1);
            const int imol1 = out ? 1 : host_choose(H.xfreq_beg, H.xfreq_end, r1);
            int imol2 = imol1;
            while (!out && imol2 == imol1) {
                out = !host_rand(rng, n_rng, cursor, &r2);
                if (!out) imol2 = host_choose(H.xfreq_beg, H.xfreq_end, r2);
            }
            if (out) { *cursor = c0; st = YAMC_ERNG_EXHAUSTED; break; }
            double du[4];
            int ov = 0;
            if ((r = xchange_eval(c, imol1, imol2, du, &ov))) return r;
            if (!ov && !(std::isfinite(du[0]) && std::isfinite(du[1]) && std::isfinite(du[2]) && std::isfinite(du[3]))) {
                xchange_commit(c, false);
                set_error("non-finite energy change of an exchange step");
                *cursor = c0; st = YAMC_ENAN; break;
            }
            bool acc = false;
            if (!ov) {  // MonteCarloMove_accept_or_decline_simple (MonteCarloMove.f90:572-597)
                const double factor = std::exp(-(du[0] + (du[1] + du[2]) + du[3]));
                double xk = 0;
                if (!host_rand(rng, n_rng, cursor, &xk)) {
                    xchange_commit(c, false);
                    *cursor = c0; st = YAMC_ERNG_EXHAUSTED; break;
                }
                acc = !(xk > factor);
            }
            if ((r = xchange_commit(c, acc))) return r;
            if (log && nlog < max_log) {
                yamc_move_record &rec = log[nlog++];
                rec.imol = imol1; rec.flags = (acc ? 1 : 0) | (ov ? 2 : 0) | 4 | (imol2 << 8); rec.cursor = *cursor;
                rec.du_real = du[0]; rec.du_k_coul = du[1]; rec.du_k_lj = du[2]; rec.du_ext = du[3];
            }
            c->sc[SC_N_MV_STEPS] += 1;
            if (acc) c->sc[SC_N_MV_ACC] += 1;
            const long long mic = c->cnt_h[CN_MOVE_IN_CYCLE] + 1;
            c->cnt_h[CN_MOVE_IN_CYCLE] = mic == H.M ? 0 : mic;
            if (mic == H.M) { host_cycle_end(c, rows, max_rows, &nrow); ++done; }
            if ((r = push_state(c))) return r;
            CUDA_TRY(cudaStreamSynchronize(c->stream));
            continue;
        }
        // a stretch of movemc steps: every move of the cycles still to run, or fewer when logging
        *cursor = c0;
        int64_t n = (n_cycles - done) * (int64_t)H.M - c->cnt_h[CN_MOVE_IN_CYCLE];
        const bool keep = log && nlog < max_log;
        if (keep) n = std::min<int64_t>(n, std::min<int64_t>((int64_t)c->log_cap, max_log - nlog));
        const bool want_rows = rows && nrow < max_rows;
        const long long icycle0 = c->cnt_h[CN_ICYCLE];
        int64_t mdone = 0;
        int32_t kr = 0;
        const int ks = run_chain_impl(c, c->d_rng, base, n_rng, cursor, n, &mdone, keep ? c->d_log : nullptr,
                                      want_rows ? c->d_rows : nullptr, want_rows ? max_rows - nrow : 0, &kr);
        if (ks != YAMC_OK && ks != YAMC_ERNG_EXHAUSTED && ks != YAMC_ENAN) return ks;
        if (keep && mdone)
            CUDA_TRY(cudaMemcpy(log + nlog, c->d_log, sizeof(yamc_move_record) * mdone, cudaMemcpyDeviceToHost));
        if (keep) nlog += mdone;
        if (want_rows && kr) {
            CUDA_TRY(cudaMemcpy(rows + 9 * (size_t)nrow, c->d_rows, sizeof(double) * 9 * kr, cudaMemcpyDeviceToHost));
            nrow += kr;
        }
        if ((r = pull_state(c))) return r;
        done += c->cnt_h[CN_ICYCLE] - icycle0;
        // a non-finite energy change: the chain stopped before deciding that move
        if (ks == YAMC_ENAN) { st = YAMC_ENAN; break; }
        // stopped with no move done although the next step is neither a volume cycle nor an
        // exchange step (both were read above): the stream ran out inside that move
        if (ks == YAMC_ERNG_EXHAUSTED && mdone == 0) { st = YAMC_ERNG_EXHAUSTED; break; }
    }
    if (cycles_done) *cycles_done = done;
    if (n_log) *n_log = nlog;
    if (n_vlog) *n_vlog = nvlog;
    if (n_rows) *n_rows = nrow;
    return st;
}

// ---------------------------------------------------------------- per-move drop-in

int yamc_move_old(yamc_ctx *c, int32_t imol, double f[3], double tau[3]) {
    YAMC_RANGE("yamc_move_old");
    if (!c || imol < 1 || imol > c->H.M) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    if (c->H.nt == 4 && is_mixed(c)) { set_error("the mixed form takes up to 3 LJ types"); return YAMC_ELIMITS; }
    int r = sync_positions(c);
    if (r) return r;
    MoveIn in{};
    in.imol = imol;
    if ((r = launch_move_pass(c, in, false))) return r;
    // the kernel writes its outputs, the scalars and the counters straight into mapped host memory
    if ((r = wait_move_pass(c, in.seq))) return r;
    const double *out = c->h_out;
    std::memcpy(c->sc, out + kNV, sizeof(double) * SC_COUNT);
    std::memcpy(c->cnt_h, out + kNV + SC_COUNT, sizeof(long long) * CN_COUNT);
    const HostSystem &H = c->H;
    const int f0 = H.first[imol - 1], na = H.natoms[imol - 1];
    for (int k = 0; k < RV_F + 3 * na; ++k)
        if (k != RV_DUC && k != RV_DUL && k != RV_OVL && !std::isfinite(out[k])) {
            set_error("non-finite old-position energy or force");
            c->api_stage = 0;
            return YAMC_ENAN;
        }
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
    YAMC_RANGE("yamc_move_eval");
    if (!c || !xn || !yn || !zn) return YAMC_EPARAMETER;
    if (c->api_stage != 1 || imol != c->api_imol) { set_error("yamc_move_eval must follow yamc_move_old for the same molecule"); return YAMC_EWRONG_FUNCTION; }
    CUDA_TRY(cudaSetDevice(c->device));
    const HostSystem &H = c->H;
    const int f0 = H.first[imol - 1], na = H.natoms[imol - 1];
    MoveIn in{};
    in.imol = imol;
    for (int a = 0; a < na; ++a) { in.x[a] = xn[a]; in.y[a] = yn[a]; in.z[a] = zn[a]; }
    int r = launch_move_pass(c, in, true);
    if (r) return r;
    if ((r = wait_move_pass(c, in.seq))) return r;
    const double *out = c->h_out;
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
    if (!ovl) {
        bool finite = std::isfinite(enew - eold) && std::isfinite(out[RV_DUC]) && std::isfinite(out[RV_DUL]) &&
                      std::isfinite(du_ext);
        for (int k = 0; k < 3; ++k) finite = finite && std::isfinite(F[k]) && std::isfinite(T[k]);
        if (!finite) {
            set_error("non-finite energy change or force at the proposed positions (the move cannot be committed)");
            c->api_stage = 0;
            return YAMC_ENAN;
        }
    }
    c->api_stage = ovl ? 0 : 2;
    return YAMC_OK;
}

int yamc_move_commit(yamc_ctx *c, int32_t accepted) {
    YAMC_RANGE("yamc_move_commit");
    if (!c) return YAMC_EPARAMETER;
    if (!accepted) { c->api_stage = 0; return YAMC_OK; }
    if (c->api_stage != 2) { set_error("yamc_move_commit(accepted) must follow a successful yamc_move_eval"); return YAMC_EWRONG_FUNCTION; }
    CUDA_TRY(cudaSetDevice(c->device));
    HostSystem &H = c->H;
    const int imol = c->api_imol, f0 = H.first[imol - 1], na = H.natoms[imol - 1];
    const int n = (1 + H.nt) * H.S;
    MoveCommit mc{};
    mc.first = f0; mc.na = na;
    for (int i = 0; i < na; ++i) {
        H.x[f0 + i] = c->api_xn[i]; H.y[f0 + i] = c->api_yn[i]; H.z[f0 + i] = c->api_zn[i];
        mc.x[i] = H.x[f0 + i]; mc.y[i] = H.y[f0 + i]; mc.z[i] = H.z[f0 + i];
    }
    c->sc[SC_UU_EW] += c->api_new[RV_EW] - c->api_eold[0];
    c->sc[SC_UU_LJ6] += c->api_new[RV_LJ6] - c->api_eold[1];
    c->sc[SC_UU_LJ12] += c->api_new[RV_LJ12] - c->api_eold[2];
    c->sc[SC_EK_C] += c->api_new[RV_DUC];
    c->sc[SC_EK_LJ] += c->api_new[RV_DUL];
    c->sc[SC_MU_X] += c->api_dmu[0]; c->sc[SC_MU_Y] += c->api_dmu[1]; c->sc[SC_MU_Z] += c->api_dmu[2];
    std::memcpy(mc.sc, c->sc, sizeof(double) * SC_COUNT);
    std::memcpy(mc.cnt, c->cnt_h, sizeof(long long) * CN_COUNT);
    // rho += the pass's deltas (scratch buffer 1, in the pass's arithmetic type), the moved atoms,
    // the scalars and the counters: one launch, the host values passed as kernel arguments
    const int nb = std::max(1, (n + 255) / 256);
    if (is_mixed(c))
        k_commit_move<<<nb, 256, 0, c->stream>>>(c->rho, scratch_buf<true>(c->scratch, 1, 1 + H.nt, H.S), n, c->hsys, mc);
    else
        k_commit_move<<<nb, 256, 0, c->stream>>>(c->rho, scratch_buf<false>(c->scratch, 1, 1 + H.nt, H.S), n, c->hsys, mc);
    CUDA_TRY(cudaGetLastError());
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
        if (params[i].pressure_step_multiplier > 0) {
            set_error("replica " + std::to_string(i) + ": batched replicas run NVT (pressure_step_multiplier 0)");
            return YAMC_EPARAMETER;
        }
        yamc_ctx *c = nullptr;
        const int r = yamc_create(&systems[i], &params[i], b->device, &c);
        if (r) {
            set_error("replica " + std::to_string(i) + ": " + last_error());
            return r;
        }
        c->in_batch = true;
        b->reps.push_back(c);
    }
    for (int i = 0; i < n; ++i) {
        const HostSystem &H = b->reps[i]->H;
        const bool split = split_variant(H);
        const bool mx = H.p.precision == YAMC_MIXED;
        const int cls = H.N <= 1024 ? 0 : H.N <= 2048 ? 1 : H.N <= 4096 ? 2 : H.N <= 8192 ? 3 : 4;
        size_t k = 0;
        while (k < b->groups.size() && !(b->groups[k].nt == H.nt && b->groups[k].split == split &&
                                         b->groups[k].mx == mx && b->groups[k].size_class == cls))
            ++k;
        if (k == b->groups.size()) {
            b->groups.emplace_back();
            b->groups.back().nt = H.nt;
            b->groups.back().split = split;
            b->groups.back().mx = mx;
            b->groups.back().size_class = cls;
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
    YAMC_RANGE("yamc_batch_run_device");
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
    YAMC_RANGE("yamc_batch_run");
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
    std::vector<std::array<int, 3>> keep;
    for (BatchGroup &g : b->groups) { keep.push_back({g.fG, g.fB, g.fL}); g.fG = 0; g.fB = 0; g.fL = YAMC_KSPACE_AUTO; }
    const int r = batch_configure(b);
    if (r) {
        b->force_G = oG; b->force_B = oB;
        for (size_t k = 0; k < keep.size(); ++k) { b->groups[k].fG = keep[k][0]; b->groups[k].fB = keep[k][1]; b->groups[k].fL = keep[k][2]; }
        batch_configure(b);
    }
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

int yamc_batch_last_launches(yamc_batch *b, int32_t *n) {
    if (!b || !n) return YAMC_EPARAMETER;
    *n = b->last_launches;
    return YAMC_OK;
}

int yamc_batch_last_kernel_ms(yamc_batch *b, double *ms) {
    if (!b || !ms) return YAMC_EPARAMETER;
    *ms = b->last_ms;
    return YAMC_OK;
}

int yamc_batch_tune(yamc_batch *b, const float *const *d_rng, const int64_t *n_rng, const int64_t *cursors,
                    int64_t n_moves, double *best_moves_per_s) {
    YAMC_RANGE("yamc_batch_tune");
    if (!b || !d_rng || !n_rng || !cursors || n_moves < 1) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(b->device));
    const size_t R = b->reps.size();
    BatchBackup keep;
    int r = batch_copy_state(b, keep, true);
    if (r) return r;
    for (size_t i = 0; i < R; ++i)
        if (!d_rng[i] || n_rng[i] < 0 || cursors[i] < 0 || cursors[i] > n_rng[i]) return YAMC_EPARAMETER;
    const int Bs[] = {kChainMaxThreadsWide, kChainMaxThreads, 128};
    const int Ls[] = {YAMC_KSPACE_REGISTERS, YAMC_KSPACE_STREAMED};
    std::vector<int64_t> cur(R), done(R), off(R, 0);
    double total = 0.0;
    struct Shape { double eff, rate; int G, B, L; };
    std::vector<std::vector<Shape>> shapes(b->groups.size());  // every shape that fits, per group
    // every group on its own (the others run no moves): the shape with its highest moves/s
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        BatchGroup &g = b->groups[gi];
        const int f0 = g.fG, f1 = g.fB, f2 = g.fL;
        double best = -1.0, brate = 0.0;
        int bG = 0, bB = 0, bL = 0;
        for (int L : Ls)
            for (int G = 1; G <= 16; ++G)
                for (int B : Bs) {
                    if (b->force_layout != YAMC_KSPACE_AUTO && L != b->force_layout) continue;
                    g.fG = G; g.fB = B; g.fL = L;
                    if (batch_configure(b) != YAMC_OK) continue;  // shape does not fit
                    if (g.cfg.G != G || g.cfg.B != B || g.max_clusters <= 0) continue;
                    for (size_t i = 0; i < R; ++i) cur[i] = cursors[i];
                    r = batch_step(b, d_rng, off.data(), n_rng, cur.data(), n_moves, done.data(), nullptr, nullptr,
                                   (int)gi);
                    const int rr = batch_copy_state(b, keep, false);
                    if (rr) return rr;
                    if (r != YAMC_OK && r != YAMC_ERNG_EXHAUSTED) return r;
                    double moves = 0;
                    for (int i : g.idx) moves += (double)done[i];
                    const double rate = b->last_ms > 0 ? moves / (1e-3 * b->last_ms) : 0.0;
                    // per SM occupied: the groups share the GPU, so the shape that does the most with
                    // the SMs it holds wins, not the one that is fastest on an empty GPU
                    const int nrep = (int)g.idx.size();
                    const double sms = (double)std::min(nrep, g.max_clusters) * G;
                    const double eff = rate / sms;
                    shapes[gi].push_back({eff, rate, G, B, L});
                    if (eff > best) { best = eff; bG = G; bB = B; bL = L; brate = rate; }
                }
        if (best < 0) {
            g.fG = f0; g.fB = f1; g.fL = f2;
            batch_configure(b);
            set_error("no launch shape fits the replicas of a batch group");
            return YAMC_ELIMITS;
        }
        g.fG = bG; g.fB = bB; g.fL = bL;
        total += brate;
    }
    // then the groups together: the whole batch's moves/s (its slowest group sets the time) with
    // each group's next shapes by moves/s per SM, then its fastest shapes alone (a group that
    // sets the batch's time gains from more SMs per chain), a change kept when the batch gains 2 %
    auto whole = [&](double *rate) -> int {
        for (size_t i = 0; i < R; ++i) cur[i] = cursors[i];
        int s2 = batch_step(b, d_rng, off.data(), n_rng, cur.data(), n_moves, done.data(), nullptr, nullptr, -1);
        const int rr = batch_copy_state(b, keep, false);
        if (rr) return rr;
        if (s2 != YAMC_OK && s2 != YAMC_ERNG_EXHAUSTED) return s2;
        double moves = 0;
        for (size_t i = 0; i < R; ++i) moves += (double)done[i];
        *rate = b->last_ms > 0 ? moves / (1e-3 * b->last_ms) : 0.0;
        return YAMC_OK;
    };
    if ((r = batch_configure(b))) return r;
    double best_total = 0;
    if ((r = whole(&best_total))) return r;
    constexpr int kAlternatives = 3;
    for (size_t gi = 0; gi < b->groups.size(); ++gi) {
        BatchGroup &g = b->groups[gi];
        std::vector<Shape> by_eff = shapes[gi], by_rate = shapes[gi];
        std::sort(by_eff.begin(), by_eff.end(), [](const Shape &a, const Shape &c) { return a.eff > c.eff; });
        std::sort(by_rate.begin(), by_rate.end(), [](const Shape &a, const Shape &c) { return a.rate > c.rate; });
        std::vector<Shape> cand;
        auto add = [&](const Shape &x) {
            for (const Shape &y : cand)
                if (y.G == x.G && y.B == x.B && y.L == x.L) return;
            cand.push_back(x);
        };
        for (size_t k = 0; k < by_eff.size() && (int)k < kAlternatives + 1; ++k) add(by_eff[k]);
        for (size_t k = 0; k < by_rate.size() && (int)k < kAlternatives; ++k) add(by_rate[k]);
        int tried = 0;
        for (const Shape &sh : cand) {
            if (tried >= 2 * kAlternatives) break;
            if (sh.G == g.fG && sh.B == g.fB && sh.L == g.fL) continue;
            const int k0 = g.fG, k1 = g.fB, k2 = g.fL;
            g.fG = sh.G; g.fB = sh.B; g.fL = sh.L;
            ++tried;
            double t = 0;
            if (batch_configure(b) == YAMC_OK && g.cfg.G == sh.G && g.cfg.B == sh.B && (r = whole(&t)) == YAMC_OK &&
                t > 1.02 * best_total) {
                best_total = t;
                continue;
            }
            if (r != YAMC_OK) return r;
            g.fG = k0; g.fB = k1; g.fL = k2;
            if ((r = batch_configure(b))) return r;
        }
    }
    r = batch_configure(b);
    for (yamc_ctx *c : b->reps) c->pos_valid = false;
    if (best_moves_per_s) *best_moves_per_s = best_total > 0 ? best_total : total;
    return r;
}

int yamc_batch_groups(yamc_batch *b, int32_t *n) {
    if (!b || !n) return YAMC_EPARAMETER;
    *n = (int32_t)b->groups.size();
    return YAMC_OK;
}

int yamc_batch_group_launch(yamc_batch *b, int32_t group, int32_t out[7]) {
    if (!b || !out || group < 0 || group >= (int)b->groups.size()) return YAMC_EPARAMETER;
    const BatchGroup &g = b->groups[group];
    out[0] = g.cfg.G; out[1] = g.cfg.B; out[2] = std::max(g.cfg.EPT, 0); out[3] = (int32_t)g.cfg.smem;
    out[4] = g.max_clusters; out[5] = (int32_t)g.idx.size(); out[6] = g.mx ? 1 : 0;
    return YAMC_OK;
}

// ---------------------------------------------------------------- adjoint forces

int yamc_forces(yamc_ctx *c, double *fx, double *fy, double *fz, double *mol_f, double *mol_tau) {
    YAMC_RANGE("yamc_forces");
    if (!c) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    HostSystem &H = c->H;
    const int N = H.N;
    int r;
    // real space over atom tiles x j slices (about two blocks per SM), the slices added in order
    const int T = (N + kFullTile - 1) / kFullTile;
    const int want = std::max(1, std::min(T, (2 * c->nsm + T - 1) / T));
    const int slice_tiles = (T + want - 1) / want, nslice = (T + slice_tiles - 1) / slice_tiles;
    if (!c->d_gx && ((r = dalloc(&c->d_gx, N)) || (r = dalloc(&c->d_gy, N)) || (r = dalloc(&c->d_gz, N)) ||
                     (r = dalloc(&c->d_fpart, (size_t)3 * nslice * N))))
        return r;
    if ((r = sync_positions(c)) || (r = pull_state(c))) return r;
    k_forces_real<<<dim3(T, nslice), kFullTile, 0, c->stream>>>(c->hsys, slice_tiles, c->d_fpart);
    CUDA_TRY(cudaGetLastError());
    k_forces_reduce<<<(N + 255) / 256, 256, 0, c->stream>>>(c->d_fpart, nslice, N, c->d_gx, c->d_gy, c->d_gz);
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
    bool finite = true;
    for (int i = 0; i < N; ++i) {
        gx[i] = gx[i] + m2k * H.q[i] * mx; gy[i] = gy[i] + m2k * H.q[i] * my; gz[i] = gz[i] + m2k * H.q[i] * mz;
        finite = finite && std::isfinite(gx[i]) && std::isfinite(gy[i]) && std::isfinite(gz[i]);
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
    if (!finite) { set_error("non-finite force (the outputs hold it)"); return YAMC_ENAN; }
    return YAMC_OK;
}

// ---------------------------------------------------------------- exact checkpoint

namespace {

// The state blob: a fixed header (sizes that must match the context it is loaded into), the
// parameters as they stand, the engine scalars and counters, the host-side tables that depend
// on the box length (NPT steps rescale them with rounding, so they are stored, not rebuilt),
// the positions and rho(k).  Host byte order; every field 8-byte aligned.
constexpr char kStateMagic[8] = {'Y', 'A', 'M', 'C', 'S', 'T', '0', '1'};
struct StateHeader {
    char magic[8];
    int32_t natom, nmol, ntype, nk, nsigned, npair;
    int64_t cursor;
    int64_t bytes;
};

struct StateWriter {
    unsigned char *p;
    void put(const void *v, size_t bytes) { std::memcpy(p, v, bytes); p += bytes; }
    void putv(const std::vector<double> &v) { put(v.data(), sizeof(double) * v.size()); }
};
struct StateReader {
    const unsigned char *p;
    void get(void *v, size_t bytes) { std::memcpy(v, p, bytes); p += bytes; }
    void getv(std::vector<double> &v) { get(v.data(), sizeof(double) * v.size()); }
};

size_t state_bytes(const HostSystem &H) {
    const size_t N = H.N, nt = H.nt;
    size_t b = sizeof(StateHeader) + sizeof(yamc_params) + sizeof(double) * SC_COUNT + sizeof(long long) * CN_COUNT;
    b += sizeof(double) * 4;                                   // n_vol_accepted, the three tails
    b += sizeof(double) * 5 * N;                               // x, y, z, sigma, dhs
    b += sizeof(double) * nt;                                  // type_sigma
    b += sizeof(double) * H.nk;                                // beta
    b += sizeof(double) * (size_t)H.npair * H.S;               // beta_LJ per entry
    b += sizeof(double) * 5 * nt * nt;                         // lj6, lj12, four_eps, sigma6, sigma2
    b += sizeof(double2) * (1 + nt) * (size_t)H.S;             // rho(k)
    return (b + 7) & ~size_t(7);
}

bool state_idle(const yamc_ctx *c) {
    if (c->api_stage || c->vol_stage || c->xch_stage) {
        set_error("a per-move, volume or exchange step is between its eval and commit");
        return false;
    }
    return true;
}

}  // namespace

int yamc_state_size(yamc_ctx *c, int64_t *bytes) {
    if (!c || !bytes) return YAMC_EPARAMETER;
    *bytes = (int64_t)state_bytes(c->H);
    return YAMC_OK;
}

int yamc_save_state(yamc_ctx *c, int64_t cursor, void *buf, int64_t bytes) {
    YAMC_RANGE("yamc_save_state");
    if (!c || !buf) return YAMC_EPARAMETER;
    HostSystem &H = c->H;
    const size_t need = state_bytes(H);
    if (bytes < (int64_t)need) { set_error("state buffer smaller than yamc_state_size"); return YAMC_ELIMITS; }
    if (!state_idle(c)) return YAMC_EWRONG_FUNCTION;
    CUDA_TRY(cudaSetDevice(c->device));
    int r;
    if ((r = sync_positions(c)) || (r = pull_state(c))) return r;
    const size_t nrho = (size_t)(1 + H.nt) * H.S;
    std::vector<double2> rho(nrho);
    CUDA_TRY(cudaMemcpyAsync(rho.data(), c->rho, sizeof(double2) * nrho, cudaMemcpyDeviceToHost, c->stream));
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    StateHeader h{};
    std::memcpy(h.magic, kStateMagic, 8);
    h.natom = H.N; h.nmol = H.M; h.ntype = H.nt; h.nk = H.nk; h.nsigned = H.S; h.npair = H.npair;
    h.cursor = cursor;
    h.bytes = (int64_t)need;
    std::memset(buf, 0, need);
    StateWriter w{static_cast<unsigned char *>(buf)};
    w.put(&h, sizeof h);
    w.put(&H.p, sizeof H.p);
    w.put(c->sc, sizeof(double) * SC_COUNT);
    w.put(c->cnt_h, sizeof(long long) * CN_COUNT);
    const double extra[4] = {c->n_vol_accepted, H.U_tail_coul, H.U_tail_lj6, H.U_tail_lj12};
    w.put(extra, sizeof extra);
    w.putv(H.x); w.putv(H.y); w.putv(H.z); w.putv(H.sigma); w.putv(H.dhs);
    w.putv(H.type_sigma); w.putv(H.beta); w.putv(H.ebetalj);
    w.putv(H.lj6); w.putv(H.lj12); w.putv(H.four_eps); w.putv(H.sigma6); w.putv(H.sigma2);
    w.put(rho.data(), sizeof(double2) * nrho);
    return YAMC_OK;
}

int yamc_load_state(yamc_ctx *c, const void *buf, int64_t bytes, int64_t *cursor) {
    YAMC_RANGE("yamc_load_state");
    if (!c || !buf) return YAMC_EPARAMETER;
    HostSystem &H = c->H;
    const size_t need = state_bytes(H);
    if (bytes < (int64_t)sizeof(StateHeader)) { set_error("state buffer too short"); return YAMC_EPARAMETER; }
    StateReader rd{static_cast<const unsigned char *>(buf)};
    StateHeader h{};
    rd.get(&h, sizeof h);
    if (std::memcmp(h.magic, kStateMagic, 8) != 0) { set_error("not a yamc state (bad magic or version)"); return YAMC_EPARAMETER; }
    if (h.natom != H.N || h.nmol != H.M || h.ntype != H.nt || h.nk != H.nk || h.nsigned != H.S ||
        h.npair != H.npair || h.bytes != (int64_t)need || bytes < (int64_t)need) {
        set_error("the state was saved from a context of another system (atom, molecule, LJ type or k counts differ)");
        return YAMC_EPARAMETER;
    }
    if (c->in_batch) {
        set_error("a batch replica: its batch's graph holds a copy of the replica's tables; load into a context of its own");
        return YAMC_EWRONG_FUNCTION;
    }
    if (!state_idle(c)) return YAMC_EWRONG_FUNCTION;
    CUDA_TRY(cudaSetDevice(c->device));
    const int precision = H.p.precision;  // the context's own precision stays
    rd.get(&H.p, sizeof H.p);
    H.p.precision = precision;
    rd.get(c->sc, sizeof(double) * SC_COUNT);
    rd.get(c->cnt_h, sizeof(long long) * CN_COUNT);
    double extra[4];
    rd.get(extra, sizeof extra);
    c->n_vol_accepted = extra[0];
    H.U_tail_coul = extra[1]; H.U_tail_lj6 = extra[2]; H.U_tail_lj12 = extra[3];
    rd.getv(H.x); rd.getv(H.y); rd.getv(H.z); rd.getv(H.sigma); rd.getv(H.dhs);
    rd.getv(H.type_sigma); rd.getv(H.beta); rd.getv(H.ebetalj);
    rd.getv(H.lj6); rd.getv(H.lj12); rd.getv(H.four_eps); rd.getv(H.sigma6); rd.getv(H.sigma2);
    const size_t nrho = (size_t)(1 + H.nt) * H.S;
    std::vector<double2> rho(nrho);
    rd.get(rho.data(), sizeof(double2) * nrho);
    int r;
    if ((r = upload_box(c)) || (r = upload(c->rho, rho.data(), nrho, c->stream)) || (r = push_state(c))) return r;
    CUDA_TRY(cudaStreamSynchronize(c->stream));
    c->api_stage = 0;
    if (cursor) *cursor = h.cursor;
    return YAMC_OK;
}

int yamc_set_positions(yamc_ctx *c, const double *x, const double *y, const double *z, double e[8]) {
    YAMC_RANGE("yamc_set_positions");
    if (!c || !x || !y || !z) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(c->device));
    HostSystem &H = c->H;
    for (int i = 0; i < H.N; ++i)
        if (!(std::isfinite(x[i]) && std::isfinite(y[i]) && std::isfinite(z[i]))) {
            set_error("non-finite coordinate of atom " + std::to_string(i + 1) + " (the configuration is unchanged)");
            return YAMC_ENAN;
        }
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

namespace {
// one checked read of arr[index] (arr holds 4 values): the index check of the bounds-checked
// builds on its own, so a test can see it record an out-of-bounds index and keep the access in bounds
__global__ void k_bounds_selftest(long long index, long long size, const double *arr, double *out, int *check) {
    out[0] = arr[checked_ix(index, size < 4 ? size : 4, __LINE__, check)];
}
}  // namespace

int yamc_checked_build(int32_t *checked) {
    if (!checked) return YAMC_EPARAMETER;
#ifdef YAMC_CHECKED
    *checked = 1;
#else
    *checked = 0;
#endif
    return YAMC_OK;
}

int yamc_bounds_check_selftest(int32_t device, int64_t index, int64_t size, double *value, int32_t *line) {
    if (!value || !line) return YAMC_EPARAMETER;
    CUDA_TRY(cudaSetDevice(device));
    const double h[4] = {10.0, 11.0, 12.0, 13.0};
    double *d = nullptr;
    int *chk = nullptr;
    CUDA_TRY(cudaMalloc(&d, sizeof(double) * 5));
    cudaError_t e = cudaMalloc(&chk, sizeof(int));
    if (e == cudaSuccess) e = cudaMemcpy(d, h, sizeof h, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(chk, 0, sizeof(int));
    if (e == cudaSuccess) {
        k_bounds_selftest<<<1, 1>>>((long long)index, (long long)size, d, d + 4, chk);
        e = cudaGetLastError();
    }
    int l = 0;
    double v = 0.0;
    if (e == cudaSuccess) e = cudaMemcpy(&v, d + 4, sizeof(double), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&l, chk, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (chk) cudaFree(chk);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return YAMC_ECUDA; }
    *value = v;
    *line = l;
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
