// Allocation-free real-space sums: yamc_realspace_sums_static.
//
// Who this is for.  Some hosts cannot call cudaMalloc at the point where they need an
// energy: a Fortran or C++ host whose device memory is handed out by its own pool (the pool
// holds the free HBM, so a fresh cudaMalloc fails or fragments it), a host that runs the
// call between kernels of its own and cannot afford the device-wide synchronisation that
// cudaMalloc/cudaFree may cause, or one that never creates a yamc_ctx at all because it
// already keeps the atoms on the device.  This entry point takes the caller's device arrays
// and writes the caller's device outputs, and allocates nothing: the only memory beyond its
// inputs and outputs is the per-block partial-sum buffer below, a fixed file-scope
// __device__ array.
//
// The kernel is a variant of the engine's k_realspace_full (the full real-space Ewald sum
// of EwaldSumRealSpace_calc, EwaldSumRealSpace.f90:233-500, with j0 = i+1): the same pair
// arithmetic, the same tile order and the same deterministic block reduction, but it reads
// the reference's structure-of-arrays atom data directly instead of the engine's packed
// double4 layout, and a second one-block kernel adds the block partials in block order on
// the device.  The engine's own full sum splits the pairs differently (blocks over pairs of
// atom tiles), so the totals agree with yamc_full_sums to rounding, not bit for bit.
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/yamc.h"
#include "yamc_device.cuh"
#include "yamc_internal.h"

namespace yamc {
namespace {

constexpr int kStaticTile = 256;  // threads per block = atoms per block
constexpr int kStaticParts = 8;   // ew, lj6, lj12, ew_intra, lj6_intra, lj12_intra, overlap, bad type
constexpr int kStaticMaxBlocks = (YAMC_STATIC_MAX_ATOMS + kStaticTile - 1) / kStaticTile;

// The scratch: kStaticParts doubles per block of kStaticTile atoms, for at most
// YAMC_STATIC_MAX_ATOMS atoms (64 KiB).  Every GPU that loads the library holds one copy
// until the process exits.  All calls on a device share it, and it keeps the last call's
// contents; every block writes all of its slots before the reduction kernel reads them, so
// nothing has to be cleared between calls.  In host code this name is only a handle for
// cudaGetSymbolAddress, never a device address.
static __device__ __align__(256) double g_static_parts[kStaticMaxBlocks * kStaticParts];

struct StaticIn {
    int N, nt;
    const double *x, *y, *z, *q;
    const int32_t *mol, *type;
    const double *hc;               // hard-core diameter, Angstrom
    const double *sig6, *feps;      // nt*nt, offset (t1-1)*nt + t2-1
    double box, rmax2, alpha, xclb, taosp;
};

// the engine's deterministic block reduction: warp xor tree, then the warps in order
__device__ inline void static_block_sum(double *vals, double *sh) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int v = 0; v < kStaticParts; ++v) {
        double x = vals[v];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
        if (lane == 0) sh[warp * kStaticParts + v] = x;
    }
    __syncthreads();
    if (threadIdx.x < kStaticParts) {
        double s = 0;
        for (int w = 0; w < kStaticTile / 32; ++w) s += sh[w * kStaticParts + threadIdx.x];
        sh[(kStaticTile / 32) * kStaticParts + threadIdx.x] = s;
    }
    __syncthreads();
    for (int v = 0; v < kStaticParts; ++v) vals[v] = sh[(kStaticTile / 32) * kStaticParts + v];
    __syncthreads();
}

// LJ type of an atom, 0 when it is outside 1..nt (counted as a bad input, LJ skipped)
__device__ inline int checked_type(int t, int nt, double &bad) {
    if (t < 0 || t > nt) { bad = 1.0; return 0; }
    return t;
}

// one thread per atom i, all j in tiles of kStaticTile staged in shared memory, in
// increasing j order; per-block partial sums go to part[blockIdx.x * kStaticParts + v]
__global__ void __launch_bounds__(kStaticTile) k_realspace_full_static(StaticIn in, double *uu, double *fx,
                                                                      double *fy, double *fz, double *part) {
    __shared__ double4 tp[kStaticTile];
    __shared__ int2 tm[kStaticTile];
    __shared__ double td[kStaticTile];
    __shared__ double red[(kStaticTile / 32 + 1) * kStaticParts];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < in.N;
    double acc[kStaticParts] = {0, 0, 0, 0, 0, 0, 0, 0};
    double4 pi = make_double4(0, 0, 0, 0);
    int2 mi = make_int2(-1, 0);
    double di = 0;
    if (valid) {
        pi = make_double4(in.x[i], in.y[i], in.z[i], in.q[i]);
        mi = make_int2(in.mol[i], checked_type(in.type[i], in.nt, acc[7]));
        di = in.hc[i] / in.box;
    }
    double u = 0, gx = 0, gy = 0, gz = 0;
    const int nt = in.nt;
    for (int t0 = 0; t0 < in.N; t0 += kStaticTile) {
        const int j = t0 + threadIdx.x;
        if (j < in.N) {
            double bad = 0;  // counted once, by the atom's own thread above
            tp[threadIdx.x] = make_double4(in.x[j], in.y[j], in.z[j], in.q[j]);
            tm[threadIdx.x] = make_int2(in.mol[j], checked_type(in.type[j], nt, bad));
            td[threadIdx.x] = in.hc[j] / in.box;
        }
        __syncthreads();
        const int nj = min(kStaticTile, in.N - t0);
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
                if (r2 >= in.rmax2) continue;
                const bool lj = mi.y > 0 && mj.y > 0;
                const int off = lj ? (mi.y - 1) * nt + (mj.y - 1) : 0;
                const PairTerm<double> t = pair_term<double, true>(r2, in.xclb * pi.w * pj.w, lj, lj ? in.sig6[off] : 0.0,
                                                                    lj ? in.feps[off] : 0.0, in.alpha, in.taosp, same);
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
    if (valid) {
        if (uu) uu[i] = u;
        if (fx) fx[i] = gx;
        if (fy) fy[i] = gy;
        if (fz) fz[i] = gz;
    }
    static_block_sum(acc, red);
    if (threadIdx.x < kStaticParts) part[blockIdx.x * kStaticParts + threadIdx.x] = acc[threadIdx.x];
}

// block partials -> the caller's sums, in block order (sums 0-5), or the largest flag (6-7)
__global__ void k_static_reduce(const double *part, int nblocks, double *sums) {
    const int v = threadIdx.x;
    if (v >= kStaticParts) return;
    double s = 0;
    for (int b = 0; b < nblocks; ++b) {
        const double x = part[b * kStaticParts + v];
        s = v >= 6 ? (x > s ? x : s) : s + x;
    }
    sums[v] = s;
}

int cuda_fail(cudaError_t e, const char *what) {
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    return YAMC_ECUDA;
}

// The device address of g_static_parts in the current context, looked up on every call: a
// host-side lookup that allocates nothing.  Not cached, because a host that resets the device
// (cudaDeviceReset) or re-creates its primary context gets the module loaded again, possibly
// at another address, and a cached pointer would then point at memory that is no longer mapped.
int static_parts_address(double **out) {
    void *ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_parts);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_static_parts)");
    *out = static_cast<double *>(ptr);
    return YAMC_OK;
}

// a caller's array must be device (or managed) memory usable from device dev, aligned to its element
int check_device_array(const void *p, size_t align, int dev, const char *name) {
    if (!p) { set_error(std::string(name) + " is NULL"); return YAMC_EPARAMETER; }
    if (reinterpret_cast<uintptr_t>(p) % align) { set_error(std::string(name) + " is misaligned"); return YAMC_EPARAMETER; }
    cudaPointerAttributes a;
    const cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) { cudaGetLastError(); set_error(std::string(name) + " is not a CUDA pointer"); return YAMC_EPARAMETER; }
    const bool ok = a.type == cudaMemoryTypeManaged || (a.type == cudaMemoryTypeDevice && a.device == dev);
    if (!ok) { set_error(std::string(name) + " is not device memory of the current device"); return YAMC_EPARAMETER; }
    return YAMC_OK;
}

}  // namespace
}  // namespace yamc

extern "C" int yamc_realspace_sums_static(const yamc_params *p, int32_t natom, const double *x, const double *y,
                                          const double *z, const double *charge, const int32_t *mol,
                                          const int32_t *lj_type, const double *hard_core_angstr, int32_t n_types,
                                          const double *sigma6_tab, const double *four_eps_tab, double *uu,
                                          double *fx, double *fy, double *fz, double *sums, void *stream) {
    using namespace yamc;
    if (!p) { set_error("params is NULL"); return YAMC_EPARAMETER; }
    if (natom < 1 || natom > YAMC_STATIC_MAX_ATOMS) {
        set_error("natom " + std::to_string(natom) + " outside 1.." + std::to_string(YAMC_STATIC_MAX_ATOMS) +
                  " (the fixed scratch of yamc_realspace_sums_static)");
        return YAMC_ELIMITS;
    }
    if (n_types < 0 || n_types > kMaxLJTypes) {
        set_error("n_types outside 0.." + std::to_string(kMaxLJTypes));
        return YAMC_ELIMITS;
    }
    if (!(p->BoxLength > 0) || !(p->rmax2 > 0)) {
        set_error("BoxLength and rmax2 must be positive (call yamc_params_recalc first)");
        return YAMC_EPARAMETER;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    int r;
    if ((r = check_device_array(x, 8, dev, "x")) || (r = check_device_array(y, 8, dev, "y")) ||
        (r = check_device_array(z, 8, dev, "z")) || (r = check_device_array(charge, 8, dev, "charge")) ||
        (r = check_device_array(mol, 4, dev, "mol")) || (r = check_device_array(lj_type, 4, dev, "lj_type")) ||
        (r = check_device_array(hard_core_angstr, 8, dev, "hard_core_angstr")) ||
        (r = check_device_array(sums, 8, dev, "sums")))
        return r;
    if (n_types > 0 && ((r = check_device_array(sigma6_tab, 8, dev, "sigma6_tab")) ||
                        (r = check_device_array(four_eps_tab, 8, dev, "four_eps_tab"))))
        return r;
    if ((uu && (r = check_device_array(uu, 8, dev, "uu"))) || (fx && (r = check_device_array(fx, 8, dev, "fx"))) ||
        (fy && (r = check_device_array(fy, 8, dev, "fy"))) || (fz && (r = check_device_array(fz, 8, dev, "fz"))))
        return r;
    double *parts = nullptr;
    if ((r = static_parts_address(&parts))) return r;

    StaticIn in;
    in.N = natom; in.nt = n_types;
    in.x = x; in.y = y; in.z = z; in.q = charge;
    in.mol = mol; in.type = lj_type; in.hc = hard_core_angstr;
    in.sig6 = sigma6_tab; in.feps = four_eps_tab;
    in.box = p->BoxLength; in.rmax2 = p->rmax2; in.alpha = p->alpha; in.xclb = p->xclb;
    in.taosp = p->two_alpha_over_sqrt_pi;
    const int nb = (natom + kStaticTile - 1) / kStaticTile;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_realspace_full_static<<<nb, kStaticTile, 0, st>>>(in, uu, fx, fy, fz, parts);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_realspace_full_static launch");
    k_static_reduce<<<1, 32, 0, st>>>(parts, nb, sums);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_static_reduce launch");
    return YAMC_OK;
}
