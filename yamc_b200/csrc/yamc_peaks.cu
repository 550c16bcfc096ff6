// yamc_fma_peak: the FP64 or FP32 fused-multiply-add throughput of one GPU, measured.
//
// The trial move is not a contraction, so its compute roofline is the plain FMA pipe, not the
// tensor cores.  The chain kernel's pipe fraction is stated against this measured figure
// rather than a datasheet number: each thread runs kChains independent FMA recurrences
// x <- x * a + b (independent so that the pipe, not the FMA latency, is the limit), the grid
// covers every SM with kBlocksPerSm blocks of 256 threads, and the time is the median of
// kTimed launches by CUDA events after one warm-up launch.  Each thread writes the sum of its
// chains to its own slot of a buffer sized grid x block, so nothing is optimised away.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/yamc.h"
#include "yamc_internal.h"

namespace yamc {
namespace {

constexpr int kChains = 16;
constexpr int kThreads = 256;
constexpr int kBlocksPerSm = 4;
constexpr int kTimed = 5;

template <typename T>
__global__ void __launch_bounds__(kThreads) k_fma_peak(T *out, int iters, T a, T b) {
    T x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = T(threadIdx.x) * T(1e-3) + T(k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], a, b);
    }
    T s = T(0);
#pragma unroll
    for (int k = 0; k < kChains; ++k) s += x[k];
    out[(size_t)blockIdx.x * kThreads + threadIdx.x] = s;
}

template <typename T>
int measure(int device, double *tflops) {
    int nsm = 0;
    cudaError_t e = cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); return YAMC_ECUDA; }
    const int blocks = nsm * kBlocksPerSm;
    // about 50 ms of FP64 work on a B200-class part (half that for FP32)
    const int iters = 1 << 17;
    T *out = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    std::vector<float> ms;
    int rc = YAMC_OK;
    auto fail = [&](cudaError_t err) { set_error(std::string("yamc_fma_peak: ") + cudaGetErrorString(err)); rc = YAMC_ECUDA; };
    if ((e = cudaMalloc(&out, sizeof(T) * (size_t)blocks * kThreads)) != cudaSuccess) { fail(e); goto done; }
    if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess) { fail(e); goto done; }
    if ((e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess) { fail(e); goto done; }
    for (int rep = 0; rep <= kTimed; ++rep) {
        cudaEventRecord(e0, s);
        k_fma_peak<T><<<blocks, kThreads, 0, s>>>(out, iters, T(0.9999999), T(1e-7));
        cudaEventRecord(e1, s);
        if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaEventSynchronize(e1)) != cudaSuccess) { fail(e); goto done; }
        float t = 0;
        cudaEventElapsedTime(&t, e0, e1);
        if (rep > 0) ms.push_back(t);
    }
    {
        std::sort(ms.begin(), ms.end());
        const double t = ms[ms.size() / 2] * 1e-3;
        const double flops = 2.0 * kChains * (double)iters * blocks * kThreads;
        *tflops = flops / t * 1e-12;
    }
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    if (out) cudaFree(out);
    return rc;
}

}  // namespace
}  // namespace yamc

extern "C" int yamc_fma_peak(int32_t device, int32_t fp64, double *tflops) {
    if (!tflops || device < 0) return YAMC_EPARAMETER;
    // the caller's current device is put back before returning
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    if (e != cudaSuccess) { yamc::set_error(cudaGetErrorString(e)); return YAMC_ECUDA; }
    if ((e = cudaSetDevice(device)) != cudaSuccess) { yamc::set_error(cudaGetErrorString(e)); return YAMC_ECUDA; }
    const int rc = fp64 ? yamc::measure<double>(device, tflops) : yamc::measure<float>(device, tflops);
    if ((e = cudaSetDevice(prev)) != cudaSuccess) { yamc::set_error(cudaGetErrorString(e)); return YAMC_ECUDA; }
    return rc;
}
