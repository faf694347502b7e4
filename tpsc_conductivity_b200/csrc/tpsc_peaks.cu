// tpsc_peaks.cu -- instrumentation: the FP64 and FP32 FMA throughput of the
// device, the arithmetic ceiling beside the HBM one for the transform kernels'
// roofline (the FFT/DCT stages do more arithmetic per byte than a copy).
//
// Each thread carries 8 independent FMA chains through kPeakIters steps;
// 8 blocks per SM of 256 threads; the chains' results are stored so that the
// work is kept.  Timed with CUDA events after one warm-up launch.
#include <cuda_runtime.h>

#include <string>

#include "../../include/tpsc_b200.h"
#include "tpsc_device.cuh"
#include "tpsc_host.h"

namespace tpsc {
namespace {

constexpr int kPeakIters = 4096, kPeakChains = 8, kPeakThreads = 256;

template <class F>
__global__ void __launch_bounds__(kPeakThreads) k_fma_peak(F b, F c, F *out) {
    F a[kPeakChains];
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) a[k] = (F)(threadIdx.x + k) * (F)1e-3;
#pragma unroll 4
    for (int it = 0; it < kPeakIters; ++it)
#pragma unroll
        for (int k = 0; k < kPeakChains; ++k) a[k] = fma(a[k], b, c);
    F s = 0;
#pragma unroll
    for (int k = 0; k < kPeakChains; ++k) s += a[k];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

template <class F>
int measure(double *tflops) {
    int dev = 0, sms = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return static_fail(TPSC_ERR_CUDA, std::string("fma peak: ") + cudaGetErrorString(e));
    const int blocks = 8 * sms;
    F *out = nullptr;
    cudaEvent_t a = nullptr, b = nullptr;
    float ms = 0.0f;
    if ((e = cudaMalloc(&out, (size_t)blocks * kPeakThreads * sizeof(F))) == cudaSuccess &&
        (e = cudaEventCreate(&a)) == cudaSuccess && (e = cudaEventCreate(&b)) == cudaSuccess) {
        // b = 1 - 2^-20, c small: the chains stay finite and do not flush to zero
        const F bb = (F)(1.0 - 1.0 / 1048576.0), cc = (F)1e-6;
        k_fma_peak<F><<<blocks, kPeakThreads>>>(bb, cc, out);
        e = launched();
        if (e == cudaSuccess) e = cudaEventRecord(a);
        for (int r = 0; r < 5 && e == cudaSuccess; ++r) {
            k_fma_peak<F><<<blocks, kPeakThreads>>>(bb, cc, out);
            e = launched();
        }
        if (e == cudaSuccess) e = cudaEventRecord(b);
        if (e == cudaSuccess) e = cudaEventSynchronize(b);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (out) cudaFree(out);
    if (e != cudaSuccess) return static_fail(TPSC_ERR_CUDA, std::string("fma peak: ") + cudaGetErrorString(e));
    const double flops = 5.0 * 2.0 * (double)blocks * kPeakThreads * kPeakChains * kPeakIters;
    *tflops = flops / (ms * 1e-3) / 1e12;
    return TPSC_OK;
}

}  // namespace
}  // namespace tpsc

extern "C" int tpsc_fma_peak(int bits, double *tflops) {
    if (!tflops || (bits != 32 && bits != 64)) return tpsc::static_fail(TPSC_ERR_ARG, "tpsc_fma_peak: bits 32 or 64");
    return bits == 64 ? tpsc::measure<double>(tflops) : tpsc::measure<float>(tflops);
}
