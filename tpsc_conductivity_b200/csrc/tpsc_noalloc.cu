// tpsc_noalloc.cu -- a sum-rule evaluation that allocates no memory.
//
// Some callers cannot allocate device memory at the point where they need
// the spin or charge sum rule: code running inside a memory pool or arena
// that owns all device memory, code called back from a framework that
// forbids allocation on its hot path, or a solver loop that must not call
// cudaMalloc/cudaFree because those calls synchronise the device.  For them
// tpsc_sumrule_noalloc takes only caller-owned inputs and outputs and keeps
// its per-block partial sums in a fixed array that lives in this library's
// device image (g_noalloc_scratch below): every GPU that loads the library
// holds that array until the process exits.
//
// The array is shared by every call on a device and keeps the last call's
// contents; the arrival counter it holds is cleared before each launch.
// Two calls whose work overlaps on the GPU (different streams with no
// ordering between them) race on it: order them on one stream or with events.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/tpsc_b200.h"

namespace {

constexpr int kThreads = 256;
// one block per group of four octant columns: the largest supported lattice,
// nk0 = 256, has N8 = 8385 octant points -> 2097 blocks
constexpr int kMaxLattice = 256;
constexpr int kMaxBlocks = 2100;
// partial sums (value, derivative) per block, then the arrival counter
constexpr int kScratchDoubles = 2 * kMaxBlocks + 2;

static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// device address of g_noalloc_scratch, resolved once per device and kept
// for the life of the process (a device reset would leave it stale; the
// header says that such a process must not call this entry point again)
constexpr int kMaxDevices = 64;
double *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

int scratch_for_current_device(double **out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return TPSC_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return TPSC_ERR_CUDA;
        g_scratch_addr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_addr[dev];
    return TPSC_OK;
}

__device__ __forceinline__ int octant_weight16(int o, int nbk) {
    // o = m + l(l+1)/2 with m <= l
    int l = (int)((sqrt(8.0 * o + 1.0) - 1.0) / 2.0);
    while ((l + 1) * (l + 2) / 2 <= o) ++l;
    while (l * (l + 1) / 2 > o) --l;
    const int m = o - l * (l + 1) / 2;
    int w = 16;
    if (l == 0 || l == nbk - 1) w /= 2;
    if (m == 0 || m == nbk - 1) w /= 2;
    if (m == l) w /= 2;
    return w;
}

// chi::traceDiffChispChi0 / traceDiffChichChi0 (src/chi.cpp:738-830) on
// chi0(q, iqn) in the reference's layout [j * N8 + o], j <= Nw0/2, with the
// tail Nw0/2 < n <= Nw0 summed term by term; scratch = partials + counter.
__global__ void __launch_bounds__(kThreads)
    k_sumrule_noalloc(const double *__restrict__ chiqw, const double *__restrict__ cinf,
                      const double *__restrict__ cinf2, int n8, int nb, int nbk, double Uv, double sgn, double T,
                      double scale, double *scratch, double *out) {
    const int o0 = 4 * blockIdx.x;
    const int nwmax = nb - 1;
    const double hu = sgn * Uv / 2.0;
    double w[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) w[c] = (o0 + c < n8) ? (double)octant_weight16(o0 + c, nbk) : 0.0;
    double v = 0.0, dv = 0.0;
    for (int j = threadIdx.x; j < nb; j += blockDim.x) {
        const double f = j == 0 ? 0.5 : 1.0;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (w[c] == 0.0) continue;
            const double x = chiqw[(size_t)j * n8 + o0 + c];
            const double q = x / (1.0 + hu * x);
            v += f * w[c] * (q - x);
            dv += f * w[c] * q * q;
        }
    }
    dv *= -0.5 * sgn;
    const double tw = 2.0 * 3.141592653589793 * T;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (w[c] == 0.0) continue;
        const double a = cinf[o0 + c], b = cinf2[o0 + c];
        for (int t = threadIdx.x; t < nwmax; t += blockDim.x) {
            const double wn = (nwmax + 1 + t) * tw;
            const double x = a / (wn * wn) + b / (wn * wn * wn * wn);
            const double q = x / (1.0 + hu * x);
            v += w[c] * (q - x);
            dv += w[c] * (-0.5 * sgn) * q * q;
        }
    }
    // block sums -> scratch partials; the last block to arrive adds them in
    // block order and writes out[0..1]
    __shared__ double red[kThreads / 32][2];
    __shared__ bool last;
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_down_sync(0xffffffffu, v, off);
        dv += __shfl_down_sync(0xffffffffu, dv, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5][0] = v;
        red[threadIdx.x >> 5][1] = dv;
    }
    __syncthreads();
    unsigned *ticket = reinterpret_cast<unsigned *>(scratch + 2 * kMaxBlocks);
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) {
            s0 += red[k][0];
            s1 += red[k][1];
        }
        scratch[blockIdx.x] = s0;
        scratch[kMaxBlocks + blockIdx.x] = s1;
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    double s0 = 0.0, s1 = 0.0;
    for (int b = 0; b < (int)gridDim.x; ++b) {
        s0 += __ldcg(&scratch[b]);
        s1 += __ldcg(&scratch[kMaxBlocks + b]);
    }
    out[0] = scale * s0;
    out[1] = scale * s1;
    *ticket = 0u;
}

}  // namespace

extern "C" int tpsc_sumrule_noalloc(const double *chiqw, const double *chi0_inf, const double *chi0_inf2, int nk0,
                                    int Nw0, double T, int channel, double Uv, double *out, void *stream) {
    if (!chiqw || !chi0_inf || !chi0_inf2 || !out) return TPSC_ERR_ARG;
    if (nk0 < 8 || (nk0 & (nk0 - 1)) || nk0 > kMaxLattice) return TPSC_ERR_ARG;  // beyond the fixed scratch
    if (Nw0 < 4 || (Nw0 & 1) || !(T > 0.0) || (channel != 0 && channel != 1)) return TPSC_ERR_ARG;
    const int nbk = nk0 / 2 + 1;
    const int n8 = nbk * (nbk + 1) / 2;
    const int blocks = (n8 + 3) / 4;
    if (blocks > kMaxBlocks) return TPSC_ERR_ARG;
    double *scratch = nullptr;
    if (scratch_for_current_device(&scratch) != TPSC_OK) return TPSC_ERR_CUDA;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the arrival counter must start at zero
    if (cudaMemsetAsync(scratch + 2 * kMaxBlocks, 0, sizeof(double), st) != cudaSuccess) return TPSC_ERR_CUDA;
    const double Nq = 4.0 * (nbk - 1) * (nbk - 1);
    k_sumrule_noalloc<<<blocks, kThreads, 0, st>>>(chiqw, chi0_inf, chi0_inf2, n8, Nw0 / 2 + 1, nbk, Uv,
                                                    channel == 0 ? -1.0 : 1.0, T, T / Nq, scratch, out);
    return cudaGetLastError() == cudaSuccess ? TPSC_OK : TPSC_ERR_CUDA;
}
