// tpsc_lattice.cu -- the infinite-lattice quantities the reference obtains
// by adaptive 2D quadrature, for spot checks of the finite-lattice results:
// mu0 of the infinite system (green0::find_mu_inf_syst / ddensity_mu,
// src/green0.cpp:221-287) and chi0(q, i q_n) at any q (chi0::chiqw /
// chi0IntegRe, src/chi0.cpp:211-276, 1614-1651).
//
// At T > 0 both integrands are analytic and periodic in k, so the trapezoid
// rule on an L x L grid of the Brillouin zone converges exponentially in L
// (the finite-lattice sum chiqw_discret, src/chi0.cpp:1587-1612, is that rule
// at the lattice's own L).  The host doubles L until two sums agree to
// 1e-13 relative.  Each sum is one launch: a block per (row stripe, point),
// compensated sums, and a second kernel that adds the block partials in a
// fixed order.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/tpsc_b200.h"
#include "tpsc_device.cuh"
#include "tpsc_host.h"

namespace tpsc {

namespace {

constexpr int kLatThreads = 256;
constexpr int kLatBlocks = 64;  // blocks per point (row stripes)

struct Hop {
    double tp, tpp, t3;
};

// hamiltonien::dispk (src/hamiltonien.cpp:119-122)
__device__ __forceinline__ double disp(double kx, double ky, Hop h) {
    const double cx = cos(kx), cy = cos(ky), c2x = cos(2 * kx), c2y = cos(2 * ky);
    return -2.0 * (cx + cy) - 4.0 * h.tp * cx * cy - 2.0 * h.tpp * (c2x + c2y) - 4 * h.t3 * (c2x * cy + c2y * cx);
}

// chi0::chi0IntegRe at (kx, ky) for q = (qx, qy), w_n (src/chi0.cpp:1614-1651)
__device__ double lindhard(double kx, double ky, double qx, double qy, double wn, double mu, double T, Hop h) {
    const double ek = disp(kx, ky, h), ekq = disp(kx + qx, ky + qy, h);
    double delta = ek - ekq;
    if (qx == 0.0 && qy == 0.0) delta = 0.0;
    const double expk = exp((ek - mu) / T);
    if (wn != 0.0) {
        if (delta == 0.0) return 0.0;
        return (1.0 / (expk + 1.0) - 1.0 / (exp((ekq - mu) / T) + 1.0)) * delta / (wn * wn + delta * delta);
    }
    if (fabs(delta) > 1e-12) return (1.0 / (expk + 1.0) - 1.0 / (exp((ekq - mu) / T) + 1.0)) / delta;
    if (ek - mu < 0) return -(1.0 / T) * expk / ((expk + 1.0) * (expk + 1.0));
    const double expkm = exp(-(ek - mu) / T);
    return -(1.0 / T) * expkm / ((expkm + 1.0) * (expkm + 1.0));
}

// block b of point p sums rows i = b, b + B, ... of the L x L grid k = 2 pi (i, j) / L
__device__ void block_partial(KSum &acc, double *partial) {
    __shared__ double red[kLatThreads / 32];
    double v = acc.value();
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kLatThreads / 32; ++w) s += red[w];
        partial[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(kLatThreads) k_lindhard_sum(const double *__restrict__ qw, int L, double mu,
                                                              double T, Hop h, double *partial) {
    const double3 q = reinterpret_cast<const double3 *>(qw)[blockIdx.y];
    const double dk = 2.0 * 3.141592653589793 / L;
    KSum acc;
    for (int i = blockIdx.x; i < L; i += gridDim.x)
        for (int j = threadIdx.x; j < L; j += blockDim.x) acc.add(lindhard(i * dk, j * dk, q.x, q.y, q.z, mu, T, h));
    block_partial(acc, partial);
}

// (2/L^2) sum f(eps - mu) and its mu derivative, the Fermi function of
// green0::Fermi with the reference's overflow-free branches
__global__ void __launch_bounds__(kLatThreads) k_density_sum(int L, double mu, double T, Hop h, double *partial) {
    const double dk = 2.0 * 3.141592653589793 / L;
    KSum acc;
    for (int i = blockIdx.x; i < L; i += gridDim.x)
        for (int j = threadIdx.x; j < L; j += blockDim.x) {
            const double x = (disp(i * dk, j * dk, h) - mu) / T;
            double f;
            if (x > 0) {
                const double e = exp(-x);
                f = e / (1.0 + e);
            } else {
                f = 1.0 / (1.0 + exp(x));
            }
            // blockIdx.y 0: f, 1: df/dmu
            acc.add(blockIdx.y == 0 ? f : f * (1.0 - f) / T);
        }
    block_partial(acc, partial);
}

// out[p] = scale * sum of the B partials of point p, in block order (a
// negative scale as 0 - |scale| sum, so that a zero sum gives +0 as the
// reference's accumulation 0 - ... does)
__global__ void k_lattice_finish(const double *__restrict__ partial, int B, int np, double scale, double *out) {
    const int p = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (p >= np) return;
    KSum acc;
    for (int b = lane; b < B; b += 32) acc.add(partial[(size_t)p * B + b]);
    double v = acc.value();
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) out[p] = scale < 0 ? 0.0 - (-scale) * v : scale * v;
}

struct DevBuf {
    double *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

int cuda_err(cudaError_t e, const char *what) {
    return static_fail(e == cudaErrorMemoryAllocation ? TPSC_ERR_OOM : TPSC_ERR_CUDA,
                       std::string(what) + ": " + cudaGetErrorString(e));
}

// the np sums at L on stream st into host h[np]
int lattice_sums(bool density, int L, const double *d_qw, int np, double mu, double T, Hop hop, double *d_part,
                 double *d_out, double scale, double *h, cudaStream_t st) {
    const dim3 grid(kLatBlocks, np);
    if (density)
        k_density_sum<<<grid, kLatThreads, 0, st>>>(L, mu, T, hop, d_part);
    else
        k_lindhard_sum<<<grid, kLatThreads, 0, st>>>(d_qw, L, mu, T, hop, d_part);
    cudaError_t e = launched();
    if (e != cudaSuccess) return cuda_err(e, "lattice sum");
    k_lattice_finish<<<(np + 7) / 8, 256, 0, st>>>(d_part, kLatBlocks, np, scale, d_out);
    if ((e = launched()) != cudaSuccess) return cuda_err(e, "lattice sum");
    if ((e = cudaMemcpyAsync(h, d_out, np * sizeof(double), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_err(e, "lattice sum");
    return TPSC_OK;
}

constexpr int kLatL0 = 128, kLatLMax = 8192;
constexpr double kLatTol = 1e-13;

}  // namespace

// mu of the infinite lattice for density n at T: safeguarded Newton on the
// lattice density at each L, L doubled until mu moves by < 1e-13 (1 + |mu|).
int lattice_mu0(double n, double T, double tp, double tpp, double t3, cudaStream_t st, double *mu_out, int *L_out) {
    // green0::find_mu_inf_syst: the symmetric point keeps mu0 = 0 (src/green0.cpp:267-271)
    if (n == 1.0 && tp == 0 && tpp == 0) {
        *mu_out = 0.0;
        if (L_out) *L_out = 0;
        return TPSC_OK;
    }
    const Hop hop{tp, tpp, t3};
    DevBuf part, out;
    cudaError_t e;
    if ((e = cudaMalloc(&part.p, 2 * kLatBlocks * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&out.p, 2 * sizeof(double))) != cudaSuccess)
        return cuda_err(e, "lattice mu0");
    double mu = 0.0, prev = 0.0;
    int L = kLatL0;
    for (; L <= kLatLMax; L *= 2) {
        double lo = -8.0, hi = 8.0;
        const double scale = 2.0 / ((double)L * L);
        bool done = false;
        for (int it = 0; it < 200 && !done; ++it) {
            double r[2];
            int rc = lattice_sums(true, L, nullptr, 2, mu, T, hop, part.p, out.p, scale, r, st);
            if (rc) return rc;
            const double F = r[0] - n, D = r[1];
            if (F > 0)
                hi = mu;
            else
                lo = mu;
            double mn = D > 0 ? mu - F / D : 0.5 * (lo + hi);
            if (!(mn > lo && mn < hi)) mn = 0.5 * (lo + hi);
            done = F == 0.0 || fabs(mn - mu) <= 1e-15 * (1.0 + fabs(mu));
            mu = F == 0.0 ? mu : mn;
        }
        if (!done) return static_fail(TPSC_ERR_NO_ROOT, "infinite-lattice mu0 not found");
        if (L > kLatL0 && fabs(mu - prev) <= kLatTol * (1.0 + fabs(mu))) break;
        prev = mu;
    }
    if (L > kLatLMax) return static_fail(TPSC_ERR_NO_ROOT, "infinite-lattice mu0: the lattice sums did not converge");
    *mu_out = mu;
    if (L_out) *L_out = L;
    return TPSC_OK;
}

// chi0(q, i w_n) of the infinite lattice at np points qw[p] = (qx, qy, w_n):
// -(2/L^2) sum_k chi0IntegRe, L doubled until every point moves by < 1e-13
// of the largest |chi0|.
int lattice_chi0(double mu, double T, double tp, double tpp, double t3, int np, const double *qw, int L_fixed,
                 cudaStream_t st, double *out, int *L_out) {
    const Hop hop{tp, tpp, t3};
    DevBuf part, dout, dqw;
    cudaError_t e;
    if ((e = cudaMalloc(&part.p, (size_t)np * kLatBlocks * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&dout.p, np * sizeof(double))) != cudaSuccess ||
        (e = cudaMalloc(&dqw.p, 3 * (size_t)np * sizeof(double))) != cudaSuccess ||
        (e = cudaMemcpyAsync(dqw.p, qw, 3 * (size_t)np * sizeof(double), cudaMemcpyHostToDevice, st)) != cudaSuccess)
        return cuda_err(e, "lattice chi0");
    std::vector<double> cur(np), prev(np, 0.0);
    if (L_fixed > 0) {
        // one lattice: the finite-lattice sum chi0::chiqw_discret (src/chi0.cpp:1587-1612)
        int rc = lattice_sums(false, L_fixed, dqw.p, np, mu, T, hop, part.p, dout.p, -2.0 / ((double)L_fixed * L_fixed),
                              out, st);
        if (!rc && L_out) *L_out = L_fixed;
        return rc;
    }
    int L = kLatL0;
    for (; L <= kLatLMax; L *= 2) {
        int rc = lattice_sums(false, L, dqw.p, np, mu, T, hop, part.p, dout.p, -2.0 / ((double)L * L), cur.data(), st);
        if (rc) return rc;
        double big = 0.0, diff = 0.0;
        for (int p = 0; p < np; ++p) {
            big = fmax(big, fabs(cur[p]));
            diff = fmax(diff, fabs(cur[p] - prev[p]));
        }
        prev = cur;
        if (L > kLatL0 && diff <= kLatTol * big) break;
    }
    if (L > kLatLMax) return static_fail(TPSC_ERR_NO_ROOT, "infinite-lattice chi0: the lattice sums did not converge");
    for (int p = 0; p < np; ++p) out[p] = cur[p];
    if (L_out) *L_out = L;
    return TPSC_OK;
}

}  // namespace tpsc
