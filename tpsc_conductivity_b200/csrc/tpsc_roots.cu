// tpsc_roots.cu -- the Newton form's root searches on the device.
//
// The sum-rule roots Usp and Uch (chi::find_Usp_Uch(nq0, nw0, Usc),
// src/chi.cpp:846-876) as one cooperative kernel: every block sums its share
// of the stored frequencies below the series cut, a grid barrier, block 0
// adds the high-frequency moment series and takes the safeguarded Newton
// step, a grid barrier, and so on until both roots have converged.  One
// launch and one readback replace a host round trip per evaluation.
//
// The grid barrier spins on a generation counter with an iteration bound:
// the launch is cooperative (every block resident), so the bound only ends
// a wait that could not otherwise end; it then sets the error flag, every
// block leaves, and the host reports the failure.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "tpsc_device.cuh"

namespace tpsc {

namespace {

constexpr int kRootThreads = 256;
constexpr long long kBarrierSpins = 1LL << 24;  // x ~64 ns: ~1 s before giving up

// bar[0]: arrivals, bar[1]: generation.  Returns false (and sets *err) when
// the wait ran out or another block had already failed.
__device__ bool grid_sync(unsigned *bar, int *err) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = bar + 1;
        const unsigned g0 = *gen;
        __threadfence();
        int ok = 1;
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            for (long long spin = 0; *gen == g0; ++spin) {
                if (spin > kBarrierSpins || *(volatile int *)err) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok && !*(volatile int *)err;
    }
    __syncthreads();
    return s_ok;
}

struct RootCtl {
    double x, lo, hi, prev_step, root;
    int nev, it, done, ok;
};

struct SumRootArgs {
    const double4 *chiq;
    const double *cinf, *cinf2, *w16, *tailq;
    const double *mom_suf;   // [(nb + 1) kMomP] sums of the moments over frequencies >= j
    const double *cmax_suf;  // [nb + 1] max |chi| over frequencies >= j
    const double *tailm;     // [kMomP] tail moments, [kMomP] = max |chi| over the tail
    int nb, nblk, n8;
    double T, scale, n, nsr, U, hi_sp;
    double *partial;  // [2 gridDim.x]
    unsigned *bar;    // [2], zero at launch
    int *err;         // zero at launch
    RootCtl *ctl;     // [1]
    double *out;      // Usp, Uch, evals_sp, evals_ch, ok_sp, ok_ch
};

// the (value, derivative) pair, summed in a fixed order
__device__ void block_pair_sum(double &v, double &dv, double *dst) {
    __shared__ double red[32][2];
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_down_sync(0xffffffffu, v, off);
        dv += __shfl_down_sync(0xffffffffu, dv, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5][0] = v;
        red[threadIdx.x >> 5][1] = dv;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += red[w][0];
            b += red[w][1];
        }
        dst[0] = a;
        dst[1] = b;
    }
    __syncthreads();
}

// one safeguarded Newton update of the host routine newton_root (tpsc_engine.cpp)
__device__ void newton_update(RootCtl &c, double y, double dy, double tol) {
    ++c.nev;
    if (!isfinite(y) || !isfinite(dy)) {
        c.done = 1;
        c.ok = 0;
        return;
    }
    if (fabs(y) < tol) {
        c.root = c.x;
        c.done = c.ok = 1;
        return;
    }
    if ((y > 0) == (dy > 0))
        c.hi = fmin(c.hi, c.x);
    else
        c.lo = fmax(c.lo, c.x);
    const double scale = fmax(1.0, fabs(c.x));
    double xn = (dy != 0.0) ? c.x - y / dy : 0.5 * (c.lo + c.hi);
    if (dy != 0.0 && fabs(xn - c.x) <= 1e-14 * scale) {
        c.root = xn;
        c.done = c.ok = 1;
        return;
    }
    if (!(xn >= c.lo && xn <= c.hi)) xn = 0.5 * (c.lo + c.hi);
    const double step = fabs(xn - c.x);
    if (c.it >= 2 && step < 1e-10 * scale && step > 0.5 * c.prev_step) {
        c.root = xn;
        c.done = c.ok = 1;
        return;
    }
    c.prev_step = step;
    c.x = xn;
    if (++c.it >= 60) {
        c.done = 1;
        c.ok = 0;
    }
}

__global__ void __launch_bounds__(kRootThreads) k_sumrule_roots(SumRootArgs a) {
    __shared__ int s_jdir, s_tail, s_done;
    __shared__ double s_x;
    const int nwmax = a.nb - 1;
    const double tw = 2.0 * 3.141592653589793 * a.T;
    double Usp = 0.0;
#pragma unroll 1
    for (int phase = 0; phase < 2; ++phase) {
        const double sgn = phase == 0 ? -1.0 : 1.0;
        // every block has read the previous phase's result before it is overwritten
        if (phase > 0 && !grid_sync(a.bar, a.err)) return;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            RootCtl &c = *a.ctl;
            c.lo = 0.0;
            c.hi = phase == 0 ? a.hi_sp : 1000.0 * a.U;
            // spin: U/2 (clamped inside the interval); charge: U
            const double x0 = phase == 0 ? a.U / 2.0 : a.U;
            c.x = (x0 > c.lo && x0 < c.hi) ? x0 : 0.5 * (c.lo + c.hi);
            c.prev_step = 0.0;
            c.nev = c.it = c.done = c.ok = 0;
        }
#pragma unroll 1
        for (;;) {
            if (!grid_sync(a.bar, a.err)) return;
            if (threadIdx.x == 0) {
                const volatile RootCtl *c = a.ctl;
                s_x = c->x;
                s_done = c->done;
                const double ah = fabs(s_x) / 2.0;
                // first frequency of the series (cmax_suf does not increase)
                int lo = 0, hi = a.nb;
                while (lo < hi) {
                    const int mid = (lo + hi) / 2;
                    if (ah * a.cmax_suf[mid] >= kMomSeriesMax)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                s_jdir = lo;
                s_tail = ah * a.tailm[kMomP] >= kMomSeriesMax;
            }
            __syncthreads();
            if (s_done) break;
            const double x = s_x, hu = sgn * x / 2.0;
            const int jdir = s_jdir;
            double v = 0.0, dv = 0.0;
            const long long total = (long long)a.nblk * jdir;
            for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < total;
                 it += (long long)gridDim.x * blockDim.x) {
                const int blk = (int)(it / jdir), j = (int)(it - (long long)blk * jdir);
                const double4 xq = a.chiq[(size_t)blk * a.nb + j];
                const double4 w = reinterpret_cast<const double4 *>(a.w16)[blk];
                const double f = j == 0 ? 0.5 : 1.0;
                const double xs[4] = {xq.x, xq.y, xq.z, xq.w}, ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const double q = xs[c] / (1.0 + hu * xs[c]);
                    v += f * ws[c] * (q - xs[c]);
                    dv += f * ws[c] * q * q;
                }
            }
            dv *= -0.5 * sgn;
            if (s_tail) {
                // the Matsubara tail term by term (the series does not converge there)
                for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < a.n8; o += gridDim.x * blockDim.x) {
                    const double w = a.w16[o];
                    if (w == 0.0) continue;
                    const double ca = a.cinf[o], cb = a.cinf2[o];
                    for (int t = 0; t < nwmax; ++t) {
                        const double wn = (nwmax + 1 + t) * tw;
                        const double i2 = 1.0 / (wn * wn);
                        const double xv = ca * i2 + cb * i2 * i2;
                        const double q = xv / (1.0 + hu * xv);
                        v += w * (q - xv);
                        dv += w * (-0.5 * sgn) * q * q;
                    }
                }
            }
            block_pair_sum(v, dv, a.partial + 2 * blockIdx.x);
            if (!grid_sync(a.bar, a.err)) return;
            if (blockIdx.x == 0 && threadIdx.x < 32) {
                double pv = 0.0, pd = 0.0;
                for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) {
                    pv += __ldcg(&a.partial[2 * b]);
                    pd += __ldcg(&a.partial[2 * b + 1]);
                }
                for (int off = 16; off > 0; off >>= 1) {
                    pv += __shfl_down_sync(0xffffffffu, pv, off);
                    pd += __shfl_down_sync(0xffffffffu, pd, off);
                }
                if (threadIdx.x == 0) {
                    // the series over the frequencies from jdir (and over the tail)
                    double S = 0.0, dS = 0.0, hm1 = 1.0;  // hm1 = (-h)^(m-1)
                    const double h = hu;
                    for (int m = 1; m <= kMomP; ++m) {
                        const double M = (jdir < a.nb ? a.mom_suf[(size_t)jdir * kMomP + m - 1] : 0.0) +
                                         (s_tail ? 0.0 : a.tailm[m - 1]);
                        S += -h * hm1 * M;
                        dS += -m * hm1 * M;
                        hm1 *= -h;
                    }
                    const double tr = a.scale * (pv + S), dtr = a.scale * (pd + 0.5 * sgn * dS);
                    const double n = a.n, nsr = a.nsr, U = a.U;
                    double y, dy;
                    if (phase == 0) {
                        // chi::sum_rule_sp (src/chi.cpp:833-836)
                        y = tr + n - n * n / 2.0 - nsr + x * nsr * nsr / (2.0 * U);
                        dy = dtr + nsr * nsr / (2.0 * U);
                    } else {
                        // chi::sum_rule_ch (src/chi.cpp:840-843)
                        y = tr + n - n * n / 2.0 - (nsr + Usp * nsr * nsr / (2.0 * U) - nsr * nsr);
                        dy = dtr;
                    }
                    RootCtl c = *a.ctl;
                    newton_update(c, y, dy, 1e-16);
                    *a.ctl = c;
                    __threadfence();
                }
            }
        }
        // every block leaves the loop on the same done flag; record the root
        const volatile RootCtl *vc = a.ctl;
        const double root = vc->root;
        const int nev = vc->nev, ok = vc->ok;
        if (phase == 0) Usp = root;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.out[phase] = root;
            a.out[2 + phase] = nev;
            a.out[4 + phase] = ok;
        }
        if (!ok) return;
    }
}

}  // namespace

cudaError_t launch_sumrule_roots(const GridDev &g, const double *chiq, const double *chi0_inf, const double *chi0_inf2,
                                 const double *mom_suf, const double *cmax_suf, const double *tailm, double T,
                                 double n, double nsr, double U, double hi_sp, RootScratch rs, cudaStream_t st) {
    int dev = 0, sms = 0, per = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_sumrule_roots, kRootThreads, 0)) != cudaSuccess)
        return e;
    const int grid = std::min(sms * std::max(1, std::min(per, 2)), kRootMaxBlocks);
    if ((e = cudaMemsetAsync(rs.bar, 0, 2 * sizeof(unsigned) + sizeof(int), st)) != cudaSuccess) return e;
    SumRootArgs a;
    a.chiq = reinterpret_cast<const double4 *>(chiq);
    a.cinf = chi0_inf;
    a.cinf2 = chi0_inf2;
    a.w16 = g.w16;
    a.tailq = g.tailq;
    a.mom_suf = mom_suf;
    a.cmax_suf = cmax_suf;
    a.tailm = tailm;
    a.nb = g.nb;
    a.nblk = g.n8p / 4;
    a.n8 = g.n8;
    a.T = T;
    a.scale = T / (4.0 * (g.nbk - 1) * (g.nbk - 1));
    a.n = n;
    a.nsr = nsr;
    a.U = U;
    a.hi_sp = hi_sp;
    a.partial = rs.partial;
    a.bar = rs.bar;
    a.err = reinterpret_cast<int *>(rs.bar + 2);
    a.ctl = reinterpret_cast<RootCtl *>(rs.ctl);
    a.out = rs.out;
    void *args[] = {&a};
    e = cudaLaunchCooperativeKernel((const void *)k_sumrule_roots, dim3(grid), dim3(kRootThreads), args, 0, st);
    if (e != cudaSuccess) return e;
    return launched();
}

}  // namespace tpsc
