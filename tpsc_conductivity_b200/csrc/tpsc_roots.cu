// tpsc_roots.cu -- the Newton form's root searches on the device.
//
// The sum-rule roots Usp and Uch (chi::find_Usp_Uch(nq0, nw0, Usc),
// src/chi.cpp:846-876) as one cooperative kernel: every block sums its share
// of the stored frequencies below the series cut, a grid barrier, then every
// block adds the partials and the high-frequency moment series and takes the
// same safeguarded Halley step (the pass also sums the second derivative),
// until both roots have converged.  One launch and one readback replace a
// host round trip per evaluation.
//
// The grid barrier spins on a generation counter with a wall-time bound:
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
constexpr int kRootMaxNb = 2049;  // bosonic frequencies of Nw0 = 4096
// wall time a barrier wait spins before it gives up (%globaltimer, ns)
constexpr unsigned long long kBarrierNs = 1500000000ull;

__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// bar[0]: arrivals, bar[1]: generation.  Returns false (and sets *err) when
// the wait ran out or another block had already failed.  The waiting thread
// polls the generation word without sleeping: a poll is one L2 round trip,
// so the barrier opens within about that of the last arrival.
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
            const unsigned long long t0 = globaltimer_ns();
            while (*gen == g0) {
                if (*(volatile int *)err || globaltimer_ns() - t0 > kBarrierNs) {
                    atomicExch(err, 1);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        s_ok = ok && !*(volatile int *)err;
    }
    __syncthreads();
    return s_ok;
}

// Grid-stride walk over the items it = blk * nj + j (blk a column block,
// j < nj a frequency): both indices are stepped by the stride's quotient and
// remainder, so that no item pays a 64-bit division.  nj <= 0: no items.
struct GridWalk {
    int blk, j, dblk, dj, nj;
    __device__ explicit GridWalk(int nj_) : nj(nj_) {
        if (nj <= 0) {
            blk = 0x7fffffff;
            j = dblk = dj = 0;
            return;
        }
        const long long first = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        const long long stride = (long long)gridDim.x * blockDim.x;
        blk = (int)(first / nj);
        j = (int)(first - (long long)blk * nj);
        dblk = (int)(stride / nj);
        dj = (int)(stride - (long long)dblk * nj);
    }
    // the item after (b, jj) in this thread's walk
    __device__ void after(int b, int jj, int &nb, int &nj2) const {
        nb = b + dblk;
        nj2 = jj + dj;
        if (nj2 >= nj) {
            nj2 -= nj;
            ++nb;
        }
    }
};

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
    const double *chi0max;  // device max chi0(q, 0), or null: hi_sp as given
    double hi_off;          // hi_sp = 2 / chi0max - hi_off
    double *partial;  // [2][2 kRootMaxBlocks]: two buffers of (value, derivative) per block
    unsigned *bar;    // [2], zero at launch
    int *err;         // zero at launch
    double *out;      // Usp, Uch, evals_sp, evals_ch, ok_sp, ok_ch
    Bp b;             // batched launch: point blockIdx.z, blocks blockIdx.x of gridDim.x per point
};

// the value and its derivatives, each summed in a fixed order, into
// dst[0..kRootVals)
__device__ void block_root_sums(double v, double dv, double d2v, double *dst) {
    __shared__ double red[32][kRootVals];
    for (int off = 16; off > 0; off >>= 1) {
        v += __shfl_down_sync(0xffffffffu, v, off);
        dv += __shfl_down_sync(0xffffffffu, dv, off);
        d2v += __shfl_down_sync(0xffffffffu, d2v, off);
    }
    if ((threadIdx.x & 31) == 0) {
        red[threadIdx.x >> 5][0] = v;
        red[threadIdx.x >> 5][1] = dv;
        red[threadIdx.x >> 5][2] = d2v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0, c = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
            a += red[w][0];
            b += red[w][1];
            c += red[w][2];
        }
        dst[0] = a;
        dst[1] = b;
        dst[2] = c;
    }
    __syncthreads();
}

// warp 0 adds every block's partials of one evaluation in the same order
__device__ void grid_root_sums(const double *part, double &pv, double &pd, double &p2) {
    pv = pd = p2 = 0.0;
    for (int b = threadIdx.x; b < (int)gridDim.x; b += 32) {
        pv += __ldcg(&part[kRootVals * b]);
        pd += __ldcg(&part[kRootVals * b + 1]);
        p2 += __ldcg(&part[kRootVals * b + 2]);
    }
    for (int off = 16; off > 0; off >>= 1) {
        pv += __shfl_down_sync(0xffffffffu, pv, off);
        pd += __shfl_down_sync(0xffffffffu, pd, off);
        p2 += __shfl_down_sync(0xffffffffu, p2, off);
    }
}

// One safeguarded update with the bracket, bisection fallback and stopping
// tests of the host routine newton_root (tpsc_engine.cpp).  The step is
// Halley's, x - 2 y y' / (2 y'^2 - y y''), while |y y''| <= y'^2 (it is then
// between 2/3 and 2 Newton steps); else, and with d2y = 0, Newton's.
__device__ void newton_update(RootCtl &c, double y, double dy, double tol, double d2y = 0.0) {
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
    double xn = 0.5 * (c.lo + c.hi);
    if (dy != 0.0) {
        const double yy = y * d2y, dd = dy * dy;
        xn = (d2y != 0.0 && fabs(yy) <= dd) ? c.x - 2.0 * y * dy / (2.0 * dd - yy) : c.x - y / dy;
    }
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

// One barrier per evaluation: every block writes its partial sums into the
// buffer of the iteration's parity, waits at the barrier, then adds ALL
// partials in the same order and takes the same Newton step on its own copy
// of the state (identical in every block).  A buffer is rewritten two
// iterations later, after a barrier that every reader of it has passed.
//
// The spin search iterates on s = -ln(1 - Us/hi), hi = 2/chi0max - 2 eps,
// Us = -hi expm1(-s): R_sp has the AFM pole at hi and behaves like -ln of the
// distance to it, so Newton in Us overshoots the pole and falls back to
// bisection step after step, while in s it converges in a few steps.  The
// root is the same zero of R_sp.
constexpr double kSpinSMax = 40.0;  // -hi expm1(-40) = hi (1 - 4e-18)

__device__ __forceinline__ double spin_us(double s, double hi) { return -hi * expm1(-s); }

__global__ void __launch_bounds__(kRootThreads) k_sumrule_roots(SumRootArgs a) {
    {
        const long long ar = a.b.arena;
        a.chiq = at(a.chiq, ar);
        a.cinf = at(a.cinf, ar);
        a.cinf2 = at(a.cinf2, ar);
        a.tailq = at(a.tailq, ar);
        a.mom_suf = at(a.mom_suf, ar);
        a.cmax_suf = at(a.cmax_suf, ar);
        a.tailm = at(a.tailm, ar);
        a.chi0max = at(a.chi0max, ar);
        a.partial = at(a.partial, ar);
        a.bar = at(a.bar, ar);
        a.err = at(a.err, ar);
        a.out = at(a.out, ar);
        a.T = bpar(a.b, kPpT, a.T);
        a.scale = bpar(a.b, kPpNormFact, a.scale);
        a.n = bpar(a.b, kPpN, a.n);
        a.nsr = bpar(a.b, kPpNsr, a.nsr);
        a.U = bpar(a.b, kPpU, a.U);
    }
    // the spin interval's upper end 2/chi0max - 2 eps, from the device maximum
    // when the chi0 stage left it there (no host round trip)
    const double hi_sp = a.chi0max ? 2.0 / a.chi0max[0] - a.hi_off : a.hi_sp;
    __shared__ RootCtl sc;
    __shared__ int s_jdir, s_tail;
    // cmax_suf and tailm staged once; the series moments of an evaluation's
    // cut are fetched before its pass and read after the barrier
    __shared__ double s_cmax[kRootMaxNb], s_tailm[kMomP + 1], s_M[kMomP];
    for (int j = threadIdx.x; j < a.nb; j += blockDim.x) s_cmax[j] = a.cmax_suf[j];
    for (int m = threadIdx.x; m <= kMomP; m += blockDim.x) s_tailm[m] = a.tailm[m];
    const int nwmax = a.nb - 1;
    const double tw = 2.0 * 3.141592653589793 * a.T;
    double Usp = 0.0;
    int parity = 0;
#pragma unroll 1
    for (int phase = 0; phase < 2; ++phase) {
        const double sgn = phase == 0 ? -1.0 : 1.0;
        if (threadIdx.x == 0) {
            const double hi = phase == 0 ? hi_sp : 1000.0 * a.U;
            // spin: U/2 (clamped inside the interval); charge: U
            const double x0 = phase == 0 ? a.U / 2.0 : a.U;
            const double xs = (x0 > 0.0 && x0 < hi) ? x0 : 0.5 * hi;
            sc.lo = 0.0;
            sc.hi = phase == 0 ? kSpinSMax : hi;
            sc.x = phase == 0 ? -log1p(-xs / hi) : xs;
            sc.prev_step = 0.0;
            sc.nev = sc.it = sc.done = sc.ok = 0;
        }
        __syncthreads();
#pragma unroll 1
        while (!sc.done) {
            if (threadIdx.x < 32) {
                const double ah = fabs(phase == 0 ? spin_us(sc.x, hi_sp) : sc.x) / 2.0;
                // first frequency of the series (cmax_suf does not increase):
                // every j < lo is below the cut and every j >= hi above it;
                // a round probes 32 points of [lo, hi) and keeps one step of it
                int lo = 0, hi = a.nb;
                while (hi > lo) {
                    const int step = (hi - lo + 31) / 32;
                    const int q = lo + ((int)threadIdx.x + 1) * step - 1;
                    const bool below = q < hi && ah * s_cmax[q] >= kMomSeriesMax;
                    const int t = __popc(__ballot_sync(0xffffffffu, below));
                    const int qt = lo + (t + 1) * step - 1;
                    if (t < 32 && qt < hi) hi = qt;
                    lo += t * step;
                }
                const bool tail = ah * s_tailm[kMomP] >= kMomSeriesMax;
                if (threadIdx.x < kMomP)
                    s_M[threadIdx.x] = (lo < a.nb ? a.mom_suf[(size_t)lo * kMomP + threadIdx.x] : 0.0) +
                                       (tail ? 0.0 : s_tailm[threadIdx.x]);
                if (threadIdx.x == 0) {
                    s_jdir = lo;
                    s_tail = tail;
                }
            }
            __syncthreads();
            const double x = phase == 0 ? spin_us(sc.x, hi_sp) : sc.x, hu = sgn * x / 2.0;
            const int jdir = s_jdir;
            // v = sum f w (q - x), q = x / (1 + h x), h = sgn U / 2; its U
            // derivatives: dq/dU = -sgn q^2 / 2, d2q/dU2 = q^3 / 2
            double v = 0.0, dv = 0.0, d2v = 0.0;
            // the next item's chi0 row is loaded before this item's arithmetic
            const GridWalk walk(jdir);
            int blk = walk.blk, j = walk.j;
            double4 xn = blk < a.nblk ? a.chiq[(size_t)blk * a.nb + j] : make_double4(0.0, 0.0, 0.0, 0.0);
            while (blk < a.nblk) {
                const double4 xq = xn;
                int nb, nj;
                walk.after(blk, j, nb, nj);
                if (nb < a.nblk) xn = a.chiq[(size_t)nb * a.nb + nj];
                const double4 w = reinterpret_cast<const double4 *>(a.w16)[blk];
                const double f = j == 0 ? 0.5 : 1.0;
                const double xs[4] = {xq.x, xq.y, xq.z, xq.w}, ws[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const double q = xs[c] / (1.0 + hu * xs[c]), fw = f * ws[c];
                    v += fw * (q - xs[c]);
                    dv += fw * q * q;
                    d2v += fw * q * q * q;
                }
                blk = nb;
                j = nj;
            }
            dv *= -0.5 * sgn;
            d2v *= 0.5;
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
                        d2v += w * 0.5 * q * q * q;
                    }
                }
            }
            double *part = a.partial + (size_t)parity * kRootVals * kRootMaxBlocks;
            block_root_sums(v, dv, d2v, part + kRootVals * blockIdx.x);
            if (!grid_sync(a.bar, a.err)) return;
            parity ^= 1;
            if (threadIdx.x < 32) {
                double pv, pd, p2;
                grid_root_sums(part, pv, pd, p2);
                if (threadIdx.x == 0) {
                    // the series over the frequencies from jdir (and over the
                    // tail), S = sum_m (-h)^m M_m, and its h derivatives
                    double S = 0.0, dS = 0.0, d2S = 0.0, hm1 = 1.0, hm2 = 0.0;  // (-h)^(m-1), (-h)^(m-2)
                    const double h = hu;
                    for (int m = 1; m <= kMomP; ++m) {
                        const double M = s_M[m - 1];
                        S += -h * hm1 * M;
                        dS += -m * hm1 * M;
                        d2S += m * (m - 1) * hm2 * M;
                        hm2 = hm1;
                        hm1 *= -h;
                    }
                    // dh/dU = sgn / 2
                    const double tr = a.scale * (pv + S), dtr = a.scale * (pd + 0.5 * sgn * dS),
                                 d2tr = a.scale * (p2 + 0.25 * d2S);
                    const double n = a.n, nsr = a.nsr, U = a.U;
                    double y, dy, d2y;
                    if (phase == 0) {
                        // chi::sum_rule_sp (src/chi.cpp:833-836)
                        y = tr + n - n * n / 2.0 - nsr + x * nsr * nsr / (2.0 * U);
                        // d/ds = d/dUs * dUs/ds, dUs/ds = hi e^-s = hi - Us,
                        // d2Us/ds2 = -(hi - Us)
                        dy = (dtr + nsr * nsr / (2.0 * U)) * (hi_sp - x);
                        d2y = d2tr * (hi_sp - x) * (hi_sp - x) - dy;
                    } else {
                        // chi::sum_rule_ch (src/chi.cpp:840-843)
                        y = tr + n - n * n / 2.0 - (nsr + Usp * nsr * nsr / (2.0 * U) - nsr * nsr);
                        dy = dtr;
                        d2y = d2tr;
                    }
                    newton_update(sc, y, dy, 1e-16, d2y);
                }
            }
            __syncthreads();
        }
        const double root = phase == 0 ? spin_us(sc.root, hi_sp) : sc.root;
        if (phase == 0) Usp = root;
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.out[phase] = root;
            a.out[2 + phase] = sc.nev;
            a.out[4 + phase] = sc.ok;
        }
        if (!sc.ok) return;
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// chemical potential
// ---------------------------------------------------------------------------

// One pass over Sigma for the Newton form: Tr Sigma G0 with its asymptotic
// correction (green::traceSelfG, src/green.cpp:3001-3084) over the stored
// frequencies, and the moments of the find_mu series over the stored
// frequencies n >= jc and the tail Nw0/2 <= n <= Nw0 (asymptotic Sigma, as
// green::traceDiffG sums them):
//   C_m = sum w z^-(m+1),  z = i w_n - eps + mu0 - Sigma,  m < kMuMomP,
//   G0  = sum w Re 1/(i w_n - eps + mu0),
// so that this part of Tr(G - G0) at mu is Re sum_m (mu0 - mu)^m C_m - G0 to
// a relative kMuSeriesMax^kMuMomP while |mu - mu0| <= kMuSeriesMax |z|.
//
// C_m for m >= kMuMomF64 is formed and summed in FP32 (per thread, ~32 terms;
// the block and grid sums are FP64): its term (mu0 - mu)^m C_m is at most
// kMuSeriesMax^m = 8e-7 of the leading one per point, so an FP32 relative
// error ~1e-6 on it moves Tr(G - G0) by < 1e-12 of its leading term.  The
// point constants live in shared memory and Tr Sigma G0, its Hartree part and
// G0 share one reciprocal per (k, n), so that two CTAs fit on an SM.
//
// Blocks 0 .. nblk-1 take one column block each over the stored frequencies;
// the four columns of a row are formed without a branch (a padding column
// has weight 0 and finite stand-in values), so that their chains interleave.
// Blocks nblk .. nblk + ceil(nblk / 2) - 1 take the tail, one warp per
// column, away from the Sigma stream.  Per-block partials (block_store).
constexpr int kMuMomF64 = 4;
constexpr int kTailR = 28;           // terms of the tail power series (needs kMuMomP + kTailR < kTailP)
constexpr double kTailRatio = 0.05;  // series when rho / w_NO < this: terms below 0.05^28 (~1e-36) relative
static_assert(kMuMomP + kTailR < kTailP, "tail power sums too short");
constexpr int kMomThreads = 256;
constexpr int kMomTailCols = kMomThreads / 32;  // columns of a tail block

__host__ __device__ constexpr int sigma_moment_tail_blocks(int nblk) {
    return (4 * nblk + kMomTailCols - 1) / kMomTailCols;
}

__global__ void __launch_bounds__(kMomThreads, 2)
    k_sigma_moments(const double2 *__restrict__ S, const double *__restrict__ s2, const double *__restrict__ s3,
                    const double *__restrict__ s4, const double *__restrict__ sinfp, const double *__restrict__ ek,
                    const double *__restrict__ w16, const double *__restrict__ tailP, int nw0, double mu0,
                    double T, double nk02, int jc, int nblk, double *partial, Bp b) {
    constexpr int NV = kSigmaMomNV, P64 = kMuMomF64, P32 = kMuMomP - kMuMomF64;
    __shared__ double cw[4], cx[4], c2[4], c3[4];
    __shared__ __align__(16) double2 s_row[2][kMomThreads][4];  // two stages of 64-byte Sigma rows
    S = at(S, b.arena);
    s2 = at(s2, b.arena);
    s3 = at(s3, b.arena);
    s4 = at(s4, b.arena);
    sinfp = at(sinfp, b.arena);
    ek = at(ek, b.arena);
    tailP = at(tailP, b.arena);
    partial = at(partial, b.arena);
    mu0 = bpar(b, kPpMu0, mu0);
    T = bpar(b, kPpT, T);
    jc = (int)bpar(b, kPpJc, (double)jc);
    const int blk = blockIdx.x, NO = nw0 / 2;
    const double sinf = sinfp[0];
    const double pt = 3.141592653589793 * T;
    double tsg = 0.0, har = 0.0, g0 = 0.0;
    double m64[2 * P64];
    float m32[2 * P32];
#pragma unroll
    for (int k = 0; k < 2 * P64; ++k) m64[k] = 0.0;
#pragma unroll
    for (int k = 0; k < 2 * P32; ++k) m32[k] = 0.0f;
    // z = i w_n - x - Sigma with x = eps - mu0; inv = 1 / (w_n^2 + x^2)
    // rr = 1/|z|^2 (|z| >= w_n > 0)
    auto moments_rr = [&](double zx, double zy, double rr, double x, double w, double inv) {
        const double2 zi = make_double2(zx * rr, -zy * rr);
        double2 zp = zi;
#pragma unroll
        for (int m = 0; m < P64; ++m) {
            m64[2 * m] += w * zp.x;
            m64[2 * m + 1] += w * zp.y;
            zp = cmul(zp, zi);
        }
        const float wf = (float)w;
        const float2 zf = make_float2((float)zi.x, (float)zi.y);
        float2 zq = make_float2((float)zp.x, (float)zp.y);
#pragma unroll
        for (int m = 0; m < P32; ++m) {
            m32[2 * m] += wf * zq.x;
            m32[2 * m + 1] += wf * zq.y;
            zq = make_float2(zq.x * zf.x - zq.y * zf.y, zq.x * zf.y + zq.y * zf.x);
        }
        g0 -= w * x * inv;
    };
    auto moments = [&](double wn, double rS, double iS, double x, double w, double inv) {
        const double zx = -x - rS, zy = wn - iS;
        moments_rr(zx, zy, 1.0 / (zx * zx + zy * zy), x, w, inv);
    };
    double fermi = 0.0;  // traceSelfG's Fermi-function term, threads 0..3 of a stored-frequency block
    if (blk < nblk) {
        const int o0 = 4 * blk;
        if (threadIdx.x < 4) {
            // a padding column: weight 0, x = 1 and Sigma's coefficients 0,
            // so that |z| and w_n^2 + x^2 stay away from 0 and its terms are 0
            const int c = threadIdx.x;
            const double w = w16[o0 + c];
            const bool ok = w != 0.0;
            cw[c] = w;
            cx[c] = ok ? ek[o0 + c] - mu0 : 1.0;
            c2[c] = ok ? s2[o0 + c] : 0.0;
            c3[c] = ok ? s3[o0 + c] : 0.0;
        }
        __syncthreads();
        // this thread's Sigma rows j = tid + 256 i through two shared-memory
        // stages: row i + 1 is copied (cp.async, 4 x 16 bytes) while row i is
        // formed; each thread reads back only its own copies
        const double2 *row = S + (size_t)blk * 4 * NO;
        auto issue = [&](int jj, int st) {
#pragma unroll
            for (int c = 0; c < 4; ++c) cp_async16(&s_row[st][threadIdx.x][c], row + 4 * (size_t)jj + c);
            asm volatile("cp.async.commit_group;\n" ::: "memory");
        };
        if ((int)threadIdx.x < NO) issue(threadIdx.x, 0);
        for (int j = threadIdx.x, st = 0; j < NO; j += blockDim.x, st ^= 1) {
            const double wn = (2 * j + 1) * pt, i1 = 1.0 / wn;
            if (j + (int)blockDim.x < NO) {
                issue(j + blockDim.x, st ^ 1);
                asm volatile("cp.async.wait_group 1;\n" ::: "memory");
            } else {
                asm volatile("cp.async.wait_group 0;\n" ::: "memory");
            }
            const double2 sv[4] = {s_row[st][threadIdx.x][0], s_row[st][threadIdx.x][1], s_row[st][threadIdx.x][2],
                                   s_row[st][threadIdx.x][3]};
            if (j >= jc) {
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const double w = cw[c], x = cx[c];
                    const double2 s = w != 0.0 ? sv[c] : make_double2(0.0, 0.0);
                    double rS, iS;
                    sigma_full(i1, sinf, c2[c], c3[c], s, rS, iS);
                    // one reciprocal for 1/(w_n^2 + x^2) and 1/|z|^2
                    const double b = wn * wn + x * x;
                    const double zx = -x - rS, zy = wn - iS, a = zx * zx + zy * zy;
                    const double r = 1.0 / (a * b), inv = r * a;
                    tsg += w * inv * (rS * (-x) + iS * wn);
                    har += w * inv;
                    moments_rr(zx, zy, r * b, x, w, inv);
                }
            } else {
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const double w = cw[c], x = cx[c];
                    const double2 s = w != 0.0 ? sv[c] : make_double2(0.0, 0.0);
                    double rS, iS;
                    sigma_full(i1, sinf, c2[c], c3[c], s, rS, iS);
                    const double inv = 1.0 / (wn * wn + x * x);
                    tsg += w * inv * (rS * (-x) + iS * wn);
                    har += w * inv;
                }
            }
        }
        // traceSelfG's Fermi-function term per octant point
        if (threadIdx.x < 4) {
            const int c = threadIdx.x;
            const double w8 = 0.5 * cw[c];
            if (w8 != 0.0) {
                const double x = cx[c];
                if (fabs(x) > 1.0e-12) {
                    fermi = w8 * sinf * (1.0 / (exp(x / T) + 1.0) - 0.5) / x / nk02;
                } else {
                    const double ex = (x < 0) ? exp(x / T) : exp(-x / T);
                    fermi = -w8 * sinf * ex / ((ex + 1.0) * (ex + 1.0) * nk02 * T);
                }
            }
        }
    } else {
        // The tail n = NO .. 2 NO (asymptotic Sigma), warp `warp` for column o:
        // with u = 1/(i w_n), z^-1 = u / (1 - q(u)), q(u) = x u + Sinf u^2 +
        // C2 u^3 + C3 u^4 + C4 u^5 (real coefficients), and h^(p) the
        // coefficients of (1 - q)^-p,
        //   sum_tail z^-p = sum_r h^(p)_r (-i)^(p+r) P_(p+r),
        //   sum_tail Re 1/(i w_n - x) = -x sum_k (-x^2)^k P_(2k+2),
        // P_p = sum_tail w_n^-p (tailP).  (1 - q)^-p obeys H' (1 - q) = p q' H,
        // so R h_R = sum_{s=1..5} q_s h_(R-s) (R - s + p s),   h_0 = 1:
        // lane p - 1 runs the recurrence of moment m = p - 1 in registers.  The
        // terms fall like (rho / w_NO)^r, rho a bound on q's root radius; above
        // kTailRatio the warp sums term by term.
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        const int o = (blk - nblk) * kMomTailCols + warp;
        const double w = o < 4 * nblk ? __ldg(&w16[o]) : 0.0;
        if (w != 0.0) {
            const double x = __ldg(&ek[o]) - mu0;
            const double q1 = x, q2 = sinf, q3 = __ldg(&s2[o]), q4 = __ldg(&s3[o]), q5 = __ldg(&s4[o]);
            const double rho = fabs(x) + sqrt(fabs(sinf)) + cbrt(fabs(q3)) + sqrt(sqrt(fabs(q4))) + pow(fabs(q5), 0.2);
            const double w_no = (2 * NO + 1) * pt;
            if (rho < kTailRatio * w_no) {
                double re = 0.0, im = 0.0;
                if (lane < kMuMomP) {
                    const double p = lane + 1;
                    // h_(R-1) .. h_(R-5) in a register window
                    double h1 = 1.0, h2 = 0.0, h3 = 0.0, h4 = 0.0, h5 = 0.0;
                    // r = 0 term: (-i)^p P_p
                    auto add = [&](int k, double h) {
                        const double t = h * __ldg(&tailP[k]);
                        switch (k & 3) {
                            case 0: re += t; break;
                            case 1: im -= t; break;
                            case 2: re -= t; break;
                            default: im += t; break;
                        }
                    };
                    add(lane + 1, 1.0);
                    // unrolled: 1 / R is a constant of each step
#pragma unroll
                    for (int R = 1; R <= kTailR; ++R) {
                        const double hR = (q1 * h1 * (R - 1 + p) + q2 * h2 * (R - 2 + 2 * p) +
                                           q3 * h3 * (R - 3 + 3 * p) + q4 * h4 * (R - 4 + 4 * p) +
                                           q5 * h5 * (R - 5 + 5 * p)) *
                                          (1.0 / R);
                        add(lane + 1 + R, hR);
                        h5 = h4;
                        h4 = h3;
                        h3 = h2;
                        h2 = h1;
                        h1 = hR;
                    }
                } else if (lane == kMuMomP) {
                    // G0: -x sum_k (-x^2)^k P_(2k+2)
                    double xp = 1.0;
                    for (int k = 0; 2 * k + 2 < kTailP; ++k, xp *= -x * x) re += xp * __ldg(&tailP[2 * k + 2]);
                    re *= -x;
                }
#pragma unroll
                for (int m = 0; m < kMuMomP; ++m) {
                    const double rm = __shfl_sync(0xffffffffu, re, m), imm = __shfl_sync(0xffffffffu, im, m);
                    if (lane == 0) {
                        if (m < P64) {
                            m64[2 * m] += w * rm;
                            m64[2 * m + 1] += w * imm;
                        } else {
                            m32[2 * (m - P64)] += (float)(w * rm);
                            m32[2 * (m - P64) + 1] += (float)(w * imm);
                        }
                    }
                }
                const double gt = __shfl_sync(0xffffffffu, re, kMuMomP);
                if (lane == 0) g0 += w * gt;
            } else {
                for (int t = lane; t <= NO; t += 32) {
                    const double wn = (2 * (NO + t) + 1) * pt, i1 = 1.0 / wn, i2 = i1 * i1;
                    moments(wn, -q3 * i2 + q5 * i2 * i2, -sinf * i1 + q4 * i2 * i1, x, w, 1.0 / (wn * wn + x * x));
                }
            }
        }
    }
    double acc[NV];
    acc[0] = tsg * T / nk02;
    acc[1] = har * sinf * T / nk02 + fermi;
#pragma unroll
    for (int k = 0; k < 2 * P64; ++k) acc[2 + k] = m64[k];
#pragma unroll
    for (int k = 0; k < 2 * P32; ++k) acc[2 + 2 * P64 + k] = (double)m32[k];
    acc[2 + 2 * kMuMomP] = g0;
    block_store<NV>(acc, partial);
}

struct MuRootArgs {
    const double2 *S;
    const double *s2, *s3, *s4, *sinf, *ek, *w16;
    const double *mom;  // the k_sigma_moments results
    int nw0, nblk, jc;
    double mu0, T, nk02, wc;  // wc = w_jc
    double *partial;  // [2][2 kRootMaxBlocks]
    unsigned *bar;
    int *err;
    double *out;  // mu, evals, ok, Tr Sigma G at mu
    Bp b;         // batched launch: point blockIdx.z
};

// the four octant points of column block blk at frequency j of
// green::traceSelfG2 (src/green.cpp:2929-2976): sum w8 2T/nk02 Re[Sigma G]
// with G = 1/(i w_n - e + mu - Sigma); p, q the block's Sigma row at j.  The
// four fractions K N / A share one division: sum K_c N_c / A_c =
// [(K0 N0 A1 + K1 N1 A0) A2 A3 + (K2 N2 A3 + K3 N3 A2) A0 A1] / (A0 A1 A2 A3),
// A_c lies between w_n^2 and ~w_max^2, so the products stay far inside FP64's range.
__device__ __forceinline__ double trsg_row(const MuRootArgs &a, int blk, int j, double4 p, double4 q, double mu,
                                           double sinf, double pt) {
    const int o0 = 4 * blk;
    const double2 sv[4] = {make_double2(p.x, p.y), make_double2(p.z, p.w), make_double2(q.x, q.y),
                           make_double2(q.z, q.w)};
    const double wn = (2 * j + 1) * pt, i1 = 1.0 / wn, kT = 2.0 * a.T / a.nk02;
    double K[4], N[4], A[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const double w8 = 0.5 * __ldg(&a.w16[o0 + c]);
        // a padding column: weight 0, and e - mu = 1 with Sigma's
        // coefficients 0, so that its A >= 1 and its term is 0
        double e = 1.0, c2 = 0.0, c3 = 0.0;
        double2 s = make_double2(0.0, 0.0);
        if (w8 != 0.0) {
            e = __ldg(&a.ek[o0 + c]) - mu;
            c2 = __ldg(&a.s2[o0 + c]);
            c3 = __ldg(&a.s3[o0 + c]);
            s = sv[c];
        }
        double rS, iS;
        sigma_full(i1, sinf, c2, c3, s, rS, iS);
        const double aa = e + rS;
        A[c] = (wn - iS) * (wn - iS) + aa * aa;
        N[c] = iS * wn - iS * iS - e * rS - rS * rS;
        K[c] = w8 * kT;
    }
    const double P01 = A[0] * A[1], P23 = A[2] * A[3];
    return ((K[0] * N[0] * A[1] + K[1] * N[1] * A[0]) * P23 + (K[2] * N[2] * A[3] + K[3] * N[3] * A[2]) * P01) /
           (P01 * P23);
}

// find_mu by safeguarded Halley steps (newton_update) from
// mu0 inside [-10, 10] with tolerance 1e-15, one barrier per evaluation as in
// k_sumrule_roots; then green::traceSelfG2 (src/green.cpp:2929-2976) at mu.
__global__ void __launch_bounds__(kRootThreads) k_mu_roots(MuRootArgs a) {
    {
        const long long ar = a.b.arena;
        a.S = at(a.S, ar);
        a.s2 = at(a.s2, ar);
        a.s3 = at(a.s3, ar);
        a.s4 = at(a.s4, ar);
        a.sinf = at(a.sinf, ar);
        a.ek = at(a.ek, ar);
        a.mom = at(a.mom, ar);
        a.partial = at(a.partial, ar);
        a.bar = at(a.bar, ar);
        a.err = at(a.err, ar);
        a.out = at(a.out, ar);
        a.mu0 = bpar(a.b, kPpMu0, a.mu0);
        a.T = bpar(a.b, kPpT, a.T);
        a.jc = (int)bpar(a.b, kPpJc, (double)a.jc);
        a.wc = bpar(a.b, kPpWc, a.wc);
    }
    __shared__ RootCtl sc;
    const int NO = a.nw0 / 2;
    const double sinf = a.sinf[0];
    const double pt = 3.141592653589793 * a.T;
    // the series holds while |mu - mu0| <= kMuSeriesMax |z|_min, |z|_min = w_jc - 2 |Sigma_inf| / w_jc
    const double zmin = a.wc - 2.0 * fabs(sinf) / a.wc;
    const double dmax = zmin > 0.0 ? kMuSeriesMax * zmin : 0.0;
    int parity = 0;
    if (threadIdx.x == 0) {
        sc.lo = -10.0;
        sc.hi = 10.0;
        sc.x = (a.mu0 > sc.lo && a.mu0 < sc.hi) ? a.mu0 : 0.0;
        sc.prev_step = 0.0;
        sc.nev = sc.it = sc.done = sc.ok = 0;
    }
    __syncthreads();
#pragma unroll 1
    while (!sc.done) {
        const double pmu = sc.x, delta = pmu - a.mu0;
        const bool series = fabs(delta) <= dmax;
        const int jhi = series ? a.jc : NO;
        double v = 0.0, dv = 0.0, d2v = 0.0;
        const GridWalk walk(jhi);
        for (int blk = walk.blk, j = walk.j; blk < a.nblk; walk.after(blk, j, blk, j)) {
            const int o0 = 4 * blk;
            const double4 *row = reinterpret_cast<const double4 *>(a.S + (size_t)blk * 4 * NO);
            const double4 p = ld_stream4(&row[2 * j]), q = ld_stream4(&row[2 * j + 1]);
            const double2 sv[4] = {make_double2(p.x, p.y), make_double2(p.z, p.w), make_double2(q.x, q.y),
                                   make_double2(q.z, q.w)};
            const double wn = (2 * j + 1) * pt, i1 = 1.0 / wn;
#pragma unroll
            for (int c = 0; c < 4; ++c) {
                const double w = __ldg(&a.w16[o0 + c]);
                if (w == 0.0) continue;
                double rS, iS;
                sigma_full(i1, sinf, __ldg(&a.s2[o0 + c]), __ldg(&a.s3[o0 + c]), sv[c], rS, iS);
                trdiff_term(wn, rS, iS, __ldg(&a.ek[o0 + c]), a.mu0, pmu, w, v, dv, d2v);
            }
        }
        if (!series) {
            // the tail Nw0/2 <= n <= Nw0 with the asymptotic Sigma, term by term
            const long long ttot = (long long)a.nblk * 4 * (NO + 1);
            for (long long it = (long long)blockIdx.x * blockDim.x + threadIdx.x; it < ttot;
                 it += (long long)gridDim.x * blockDim.x) {
                const int o = (int)(it / (NO + 1)), t = (int)(it - (long long)o * (NO + 1));
                const double w = __ldg(&a.w16[o]);
                if (w == 0.0) continue;
                const double wn = (2 * (NO + t) + 1) * pt, i1 = 1.0 / wn, i2 = i1 * i1;
                const double rS = -__ldg(&a.s2[o]) * i2 + __ldg(&a.s4[o]) * i2 * i2;
                const double iS = -sinf * i1 + __ldg(&a.s3[o]) * i2 * i1;
                trdiff_term(wn, rS, iS, __ldg(&a.ek[o]), a.mu0, pmu, w, v, dv, d2v);
            }
        }
        double *part = a.partial + (size_t)parity * kRootVals * kRootMaxBlocks;
        block_root_sums(v, dv, d2v, part + kRootVals * blockIdx.x);
        if (!grid_sync(a.bar, a.err)) return;
        parity ^= 1;
        if (threadIdx.x < 32) {
            double pv, pd, p2;
            grid_root_sums(part, pv, pd, p2);
            if (threadIdx.x == 0) {
                if (series) {
                    // Re sum_m (-delta)^m C_m - G0 and its first two mu derivatives
                    double sr = 0.0, dsr = 0.0, d2sr = 0.0, pr = 1.0, pm = 0.0, pmm = 0.0;
                    for (int m = 0; m < kMuMomP; ++m) {  // pr, pm, pmm = (-delta)^(m, m-1, m-2)
                        const double C = a.mom[2 + 2 * m];
                        sr += pr * C;
                        dsr += -m * pm * C;
                        d2sr += m * (m - 1) * pmm * C;
                        pmm = pm;
                        pm = pr;
                        pr *= -delta;
                    }
                    pv += sr - a.mom[2 + 2 * kMuMomP];
                    pd += dsr;
                    p2 += d2sr;
                }
                newton_update(sc, pv, pd, 1e-15, p2);
            }
        }
        __syncthreads();
    }
    if (!sc.ok) {
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.out[0] = sc.x;
            a.out[1] = sc.nev;
            a.out[2] = 0.0;
            a.out[3] = 0.0;
        }
        return;
    }
    // Tr Sigma G at mu over the stored frequencies; the next item's Sigma
    // row is loaded before this item's arithmetic.
    const double mu = sc.root;
    double v = 0.0;
    {
        const GridWalk walk(NO);
        int blk = walk.blk, j = walk.j;
        auto load = [&](int bk, int jj, double4 &p, double4 &q) {
            const double4 *row = reinterpret_cast<const double4 *>(a.S + (size_t)bk * 4 * NO);
            p = ld_stream4(&row[2 * jj]);
            q = ld_stream4(&row[2 * jj + 1]);
        };
        double4 p = make_double4(0.0, 0.0, 0.0, 0.0), q = p;
        if (blk < a.nblk) load(blk, j, p, q);
        while (blk < a.nblk) {
            int nb, nj;
            walk.after(blk, j, nb, nj);
            double4 pn = p, qn = q;
            if (nb < a.nblk) load(nb, nj, pn, qn);
            v += trsg_row(a, blk, j, p, q, mu, sinf, pt);
            blk = nb;
            j = nj;
            p = pn;
            q = qn;
        }
    }
    double *part = a.partial + (size_t)parity * kRootVals * kRootMaxBlocks;
    block_root_sums(v, 0.0, 0.0, part + kRootVals * blockIdx.x);
    if (!grid_sync(a.bar, a.err)) return;
    if (blockIdx.x == 0 && threadIdx.x < 32) {
        double pv, pd, p2;
        grid_root_sums(part, pv, pd, p2);
        if (threadIdx.x == 0) {
            a.out[0] = mu;
            a.out[1] = sc.nev;
            a.out[2] = 1.0;
            a.out[3] = pv;
        }
    }
}

// The barrier's bound, exercised: block `withhold` never arrives (negative:
// every block does), so every other block's wait runs out after
// kBarrierNs and leaves with the error flag set.  words[0..1] the barrier,
// words[2] the error flag, words[3] the number of blocks that left with it;
// all zero at launch.
__global__ void __launch_bounds__(kRootThreads) k_barrier_probe(unsigned *words, int withhold) {
    if ((int)blockIdx.x == withhold) return;
    const bool ok = grid_sync(words, reinterpret_cast<int *>(words + 2));
    if (threadIdx.x == 0 && !ok) atomicAdd(words + 3, 1u);
}

// the cooperative grid of the root searches: up to two blocks per SM, or
// `cap` blocks when the caller runs several root searches at once (solver
// streams of a batch), so that all of them fit on the GPU together
template <typename K>
cudaError_t root_grid(K kernel, int *grid, int cap) {
    int dev = 0, sms = 0, per = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, kRootThreads, 0)) != cudaSuccess) return e;
    *grid = std::min(sms * std::max(1, std::min(per, 2)), kRootMaxBlocks);
    if (cap > 0) *grid = std::min(*grid, cap);
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_sigma_moments(const GridDev &g, const double2 *S, const double *s2, const double *s3,
                                 const double *s4, const double *sinf, double mu0, double T, int jc, Reduce r,
                                 cudaStream_t st, const Bp &b) {
    const int nblk = g.n8p / 4, nb = nblk + sigma_moment_tail_blocks(nblk);
    if (nb > kMaxBlocks) return cudaErrorInvalidValue;
    const double nk02 = 4.0 * (g.nbk - 1) * (g.nbk - 1);
    k_sigma_moments<<<dim3(nb, 1, b.P), kMomThreads, 0, st>>>(S, s2, s3, s4, sinf, g.ek, g.w16, g.tailP, g.nw0, mu0,
                                                               T, nk02, jc, nblk, r.partial, b);
    cudaError_t e = launched();
    if (e != cudaSuccess) return e;
    return finish<kSigmaMomNV>(r, nb, 0.0, st, b);
}

cudaError_t launch_mu_roots(const GridDev &g, const double2 *S, const double *s2, const double *s3, const double *s4,
                            const double *sinf, const double *mom, double mu0, double T, int jc, double wc,
                            RootScratch rs, cudaStream_t st, const Bp &b) {
    int grid = 0;
    cudaError_t e = root_grid(k_mu_roots, &grid, rs.max_blocks);
    if (e != cudaSuccess) return e;
    // a batched search: the resident grid shared out between the points
    // (the caller keeps P at most the resident grid)
    if (b.P > 1) grid = std::max(1, grid / b.P);
    // words 4..6 of rs.bar: the sum-rule search's error flag (word 2) stays readable
    if (rs.reset_mu) {
        e = b.P > 1 ? cudaMemset2DAsync(rs.bar + 4, (size_t)b.arena, 0, 2 * sizeof(unsigned) + sizeof(int), b.P, st)
                    : cudaMemsetAsync(rs.bar + 4, 0, 2 * sizeof(unsigned) + sizeof(int), st);
        if (e != cudaSuccess) return e;
    }
    MuRootArgs a;
    a.S = S;
    a.s2 = s2;
    a.s3 = s3;
    a.s4 = s4;
    a.sinf = sinf;
    a.ek = g.ek;
    a.w16 = g.w16;
    a.mom = mom;
    a.nw0 = g.nw0;
    a.nblk = g.n8p / 4;
    a.jc = jc;
    a.mu0 = mu0;
    a.T = T;
    a.nk02 = 4.0 * (g.nbk - 1) * (g.nbk - 1);
    a.wc = wc;
    a.partial = rs.partial;
    a.bar = rs.bar + 4;
    a.err = reinterpret_cast<int *>(rs.bar + 6);
    a.out = rs.out;
    a.b = b;
    void *args[] = {&a};
    e = cudaLaunchCooperativeKernel((const void *)k_mu_roots, dim3(grid, 1, b.P), dim3(kRootThreads), args, 0, st);
    if (e != cudaSuccess) return e;
    return launched();
}

cudaError_t launch_sumrule_roots(const GridDev &g, const double *chiq, const double *chi0_inf, const double *chi0_inf2,
                                 const double *mom_suf, const double *cmax_suf, const double *tailm, double T,
                                 double n, double nsr, double U, double hi_sp, RootScratch rs, cudaStream_t st,
                                 const double *chi0max, double hi_off, const Bp &b) {
    if (g.nb > kRootMaxNb) return cudaErrorInvalidValue;
    int grid = 0;
    cudaError_t e = root_grid(k_sumrule_roots, &grid, rs.max_blocks);
    if (e != cudaSuccess) return e;
    if (b.P > 1) grid = std::max(1, grid / b.P);
    if (rs.reset_sr) {
        e = b.P > 1 ? cudaMemset2DAsync(rs.bar, (size_t)b.arena, 0, 2 * sizeof(unsigned) + sizeof(int), b.P, st)
                    : cudaMemsetAsync(rs.bar, 0, 2 * sizeof(unsigned) + sizeof(int), st);
        if (e != cudaSuccess) return e;
    }
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
    a.chi0max = chi0max;
    a.hi_off = hi_off;
    a.partial = rs.partial;
    a.bar = rs.bar;
    a.err = reinterpret_cast<int *>(rs.bar + 2);
    a.out = rs.out;
    a.b = b;
    void *args[] = {&a};
    e = cudaLaunchCooperativeKernel((const void *)k_sumrule_roots, dim3(grid, 1, b.P), dim3(kRootThreads), args, 0,
                                    st);
    if (e != cudaSuccess) return e;
    return launched();
}

cudaError_t launch_barrier_probe(unsigned *words, int withhold, int *blocks, cudaStream_t st) {
    int grid = 0;
    cudaError_t e = root_grid(k_barrier_probe, &grid, 0);
    if (e != cudaSuccess) return e;
    *blocks = grid;
    if ((e = cudaMemsetAsync(words, 0, 4 * sizeof(unsigned), st)) != cudaSuccess) return e;
    void *args[] = {&words, &withhold};
    e = cudaLaunchCooperativeKernel((const void *)k_barrier_probe, dim3(grid), dim3(kRootThreads), args, 0, st);
    if (e != cudaSuccess) return e;
    return launched();
}

}  // namespace tpsc
