// tpsc_device.cuh -- device helpers shared by the kernel translation units
// (tpsc_kernels.cu: chi0, vertex, self-energy, traces; tpsc_cond.cu: the
// current-current correlator).  Everything here is internal to the library.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "tpsc_fft.cuh"
#include "tpsc_kernels.cuh"

namespace tpsc {

// counts one (or n) kernel launches for the instrumentation ABI and returns
// the launch status
cudaError_t launched(int n = 1);

// Dynamic shared memory above 48 KB needs the function's opt-in attribute,
// which is process-wide: it is raised once per kernel and device to the
// largest size the device allows and never lowered, so that launches from
// concurrent host threads with different sizes all see a cap they fit under.
cudaError_t smem_optin(const void *fn);

namespace {

constexpr double kPi = 3.141592653589793;  // == acos(-1.0) in double

// point blockIdx.z's copy of a per-point array (see Bp)
template <class T>
__device__ __forceinline__ T *at(T *ptr, long long arena) {
    using Ch = typename std::conditional<std::is_const<T>::value, const char, char>::type;
    return ptr ? reinterpret_cast<T *>(reinterpret_cast<Ch *>(ptr) + (long long)blockIdx.z * arena) : ptr;
}
// the point's scalar `slot`, or v for a plain launch
__device__ __forceinline__ double bpar(const Bp &b, int slot, double v) {
    return b.pp ? at(b.pp, b.arena)[slot] : v;
}
constexpr int kSliceThreads = 352;  // 22 groups of 16: the 65 line pairs of a 129-point pass in 3 rounds
constexpr int kTauThreads = 256;
constexpr int kWarm = 30;  // spline sweep warm-up: carry error <= 0.268^30 < 1e-17

// octant index o = m + l (l + 1) / 2, 0 <= m <= l -> (l, m) without a
// table: 8 o + 1 < 2^24 is exact in float and its square root correctly
// rounded, so the estimate of l is off by at most one and the two checks
// correct it
__device__ __forceinline__ void oct_lm(int o, int &l, int &m) {
    int a = (int)((sqrtf((float)(8 * o + 1)) - 1.0f) * 0.5f);
    if ((a + 1) * (a + 2) / 2 <= o) ++a;
    if (a * (a + 1) / 2 > o) --a;
    l = a;
    m = o - a * (a + 1) / 2;
}

// integer multiplicity weight of octant point (l, m) as in the reference
// loops: `base` halved on the l edges, m edges and the diagonal
__device__ __forceinline__ int oct_weight(int base, int l, int m, int nbk) {
    int w = base;
    if (l == 0 || l == nbk - 1) w /= 2;
    if (m == 0 || m == nbk - 1) w /= 2;
    if (m == l) w /= 2;
    return w;
}

// ---------------------------------------------------------------------------
// compensated (Kahan-Babuska) summation
// ---------------------------------------------------------------------------
struct KSum {
    double s = 0.0, c = 0.0;
    __device__ __forceinline__ void add(double x) {
        const double t = s + x;
        if (fabs(s) >= fabs(x))
            c += (s - t) + x;
        else
            c += (x - t) + s;
        s = t;
    }
    __device__ __forceinline__ double value() const { return s + c; }
};

// ---------------------------------------------------------------------------
// two-pass reductions: per-block partials, then one block adds them in order
// ---------------------------------------------------------------------------
template <int NV>
__device__ void block_store(double (&v)[NV], double *partial) {
    __shared__ double red[32][NV];
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) red[warp][k] = v[k];
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? red[lane][k] : 0.0;
            for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
            if (lane == 0) partial[k * kMaxBlocks + blockIdx.x] = x;
        }
    }
}

// Sum of the per-block partials in a fixed order: block k adds value k, each
// thread a lane-strided compensated sum, then a shuffle tree per warp and the
// warps' totals in order (deterministic).
constexpr int kFinishThreads = 256;
template <int NV>
__global__ void __launch_bounds__(kFinishThreads) k_finish(const double *partial, int nblocks, double *result,
                                                           double offset0, Bp bp) {
    __shared__ double wsum[kFinishThreads / 32];
    const int k = blockIdx.x, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    partial = at(partial, bp.arena);
    result = at(result, bp.arena);
    KSum acc;
    for (int b = threadIdx.x; b < nblocks; b += kFinishThreads) acc.add(partial[k * kMaxBlocks + b]);
    double v = acc.value();
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) wsum[warp] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < kFinishThreads / 32; ++w) t += wsum[w];
        result[k] = t + (k == 0 ? offset0 : 0.0);
    }
}

__global__ void k_max_finish(const double *partial, int nblocks, double *result, Bp bp) {
    partial = at(partial, bp.arena);
    result = at(result, bp.arena);
    double m = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += 32) m = fmax(m, partial[b]);
    for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
    if (threadIdx.x == 0) result[0] = m;
}

template <int NV>
cudaError_t finish(Reduce r, int nblocks, double offset0, cudaStream_t st, const Bp &b = Bp{}) {
    k_finish<NV><<<dim3(NV, 1, b.P), kFinishThreads, 0, st>>>(r.partial, nblocks, r.result, offset0, b);
    return launched();
}

// ---------------------------------------------------------------------------
// slice kernels: shared-memory plan of one nbk x nbk slice + FFT scratch
// ---------------------------------------------------------------------------
template <int NBK>
struct SliceSmem {
    static constexpr int L = 2 * (NBK - 1);
    static constexpr int G = FftPlan<L>::G;
    static constexpr int NGRP = kSliceThreads / G;
    static constexpr size_t slice_bytes = (size_t)NBK * NBK * sizeof(double);
    static constexpr size_t scr_off = (slice_bytes + 15) & ~(size_t)15;
    static constexpr size_t tw_off = scr_off + (size_t)NGRP * padded_len(L) * sizeof(double2);
    // the full L-point twiddle table when it fits behind the slice and the
    // groups' FFT scratch, else the two-level table (2 KB)
    static constexpr bool smem_tw = tw_off + (size_t)L * sizeof(double2) <= 232448;
    static constexpr size_t bytes = tw_off + (smem_tw ? (size_t)L * sizeof(double2) : sizeof(TwoLevelTw));
    static_assert(bytes <= 232448, "slice does not fit in shared memory");
};

template <int NBK>
__device__ __forceinline__ double2 *slice_scratch(double *S) {
    return reinterpret_cast<double2 *>(reinterpret_cast<char *>(S) + SliceSmem<NBK>::scr_off);
}

// The L-point twiddles exp(-2 pi i m / L) staged in shared memory behind the
// FFT scratch -- the full table, or where that does not fit the two-level
// table (entry m = hi[m >> 6] lo[m & 63]); the first __syncthreads of the
// kernel publishes it.
template <int NBK>
__device__ __forceinline__ auto slice_twiddles(double *S, const double2 *__restrict__ tw) {
    constexpr int L = SliceSmem<NBK>::L;
    char *base = reinterpret_cast<char *>(S) + SliceSmem<NBK>::tw_off;
    if constexpr (SliceSmem<NBK>::smem_tw) {
        double2 *t = reinterpret_cast<double2 *>(base);
        for (int i = threadIdx.x; i < L; i += blockDim.x) t[i] = __ldg(&tw[i]);
        return (const double2 *)t;
    } else {
        TwoLevelTw *t = reinterpret_cast<TwoLevelTw *>(base);
        for (int i = threadIdx.x; i < 64; i += blockDim.x) {
            t->hi[i] = 64 * i < L ? __ldg(&tw[64 * i]) : make_double2(1.0, 0.0);
            t->lo[i] = i < L ? __ldg(&tw[i]) : make_double2(1.0, 0.0);
        }
        return (const TwoLevelTw *)t;
    }
}

// L2 prefetch by the CTA of [p, p + bytes), one request per 128-byte line,
// every address inside the range
// U (3 Usp + Uch) / 8 from the device pair Usc = (Usp, Uch), rounded as the
// host expression is (no contraction into an FMA)
__device__ __forceinline__ double vertex_fact(double U, const double *Usc) {
    return __dmul_rn(U, __dadd_rn(__dmul_rn(3.0, Usc[0]), Usc[1])) / 8.0;
}

// c[a] = cos(pi a t / N), a = 0..R, from c1 = cos(pi t / N) (tw64[t].x of the
// table tw64[m] = exp(-2 pi i m / 2N)) by the Chebyshev recurrence
// c[a + 1] = 2 c1 c[a] - c[a - 1]: one table read for all R + 1 cosines, a
// few ulp for R <= 4
template <int R>
__device__ __forceinline__ void cheb_cos(double c1, double (&c)[R + 1]) {
    c[0] = 1.0;
    if constexpr (R >= 1) c[1] = c1;
#pragma unroll
    for (int a = 2; a <= R; ++a) c[a] = fma(2.0 * c1, c[a - 1], -c[a - 2]);
}

__device__ __forceinline__ void prefetch_l2_range(const void *p, size_t bytes) {
    const char *c = static_cast<const char *>(p);
    for (size_t off = (size_t)threadIdx.x * 128; off < bytes; off += (size_t)blockDim.x * 128)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(c + off));
}
// L2 prefetch by the CTA of row j of a four-column-block array (NJ rows per
// block, nblk blocks): one 32-byte piece per block
__device__ __forceinline__ void prefetch_l2_blockrow(const double *a, int j, int NJ, int nblk) {
    for (int b = threadIdx.x; b < nblk; b += blockDim.x)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a + ((size_t)b * NJ + j) * 4));
}

// CTAs that one launch of `kernel` holds on the GPU at once: a slice kernel's
// CTA j prefetches the inputs of slice j + this, which the same launch reaches
// about one wave later
template <class K>
int resident_ctas(K kernel, int threads, size_t smem) {
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, smem) != cudaSuccess) return 0;
    return sms * per;
}

// Fill a symmetric NBK x NBK slice from the octant points: value(o) does all
// global reads of point o and returns its value.  Each thread takes KB points
// at a time and issues all their reads before storing any of them, so that
// KB memory round trips overlap instead of running one after the other.
template <int NBK, int KB = 8, class T, class Value>
__device__ __forceinline__ void fill_octant(T *S, int n8, const Value &value) {
    for (int base = threadIdx.x; base < n8; base += KB * blockDim.x) {
        T v[KB];
#pragma unroll
        for (int b = 0; b < KB; ++b) {
            const int o = base + b * blockDim.x;
            if (o < n8) v[b] = value(o);
        }
#pragma unroll
        for (int b = 0; b < KB; ++b) {
            const int o = base + b * blockDim.x;
            if (o < n8) {
                int l, m;
                oct_lm(o, l, m);
                S[l * NBK + m] = v[b];
                S[m * NBK + l] = v[b];
            }
        }
    }
}

// write octant value v of point (l, m) into both triangles of the slice
template <int NBK>
__device__ __forceinline__ void put_sym(double *S, int l, int m, double v) {
    S[l * NBK + m] = v;
    S[m * NBK + l] = v;
}

// ---------------------------------------------------------------------------
// tau kernels: clamped spline along a column, staging
// ---------------------------------------------------------------------------
// Clamped cubic spline through y[0..NJ) on a uniform grid of step h with end
// slopes d0, dN: on exit y holds the node second derivatives M_j.  Solves
//   2 M_0 + M_1 = 6/h ((V_1 - V_0)/h - d0)
//   M_{i-1} + 4 M_i + M_{i+1} = 6/h^2 (V_{i+1} - 2 V_i + V_{i-1})
//   M_{N-1} + 2 M_N = 6/h (dN - (V_N - V_{N-1})/h)
// -- the same interpolant as generique::spline_coeffs_rel
// (src/generique.cpp:214-322), S_j''' = 6 a_j = (M_{j+1} - M_j)/h -- by the
// Thomas algorithm with pivots invp = 1/p_i and multipliers cp_i (cp_N = 0)
// precomputed on the host.  The sweeps are split over TPC threads per column:
// each chunk starts its carry kWarm rows early from zero; the carry decays
// by 1/p_i <= 1/(2+sqrt3) per row, so the truncation error is below 1e-17 of
// the local magnitude.  All threads of the block must call.
// RAW: y already holds the right-hand side (the adjoint of the spline solves
// the same symmetric system); h, d0 and dN are not used.
template <int NC = 4, bool RAW = false>
__device__ void spline_second_derivatives(double *A, int lda, int NJ, double h, const double *d0, const double *dN,
                                          const double *__restrict__ invp, const double *__restrict__ cp) {
    const int TPC = blockDim.x / NC;
    const int c = threadIdx.x / TPC, k = threadIdx.x % TPC;
    double *y = A + c * lda;
    const int C = (NJ + TPC - 1) / TPC;
    const int s = min(k * C, NJ), e = min(s + C, NJ);
    const int N = NJ - 1;
    const double a6 = 6.0 / (h * h), b6 = 6.0 / h, ih = 1.0 / h;
    const double dl = RAW ? 0.0 : d0[c], dr = RAW ? 0.0 : dN[c];
    // interior rows kSplinePivotConst <= i < N share one pivot, 1/p = cp: a
    // register instead of a load in the sweeps' dependent chains
    const double cpiv = N > kSplinePivotConst ? __ldg(&invp[kSplinePivotConst]) : 0.0;
    auto piv = [&](int i) -> double { return (i >= kSplinePivotConst && i < N) ? cpiv : __ldg(&invp[i]); };
    auto sup = [&](int i) -> double { return (i >= kSplinePivotConst && i < N) ? cpiv : __ldg(&cp[i]); };
    auto rhs = [&](int i, double vm, double v0, double vp) -> double {
        if (RAW) return v0;
        if (i == 0) return b6 * ((vp - v0) * ih - dl);
        if (i == N) return b6 * (dr - (v0 - vm) * ih);
        return a6 * (vp - 2.0 * v0 + vm);
    };
    double carry = 0.0, vm_h = 0.0, vs_h = 0.0, ve_h = 0.0;
    if (s < e) {
        if (s > 0) {
            const int i0 = max(0, s - kWarm);
            double cc = 0.0;
            double vm = i0 > 0 ? y[i0 - 1] : 0.0, v0 = y[i0];
            for (int i = i0; i < s; ++i) {
                const double vp = y[i + 1];
                cc = (rhs(i, vm, v0, vp) - cc) * piv(i);
                vm = v0;
                v0 = vp;
            }
            carry = cc;
            vm_h = y[s - 1];
        }
        vs_h = y[s];
        ve_h = e < NJ ? y[e] : 0.0;
    }
    __syncthreads();
    if (s < e) {
        double vm = vm_h, v0 = vs_h;
        for (int i = s; i < e; ++i) {
            const double vp = (i + 1 < e) ? y[i + 1] : ve_h;
            const double dp = (rhs(i, vm, v0, vp) - carry) * piv(i);
            y[i] = dp;
            carry = dp;
            vm = v0;
            v0 = vp;
        }
    }
    __syncthreads();
    double mc = 0.0;
    if (s < e && e < NJ) {
        const int i1 = min(N, e - 1 + kWarm);
        double mm = 0.0;
        for (int i = i1; i >= e; --i) mm = y[i] - sup(i) * mm;
        mc = mm;
    }
    __syncthreads();
    if (s < e) {
        double mm = mc;
        for (int i = e - 1; i >= s; --i) {
            mm = y[i] - sup(i) * mm;
            y[i] = mm;
        }
    }
    __syncthreads();
}

// error-free sum of two doubles (Knuth's TwoSum): a + b = s + e exactly
__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
    s = a + b;
    const double bp = s - a;
    e = (a - (s - bp)) + (b - bp);
}

// per-column sum of y[i0..i1) over the TPC threads of each column -> out[c]:
// compensated per-thread sums, then a fixed shuffle tree that adds the pairs
// (sum, compensation) with TwoSum, then the column's warps in order.  TPC is
// a multiple of 32 (blockDim.x = 32 NC k).
template <int NC = 4>
__device__ void column_sums(const double *A, int lda, int i0, int i1, double *out) {
    const int TPC = blockDim.x / NC;
    const int c = threadIdx.x / TPC, k = threadIdx.x % TPC;
    KSum acc;
    for (int i = i0 + k; i < i1; i += TPC) acc.add(A[c * lda + i]);
    double s = acc.s, e = acc.c;
    for (int off = 16; off > 0; off >>= 1) {
        const double s2 = __shfl_down_sync(0xffffffffu, s, off);
        const double e2 = __shfl_down_sync(0xffffffffu, e, off);
        double t, r;
        two_sum(s, s2, t, r);
        s = t;
        e += e2 + r;
    }
    __shared__ double2 part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = make_double2(s, e);
    __syncthreads();
    if (k == 0) {
        const int w0 = threadIdx.x >> 5, nw = TPC >> 5;
        double S = part[w0].x, E = part[w0].y;
        for (int q = 1; q < nw; ++q) {
            double t, r;
            two_sum(S, part[w0 + q].x, t, r);
            S = t;
            E += part[w0 + q].y + r;
        }
        out[c] = S + E;
    }
    __syncthreads();
}

template <int N>
struct TauSmem {
    static constexpr int threads = (N / 16) > kTauThreads ? (N / 16) : kTauThreads;
    // four staged columns, the FFT scratch, then the two-level twiddle tables
    __host__ __device__ static size_t tables_off(int NJ) {
        return (((size_t)4 * NJ * sizeof(double) + 15) & ~(size_t)15) + (size_t)padded_len(N) * sizeof(double2);
    }
    __host__ __device__ static size_t bytes(int NJ) { return tables_off(NJ) + 2 * sizeof(TwoLevelTw); }
};

// Two-level tables (shared memory) of the N-point FFT twiddles tw[m] =
// exp(-2 pi i m/N) and of the pre-twiddles ht[m] = exp(+i pi m/N), m < N,
// from the global tables; entry m is hi[m >> 6] * lo[m & 63].  The caller's
// next barrier publishes them.
__device__ __forceinline__ void tau_tables(TwoLevelTw *tw2, TwoLevelTw *ht2, const double2 *__restrict__ tw,
                                           const double2 *__restrict__ ht, int N) {
    for (int t = threadIdx.x; t < 64; t += blockDim.x) {
        const double2 one = make_double2(1.0, 0.0);
        tw2->hi[t] = 64 * t < N ? __ldg(&tw[64 * t]) : one;
        tw2->lo[t] = t < N ? __ldg(&tw[t]) : one;
        ht2->hi[t] = 64 * t < N ? __ldg(&ht[64 * t]) : one;
        ht2->lo[t] = t < N ? __ldg(&ht[t]) : one;
    }
}
__device__ __forceinline__ double2 tw_at(const TwoLevelTw *t, int m) { return cmul(t->hi[m >> 6], t->lo[m & 63]); }

// Asynchronous 8-byte global -> shared copy (cp.async); the issuing thread
// waits for its own copies with cp_async_wait_all, a barrier then publishes
// them.  A thread keeps all its copies in flight at once, which is what
// streams a column block in at HBM speed with one CTA per SM.
__device__ __forceinline__ void cp_async8(double *smem, const double *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// ---------------------------------------------------------------------------
// input staging of the slice kernels whose inputs are rows of global arrays:
// the slice and the FFT scratch are idle until the fill, so a CTA first copies
// its input rows there with asynchronous copies (all in flight at once: one
// memory latency per slice instead of one per batch of loads), waits for its
// own copies, and forms the slice from shared memory
// ---------------------------------------------------------------------------
template <int NBK>
struct StageRows {
    static constexpr int N8 = NBK * (NBK + 1) / 2;
    static constexpr int N8P = (N8 + 3) & ~3;
    static constexpr size_t blockrow_bytes = (size_t)N8P * sizeof(double);  // one row of a column-block array
    static constexpr size_t drow_bytes = ((size_t)N8 * sizeof(double) + 15) & ~(size_t)15;  // one FP64 row
};

__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// row j of a column-block array a (NJ rows) -> dst[o], o < N8P (16-byte copies)
template <int NBK>
__device__ __forceinline__ void stage_blockrow(double *dst, const double *__restrict__ a, int j, int NJ) {
    for (int i = threadIdx.x; i < StageRows<NBK>::N8P / 2; i += blockDim.x) {
        const int b = i >> 1, h = i & 1;
        cp_async16(dst + 4 * b + 2 * h, a + ((size_t)b * NJ + j) * 4 + 2 * h);
    }
}
// n8 doubles from src -> dst (8-byte copies: rows of an [j][o] array are
// 16-byte aligned only for even j)
template <int NBK>
__device__ __forceinline__ void stage_drow(double *dst, const double *__restrict__ src) {
    for (int o = threadIdx.x; o < StageRows<NBK>::N8; o += blockDim.x) cp_async8(dst + o, src + o);
}
// Form the symmetric slice from value(o), which reads the staged inputs:
// every thread computes its octant points into registers, then a barrier (the
// staging area overlaps the slice), then the writes of both triangles.
// THREADS: the block size the kernel is launched with.
template <int NBK, int THREADS, class T, class Value>
__device__ __forceinline__ void fill_from_staged(T *S, const Value &value) {
    constexpr int N8 = StageRows<NBK>::N8, PER = (N8 + THREADS - 1) / THREADS;
    T v[PER];
#pragma unroll
    for (int b = 0; b < PER; ++b) {
        const int o = threadIdx.x + b * THREADS;
        if (o < N8) v[b] = value(o);
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < PER; ++b) {
        const int o = threadIdx.x + b * THREADS;
        if (o < N8) {
            int l, m;
            oct_lm(o, l, m);
            S[l * NBK + m] = v[b];
            S[m * NBK + l] = v[b];
        }
    }
}


// Load one column block into shared memory, column-major (the caller's next
// __syncthreads publishes it).  Padding columns (octant index >= n8, present
// because N8 is rounded up to a multiple of 4) load as zeros: they share
// packed FFTs with real columns, so stale values there would leak into real
// outputs through rounding.
__device__ __forceinline__ void stage_in(double *A, const double *g, int NJ, int nvalid) {
    for (int i = threadIdx.x; i < 4 * NJ; i += blockDim.x) {
        double *dst = &A[(i & 3) * NJ + (i >> 2)];
        if ((i & 3) < nvalid)
            cp_async8(dst, g + i);
        else
            *dst = 0.0;
    }
    cp_async_wait_all();
}
__device__ __forceinline__ void stage_out(const double *A, double *g, int NJ) {
    for (int i = threadIdx.x; i < 4 * NJ; i += blockDim.x) g[i] = A[(i & 3) * NJ + (i >> 2)];
}

// full Sigma(k, i w_n) = Sinf/z + C2/z^2 + C3/z^3 + S/z^4, z = i w_n, from the
// reciprocal powers of w_n
__device__ __forceinline__ void sigma_full(double i1, double sinf, double c2, double c3, double2 Sv, double &rS,
                                           double &iS) {
    const double i2 = i1 * i1, i4 = i2 * i2;
    rS = -c2 * i2 + Sv.x * i4;
    iS = -sinf * i1 + c3 * i2 * i1 + Sv.y * i4;
}

// 32-byte streaming load (two 16-byte evict-first loads)
__device__ __forceinline__ double4 ld_stream4(const double4 *p) {
    const double2 *q = reinterpret_cast<const double2 *>(p);
    const double2 a = __ldcs(q), b = __ldcs(q + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// one term of Tr(G - G0) (green::traceDiffG, src/green.cpp:3108-3182) and its
// derivative with respect to the chemical potential pmu: w Re[G - G0] with
// G = 1/(i w_n - e + pmu - Sigma), G0 = 1/(i w_n - e + mu0)
__device__ __forceinline__ void trdiff_term(double wn, double rS, double iS, double e, double mu0, double pmu,
                                            double w, double &v, double &dv) {
    const double a = e - pmu + rS, d = e - mu0, g = mu0 - pmu + rS;
    const double A2 = (wn - iS) * (wn - iS) + a * a;
    const double num = g * a * d + iS * (iS - 2 * wn) * d - wn * wn * g;
    const double inv = w / (A2 * (wn * wn + d * d));
    v += inv * num;
    dv += inv * (wn * wn - (a + g) * d + num * 2.0 * a / A2);
}
// the same with the second derivative: d2/dpmu2 w Re G = 2 w Re G^3, and
// with z = x + i y (x = -a, y = w_n - Im Sigma), Re conj(z)^3 = x^3 - 3 x y^2
__device__ __forceinline__ void trdiff_term(double wn, double rS, double iS, double e, double mu0, double pmu,
                                            double w, double &v, double &dv, double &d2v) {
    trdiff_term(wn, rS, iS, e, mu0, pmu, w, v, dv);
    const double x = pmu - e - rS, y = wn - iS, r = 1.0 / (x * x + y * y);
    d2v += 2.0 * w * x * (x * x - 3.0 * y * y) * (r * r * r);
}

// complex division
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    // Smith's algorithm
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        const double r = b.x / b.y, d = b.y + b.x * r;
        return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}

// ---------------------------------------------------------------------------
// helpers of the current-current correlator kernels (tpsc_cond.cu, tpsc_al.cu)
// ---------------------------------------------------------------------------
// two-column-block layout of the h V and f0 V tau arrays: element (j, c)
__host__ __device__ __forceinline__ size_t bidx2(int j, int c, int NJ) {
    return ((size_t)(c >> 1) * NJ + j) * 2 + (c & 1);
}

// octant index of lattice point (x, y), 0 <= x, y < nbk
__device__ __forceinline__ int oct_index(int x, int y) {
    const int a = max(x, y), b = min(x, y);
    return b + a * (a + 1) / 2;
}

__device__ __forceinline__ double2 cexp2(double2 z) {
    const double ea = exp(z.x);
    if (z.y == 0.0) return make_double2(ea, 0.0);
    double s, c;
    sincos(z.y, &s, &c);
    return make_double2(ea * c, ea * s);
}

__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// block-wide sum of NV values per thread -> out[0..NV) (all threads must call;
// out visible to every thread on return)
template <int NV>
__device__ void block_sum(double (&v)[NV], double *out) {
    __shared__ double red[32][NV];
#pragma unroll
    for (int k = 0; k < NV; ++k)
        for (int off = 16; off > 0; off >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) red[warp][k] = v[k];
    __syncthreads();
    if (threadIdx.x < NV) {
        const int nw = (blockDim.x + 31) >> 5;
        double s = 0.0;
        for (int w = 0; w < nw; ++w) s += red[w][threadIdx.x];
        out[threadIdx.x] = s;
    }
    __syncthreads();
}

// split of a packed FFT of two real sequences at bins n and N - n
__device__ __forceinline__ void split_real(double2 Z, double2 Zc, double2 &Fa, double2 &Fb) {
    Fa = make_double2(0.5 * (Z.x + Zc.x), 0.5 * (Z.y - Zc.y));
    Fb = make_double2(0.5 * (Z.y + Zc.y), -0.5 * (Z.x - Zc.x));
}

// Stage the two columns of pair p (contiguous in the two-column-block layout)
// column-major into R; a padding column loads zeros.
__device__ __forceinline__ void stage_pair(double *R, const double *g, int NJ, bool two) {
    for (int i = threadIdx.x; i < 2 * NJ; i += blockDim.x) {
        double *dst = &R[(i & 1) * NJ + (i >> 1)];
        if ((i & 1) && !two)
            *dst = 0.0;
        else
            cp_async8(dst, g + i);
    }
    cp_async_wait_all();
}

// ---------------------------------------------------------------------------
// dispatch over the compiled sizes
// ---------------------------------------------------------------------------
template <template <int> class F, typename... Args>
cudaError_t dispatch_nbk(int nbk, Args... args) {
    switch (nbk) {
        case 5: return F<5>::run(args...);
        case 9: return F<9>::run(args...);
        case 17: return F<17>::run(args...);
        case 33: return F<33>::run(args...);
        case 65: return F<65>::run(args...);
        case 129: return F<129>::run(args...);
        default: return cudaErrorInvalidValue;
    }
}
template <template <int> class F, typename... Args>
cudaError_t dispatch_nw(int nw0, Args... args) {
    switch (nw0) {
        case 16: return F<16>::run(args...);
        case 32: return F<32>::run(args...);
        case 64: return F<64>::run(args...);
        case 128: return F<128>::run(args...);
        case 256: return F<256>::run(args...);
        case 512: return F<512>::run(args...);
        case 1024: return F<1024>::run(args...);
        case 2048: return F<2048>::run(args...);
        case 4096: return F<4096>::run(args...);
        default: return cudaErrorInvalidValue;
    }
}

template <typename K>
cudaError_t set_smem(K kernel, size_t bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return smem_optin((const void *)kernel);
}

}  // namespace
}  // namespace tpsc
