// tpsc_tcdct.cu -- the "tensor" slice plan: the folded matrix DCT-I of the
// mixed form's Sigma slice (tpsc_dct.cuh) with both matrix products on the
// tcgen05 tensor cores, 3xTF32 (each FP32 operand split into a TF32 high part
// and its remainder; hi*hi + hi*lo + lo*hi accumulated in FP32 in tensor
// memory).  Lattice 256 x 256 (nbk = 129, H = 64).
//
// One slice at a time per CTA (persistent, one CTA per SM, 384 threads):
//   1. the V(r, tau_j) block row by TMA (a 4-D tensor map over this GPU's
//      V), the FP32 G(r, tau_j) row by one bulk copy, both on an mbarrier;
//   2. x = G V in FP64: the near field |rx|, |ry| <= 4 kept in FP64, the rest rounded to FP32;
//   3. fold x into SS, SD, DD (tpsc_dct.cuh) as K-major hi/lo TF32 operands;
//   4. T = K . fold^T on the tensor cores (M = 64 output rows of the DCT
//      tables Ks, Kd; N = the fold's rows; K = its columns);
//   5. T from tensor memory into the second products' operands (hi/lo);
//   6. Z = K . T^T on the tensor cores; Z from tensor memory into shared memory
//      in octant order; the next slice's inputs are staged from here on;
//   7. Sigma(k, tau_j) = Z + the near field's FP64 transform, to HBM.
// Row and column H = 64 of the blocks, which the M = 64 products leave out,
// are alternating sums (Ks[H][k] = w_k (-1)^k) formed on the CUDA cores while
// the tensor cores run.  Every mbarrier wait is bounded: a wait that runs
// out sets the error word, the CTA waits (bounded) once more, frees its
// tensor memory and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <math.h>
#include <stdint.h>

#include <cstring>
#include <mutex>
#include <vector>

#include "tpsc_dct.cuh"
#include "tpsc_tc.cuh"

namespace tpsc {

// the A-operand tables of the tensor plan for H = 64 (host side): Ks rows
// n < 64 (K = 72, k > 64 zero) and Kd (64 x 64) as K-major TF32 hi / lo
// pairs, then Ks[64][k] = w_k (-1)^k (72 floats); 69,920 bytes
void dct_tc_table(int nbk, std::vector<float> &out) {
    out.clear();
    if (nbk != 129) return;
    constexpr int H = 64, N = 128, KS = 72;
    const long double pi = 3.141592653589793238462643383279502884L;
    out.assign((2 * 64 * KS + 2 * 64 * 64 + KS), 0.0f);
    auto rna = [](float x) {
        uint32_t b;
        memcpy(&b, &x, 4);
        b = (b + 0x1000u) & ~0x1FFFu;
        float y;
        memcpy(&y, &b, 4);
        return y;
    };
    auto put = [&](size_t base_hi, size_t base_lo, int r, int k, int R, long double v) {
        const float hi = rna((float)v);
        const float lo = (float)(v - (long double)hi);
        out[base_hi + kmaj_off(r, k, R) / 4] = hi;
        out[base_lo + kmaj_off(r, k, R) / 4] = lo;
    };
    const size_t ks_hi = 0, ks_lo = 64 * KS, kd_hi = 2 * 64 * KS, kd_lo = kd_hi + 64 * 64, k64 = kd_lo + 64 * 64;
    for (int n = 0; n < 64; ++n)
        for (int k = 0; k <= H; ++k)
            put(ks_hi, ks_lo, n, k, 64, (k == 0 ? 1.0L : 2.0L) * cosl(pi * ((k * n) % (2 * H)) / H));
    for (int n = 0; n < 64; ++n)
        for (int k = 0; k < H; ++k)
            put(kd_hi, kd_lo, n, k, 64, (k == 0 ? 1.0L : 2.0L) * cosl(pi * ((k * (2 * n + 1)) % (2 * N)) / N));
    for (int k = 0; k <= H; ++k) out[k64 + k] = (k == 0 ? 1.0f : 2.0f) * ((k & 1) ? -1.0f : 1.0f);
}

namespace {

__device__ unsigned g_tc_err;  // set by a wait that ran out (never cleared by the kernel)

template <class T>
__device__ __forceinline__ T *tc_point(T *ptr, long long arena, int p) {
    using Ch = typename std::conditional<std::is_const<T>::value, const char, char>::type;
    return reinterpret_cast<T *>(reinterpret_cast<Ch *>(ptr) + (long long)p * arena);
}

// shared memory of k_sigma_slice_tc (bytes)
struct TcSmem {
    static constexpr int N8 = 8385, N8P = 8388, NBK = 129, KS = 72;
    // A tables: Ks hi | Ks lo (64 x 72) | Kd hi | Kd lo (64 x 64) | Ks row 64
    static constexpr uint32_t ks_hi = 0, ks_lo = 64 * KS * 4, kd_hi = 2 * 64 * KS * 4, kd_lo = kd_hi + 64 * 64 * 4;
    static constexpr uint32_t k64 = kd_lo + 64 * 64 * 4;  // 72 floats
    static constexpr uint32_t tab_bytes = k64 + KS * 4;   // 69,920
    // B operands, hi | lo each.  First products: SS (72 rows x K 72) and
    // [SD; DD] (72 + 64 rows x K 64, one MMA for both, A = Kd).  Second
    // products: [T_ee^T; T_eo^T] (72 + 64 rows x K 72, one MMA, A = Ks) and
    // T_oo^T (64 x 64).  Both stages span the same 111,104 bytes.
    static constexpr uint32_t b0 = tab_bytes;
    static constexpr uint32_t ss_hi = b0, ss_lo = ss_hi + 72 * 72 * 4;
    static constexpr uint32_t sddd_hi = ss_lo + 72 * 72 * 4, sddd_lo = sddd_hi + 136 * 64 * 4;
    static constexpr uint32_t b_end = sddd_lo + 136 * 64 * 4;  // b0 + 111,104
    static constexpr uint32_t t_hi = b0, t_lo = t_hi + 136 * 72 * 4;
    static constexpr uint32_t too_hi = t_lo + 136 * 72 * 4, too_lo = too_hi + 64 * 64 * 4;
    static_assert(too_lo + 64 * 64 * 4 == b_end, "both stages' operands span the same bytes");
    static constexpr uint32_t xs = b_end;                    // N8 floats
    static constexpr uint32_t xn = xs + ((N8 * 4 + 15) & ~15);
    static constexpr uint32_t u = xn + 16 * 8;
    static constexpr int R = 4, NOCT = 15;
    static constexpr uint32_t zx = u + (R + 1) * NBK * 8;  // 129 floats: rows 64 of Z_ee, Z_eo
    static constexpr uint32_t t64 = zx + 132 * 4;          // 72 floats: column 64 of T_ee
    static constexpr uint32_t bar = t64 + 72 * 4;           // mbarrier (8-byte aligned)
    static constexpr uint32_t misc = bar + 8;               // tensor-memory base, error flag
    static constexpr uint32_t cf = misc + 16;               // 2 cos(pi a l / N), a = 1..R, l < NBK (doubles)
    static constexpr uint32_t tbar = cf + R * NBK * 8;      // mbarrier of the input copies
    static constexpr uint32_t bytes = tbar + 8;
    // the raw inputs over the B operands: the V block row as 9 TMA boxes of
    // 256 four-double blocks (the last one partly beyond the row, filled with
    // zeros), then the FP32 G row as one bulk copy of its 16-byte-aligned cover
    static constexpr int VBOX = 256, NVBOX = (N8P / 4 + VBOX - 1) / VBOX;
    static constexpr uint32_t vst = (b0 + 127) & ~127u;
    static constexpr uint32_t gst = vst + NVBOX * VBOX * 32;
    static constexpr uint32_t gmax = ((N8 * 4 + 15) & ~15) + 16;  // the cover of a row: at most 12 bytes each side
    static_assert(gst + gmax <= b_end, "raw inputs fit over the B operands");
    static_assert(vst + 2 * gmax <= b_end && gmax % 16 == 0, "two G rows fit over the B operands");
    static_assert(tbar % 8 == 0, "mbarrier alignment");
    static_assert(bar % 8 == 0, "mbarrier alignment");
    static_assert(DctPlan<64>::REG * 4 <= b_end - b0, "Z fits over the B operands");
};

constexpr int kTcThreads = 384;
constexpr uint32_t kTmemCols = 256;
constexpr uint64_t kWaitNs = 2000000000ull;  // 2 s: the products of one slice take microseconds

// The butterfly at position (r, k) of the three blocks at once, from the
// octant values xs: with A = X(r, k), B = X(N-r, k), C = X(r, N-k),
// D = X(N-r, N-k),
//   SS = A + B + C + D,  SD = (A - C) + (B - D),  DD = (A - C) - (B - D),
// row or column H taking its point once (s_H = x_H, no d_H); positions
// beyond the blocks are the operands' zero padding.
__device__ __forceinline__ void fold_at(const float *__restrict__ xs, int r, int k, float &ss, float &sd, float &dd) {
    constexpr int H = 64, N = 128;
    auto X = [&](int p, int q) -> float {
        const int l = p > q ? p : q, m = p > q ? q : p;
        return xs[l * (l + 1) / 2 + m];
    };
    ss = sd = dd = 0.0f;
    if (r > H || k > H) return;
    const float a = X(r, k);
    if (r < H && k < H) {
        const float bq = X(N - r, k), c = X(r, N - k), d = X(N - r, N - k);
        ss = (a + bq) + (c + d);
        sd = (a - c) + (bq - d);
        dd = (a - c) - (bq - d);
    } else if (r < H) {  // k = H
        ss = a + X(N - r, k);
    } else if (k < H) {  // r = H
        const float c = X(r, N - k);
        ss = a + c;
        sd = a - c;
    } else {
        ss = a;
    }
}

// The MMAs of one block: D (tensor-memory column COL) = A B^T over KSTEPS
// steps of K = 8, 3xTF32 (the two cross terms first, then hi * hi); A is a
// table of 64 rows, B has BROWS rows (= N).  Fully unrolled: every
// descriptor is the base descriptor plus a constant start-address offset.
template <uint32_t A_HI, uint32_t A_LO, uint32_t B_HI, uint32_t B_LO, int BROWS, int KSTEPS, int COL>
__device__ __forceinline__ void issue_block(uint64_t dbase_a, uint64_t dbase_b, uint32_t tmem) {
    constexpr uint32_t a_lbo = 64 * 16, b_lbo = BROWS * 16;
    constexpr uint32_t id = idesc_tf32(64, BROWS);
    const uint64_t a0 = dbase_a | ((uint64_t)(a_lbo >> 4) << 16), b0 = dbase_b | ((uint64_t)(b_lbo >> 4) << 16);
#pragma unroll
    for (int pass = 0; pass < 3; ++pass) {
        const uint32_t a = pass == 1 ? A_LO : A_HI;
        const uint32_t bb = pass == 0 ? B_LO : B_HI;
#pragma unroll
        for (int s = 0; s < KSTEPS; ++s)
            mma_tf32(tmem + COL, a0 + ((a + 2 * a_lbo * s) >> 4), b0 + ((bb + 2 * b_lbo * s) >> 4), id,
                     (pass | s) != 0);
    }
}

// the first products (T = K . fold^T) or the second (Z = K . T^T); sdesc: the
// descriptor of shared-memory offset 0 (start address field only, SBO 128)
template <bool SECOND>
__device__ __forceinline__ void issue_stage(uint64_t sdesc, uint32_t tmem) {
    using S = TcSmem;
    if constexpr (SECOND) {
        // Z_ee and Z_eo in one MMA chain (columns 0..71 and 72..135), Z_oo (136..199)
        issue_block<S::ks_hi, S::ks_lo, S::t_hi, S::t_lo, 136, 9, 0>(sdesc, sdesc, tmem);
        issue_block<S::kd_hi, S::kd_lo, S::too_hi, S::too_lo, 64, 8, 136>(sdesc, sdesc, tmem);
    } else {
        // T_ee (columns 0..71), then T_eo and T_oo in one MMA chain (72..143 and 144..207)
        issue_block<S::ks_hi, S::ks_lo, S::ss_hi, S::ss_lo, 72, 9, 0>(sdesc, sdesc, tmem);
        issue_block<S::kd_hi, S::kd_lo, S::sddd_hi, S::sddd_lo, 136, 8, 72>(sdesc, sdesc, tmem);
    }
}

// the 16-byte-aligned cover of the FP32 G row j of point p: its start and
// bytes, and the row's offset in floats inside it
struct GCover {
    const unsigned char *src;
    uint32_t bytes;
    int shift;
};
__device__ __forceinline__ GCover g_cover(const float *__restrict__ Grt, int p, int j, long long arena) {
    using S = TcSmem;
    const uintptr_t a = reinterpret_cast<uintptr_t>(tc_point(Grt, arena, p) + (size_t)j * S::N8);
    const uintptr_t a0 = a & ~(uintptr_t)15, a1 = (a + S::N8 * 4 + 15) & ~(uintptr_t)15;
    return GCover{reinterpret_cast<const unsigned char *>(a0), (uint32_t)(a1 - a0), (int)((a - a0) >> 2)};
}
// the kinds of slice the tensor plan transforms (kSliceVertex, kSliceSigma) and
// their arguments (the pointers are point 0's; a batched launch adds
// p * arena for point p)
struct TcArgs {
    const float *Grt = nullptr;     // Sigma: G(r, tau) in FP32, [j][o]
    const double *Usc = nullptr;    // V: the device pair (Usp, Uch)
    const double2 *tw64 = nullptr;  // Sigma: exp(-2 pi i m / 2N), m < 2N
    double *out = nullptr;          // Sigma: Sigma(k, tau); V: V(r, tau) (column blocks)
    double normFact = 0.0, U = 0.0;
    int nw0 = 0;
};
template <int KIND>
__host__ __device__ constexpr int tc_slices(int nw0) {
    static_assert(KIND == kSliceSigma || KIND == kSliceVertex, "the tensor plan's slice kinds");
    return KIND == kSliceSigma ? nw0 + 1 : nw0 / 2 + 1;
}
// (one thread) the raw inputs of slice j of point p into shared memory, on tbar:
//   Sigma: the V(r, tau_jv) block row by TMA and the G(r, tau_j) row by one bulk copy;
//   V:     the chi0(q, iq_j) block row by TMA.
template <int KIND>
__device__ __forceinline__ void tc_stage(unsigned char *smem, const void *tmIn, const TcArgs &a, int p, int j,
                                         long long arena) {
    using S = TcSmem;
    const int nb = a.nw0 / 2 + 1;
    uint64_t *tbar = reinterpret_cast<uint64_t *>(smem + S::tbar);
    fence_async_smem();
    if constexpr (KIND == kSliceSigma) {
        const int jv = j < nb ? j : a.nw0 - j;
        const GCover gc = g_cover(a.Grt, p, j, arena);
        mbar_expect_tx(tbar, (uint32_t)(S::NVBOX * S::VBOX * 32) + gc.bytes);
#pragma unroll 1
        for (int c = 0; c < S::NVBOX; ++c)
            tma_load_4d(smem + S::vst + c * S::VBOX * 32, tmIn, 0, jv, c * S::VBOX, p, tbar);
        bulk_load(smem + S::gst, gc.src, gc.bytes, tbar);
    } else if constexpr (KIND == kSliceVertex) {
        mbar_expect_tx(tbar, (uint32_t)(S::NVBOX * S::VBOX * 32));
#pragma unroll 1
        for (int c = 0; c < S::NVBOX; ++c)
            tma_load_4d(smem + S::vst + c * S::VBOX * 32, tmIn, 0, j, c * S::VBOX, p, tbar);
    }
}

__device__ __forceinline__ int oct_of(int l, int m) { return l * (l + 1) / 2 + m; }

// point p's scalar `slot` of a batched launch, or v for a plain launch
__device__ __forceinline__ double tc_par(const Bp &b, int slot, double v, int p) {
    return b.pp ? tc_point(b.pp, b.arena, p)[slot] : v;
}

template <int KIND>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_slice_tc(const __grid_constant__ CUtensorMap tmIn, const float *__restrict__ tab, const TcArgs a, Bp b) {
    using S = TcSmem;
    constexpr int H = 64, N8 = S::N8, NBK = S::NBK, L = 256, R = S::R, NOCT = S::NOCT;
    constexpr int PER = (N8 + kTcThreads - 1) / kTcThreads;
    extern __shared__ __align__(1024) unsigned char smem[];
    const uint32_t sbase = smem_u32(smem);
    const uint64_t sdesc0 = smem_desc(sbase, 0, 128);
    float *xs = reinterpret_cast<float *>(smem + S::xs);  // the slice's octant values, later its transform
    double *xn = reinterpret_cast<double *>(smem + S::xn);
    double *u = reinterpret_cast<double *>(smem + S::u);
    float *zx = reinterpret_cast<float *>(smem + S::zx);
    float *t64 = reinterpret_cast<float *>(smem + S::t64);
    const float *k64 = reinterpret_cast<const float *>(smem + S::k64);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + S::bar);
    uint64_t *tbar = reinterpret_cast<uint64_t *>(smem + S::tbar);
    uint32_t *s_tmem = reinterpret_cast<uint32_t *>(smem + S::misc);
    volatile uint32_t *s_err = reinterpret_cast<volatile uint32_t *>(smem + S::misc + 4);
    double *cf = reinterpret_cast<double *>(smem + S::cf);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    if (warp == 0) {
        tmem_alloc(s_tmem, kTmemCols);
        tmem_relinquish();
    }
    if (tid == 0) {
        mbar_init(bar, 1);
        mbar_init(tbar, 1);
        *s_err = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < (int)(S::tab_bytes / 16); i += blockDim.x)
        cp_async16(smem + 16 * i, reinterpret_cast<const unsigned char *>(tab) + 16 * i);
    if constexpr (KIND == kSliceSigma)
        for (int i = tid; i < R * NBK; i += blockDim.x)
            cf[i] = 2.0 * __ldg(&a.tw64[((i / NBK + 1) * (i % NBK)) % L]).x;
    cp_async_wait_all();
    const int nw0 = a.nw0, nb = nw0 / 2 + 1, ns = tc_slices<KIND>(nw0);
    const long long items = (long long)ns * b.P;
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (tid == 0 && blockIdx.x < items)
        tc_stage<KIND>(smem, &tmIn, a, (int)(blockIdx.x / ns), (int)(blockIdx.x % ns), b.arena);
    const uint32_t tmem = *s_tmem;
    uint32_t phase = 0, tphase = 0;

    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int p = (int)(it / ns), j = (int)(it % ns);
        const long long nx = it + gridDim.x;
        __syncthreads();  // the previous slice's reads of xs are done
        // 1. this slice's raw inputs (copied in during the previous slice's output)
        if (!mbar_wait(tbar, tphase, kWaitNs)) *s_err = 1;
        __syncthreads();
        if (*s_err) break;
        tphase ^= 1;
        if (KIND == kSliceSigma && nx < items) {
            const int pn = (int)(nx / ns), jn = (int)(nx % ns);
            prefetch_l2_range(tc_point(a.Grt, b.arena, pn) + (size_t)jn * N8, (size_t)N8 * sizeof(float));
        }
        // 2. the slice's octant values, formed in FP64 and rounded once
        if constexpr (KIND == kSliceSigma) {
            // x = G V; the near field stays in FP64
            const double *vs = reinterpret_cast<const double *>(smem + S::vst);
            const float *gs = reinterpret_cast<const float *>(smem + S::gst) + g_cover(a.Grt, p, j, b.arena).shift;
#pragma unroll
            for (int i = 0; i < PER; ++i) {
                const int o = tid + i * kTcThreads;
                if (o < N8) {
                    const double x = (double)gs[o] * vs[o];
                    if (o < NOCT) xn[o] = x;
                    xs[o] = o < NOCT ? 0.0f : (float)x;
                }
            }
        } else if constexpr (KIND == kSliceVertex) {
            // V(q, iq_j) from chi0(q, iq_j): with a = Usp/2, b = Uch/2 one division per point
            const double *cs = reinterpret_cast<const double *>(smem + S::vst);
            const double *us = tc_point(a.Usc, b.arena, p);
            const double Usp = us[0], Uch = us[1];
            const double nf = tc_par(b, kPpNormFact, a.normFact, p), Up = tc_par(b, kPpU, a.U, p);
#pragma unroll
            for (int i = 0; i < PER; ++i) {
                const int o = tid + i * kTcThreads;
                if (o < N8) {
                    const double c0 = cs[o];
                    const double as = 0.5 * Usp, bc = 0.5 * Uch;
                    const double ds = 1.0 - as * c0, dc = 1.0 + bc * c0;
                    const double num = 3.0 * Usp * as * dc - Uch * bc * ds;
                    xs[o] = (float)(0.125 * nf * Up * c0 * c0 * num / (ds * dc));
                }
            }
        }
        __syncthreads();
        // 3. the fold as K-major hi/lo operands, 8 rows x 4 columns per warp pass
#pragma unroll 2
        for (int un = warp; un < 9 * 18; un += kTcThreads / 32) {
            const int r = 8 * (un / 18) + (lane >> 2), k = 4 * (un % 18) + (lane & 3);
            float v[3];
            fold_at(xs, r, k, v[0], v[1], v[2]);
            const uint32_t off72 = kmaj_off(r, k, 72);
            float h = tf32_hi(v[0]);
            *reinterpret_cast<float *>(smem + S::ss_hi + off72) = h;
            *reinterpret_cast<float *>(smem + S::ss_lo + off72) = v[0] - h;
            if (k < 64) {
                const uint32_t offsd = kmaj_off(r, k, 136);
                h = tf32_hi(v[1]);
                *reinterpret_cast<float *>(smem + S::sddd_hi + offsd) = h;
                *reinterpret_cast<float *>(smem + S::sddd_lo + offsd) = v[1] - h;
                if (r < 64) {
                    const uint32_t offdd = kmaj_off(72 + r, k, 136);
                    h = tf32_hi(v[2]);
                    *reinterpret_cast<float *>(smem + S::sddd_hi + offdd) = h;
                    *reinterpret_cast<float *>(smem + S::sddd_lo + offdd) = v[2] - h;
                }
            }
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        // 4. first products
        if (tid == 0) {
            tc_fence_after();
            issue_stage<false>(sdesc0, tmem);
            mma_commit(bar);
        }
        // (while the tensor cores run) near field of the Sigma slice:
        // u_r(k2) = sum_c w_c x(r, c) cos(pi c k2 / N)
        if constexpr (KIND == kSliceSigma)
            for (int i = tid; i < (R + 1) * NBK; i += blockDim.x) {
                const int r = i / NBK, k2 = i % NBK;
                double cs[R + 1];
                cheb_cos<R>(__ldg(&a.tw64[k2]).x, cs);
                double acc = 0.0;
#pragma unroll
                for (int c = 0; c <= R; ++c) {
                    const int hi = r > c ? r : c, lo = r > c ? c : r;
                    acc = fma((c == 0 ? 1.0 : 2.0) * xn[lo + hi * (hi + 1) / 2], cs[c], acc);
                }
                u[i] = acc;
            }
        // column 64 of T_ee: t64[m] = sum_{k<=64} SS[m][k] Ks[64][k], m <= 64;
        // four threads per m (warps 2..10), k = sub, sub + 4, ...
        if (warp >= 2 && warp <= 10) {
            const int i = tid - 64, m = i >> 2, sub = i & 3;
            float acc = 0.0f;
            if (m <= H)
                for (int k = sub; k <= H; k += 4) {
                    const uint32_t off = kmaj_off(m, k, 72);
                    const float sv = *reinterpret_cast<const float *>(smem + S::ss_hi + off) +
                                     *reinterpret_cast<const float *>(smem + S::ss_lo + off);
                    acc = fmaf(sv, k64[k], acc);
                }
            acc += __shfl_xor_sync(0xffffffffu, acc, 1);
            acc += __shfl_xor_sync(0xffffffffu, acc, 2);
            if (sub == 0 && m <= H) t64[m] = acc;
        }
        if (!mbar_wait(bar, phase, kWaitNs)) *s_err = 1;
        tc_fence_after();
        __syncthreads();
        if (*s_err) break;
        phase ^= 1;
        // 5. T from tensor memory into the second products' B operands:
        // rows n of [T_ee^T; T_eo^T] (row n: T_ee[.][n], n < 64 from the
        // accumulator, row 64 = t64; row 72 + n: T_eo[.][n]) and of T_oo^T
        {
            const int q = warp & 3, blk = warp >> 2;
            const int n = 16 * q + (lane & 15) + (blk == 1 ? 72 : 0);
            const int col0 = blk == 0 ? 0 : (blk == 1 ? 72 : 144);
            const int ncol = blk == 2 ? 64 : 72;
            const uint32_t hi_off = blk == 2 ? S::too_hi : S::t_hi;
            const uint32_t lo_off = blk == 2 ? S::too_lo : S::t_lo;
            const int R2 = blk == 2 ? 64 : 136;
            uint32_t rr[72];
            tmem_ld_row72(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)col0, rr, ncol == 72);
            if (lane < 16) {
#pragma unroll
                for (int c = 0; c < 72; c += 4) {
                    if (c < ncol) {
                        float4 hv, lv;
                        float *hp = &hv.x, *lp = &lv.x;
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float v = __uint_as_float(rr[c + e]);
                            hp[e] = tf32_hi(v);
                            lp[e] = v - hp[e];
                        }
                        const uint32_t off = kmaj_off(n, c, R2);
                        *reinterpret_cast<float4 *>(smem + hi_off + off) = hv;
                        *reinterpret_cast<float4 *>(smem + lo_off + off) = lv;
                    }
                }
            }
        }
        // rows 64..71 of the T_ee^T part: row 64 = t64 (k <= 64), the rest zero
        for (int i = tid; i < 8 * 72; i += blockDim.x) {
            const int n = 64 + i / 72, k = i % 72;
            const float v = (n == 64 && k <= H) ? t64[k] : 0.0f;
            const float h = tf32_hi(v);
            const uint32_t off = kmaj_off(n, k, 136);
            *reinterpret_cast<float *>(smem + S::t_hi + off) = h;
            *reinterpret_cast<float *>(smem + S::t_lo + off) = v - h;
        }
        fence_async_smem();
        tc_fence_before();
        __syncthreads();
        // 6. second products
        if (tid == 0) {
            tc_fence_after();
            issue_stage<true>(sdesc0, tmem);
            mma_commit(bar);
        }
        // rows 64 of Z_ee (n <= 64) and Z_eo (n < 64): sum_{k<=64} Ks[64][k] T[k][n];
        // two threads per sum (warps 2..10), k = sub, sub + 2, ...
        if (warp >= 2 && warp <= 10) {
            const int i = tid - 64, d = i >> 1, sub = i & 1;
            const bool ee = d <= H;
            const int row = ee ? d : 72 + (d - H - 1);  // T_ee^T row d, T_eo^T row d - 65
            float acc = 0.0f;
            if (d <= 2 * H)
                for (int k = sub; k <= H; k += 2) {
                    const uint32_t off = kmaj_off(row, k, 136);
                    const float tv = *reinterpret_cast<const float *>(smem + S::t_hi + off) +
                                     *reinterpret_cast<const float *>(smem + S::t_lo + off);
                    acc = fmaf(k64[k], tv, acc);
                }
            acc += __shfl_xor_sync(0xffffffffu, acc, 1);
            if (sub == 0 && d <= 2 * H) zx[d] = acc;
        }
        if (!mbar_wait(bar, phase, kWaitNs)) *s_err = 1;
        tc_fence_after();
        __syncthreads();
        if (*s_err) break;
        phase ^= 1;
        // Z from tensor memory straight into octant order over xs:
        //   Z_ee[m][n] -> (2m, 2n), n <= m;  Z_oo[m][n] -> (2m+1, 2n+1), n <= m;
        //   Z_eo[m][n] -> (2m, 2n+1) for n < m, (2n+1, 2m) for n >= m
        // rows 64 of Z_ee and Z_eo (zx) -> (128, 2n) and (128, 2n+1)
        {
            const int q = warp & 3, blk = warp >> 2;
            const int m = 16 * q + (lane & 15);
            const int col0 = blk == 0 ? 0 : (blk == 1 ? 72 : 136);
            uint32_t rr[72];
            tmem_ld_row72(tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)col0, rr, blk == 0);
            if (lane < 16) {
#pragma unroll
                for (int n = 0; n < 64; ++n) {
                    const float v = __uint_as_float(rr[n]);
                    if (blk == 0) {
                        if (n <= m) xs[oct_of(2 * m, 2 * n)] = v;
                    } else if (blk == 1) {
                        xs[n < m ? oct_of(2 * m, 2 * n + 1) : oct_of(2 * n + 1, 2 * m)] = v;
                    } else {
                        if (n <= m) xs[oct_of(2 * m + 1, 2 * n + 1)] = v;
                    }
                }
            }
        }
        for (int i = tid; i < 2 * H + 1; i += blockDim.x)
            xs[oct_of(2 * H, i <= H ? 2 * i : 2 * (i - H - 1) + 1)] = zx[i];
        fence_async_smem();  // this slice's accesses to the B operands come before the next copies
        tc_fence_before();
        __syncthreads();
        // the next slice's raw inputs (the B operands are free again)
        if (tid == 0 && nx < items)
            tc_stage<KIND>(smem, &tmIn, a, (int)(nx / ns), (int)(nx % ns), b.arena);
        // 7. output (consecutive lanes on consecutive octant points: a warp
        // writes whole 32-byte blocks of the column-block layout)
        if constexpr (KIND == kSliceSigma) {
            double *out = tc_point(a.out, b.arena, p);
            for (int o = tid; o < N8; o += blockDim.x) {
                int l, m;
                oct_lm(o, l, m);
                double nf = u[m];
#pragma unroll
                for (int r = 1; r <= R; ++r) nf = fma(cf[(r - 1) * NBK + l], u[r * NBK + m], nf);
                out[bidx(j, o, nw0 + 1)] = (double)xs[o] + nf;
            }
        } else {
            double *out = tc_point(a.out, b.arena, p);
            for (int o = tid; o < N8; o += blockDim.x) out[bidx(j, o, nb)] = xs[o];
        }
    }
    if (*s_err) {
        // let the MMAs and copies in flight (the phases whose wait ran out)
        // finish, bounded, before the tensor memory is freed and the CTA leaves
        if (tid == 0) {
            atomicOr(&g_tc_err, 1u);
            mbar_wait(bar, phase, kWaitNs);
            mbar_wait(tbar, tphase, kWaitNs);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, kTmemCols);
    }
}

}  // namespace

namespace {
// cuTensorMapEncodeTiled from the driver, looked up once through the runtime
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static std::once_flag once;
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// a 4-D tensor map over a column-block array of nb rows (4 doubles of a block,
// row, block, point): box (4, 1, 256, 1) = one row of 256 column blocks, 8 KB
cudaError_t block_row_map(const double *base, const GridDev &g, const Bp &b, CUtensorMap *m) {
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return cudaErrorNotSupported;
    const cuuint64_t nblk = (cuuint64_t)g.n8p / 4;
    const cuuint64_t dims[4] = {4, (cuuint64_t)g.nb, nblk, (cuuint64_t)b.P};
    const cuuint64_t strides[3] = {32, (cuuint64_t)g.nb * 32,
                                   b.P > 1 ? (cuuint64_t)b.arena : (cuuint64_t)g.nb * 32 * nblk};
    const cuuint32_t box[4] = {4, 1, TcSmem::VBOX, 1}, estr[4] = {1, 1, 1, 1};
    if (encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double *>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    return cudaSuccess;
}

template <int KIND>
cudaError_t run_slice_tc(const GridDev &g, const CUtensorMap &m, const TcArgs &a, const Bp &b, cudaStream_t st) {
    if (g.nbk != 129 || !g.dct_tc) return cudaErrorInvalidValue;
    const size_t sm = TcSmem::bytes;
    cudaError_t e = set_smem(k_slice_tc<KIND>, sm);
    if (e != cudaSuccess) return e;
    const int ctas = resident_ctas(k_slice_tc<KIND>, kTcThreads, sm);
    if (ctas <= 0) return cudaErrorInvalidConfiguration;
    const long long items = (long long)tc_slices<KIND>(g.nw0) * b.P;
    const int grid = (int)(items < ctas ? items : ctas);
    k_slice_tc<KIND><<<grid, kTcThreads, sm, st>>>(m, g.dct_tc, a, b);
    return launched();
}
}  // namespace

cudaError_t launch_sigma_slice_tc(const GridDev &g, const float *Grt, const double *V, double *sigt, cudaStream_t st,
                                  const Bp &b) {
    CUtensorMap m;
    cudaError_t e = block_row_map(V, g, b, &m);
    if (e != cudaSuccess) return e;
    TcArgs a;
    a.Grt = Grt;
    a.tw64 = g.tw_k;
    a.out = sigt;
    a.nw0 = g.nw0;
    return run_slice_tc<kSliceSigma>(g, m, a, b, st);
}

cudaError_t launch_vertex_q_tc(const GridDev &g, const double *chiq, double *Vr, double U, const double *Usc,
                               double T, cudaStream_t st, const Bp &b) {
    CUtensorMap m;
    cudaError_t e = block_row_map(chiq, g, b, &m);
    if (e != cudaSuccess) return e;
    TcArgs a;
    a.Usc = Usc;
    a.normFact = T / ((double)g.nk0 * g.nk0);
    a.U = U;
    a.out = Vr;
    a.nw0 = g.nw0;
    return run_slice_tc<kSliceVertex>(g, m, a, b, st);
}

// the error word of the tensor plan's kernels: nonzero once an mbarrier wait
// ran out (the context stays usable; the affected outputs are not valid)
int tensor_plan_errors(unsigned *out, bool clear) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyFromSymbol(&v, g_tc_err, sizeof(v));
    if (e != cudaSuccess) return -1;
    if (clear && v) {
        const unsigned z = 0;
        if (cudaMemcpyToSymbol(g_tc_err, &z, sizeof(z)) != cudaSuccess) return -1;
    }
    *out = v;
    return 0;
}

}  // namespace tpsc
