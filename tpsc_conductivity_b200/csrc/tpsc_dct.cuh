// tpsc_dct.cuh -- the 2D DCT-I of a symmetric slice as folded matrix
// products on the FP32 pipe (the "direct" slice plan of the mixed form).
//
// A slice X is symmetric, (N+1) x (N+1), N = 2H, and its DCT-I (FFTW's
// REDFT00 along both axes) Z = C X C^T, C[k][j] = w_j cos(pi j k / N) with
// w_j = 1 at j = 0, N and 2 elsewhere.  One radix-2 butterfly on the input
// index splits C:
//   even k = 2m:   Z_k = sum_{j<=H} Ks[m][j] s_j,  s_0 = x_0 + x_N,
//                  s_j = x_j + x_{N-j} (0 < j < H), s_H = x_H,
//                  Ks[m][j] = w'_j cos(pi j m / H)          (a DCT-I of length H+1)
//   odd k = 2m+1:  Z_k = sum_{j<H} Kd[m][j] d_j,   d_j = x_j - x_{N-j},
//                  Kd[m][j] = w'_j cos(pi j (2m+1) / N)     (a DCT-III of length H)
// with w'_0 = 1 and w'_j = 2 otherwise.  Folding both axes of X gives three
// blocks (the fourth is the transpose of one of them because X is symmetric):
//   SS = s-fold x s-fold  ((H+1) x (H+1), symmetric),
//   SD = s-fold x d-fold  ((H+1) x H),
//   DD = d-fold x d-fold  (H x H, symmetric),
// and Z_ee = Ks SS Ks^T, Z_eo = Ks SD Kd^T, Z_oo = Kd DD Kd^T, Z_oe = Z_eo^T.
// Each block is two small matrix products (T = block K^T, then Z = K T):
// register tiles of TM x TN outputs per thread, operands read as float4 rows
// of k-major tables, every product an FMA into an FP32 accumulator.  One
// slice is about 1.4 M FMAs at H = 64; the FFT plan (tpsc_fft.cuh) does
// fewer operations but exchanges every radix pass through shared memory, and
// that exchange, not arithmetic, bounds it.
//
// Shared-memory regions (floats, rows of LD = H + 4 so that rows start on
// 16-byte boundaries):
//   tab: KsT (H+1 rows), KdT (H rows); KsT[k][n] = Ks[n][k], KdT[k][n] = Kd[n][k]
//   F:   SS (H+1 rows) | SDT (H+1 rows, SDT[k][m] = SD[m][k], row H unused) | DD (H rows);
//        the second product writes Z_ee, Z_eo (H+1 rows x H), Z_oo over them
//   T:   T_ee (H+1 x H+1) | T_eo (H+1 x H) | T_oo (H x H)
// The table is built on the host from long double cosines rounded once.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tpsc_device.cuh"

namespace tpsc {
namespace {

constexpr int kDctThreads = 384;  // 3 blocks x 128 register tiles

template <int H>
struct DctPlan {
    static_assert(H == 16 || H == 32 || H == 64, "H in {16, 32, 64}");
    static constexpr int N = 2 * H, NBK = N + 1, N8 = NBK * (NBK + 1) / 2;
    static constexpr int LD = H + 4;
    static constexpr int EE = 0, EO = (H + 1) * LD, OO = 2 * (H + 1) * LD;  // block offsets in F and T
    static constexpr int REG = (3 * H + 2) * LD;                             // floats of F (and of T)
    static constexpr int KS = 0, KD = (H + 1) * LD, TAB = (2 * H + 1) * LD;  // table offsets, size
    static constexpr int TM = H / 8, TN = H / 16;  // thread tile: 8 x 16 tiles cover an H x H block
    static constexpr int NSS = (H + 1) * (H + 1), NSD = (H + 1) * H, NDD = H * H;
};

// r[0..R) <- p[0..R) (p 4R-byte aligned for R = 2, 16-byte aligned for R % 4 == 0)
template <int R>
__device__ __forceinline__ void lds_vec(float (&r)[R], const float *p) {
    if constexpr (R % 4 == 0) {
#pragma unroll
        for (int q = 0; q < R / 4; ++q) {
            const float4 v = reinterpret_cast<const float4 *>(p)[q];
            r[4 * q] = v.x;
            r[4 * q + 1] = v.y;
            r[4 * q + 2] = v.z;
            r[4 * q + 3] = v.w;
        }
    } else if constexpr (R == 2) {
        const float2 v = *reinterpret_cast<const float2 *>(p);
        r[0] = v.x;
        r[1] = v.y;
    } else {
        r[0] = p[0];
    }
}
template <int R>
__device__ __forceinline__ void sts_vec(float *p, const float (&r)[R]) {
    if constexpr (R % 4 == 0) {
#pragma unroll
        for (int q = 0; q < R / 4; ++q)
            reinterpret_cast<float4 *>(p)[q] = make_float4(r[4 * q], r[4 * q + 1], r[4 * q + 2], r[4 * q + 3]);
    } else if constexpr (R == 2) {
        *reinterpret_cast<float2 *>(p) = make_float2(r[0], r[1]);
    } else {
        p[0] = r[0];
    }
}

// out[i][j] = sum_{k<K} A[k LD + i] B[k LD + j], i < TM, j < TN, stored at
// out[i LD + j]: one register tile of a k-major product
template <int H>
__device__ __forceinline__ void dct_tile(const float *__restrict__ A, const float *__restrict__ B, int K,
                                         float *__restrict__ out) {
    using P = DctPlan<H>;
    constexpr int TM = P::TM, TN = P::TN, LD = P::LD;
    float acc[TM][TN];
#pragma unroll
    for (int i = 0; i < TM; ++i)
#pragma unroll
        for (int j = 0; j < TN; ++j) acc[i][j] = 0.0f;
#pragma unroll 4
    for (int k = 0; k < K; ++k) {
        float a[TM], b[TN];
        lds_vec(a, A + k * LD);
        lds_vec(b, B + k * LD);
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
    }
#pragma unroll
    for (int i = 0; i < TM; ++i) sts_vec(out + i * LD, acc[i]);
}

// sum_{k<K} a[k sa] b[k sb] (the H-th row and column of the blocks)
__device__ __forceinline__ float dct_dot(const float *__restrict__ a, int sa, const float *__restrict__ b, int sb,
                                         int K) {
    float acc = 0.0f;
#pragma unroll 5
    for (int k = 0; k < K; ++k) acc = fmaf(a[k * sa], b[k * sb], acc);
    return acc;
}

// thread's block (0 ee, 1 eo, 2 oo) and register tile origin (m0, n0)
template <int H>
__device__ __forceinline__ void dct_tile_of(int t, int &blk, int &m0, int &n0) {
    blk = t >> 7;
    const int tt = t & 127;
    m0 = (tt >> 4) * DctPlan<H>::TM;
    n0 = (tt & 15) * DctPlan<H>::TN;
}

// The butterfly: F <- SS, SDT, DD of the slice whose octant values are
// xs[l (l + 1)/2 + m], m <= l (X(p, q) = X(q, p)).
template <int H>
__device__ __forceinline__ void dct_fold(const float *__restrict__ xs, float *__restrict__ F) {
    using P = DctPlan<H>;
    constexpr int N = P::N, LD = P::LD;
    auto X = [&](int p, int q) -> float {
        const int l = p > q ? p : q, m = p > q ? q : p;
        return xs[l * (l + 1) / 2 + m];
    };
    for (int e = threadIdx.x; e < P::NSS + P::NSD + P::NDD; e += blockDim.x) {
        if (e < P::NSS) {
            const int a = e / (H + 1), b = e % (H + 1);
            float v = X(a, b);
            if (a < H) v += X(N - a, b);
            if (b < H) {
                float w = X(a, N - b);
                if (a < H) w += X(N - a, N - b);
                v += w;
            }
            F[P::EE + a * LD + b] = v;
        } else if (e < P::NSS + P::NSD) {
            const int f = e - P::NSS;
            const int k = f / (H + 1), m = f % (H + 1);  // SDT[k][m] = SD[m][k]: s-fold m, d-fold k
            float v = X(m, k) - X(m, N - k);
            if (m < H) v += X(N - m, k) - X(N - m, N - k);
            F[P::EO + k * LD + m] = v;
        } else {
            const int f = e - P::NSS - P::NSD;
            const int a = f / H, b = f % H;
            F[P::OO + a * LD + b] = (X(a, b) - X(a, N - b)) - (X(N - a, b) - X(N - a, N - b));
        }
    }
}

// first products: T_ee = SS Ks^T, T_eo = SD Kd^T, T_oo = DD Kd^T (F -> T)
template <int H>
__device__ __forceinline__ void dct_stage1(const float *__restrict__ F, float *__restrict__ T,
                                           const float *__restrict__ tab) {
    using P = DctPlan<H>;
    constexpr int LD = P::LD;
    const int t = threadIdx.x;
    if (t < kDctThreads) {
        int blk, m0, n0;
        dct_tile_of<H>(t, blk, m0, n0);
        const int off = blk == 0 ? P::EE : (blk == 1 ? P::EO : P::OO);
        const float *B = tab + (blk == 0 ? P::KS : P::KD);
        dct_tile<H>(F + off + m0, B + n0, blk == 0 ? H + 1 : H, T + off + m0 * LD + n0);
    }
    // row H and column H of T_ee, row H of T_eo: 3H + 1 dot products
    for (int i = t; i < 3 * H + 1; i += blockDim.x) {
        if (i <= H)
            T[P::EE + H * LD + i] = dct_dot(F + P::EE + H, LD, tab + P::KS + i, LD, H + 1);
        else if (i <= 2 * H)
            T[P::EE + (i - H - 1) * LD + H] = dct_dot(F + P::EE + (i - H - 1), LD, tab + P::KS + H, LD, H + 1);
        else
            T[P::EO + H * LD + (i - 2 * H - 1)] = dct_dot(F + P::EO + H, LD, tab + P::KD + (i - 2 * H - 1), LD, H);
    }
}

// second products: Z_ee = Ks T_ee, Z_eo = Ks T_eo, Z_oo = Kd T_oo (T -> F)
template <int H>
__device__ __forceinline__ void dct_stage2(const float *__restrict__ T, float *__restrict__ F,
                                           const float *__restrict__ tab) {
    using P = DctPlan<H>;
    constexpr int LD = P::LD;
    const int t = threadIdx.x;
    if (t < kDctThreads) {
        int blk, m0, n0;
        dct_tile_of<H>(t, blk, m0, n0);
        const int off = blk == 0 ? P::EE : (blk == 1 ? P::EO : P::OO);
        const float *A = tab + (blk == 2 ? P::KD : P::KS);
        dct_tile<H>(A + m0, T + off + n0, blk == 2 ? H : H + 1, F + off + m0 * LD + n0);
    }
    // row H of Z_ee (H + 1 values) and of Z_eo (H values)
    for (int i = t; i < 2 * H + 1; i += blockDim.x) {
        if (i <= H)
            F[P::EE + H * LD + i] = dct_dot(tab + P::KS + H, LD, T + P::EE + i, LD, H + 1);
        else
            F[P::EO + H * LD + (i - H - 1)] = dct_dot(tab + P::KS + H, LD, T + P::EO + (i - H - 1), LD, H + 1);
    }
}

// Z(l, m) of the transformed slice, read from F after dct_stage2
template <int H>
__device__ __forceinline__ float dct_z(const float *__restrict__ F, int l, int m) {
    using P = DctPlan<H>;
    constexpr int LD = P::LD;
    const int a = l >> 1, b = m >> 1;
    if (((l | m) & 1) == 0) return F[P::EE + a * LD + b];
    if (l & m & 1) return F[P::OO + a * LD + b];
    return (l & 1) ? F[P::EO + b * LD + a] : F[P::EO + a * LD + b];
}

// 2D DCT-I of the slice in xs (octant values) into F; T is scratch.  All
// threads of the block call; the block has kDctThreads threads.  Ends with
// a barrier: dct_z(F, ...) may be read right after.
template <int H>
__device__ __forceinline__ void dct2_direct(const float *xs, float *F, float *T, const float *tab) {
    dct_fold<H>(xs, F);
    __syncthreads();
    dct_stage1<H>(F, T, tab);
    __syncthreads();
    dct_stage2<H>(T, F, tab);
    __syncthreads();
}

}  // namespace
}  // namespace tpsc
