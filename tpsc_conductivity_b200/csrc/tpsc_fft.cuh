// tpsc_fft.cuh -- FFT building blocks for sm_100a, FP64 (double2) and FP32
// (float2) complex data.
//
// * in-register radix-2/4/8/16 DFTs (exact constants, standard split-radix
//   style recursion);
// * a Stockham auto-sort FFT executed by a group of G threads, each thread
//   holding 16 points, over a padded shared-memory buffer;
// * a 2D DCT-I of a symmetric nbk x nbk slice held in shared memory.  Two
//   real rows (columns) are packed into one complex FFT of their even
//   extension of length L = 2(nbk-1): a real even sequence has a real
//   spectrum, so Re/Im of the packed transform are the two DCT-I outputs.
//
// DCT-I here is FFTW's REDFT00 (unnormalised):
//   Y_k = X_0 + (-1)^k X_{n-1} + 2 sum_{j=1}^{n-2} X_j cos(pi j k/(n-1)).
//
// FP32 transforms take their inter-pass twiddles from a float4 table
// (cos_hi, sin_hi, cos_lo, sin_lo) with hi + lo the twiddle to ~48 bits and
// form the twiddle product with FMAs around the lo correction, so the
// twiddle enters to full FP32 accuracy of the product (compensated twiddles);
// the radix-16 constants and the butterfly sums are plain FP32.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tpsc {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
// multiply by -i (SIGN = -1) or +i (SIGN = +1)
template <int SIGN, class C>
__device__ __forceinline__ C mul_i(C a) {
    return SIGN < 0 ? C{a.y, -a.x} : C{-a.y, a.x};
}

// real type of a complex type
template <class C>
struct real_of;
template <>
struct real_of<double2> {
    using type = double;
};
template <>
struct real_of<float2> {
    using type = float;
};

// the twiddle product v * w (conj(w) for SIGN > 0), w from the table of the
// transform's precision: double2 for FP64; float4 (hi, lo) for FP32
template <int SIGN, bool SMEM>
__device__ __forceinline__ double2 twiddle(double2 v, const double2 *__restrict__ tw, int m) {
    double2 w = SMEM ? tw[m] : __ldg(&tw[m]);
    if (SIGN > 0) w.y = -w.y;
    return cmul(v, w);
}
template <int SIGN, bool SMEM>
__device__ __forceinline__ float2 twiddle(float2 v, const float4 *__restrict__ tw, int m) {
    float4 w = SMEM ? tw[m] : __ldg(&tw[m]);
    if (SIGN > 0) {
        w.y = -w.y;
        w.w = -w.w;
    }
    // (a + i b)(c + i d) with c = w.x + w.z, d = w.y + w.w: the lo parts as a
    // correction term, the hi parts fused into it
    const float cr = fmaf(v.x, w.z, -v.y * w.w), ci = fmaf(v.x, w.w, v.y * w.z);
    return make_float2(fmaf(v.x, w.x, fmaf(-v.y, w.y, cr)), fmaf(v.x, w.y, fmaf(v.y, w.x, ci)));
}

// Two-level twiddle table for FFT lengths N <= 4096 kept in shared memory:
// exp(-2 pi i m / N) = hi[m >> 6] * lo[m & 63] with hi[a] = exp(-2 pi i 64 a/N)
// and lo[b] = exp(-2 pi i b/N) (2 KB instead of 16 N bytes; the product adds
// about one ulp to the twiddle).
struct TwoLevelTw {
    double2 hi[64], lo[64];
};
template <int SIGN, bool SMEM>
__device__ __forceinline__ double2 twiddle(double2 v, const TwoLevelTw *__restrict__ tw, int m) {
    double2 w = cmul(tw->hi[m >> 6], tw->lo[m & 63]);
    if (SIGN > 0) w.y = -w.y;
    return cmul(v, w);
}

// exp(sign * 2 pi i m / 16) for the constant twiddles of the radix-8/16
// kernels; m is a compile-time constant after unrolling, so the switch folds.
__device__ __forceinline__ double2 w16(int m, int sign) {
    const double c1 = 0.92387953251128675613;  // cos(pi/8)
    const double s1 = 0.38268343236508977173;  // sin(pi/8)
    const double c2 = 0.70710678118654752440;  // cos(pi/4)
    double c, s;
    switch (m & 15) {
        case 0: c = 1; s = 0; break;
        case 1: c = c1; s = s1; break;
        case 2: c = c2; s = c2; break;
        case 3: c = s1; s = c1; break;
        case 4: c = 0; s = 1; break;
        case 5: c = -s1; s = c1; break;
        case 6: c = -c2; s = c2; break;
        case 7: c = -c1; s = s1; break;
        case 8: c = -1; s = 0; break;
        case 9: c = -c1; s = -s1; break;
        case 10: c = -c2; s = -c2; break;
        case 11: c = -s1; s = -c1; break;
        case 12: c = 0; s = -1; break;
        case 13: c = s1; s = -c1; break;
        case 14: c = c2; s = -c2; break;
        default: c = c1; s = -s1; break;
    }
    return make_double2(c, sign * s);
}

template <class C>
__device__ __forceinline__ C w16c(int m, int sign) {
    const double2 w = w16(m, sign);
    using T = typename real_of<C>::type;
    return C{(T)w.x, (T)w.y};
}

// In-register DFT of length R on v[0..R) with stride S inside the array
// (elements v[OFF + k*S]).  X_k = sum_j x_j exp(SIGN 2 pi i jk/R).
template <int SIGN, int R, int S = 1, int OFF = 0, int NV, class C>
__device__ __forceinline__ void dft(C (&v)[NV]) {
    if constexpr (R == 1) {
        return;
    } else if constexpr (R == 2) {
        C a = v[OFF], b = v[OFF + S];
        v[OFF] = cadd(a, b);
        v[OFF + S] = csub(a, b);
    } else if constexpr (R == 4) {
        C a = v[OFF], b = v[OFF + S], c = v[OFF + 2 * S], d = v[OFF + 3 * S];
        C t0 = cadd(a, c), t1 = csub(a, c), t2 = cadd(b, d), t3 = mul_i<SIGN>(csub(b, d));
        v[OFF] = cadd(t0, t2);
        v[OFF + 2 * S] = csub(t0, t2);
        v[OFF + S] = cadd(t1, t3);
        v[OFF + 3 * S] = csub(t1, t3);
    } else {
        // radix-2 decimation in time: even/odd halves are DFTs of length R/2
        // taken on the sub-sequences at stride 2S; results interleaved back.
        constexpr int H = R / 2;
        C e[H], o[H];
#pragma unroll
        for (int k = 0; k < H; ++k) {
            e[k] = v[OFF + (2 * k) * S];
            o[k] = v[OFF + (2 * k + 1) * S];
        }
        dft<SIGN, H, 1, 0>(e);
        dft<SIGN, H, 1, 0>(o);
#pragma unroll
        for (int k = 0; k < H; ++k) {
            const C w = w16c<C>((16 / R) * k, SIGN);
            C t = cmul(o[k], w);
            v[OFF + k * S] = cadd(e[k], t);
            v[OFF + (k + H) * S] = csub(e[k], t);
        }
    }
}

// padded index into an FFT scratch buffer: one complex of padding every 16
__device__ __forceinline__ int pidx(int i) { return i + (i >> 4); }
__host__ __device__ constexpr int padded_len(int n) { return n + n / 16; }

// Group barrier: G threads with consecutive thread ids starting at a multiple
// of G.  Groups inside one warp use a lane mask; a group spanning the whole
// block uses __syncthreads; otherwise a named barrier per group.
template <int G>
__device__ __forceinline__ void group_sync(int grp) {
    if constexpr (G < 32) {
        const unsigned lane0 = (threadIdx.x & 31) & ~(G - 1);
        const unsigned mask = ((G == 32) ? 0xffffffffu : ((1u << G) - 1u)) << lane0;
        __syncwarp(mask);
    } else if constexpr (G == 32) {
        __syncwarp();
    } else {
        asm volatile("bar.sync %0, %1;" ::"r"(grp + 1), "r"(G) : "memory");
    }
}

// The twiddle w_m = exp(-2 pi i m / N) itself, from a FP64 table.
template <bool SMEM>
__device__ __forceinline__ double2 tw_value(const double2 *__restrict__ tw, int m) {
    return SMEM ? tw[m] : __ldg(&tw[m]);
}
template <bool SMEM>
__device__ __forceinline__ double2 tw_value(const TwoLevelTw *__restrict__ tw, int m) {
    return cmul(tw->hi[m >> 6], tw->lo[m & 63]);
}

// v[q] *= w^q (conj(w)^q for SIGN > 0), q = 1..15, w = w_step, in FP64: the
// table gives w, w^2, w^4 and w^8, and every other power is a product of at
// most four of them (a few ulp), so a radix-16 butterfly reads 4 twiddles
// instead of 15.  The table entries read are w_{step q mod N}, q = 1, 2, 4, 8.
template <int N, int SIGN, bool SMEM, class TW>
__device__ __forceinline__ void twiddle16_powers(double2 *v, const TW *__restrict__ tw, int step) {
    double2 w1 = tw_value<SMEM>(tw, step & (N - 1)), w2 = tw_value<SMEM>(tw, (2 * step) & (N - 1));
    double2 w4 = tw_value<SMEM>(tw, (4 * step) & (N - 1)), w8 = tw_value<SMEM>(tw, (8 * step) & (N - 1));
    if (SIGN > 0) {
        w1.y = -w1.y;
        w2.y = -w2.y;
        w4.y = -w4.y;
        w8.y = -w8.y;
    }
    const double2 w3 = cmul(w2, w1), w5 = cmul(w4, w1), w6 = cmul(w4, w2), w7 = cmul(w4, w3);
    v[1] = cmul(v[1], w1);
    v[2] = cmul(v[2], w2);
    v[3] = cmul(v[3], w3);
    v[4] = cmul(v[4], w4);
    v[5] = cmul(v[5], w5);
    v[6] = cmul(v[6], w6);
    v[7] = cmul(v[7], w7);
    v[8] = cmul(v[8], w8);
    v[9] = cmul(v[9], cmul(w8, w1));
    v[10] = cmul(v[10], cmul(w8, w2));
    v[11] = cmul(v[11], cmul(w8, w3));
    v[12] = cmul(v[12], cmul(w8, w4));
    v[13] = cmul(v[13], cmul(w8, w5));
    v[14] = cmul(v[14], cmul(w8, w6));
    v[15] = cmul(v[15], cmul(w8, w7));
}
template <int N, int SIGN, bool SMEM, class TW>
__device__ __forceinline__ void twiddle16_powers(float2 *, const TW *__restrict__, int) {}

// Loaders / storers for the first and last FFT pass.  `In` returns input
// element j of the sequence; `Out` receives output element k.
template <class C>
struct ScratchIOT {
    C *x;
    __device__ __forceinline__ C operator()(int j) const { return x[pidx(j)]; }
    __device__ __forceinline__ void operator()(int k, C v) const { x[pidx(k)] = v; }
};
using ScratchIO = ScratchIOT<double2>;

// One Stockham pass of radix R over a length-N sequence, performed by a group
// of G threads holding E points each; thread t does E/R butterflies
// b = t + G u.  tw[m] = exp(-2 pi i m / N), m < N.  The first pass reads its
// inputs through `in` (FIRST), the last pass hands its outputs, in natural
// order, to `out` (LAST); every other pass reads and writes the padded
// scratch x in place, with group barriers around the writes.  SYNC_IN puts
// a barrier between the first pass's reads and its writes, for an `in` that
// reads x itself.
template <int N, int G, int R, int SIGN, int E, bool SMEM_TW, bool FIRST, bool LAST, bool SYNC_IN, class In,
          class Out, class C, class TW>
__device__ __forceinline__ void stockham_pass(C *x, int t, int Ns, const TW *__restrict__ tw, int grp, const In &in,
                                              const Out &out) {
    constexpr int NB = E / R;  // butterflies per thread
    C v[E];
#pragma unroll
    for (int u = 0; u < NB; ++u) {
        const int b = t + G * u;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const int j = b + q * (N / R);
            v[u * R + q] = FIRST ? in(j) : x[pidx(j)];
        }
    }
    if (!FIRST || SYNC_IN) group_sync<G>(grp);
#pragma unroll
    for (int u = 0; u < NB; ++u) {
        const int b = t + G * u;
        const int k = b % Ns;
        if (Ns > 1) {
            // twiddle exp(SIGN 2 pi i k q / (Ns R)) = tw[k q N/(Ns R)] (conjugated for SIGN>0)
            const int step = k * (N / (Ns * R));
            if constexpr (N == 256 && R == 16 && !FIRST && sizeof(C) == sizeof(float2)) {
                // the FP32 256-point transform's second pass (Ns = 16, step = k):
                // its twiddles tw[k q], q = 1..15, are read from the transposed
                // copy behind the table, entry 256 + (q - 1) 16 + k, so that the
                // 16 threads of a group read 16 consecutive entries (no bank
                // conflicts; strided reads tw[k q] are up to 16-way for even q)
#pragma unroll
                for (int q = 1; q < R; ++q)
                    v[u * R + q] = twiddle<SIGN, SMEM_TW>(v[u * R + q], tw, 256 + (q - 1) * 16 + k);
            } else if constexpr (R == 16 && sizeof(C) == sizeof(double2)) {
                twiddle16_powers<N, SIGN, SMEM_TW>(&v[u * R], tw, step);
            } else {
#pragma unroll
                for (int q = 1; q < R; ++q)
                    v[u * R + q] = twiddle<SIGN, SMEM_TW>(v[u * R + q], tw, (step * q) & (N - 1));
            }
        }
        C r[R];
#pragma unroll
        for (int q = 0; q < R; ++q) r[q] = v[u * R + q];
        dft<SIGN, R>(r);
#pragma unroll
        for (int q = 0; q < R; ++q) v[u * R + q] = r[q];
    }
#pragma unroll
    for (int u = 0; u < NB; ++u) {
        const int b = t + G * u;
        const int k = b % Ns;
        const int base = (b / Ns) * Ns * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) {
            if (LAST)
                out(base + q * Ns, v[u * R + q]);
            else
                x[pidx(base + q * Ns)] = v[u * R + q];
        }
    }
    if (!LAST) group_sync<G>(grp);
}

// EP points per thread (16 or 8): radix-EP passes followed by one pass of
// radix N / EP^P16 (if > 1); each of the G threads holds E = min(EP, N)
// points.  EP = 8 takes twice the threads and one more pass for N >= 512.
template <int N, int EP = 16>
struct FftPlan {
    static_assert(EP == 16 || EP == 8, "16 or 8 points per thread");
    static constexpr int log2n() {
        int l = 0;
        while ((1 << l) < N) ++l;
        return l;
    }
    static constexpr int LE = EP == 16 ? 4 : 3;
    static constexpr int P16 = log2n() / LE;
    static constexpr int RLAST = 1 << (log2n() % LE);
    static constexpr int E = N < EP ? N : EP;
    static constexpr int G = N / E;
    static constexpr int NPASS = P16 + (RLAST > 1 ? 1 : 0);
};

template <int N, int SIGN, bool SMEM_TW, bool INPLACE, int P, int EP, class In, class Out, class C, class TW>
__device__ __forceinline__ void fft_passes(C *x, int t, int Ns, const TW *__restrict__ tw, int grp, const In &in,
                                           const Out &out) {
    using Plan = FftPlan<N, EP>;
    constexpr int G = Plan::G;
    constexpr int E = Plan::E;
    constexpr int NP = Plan::NPASS;
    constexpr int R = (P < Plan::P16) ? EP : Plan::RLAST;
    if constexpr (N <= EP) {
        // one in-register DFT, single pass
        stockham_pass<N, G, N, SIGN, E, SMEM_TW, true, true, INPLACE>(x, t, 1, tw, grp, in, out);
    } else {
        stockham_pass<N, G, R, SIGN, E, SMEM_TW, P == 0, P == NP - 1, INPLACE && P == 0>(x, t, Ns, tw, grp, in,
                                                                                        out);
        if constexpr (P + 1 < NP) fft_passes<N, SIGN, SMEM_TW, INPLACE, P + 1, EP>(x, t, Ns * R, tw, grp, in, out);
    }
}

// FFT of a length-N sequence by a group of G = FftPlan<N>::G threads: inputs
// from in(j), outputs (natural order) to out(k, value); x is the group's
// padded scratch of padded_len(N) complex.  All G threads must call.  When
// the FFT has more than one pass, x is free again when the call returns.
// INPLACE: `in` reads x (the first pass then holds its writes back until
// every thread of the group has read its inputs).
template <int N, int SIGN, bool SMEM_TW = false, bool INPLACE = false, int EP = 16, class In, class Out, class C,
          class TW>
__device__ __forceinline__ void group_fft_io(C *x, int t, const TW *__restrict__ tw, int grp, const In &in,
                                             const Out &out) {
    static_assert(N >= 4 && (N & (N - 1)) == 0, "power of two >= 4");
    fft_passes<N, SIGN, SMEM_TW, INPLACE, 0, EP>(x, t, 1, tw, grp, in, out);
    if constexpr (FftPlan<N, EP>::NPASS > 1) group_sync<FftPlan<N, EP>::G>(grp);
}

// In-place FFT of x[0..N) (padded layout).
template <int N, int SIGN, bool SMEM_TW = false, class C, class TW>
__device__ __forceinline__ void group_fft(C *x, int t, const TW *__restrict__ tw, int grp) {
    const ScratchIOT<C> io{x};
    group_fft_io<N, SIGN, SMEM_TW, true>(x, t, tw, grp, io, io);
}

// 2D DCT-I (REDFT00 x REDFT00) in place on a symmetric NBK x NBK slice S
// (row-major, leading dimension NBK, which is odd so that column accesses
// are bank-conflict free).  scr: per-group FFT scratch, group g at
// scr + g * padded_len(L); tw: the L twiddles (shared or global memory).  All
// threads of the block must call.  Two lines (rows, then columns) go through
// one complex FFT of their even extension; the first FFT pass reads the
// lines straight from S and the last pass writes outputs k < NBK back.
template <int NBK, class T, class C, class TW>
__device__ void dct2_slice(T *S, C *scr, const TW *tw) {
    constexpr int L = 2 * (NBK - 1);
    constexpr int G = FftPlan<L>::G;
    constexpr int NPAIR = (NBK + 1) / 2;
    const int tid = threadIdx.x;
    const int grp = tid / G;
    const int t = tid % G;
    const int ngrp = blockDim.x / G;
    C *x = scr + grp * padded_len(L);
#pragma unroll 1
    for (int pass = 0; pass < 2; ++pass) {
        // pass 0: rows (stride 1 along the line, NBK between lines)
        // pass 1: columns (stride NBK along the line, 1 between lines)
        const int es = pass == 0 ? 1 : NBK;
        const int ls = pass == 0 ? NBK : 1;
#pragma unroll 1
        for (int p = grp; p < NPAIR; p += ngrp) {
            const int r0 = 2 * p, r1 = 2 * p + 1;
            const bool two = r1 < NBK;
            T *a = S + r0 * ls;
            T *b = S + (two ? r1 : r0) * ls;
            auto in = [&](int j) -> C {
                const int c = j < NBK ? j : L - j;
                return C{a[c * es], two ? b[c * es] : (T)0};
            };
            auto out = [&](int k, C z) {
                if (k < NBK) {
                    a[k * es] = z.x;
                    if (two) b[k * es] = z.y;
                }
            };
            group_fft_io<L, -1, true>(x, t, tw, grp, in, out);
            if constexpr (FftPlan<L>::NPASS == 1) group_sync<G>(grp);
        }
        __syncthreads();
    }
}

// 2D RODFT00 x REDFT00 in place on an (NBK-2) x NBK slice S (row l, column
// m, leading dimension NBK): DCT-I of length NBK along m, DST-I of length
// NBK-2 along l -- the transform of functions odd in kx and even in ky on the
// interior kx points (FFTW's RODFT00: Y_k = 2 sum_j X_j sin(pi (j+1)(k+1)/(n+1))).
// Both lengths use complex FFTs of L = 2(NBK-1): the DCT through the even
// extension of two packed lines, the DST through the odd extension
// z = [0, X, 0, -reverse(X)], whose transform is -i Y_a + Y_b for the packed
// pair a + i b.  Same calling rules as dct2_slice.
template <int NBK, class T, class C, class TW>
__device__ void dst_dct_slice(T *S, C *scr, const TW *tw) {
    constexpr int L = 2 * (NBK - 1);
    constexpr int NR = NBK - 2;
    constexpr int G = FftPlan<L>::G;
    const int tid = threadIdx.x;
    const int grp = tid / G;
    const int t = tid % G;
    const int ngrp = blockDim.x / G;
    C *x = scr + grp * padded_len(L);
    // rows: DCT-I along m, NR lines
#pragma unroll 1
    for (int p = grp; p < (NR + 1) / 2; p += ngrp) {
        const int r0 = 2 * p, r1 = 2 * p + 1;
        const bool two = r1 < NR;
        T *a = S + r0 * NBK;
        T *b = S + (two ? r1 : r0) * NBK;
        auto in = [&](int j) -> C {
            const int c = j < NBK ? j : L - j;
            return C{a[c], two ? b[c] : (T)0};
        };
        auto out = [&](int k, C z) {
            if (k < NBK) {
                a[k] = z.x;
                if (two) b[k] = z.y;
            }
        };
        group_fft_io<L, -1, true>(x, t, tw, grp, in, out);
        if constexpr (FftPlan<L>::NPASS == 1) group_sync<G>(grp);
    }
    __syncthreads();
    // columns: DST-I along l, NBK lines
#pragma unroll 1
    for (int p = grp; p < (NBK + 1) / 2; p += ngrp) {
        const int c0 = 2 * p, c1 = 2 * p + 1;
        const bool two = c1 < NBK;
        T *a = S + c0;
        T *b = S + (two ? c1 : c0);
        auto in = [&](int j) -> C {
            if (j == 0 || j == NR + 1) return C{(T)0, (T)0};
            if (j <= NR) return C{a[(j - 1) * NBK], two ? b[(j - 1) * NBK] : (T)0};
            const int r = L - j - 1;
            return C{-a[r * NBK], two ? -b[r * NBK] : (T)0};
        };
        auto out = [&](int k, C z) {
            if (k >= 1 && k <= NR) {
                a[(k - 1) * NBK] = -z.y;
                if (two) b[(k - 1) * NBK] = z.x;
            }
        };
        group_fft_io<L, -1, true>(x, t, tw, grp, in, out);
        if constexpr (FftPlan<L>::NPASS == 1) group_sync<G>(grp);
    }
    __syncthreads();
}

}  // namespace tpsc
