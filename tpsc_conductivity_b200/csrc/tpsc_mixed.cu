// tpsc_mixed.cu -- the FP32 slice transforms of the mixed-precision form.
//
// The G(r, tau), chi0, V(q) and Sigma(k, tau) stages of the solve transform
// in FP32 (the slice and its DCT-I in float, twiddles compensated, see
// tpsc_fft.cuh); their inputs are formed and their outputs kept in FP64 where
// the next stage needs it: chi0(r, tau) and chi0(q, tau) feed the FP64 tau
// transforms and sum rules, V(r, tau) the self-energy, Sigma(k, tau) the
// FP64 spline and FFT along tau.  G(r, tau) is stored in FP32 (half the
// bytes).  Every tau transform, the tail moments, the sum rules, the root
// searches and the continuation stay FP64.
//
// The Sigma slice compensates for its size: a plain FP32 transform of
// G(r, tau) V(r, tau) costs ~6e-6 of Sigma(k, i w_n), because the few
// points nearest r = 0 dominate the product and their FP32 rounding
// survives the tau integral.  The slice therefore transforms in FP32 only
// the product beyond the near field |rx|, |ry| <= kNear and adds the near
// field's exact DCT-I in FP64: with u_a(k2) = sum_b w_b x(a, b) cos(pi b k2/(nbk-1)),
// the near field contributes sum_a w_a cos(pi a k1/(nbk-1)) u_a(k2) at
// (k1, k2), kNear + 1 FMAs per output point.
//
// Each FP32 slice needs ~105 KB of shared memory (the 129 x 129 float slice,
// 16 groups' float2 FFT scratch and the hi/lo twiddles), so two CTAs run on
// an SM where the FP64 slice kernels fit one.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tpsc_device.cuh"

namespace tpsc {

namespace {

constexpr int kSlice32Threads = 256;

template <int NBK>
struct Slice32Smem {
    static constexpr int L = 2 * (NBK - 1);
    static constexpr int G = FftPlan<L>::G;
    static constexpr int NGRP = kSlice32Threads / G;
    static constexpr size_t slice_bytes = (size_t)NBK * NBK * sizeof(float);
    static constexpr size_t scr_off = (slice_bytes + 15) & ~(size_t)15;
    static constexpr size_t tw_off = scr_off + (size_t)NGRP * padded_len(L) * sizeof(float2);
    // the L twiddles, and for L = 256 the second pass's twiddles transposed
    // behind them (15 x 16, see stockham_pass)
    static constexpr int NTW = L + (L == 256 ? 15 * 16 : 0);
    static constexpr size_t bytes = tw_off + (size_t)NTW * sizeof(float4);
};

// Input staging (see stage_blockrow / fill_from_staged): the FP32 slices'
// input rows fit in the slice and FFT scratch, which are idle until the fill
template <int NBK>
struct Stage32 {
    static constexpr int N8 = NBK * (NBK + 1) / 2;
    static constexpr size_t blockrow_bytes = StageRows<NBK>::blockrow_bytes;
    static constexpr size_t frow_bytes = ((size_t)N8 * sizeof(float) + 15) & ~(size_t)15;  // one FP32 G row
    static_assert(blockrow_bytes + frow_bytes <= Slice32Smem<NBK>::tw_off, "inputs must fit before the twiddles");
    static_assert(2 * frow_bytes <= Slice32Smem<NBK>::tw_off, "inputs must fit before the twiddles");
};

// n8 floats from src -> dst (4-byte copies: the FP32 G rows are not 16-byte aligned)
template <int NBK>
__device__ __forceinline__ void stage_frow(float *dst, const float *__restrict__ src) {
    for (int o = threadIdx.x; o < StageRows<NBK>::N8; o += blockDim.x) cp_async4(dst + o, src + o);
}

template <int NBK>
__device__ __forceinline__ float2 *scratch32(float *S) {
    return reinterpret_cast<float2 *>(reinterpret_cast<char *>(S) + Slice32Smem<NBK>::scr_off);
}

// the hi/lo twiddles in shared memory, and for L = 256 entry 256 + (q-1) 16 + k
// = tw[k q] (q = 1..15, k < 16); the kernel's first barrier publishes them
template <int NBK>
__device__ __forceinline__ const float4 *twiddles32(float *S, const float4 *__restrict__ tw) {
    constexpr int L = Slice32Smem<NBK>::L;
    float4 *t = reinterpret_cast<float4 *>(reinterpret_cast<char *>(S) + Slice32Smem<NBK>::tw_off);
    for (int i = threadIdx.x; i < Slice32Smem<NBK>::NTW; i += blockDim.x) {
        const int m = i < L ? i : (((i - L) & 15) * ((i - L) / 16 + 1)) & (L - 1);
        t[i] = __ldg(&tw[m]);
    }
    return t;
}

// G(r, tau_j) = DCT-I[ G0(k, tau_j) / L^2 ] in FP32 (the FP64 k_gslice's
// stage, src/green.cpp:1830-1841 and src/chi0.cpp:462-495): G0 formed in
// FP64, rounded once to float; Grt32[j * n8 + o].
template <int NBK>
__global__ void __launch_bounds__(kSlice32Threads, 2)
    k_gslice32(const double2 *__restrict__ gk, const float4 *__restrict__ tw,
               int n8, int nw0, double T, float *__restrict__ Grt, Bp b) {
    extern __shared__ __align__(16) float S32[];
    const float4 *tws = twiddles32<NBK>(S32, tw);
    gk = at(gk, b.arena);
    Grt = at(Grt, b.arena);
    T = bpar(b, kPpT, T);
    const int j = blockIdx.x;
    const double t = j / (nw0 * T);
    const double bt = 1.0 / T - t;
    fill_octant<NBK>(S32, n8, [&](int o) -> float {
        const double2 c = __ldg(&gk[o]);
        return (float)(c.y * exp((c.x > 0 ? -t : bt) * c.x));
    });
    __syncthreads();
    dct2_slice<NBK>(S32, scratch32<NBK>(S32), tws);
    float *out = Grt + (size_t)j * n8;
    for (int o = threadIdx.x; o < n8; o += blockDim.x) {
        int l, m;
        oct_lm(o, l, m);
        out[o] = S32[l * NBK + m];
    }
}

// chi0(r, tau_j) = -2 G(r, tau_j) G(r, -tau_j) from the FP32 G (the product
// is exact in FP64 and kept there for the tau transforms), its DCT-I in FP32
// -> chi0(q, tau_j) in FP64 (src/chi0.cpp:393-418, 497-517, 545-558).
template <int NBK>
__global__ void __launch_bounds__(kSlice32Threads, 2)
    k_chi0_slice32(const float *__restrict__ Grt, const float4 *__restrict__ tw,
                   int n8, int nw0, int ahead, double *__restrict__ chirt, double *__restrict__ chiq, Bp b) {
    extern __shared__ __align__(16) float S32[];
    const float4 *tws = twiddles32<NBK>(S32, tw);
    Grt = at(Grt, b.arena);
    chirt = at(chirt, b.arena);
    chiq = at(chiq, b.arena);
    const int j = blockIdx.x;
    const int nb = nw0 / 2 + 1;
    if (ahead > 0 && j + ahead < nb) {
        const int jn = j + ahead;
        prefetch_l2_range(Grt + (size_t)jn * n8, (size_t)n8 * sizeof(float));
        prefetch_l2_range(Grt + (size_t)(nw0 - jn) * n8, (size_t)n8 * sizeof(float));
    }
    // G(r, tau_j) and G(r, beta - tau_j) staged in the slice / scratch area
    float *gp = S32;
    float *gm = S32 + Stage32<NBK>::frow_bytes / sizeof(float);
    stage_frow<NBK>(gp, Grt + (size_t)j * n8);
    stage_frow<NBK>(gm, Grt + (size_t)(nw0 - j) * n8);
    cp_async_wait_all();
    __syncthreads();
    fill_from_staged<NBK, kSlice32Threads>(S32, [&](int o) -> float {
        const double a = gp[o];
        double c;
        if (j == 0)
            c = (o == 0) ? -2.0 * a * (a + 1.0) : -2.0 * a * a;
        else if (j == nb - 1)
            c = 2.0 * a * a;
        else
            c = -2.0 * (-(double)gm[o]) * a;
        chirt[bidx(j, o, nb)] = c;
        return (float)c;
    });
    __syncthreads();
    dct2_slice<NBK>(S32, scratch32<NBK>(S32), tws);
    for (int o = threadIdx.x; o < n8; o += blockDim.x) {
        int l, m;
        oct_lm(o, l, m);
        chiq[bidx(j, o, nb)] = S32[l * NBK + m];
    }
}

// V(q, iqn) in FP64 from chi0(q, iqn), its DCT-I over q in FP32
// (src/chi.cpp:89-115).  With a = Usp/2, b = Uch/2,
//   chi_sp - chi0 = a chi0^2 / (1 - a chi0),  chi_ch - chi0 = -b chi0^2 / (1 + b chi0),
// so that V takes one FP64 division per point.
template <int NBK>
__global__ void __launch_bounds__(kSlice32Threads, 2)
    k_vertex_q32(const double *__restrict__ chiq, const float4 *__restrict__ tw,
                 int n8, int nb, int ahead, double normFact, double U, const double *__restrict__ Usc,
                 double *__restrict__ Vr, Bp b) {
    extern __shared__ __align__(16) float S32[];
    const float4 *tws = twiddles32<NBK>(S32, tw);
    chiq = at(chiq, b.arena);
    Usc = at(Usc, b.arena);
    Vr = at(Vr, b.arena);
    normFact = bpar(b, kPpNormFact, normFact);
    U = bpar(b, kPpU, U);
    const int j = blockIdx.x;
    const double Usp = Usc[0], Uch = Usc[1];
    if (ahead > 0 && j + ahead < nb) prefetch_l2_blockrow(chiq, j + ahead, nb, (n8 + 3) / 4);
    // chi0(q, iq_j) staged in the slice / scratch area
    double *cs = reinterpret_cast<double *>(S32);
    stage_blockrow<NBK>(cs, chiq, j, nb);
    cp_async_wait_all();
    __syncthreads();
    fill_from_staged<NBK, kSlice32Threads>(S32, [&](int o) -> float {
        const double c0 = cs[o];
        const double a = 0.5 * Usp, b = 0.5 * Uch;
        const double ds = 1.0 - a * c0, dc = 1.0 + b * c0;
        const double num = 3.0 * Usp * a * dc - Uch * b * ds;
        return (float)(0.125 * normFact * U * c0 * c0 * num / (ds * dc));
    });
    __syncthreads();
    dct2_slice<NBK>(S32, scratch32<NBK>(S32), tws);
    for (int o = threadIdx.x; o < n8; o += blockDim.x) {
        int l, m;
        oct_lm(o, l, m);
        Vr[bidx(j, o, nb)] = S32[l * NBK + m];
    }
}

// near field of the FP32 Sigma slice: the points with both lattice
// coordinates <= R (R = kNear, or nbk - 2 on the smallest lattices, so that
// the near field never reaches the slice's last line, whose DCT-I weight
// is 1), (R + 1)(R + 2)/2 of them in the octant
constexpr int kNear = 4;

// shared memory of k_sigma_slice32: the FP32 slice plan, then the near
// field's FP64 values x(o), o < NOCT, and its partial sums u_a(k2)
template <int NBK>
struct SigmaSlice32Smem {
    static constexpr int R = kNear < NBK - 1 ? kNear : NBK - 2;
    static constexpr int NOCT = (R + 1) * (R + 2) / 2;
    static constexpr size_t near_off = (Slice32Smem<NBK>::bytes + 15) & ~(size_t)15;
    static constexpr size_t u_off = near_off + (size_t)NOCT * sizeof(double);
    static constexpr size_t bytes = u_off + (size_t)(R + 1) * NBK * sizeof(double);
};

// Sigma(k, tau_j) = DCT-I[ G(r, tau_j) V(r, tau_j) ], j = 0..Nw0, with
// V(r, tau_j) = V(r, beta - tau_j) for tau_j > beta/2 (src/green.cpp:1822-1885):
// the product in FP64 from the FP32 G; beyond the near field transformed in
// FP32, the near field's transform added in FP64 (cos(pi a t / (nbk - 1)) by
// the Chebyshev recurrence from the FP64 twiddle table entry tw64[t],
// tw64[m] = exp(-2 pi i m / L), L = 2 (nbk - 1)).
template <int NBK>
__global__ void __launch_bounds__(kSlice32Threads, 2)
    k_sigma_slice32(const float *__restrict__ Grt, const double *__restrict__ V, const float4 *__restrict__ tw,
                    const double2 *__restrict__ tw64, int n8, int nw0, int ahead, double *__restrict__ sigt, Bp b) {
    Grt = at(Grt, b.arena);
    V = at(V, b.arena);
    sigt = at(sigt, b.arena);
    constexpr int R = SigmaSlice32Smem<NBK>::R;
    constexpr int NOCT = SigmaSlice32Smem<NBK>::NOCT;
    extern __shared__ __align__(16) float S32[];
    double *xn = reinterpret_cast<double *>(reinterpret_cast<char *>(S32) + SigmaSlice32Smem<NBK>::near_off);
    double *u = reinterpret_cast<double *>(reinterpret_cast<char *>(S32) + SigmaSlice32Smem<NBK>::u_off);
    const float4 *tws = twiddles32<NBK>(S32, tw);
    const int j = blockIdx.x;
    const int nb = nw0 / 2 + 1;
    const int jv = j < nb ? j : nw0 - j;
    if (ahead > 0 && j + ahead <= nw0) {
        const int jn = j + ahead;
        prefetch_l2_range(Grt + (size_t)jn * n8, (size_t)n8 * sizeof(float));
        prefetch_l2_blockrow(V, jn < nb ? jn : nw0 - jn, nb, (n8 + 3) / 4);
    }
    // V(r, tau_j) and G(r, tau_j) staged in the slice / scratch area
    double *vs = reinterpret_cast<double *>(S32);
    float *gs = reinterpret_cast<float *>(reinterpret_cast<char *>(S32) + Stage32<NBK>::blockrow_bytes);
    stage_blockrow<NBK>(vs, V, jv, nb);
    stage_frow<NBK>(gs, Grt + (size_t)j * n8);
    cp_async_wait_all();
    __syncthreads();
    // octant points o < NOCT are exactly those with l <= R
    fill_from_staged<NBK, kSlice32Threads>(S32, [&](int o) -> float {
        const double x = (double)gs[o] * vs[o];
        if (o < NOCT) {
            xn[o] = x;
            return 0.0f;
        }
        return (float)x;
    });
    __syncthreads();
    // u_a(k2) = sum_b w_b x(a, b) cos(pi b k2 / (nbk - 1)), w_0 = 1, w_b = 2
    for (int i = threadIdx.x; i < (R + 1) * NBK; i += blockDim.x) {
        const int a = i / NBK, k2 = i % NBK;
        double cs[R + 1];
        cheb_cos<R>(__ldg(&tw64[k2]).x, cs);
        double acc = 0.0;
#pragma unroll
        for (int b = 0; b <= R; ++b) {
            const int hi = a > b ? a : b, lo = a > b ? b : a;
            const double wb = b == 0 ? 1.0 : 2.0;
            acc = fma(wb * xn[lo + hi * (hi + 1) / 2], cs[b], acc);
        }
        u[i] = acc;
    }
    // (the transform's barriers publish u)
    dct2_slice<NBK>(S32, scratch32<NBK>(S32), tws);
    for (int o = threadIdx.x; o < n8; o += blockDim.x) {
        int l, m;
        oct_lm(o, l, m);
        double cs[R + 1];
        cheb_cos<R>(__ldg(&tw64[l]).x, cs);
        double nf = u[m];
#pragma unroll
        for (int a = 1; a <= R; ++a) nf = fma(2.0 * cs[a], u[a * NBK + m], nf);
        sigt[bidx(j, o, nw0 + 1)] = (double)S32[l * NBK + m] + nf;
    }
}

// h V(r, tau) and f0 V(r, tau) of the correlator (k_cond_slice's stage,
// src/cond_opt.cpp:2696-2908) with both DST x DCT transforms in FP32: the
// slice formed in FP64 from the (x, A, B) table and rounded once, the
// product with 2 V(r, tau) formed in FP64 from the FP32 transform and rounded
// once; outputs kept in FP64 for the FP64 tau kernel.  h V enters only the
// Maki-Thompson part of chi_jj and f0 V only its q_n = 0 value.
template <int NBK>
__global__ void __launch_bounds__(kSlice32Threads, 2)
    k_cond_slice32(const double *__restrict__ tab, const double *__restrict__ V, const float4 *__restrict__ tw,
                   int nw0, double T, int K4p, double *__restrict__ hV, double *__restrict__ f0V,
                   double *__restrict__ pre) {
    constexpr int K4 = (NBK - 2) * NBK;
    extern __shared__ __align__(16) float S32[];
    const float4 *tws = twiddles32<NBK>(S32, tw);
    const int j = blockIdx.x, y = blockIdx.y;
    const int nb = nw0 / 2 + 1;
    const double t = j / (nw0 * T);
    const double bt = 1.0 / T - t;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const double2 xa = *reinterpret_cast<const double2 *>(tab + 4 * c);
        const double b = tab[4 * c + 2];
        const double E = exp(xa.x > 0 ? -xa.x * t : xa.x * bt);
        S32[c] = (float)((y == 0) ? xa.y * E : (xa.y * t + b) * E);
    }
    __syncthreads();
    dst_dct_slice<NBK>(S32, scratch32<NBK>(S32), tws);
    const int jv = j < nb ? j : nw0 - j;
    const bool edge = (j == 0 || j == nw0);
    double *pe = pre + (size_t)(2 * y + (j == nw0 ? 1 : 0)) * K4p;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const int l = c / NBK, m = c % NBK;
        const double v = S32[c];
        if (edge) pe[c] = v;
        S32[c] = (float)(v * (2.0 * V[bidx(jv, oct_index(l + 1, m), nb)]));
    }
    __syncthreads();
    dst_dct_slice<NBK>(S32, scratch32<NBK>(S32), tws);
    double *out = (y == 0) ? hV : f0V;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) out[bidx2(j, c, nw0 + 1)] = S32[c];
}

template <int NBK>
struct RunCondSlice32 {
    static cudaError_t run(const GridDev *g, const CondDev *c, const double *V, double T, int ny, cudaStream_t st) {
        const size_t sm = Slice32Smem<NBK>::bytes;
        cudaError_t e = set_smem(k_cond_slice32<NBK>, sm);
        if (e != cudaSuccess) return e;
        k_cond_slice32<NBK><<<dim3(g->nw0 + 1, ny), kSlice32Threads, sm, st>>>(c->tab, V, g->tw_k32, g->nw0, T,
                                                                               c->K4p, c->hV, c->f0V, c->pre);
        return launched();
    }
};

// (a batched launch, b.P > 1, skips the L2 prefetch of the slice ahead: its
// blocks of one slice index belong to different points)
template <int NBK>
struct RunGslice32 {
    static cudaError_t run(const GridDev *g, float *Grt, double mu0, double T, const Bp *b, cudaStream_t st) {
        const int plan = slice_plan(kSliceG, NBK);
        if (plan == kSliceDirect && g->dct32) return launch_gslice_dct(*g, Grt, mu0, T, st, *b);
        const size_t sm = Slice32Smem<NBK>::bytes;
        cudaError_t e = set_smem(k_gslice32<NBK>, sm);
        if (e != cudaSuccess) return e;
        if ((e = launch_gk_table(*g, mu0, T, st, *b)) != cudaSuccess) return e;
        k_gslice32<NBK><<<dim3(g->nw0 + 1, 1, b->P), kSlice32Threads, sm, st>>>(g->gk, g->tw_k32, g->n8, g->nw0, T,
                                                                               Grt, *b);
        return launched();
    }
};
template <int NBK>
struct RunChi0Slice32 {
    static cudaError_t run(const GridDev *g, const float *Grt, double *chirt, double *chiq, const Bp *b,
                           cudaStream_t st) {
        const int plan = slice_plan(kSliceChi0, NBK);
        if (plan == kSliceDirect && g->dct32) return launch_chi0_slice_dct(*g, Grt, chirt, chiq, st, *b);
        const size_t sm = Slice32Smem<NBK>::bytes;
        cudaError_t e = set_smem(k_chi0_slice32<NBK>, sm);
        if (e != cudaSuccess) return e;
        const int ahead = b->P > 1 ? 0 : resident_ctas(k_chi0_slice32<NBK>, kSlice32Threads, sm);
        k_chi0_slice32<NBK><<<dim3(g->nb, 1, b->P), kSlice32Threads, sm, st>>>(Grt, g->tw_k32, g->n8, g->nw0, ahead,
                                                                              chirt, chiq, *b);
        return launched();
    }
};
template <int NBK>
struct RunVertexQ32 {
    static cudaError_t run(const GridDev *g, const double *chiq, double *Vr, double U, const double *Usc, double T,
                           const Bp *b, cudaStream_t st) {
        const int plan = slice_plan(kSliceVertex, NBK);
        if (plan == kSliceTensor && g->dct_tc) return launch_vertex_q_tc(*g, chiq, Vr, U, Usc, T, st, *b);
        if (plan == kSliceDirect && g->dct32) return launch_vertex_q_dct(*g, chiq, Vr, U, Usc, T, st, *b);
        const size_t sm = Slice32Smem<NBK>::bytes;
        cudaError_t e = set_smem(k_vertex_q32<NBK>, sm);
        if (e != cudaSuccess) return e;
        const double normFact = T / ((double)g->nk0 * g->nk0);
        const int ahead = b->P > 1 ? 0 : resident_ctas(k_vertex_q32<NBK>, kSlice32Threads, sm);
        k_vertex_q32<NBK><<<dim3(g->nb, 1, b->P), kSlice32Threads, sm, st>>>(chiq, g->tw_k32, g->n8, g->nb, ahead,
                                                                            normFact, U, Usc, Vr, *b);
        return launched();
    }
};

template <int NBK>
struct RunSigmaSlice32 {
    static cudaError_t run(const GridDev *g, const float *Grt, const double *V, double *sigt, const Bp *b,
                           cudaStream_t st) {
        const int plan = slice_plan(kSliceSigma, NBK);
        if (plan == kSliceTensor && g->dct_tc) return launch_sigma_slice_tc(*g, Grt, V, sigt, st, *b);
        if (plan == kSliceDirect && g->dct32) return launch_sigma_slice_dct(*g, Grt, V, sigt, st, *b);
        const size_t sm = SigmaSlice32Smem<NBK>::bytes;
        cudaError_t e = set_smem(k_sigma_slice32<NBK>, sm);
        if (e != cudaSuccess) return e;
        const int ahead = b->P > 1 ? 0 : resident_ctas(k_sigma_slice32<NBK>, kSlice32Threads, sm);
        k_sigma_slice32<NBK><<<dim3(g->nw0 + 1, 1, b->P), kSlice32Threads, sm, st>>>(Grt, V, g->tw_k32, g->tw_k, g->n8,
                                                                                    g->nw0, ahead, sigt, *b);
        return launched();
    }
};

}  // namespace

cudaError_t launch_cond_slice32(const GridDev &g, const CondDev &c, const double *V, double T, int ny,
                                cudaStream_t st) {
    return dispatch_nbk<RunCondSlice32>(g.nbk, &g, &c, V, T, ny, st);
}

cudaError_t launch_sigma_slice32(const GridDev &g, const float *Grt, const double *V, double *sigt, cudaStream_t st,
                                 const Bp &b) {
    return dispatch_nbk<RunSigmaSlice32>(g.nbk, &g, Grt, V, sigt, &b, st);
}

cudaError_t launch_gslice32(const GridDev &g, float *Grt, double mu0, double T, cudaStream_t st, const Bp &b) {
    return dispatch_nbk<RunGslice32>(g.nbk, &g, Grt, mu0, T, &b, st);
}

cudaError_t launch_chi0_slice32(const GridDev &g, const float *Grt, double *chirt, double *chiq, cudaStream_t st,
                                const Bp &b) {
    return dispatch_nbk<RunChi0Slice32>(g.nbk, &g, Grt, chirt, chiq, &b, st);
}

cudaError_t launch_vertex_q32(const GridDev &g, const double *chiq, double *Vr, double U, const double *Usc, double T,
                              cudaStream_t st, const Bp &b) {
    return dispatch_nbk<RunVertexQ32>(g.nbk, &g, chiq, Vr, U, Usc, T, &b, st);
}

}  // namespace tpsc
