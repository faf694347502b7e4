// tpsc_direct.cu -- slice kernels of the mixed form on the folded matrix
// DCT-I (tpsc_dct.cuh): the "direct" slice plan.
//
// k_sigma_slice_dct: Sigma(k, tau_j) = DCT-I[ G(r, tau_j) V(r, tau_j) ], the
// stage of src/green.cpp:1822-1885, for the slices j and Nw0 - j together:
// both use the same V(r, tau_j) row (V(r, beta - tau) = V(r, tau)), which is
// then read once.  The product is formed in FP64 from the FP32 G; the near
// field |rx|, |ry| <= 4 is transformed in FP64 (its values dominate the
// product, and their FP32 rounding would survive the tau integral), the rest
// by the FP32 matrix DCT.  The kernel is persistent: one CTA per SM keeps the
// DCT tables in shared memory and walks the slice pairs (of every point of a
// batched launch), prefetching the next pair's rows into L2.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <atomic>
#include <vector>

#include "tpsc_dct.cuh"

namespace tpsc {

// slice plan per kind (kSliceG, kSliceChi0, kSliceVertex, kSliceSigma) and
// lattice: 0 = the library default, else 1 + plan
static std::atomic<int> g_slice_plan[4][8];
static int plan_index(int nbk) {
    int k = 0;
    while ((1 << k) < nbk - 1 && k < 7) ++k;
    return k;
}
int slice_plan(int kind, int nbk) {
    const int v = g_slice_plan[kind][plan_index(nbk)].load(std::memory_order_relaxed);
    if (v > 0) return v - 1;
    (void)kind;
    return kSliceFft;
}
void set_slice_plan(int kind, int nbk, int plan) {
    if (g_slice_plan[kind][plan_index(nbk)].exchange(plan + 1) != plan + 1) bump_plans_version();
}
bool slice_plan_supported(int kind, int plan, int nbk) {
    if (plan == kSliceFft) return true;
    if (plan == kSliceDirect) return nbk == 33 || nbk == 65 || nbk == 129;
    // the tensor plan for the Sigma and V slices only: on the G and chi0
    // slices, whose values have no large near field split off, its 3xTF32
    // products leave chi0 8e-7 and Sigma 1e-6 to 3e-6 from FP64 (the FFT
    // plan: 1e-7, 5e-7), outside the mixed form's bound
    return plan == kSliceTensor && (kind == kSliceSigma || kind == kSliceVertex) && nbk == 129;
}

// KsT[k][n] = w_k cos(pi k n / H) (rows k <= H) and KdT[k][n] = w_k cos(pi k (2n + 1) / N)
// (rows H + 1 + k, k < H), rows of H + 4 floats, w_0 = 1, w_k = 2: each angle
// reduced exactly (the integer product modulo the period) and its cosine
// taken in long double, then rounded once
void dct_table(int nbk, std::vector<float> &out) {
    out.clear();
    if (!slice_plan_supported(kSliceG, kSliceDirect, nbk)) return;
    const int N = nbk - 1, H = N / 2, LD = H + 4;
    const long double pi = 3.141592653589793238462643383279502884L;
    out.assign((size_t)(2 * H + 1) * LD, 0.0f);
    for (int k = 0; k <= H; ++k)
        for (int n = 0; n <= H; ++n)
            out[(size_t)k * LD + n] = (float)((k == 0 ? 1.0L : 2.0L) * cosl(pi * ((k * n) % (2 * H)) / H));
    for (int k = 0; k < H; ++k)
        for (int n = 0; n < H; ++n)
            out[(size_t)(H + 1 + k) * LD + n] =
                (float)((k == 0 ? 1.0L : 2.0L) * cosl(pi * ((k * (2 * n + 1)) % (2 * N)) / N));
}

namespace {

// point p's copy of a per-point array of a batched launch (see Bp)
template <class T>
__device__ __forceinline__ T *at_point(T *ptr, long long arena, int p) {
    using Ch = typename std::conditional<std::is_const<T>::value, const char, char>::type;
    return reinterpret_cast<T *>(reinterpret_cast<Ch *>(ptr) + (long long)p * arena);
}

// point p's scalar `slot` of a batched launch, or v for a plain launch
__device__ __forceinline__ double bpar_point(const Bp &b, int slot, double v, int p) {
    return b.pp ? at_point(b.pp, b.arena, p)[slot] : v;
}

constexpr int kNearDirect = 4;  // near field |rx|, |ry| <= 4 in FP64

// shared memory of the one-slice kernels (G, chi0, V): tables, F, T; their
// raw inputs are staged over F and T, the slice's values written to T
template <int H>
struct SliceDctSmem {
    using P = DctPlan<H>;
    static constexpr int N8 = P::N8, N8P = (N8 + 3) & ~3;
    static constexpr size_t f_off = (size_t)P::TAB * 4;
    static constexpr size_t t_off = f_off + (size_t)P::REG * 4;
    static constexpr size_t bytes = t_off + (size_t)P::REG * 4;
    static_assert((size_t)N8P * 8 <= 2 * (size_t)P::REG * 4, "raw inputs must fit over F and T");
};

template <int H>
__device__ __forceinline__ void load_dct_tables(float *tabs, const float *__restrict__ tab) {
    for (int i = threadIdx.x; i < DctPlan<H>::TAB / 4; i += blockDim.x) cp_async16(tabs + 4 * i, tab + 4 * i);
}

template <int H>
struct SigmaDctSmem {
    using P = DctPlan<H>;
    static constexpr int NBK = P::NBK, N8 = P::N8, N8P = (N8 + 3) & ~3;
    static constexpr int R = kNearDirect < NBK - 1 ? kNearDirect : NBK - 2;
    static constexpr int NOCT = (R + 1) * (R + 2) / 2;  // octant points with l <= R
    static_assert(NOCT <= 16, "near field");
    static constexpr size_t f_off = (size_t)P::TAB * 4;
    static constexpr size_t t_off = f_off + (size_t)P::REG * 4;
    static constexpr size_t x2_off = t_off + (size_t)P::REG * 4;
    static constexpr size_t xn_off = x2_off + (((size_t)N8 * 4 + 15) & ~(size_t)15);
    static constexpr size_t u_off = xn_off + 2 * 16 * sizeof(double);
    static constexpr size_t bytes = u_off + (size_t)2 * (R + 1) * NBK * sizeof(double);
    // the raw inputs of a pair (V block row, two FP32 G rows) staged over F, T and X2
    static constexpr size_t raw_bytes = (size_t)N8P * 8 + (size_t)2 * N8 * 4;
    static_assert(raw_bytes <= xn_off - f_off, "raw inputs must fit over F, T and X2");
    static_assert(P::N8 <= P::REG, "the first slice's values must fit in T");
};

template <int N8>
__device__ __forceinline__ void stage_frow32(float *dst, const float *__restrict__ src) {
    for (int o = threadIdx.x; o < N8; o += blockDim.x) cp_async4(dst + o, src + o);
}

template <int H>
__global__ void __launch_bounds__(kDctThreads, 1)
    k_sigma_slice_dct(const float *__restrict__ Grt, const double *__restrict__ V, const float *__restrict__ tab,
                      const double2 *__restrict__ tw64, int nw0, double *__restrict__ sigt, Bp b) {
    using P = DctPlan<H>;
    using SM = SigmaDctSmem<H>;
    constexpr int NBK = P::NBK, N8 = P::N8, R = SM::R, NOCT = SM::NOCT;
    constexpr int PER = (N8 + kDctThreads - 1) / kDctThreads;
    extern __shared__ __align__(16) unsigned char smem[];
    float *tabs = reinterpret_cast<float *>(smem);
    float *F = reinterpret_cast<float *>(smem + SM::f_off);
    float *Tr = reinterpret_cast<float *>(smem + SM::t_off);
    float *X2 = reinterpret_cast<float *>(smem + SM::x2_off);
    double *xn = reinterpret_cast<double *>(smem + SM::xn_off);
    double *u = reinterpret_cast<double *>(smem + SM::u_off);
    const int tid = threadIdx.x;
    // the DCT tables, once per CTA (waited for with the first pair's inputs)
    for (int i = tid; i < P::TAB / 4; i += blockDim.x) cp_async16(tabs + 4 * i, tab + 4 * i);
    const int nb = nw0 / 2 + 1;
    const long long items = (long long)nb * b.P;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int p = (int)(it / nb), j = (int)(it % nb);
        const float *G = at_point(Grt, b.arena, p);
        const double *Vp = at_point(V, b.arena, p);
        double *out = at_point(sigt, b.arena, p);
        const int j2 = nw0 - j;
        const bool two = j2 != j;
        const long long nx = it + gridDim.x;
        if (nx < items) {
            const int pn = (int)(nx / nb), jn = (int)(nx % nb);
            const float *Gn = at_point(Grt, b.arena, pn);
            prefetch_l2_blockrow(at_point(V, b.arena, pn), jn, nb, SM::N8P / 4);
            prefetch_l2_range(Gn + (size_t)jn * N8, (size_t)N8 * sizeof(float));
            if (nw0 - jn != jn) prefetch_l2_range(Gn + (size_t)(nw0 - jn) * N8, (size_t)N8 * sizeof(float));
        }
        __syncthreads();  // the previous pair's reads of F are done
        double *vs = reinterpret_cast<double *>(F);
        float *g1 = reinterpret_cast<float *>(vs + SM::N8P);
        float *g2 = g1 + N8;
        stage_blockrow<NBK>(vs, Vp, j, nb);
        stage_frow32<N8>(g1, G + (size_t)j * N8);
        if (two) stage_frow32<N8>(g2, G + (size_t)j2 * N8);
        cp_async_wait_all();
        __syncthreads();
        // the products G V in FP64; the near field kept in FP64, the rest rounded once
        float r1[PER], r2[PER];
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int o = tid + i * kDctThreads;
            r1[i] = 0.0f;
            r2[i] = 0.0f;
            if (o < N8) {
                const double v = vs[o];
                const double x1 = (double)g1[o] * v;
                const double x2 = two ? (double)g2[o] * v : 0.0;
                if (o < NOCT) {
                    xn[o] = x1;
                    xn[16 + o] = x2;
                } else {
                    r1[i] = (float)x1;
                    r2[i] = (float)x2;
                }
            }
        }
        __syncthreads();
        float *xs1 = Tr;
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int o = tid + i * kDctThreads;
            if (o < N8) {
                xs1[o] = r1[i];
                X2[o] = r2[i];
            }
        }
        __syncthreads();
        for (int s = 0; s < (two ? 2 : 1); ++s) {
            const double *xns = xn + 16 * s;
            double *us = u + s * (R + 1) * NBK;
            // near field: u_a(k2) = sum_b w_b x(a, b) cos(pi b k2 / N), w_0 = 1, w_b = 2
            for (int i = tid; i < (R + 1) * NBK; i += blockDim.x) {
                const int a = i / NBK, k2 = i % NBK;
                double cs[R + 1];
                cheb_cos<R>(__ldg(&tw64[k2]).x, cs);
                double acc = 0.0;
#pragma unroll
                for (int c = 0; c <= R; ++c) {
                    const int hi = a > c ? a : c, lo = a > c ? c : a;
                    const double wb = c == 0 ? 1.0 : 2.0;
                    acc = fma(wb * xns[lo + hi * (hi + 1) / 2], cs[c], acc);
                }
                us[i] = acc;
            }
            // (the transform's barriers publish u)
            dct2_direct<H>(s ? X2 : xs1, F, Tr, tabs);
            const int js = s ? j2 : j;
            for (int o = tid; o < N8; o += blockDim.x) {
                int l, m;
                oct_lm(o, l, m);
                double cs[R + 1];
                cheb_cos<R>(__ldg(&tw64[l]).x, cs);
                double nf = us[m];
#pragma unroll
                for (int a = 1; a <= R; ++a) nf = fma(2.0 * cs[a], us[a * NBK + m], nf);
                out[bidx(js, o, nw0 + 1)] = (double)dct_z<H>(F, l, m) + nf;
            }
            if (s == 0 && two) __syncthreads();  // the next fold overwrites F
        }
    }
}

// G(r, tau_j) = DCT-I[ G0(k, tau_j) / L^2 ] (k_gslice32's stage, src/green.cpp:1830-1841
// and src/chi0.cpp:462-495): G0 formed in FP64 from the (eps - mu0, prefactor)
// table, rounded once; the transform FP32; Grt32[j n8 + o]
template <int H>
__global__ void __launch_bounds__(kDctThreads, 1)
    k_gslice_dct(const double2 *__restrict__ gk, const float *__restrict__ tab, int nw0, double T,
                 float *__restrict__ Grt, Bp b) {
    using P = DctPlan<H>;
    using SM = SliceDctSmem<H>;
    constexpr int N8 = P::N8;
    extern __shared__ __align__(16) unsigned char smem[];
    float *tabs = reinterpret_cast<float *>(smem);
    float *F = reinterpret_cast<float *>(smem + SM::f_off);
    float *Tr = reinterpret_cast<float *>(smem + SM::t_off);
    load_dct_tables<H>(tabs, tab);
    cp_async_wait_all();
    const long long items = (long long)(nw0 + 1) * b.P;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int p = (int)(it / (nw0 + 1)), j = (int)(it % (nw0 + 1));
        const double2 *gkp = at_point(gk, b.arena, p);
        float *out = at_point(Grt, b.arena, p) + (size_t)j * N8;
        const double Tp = bpar_point(b, kPpT, T, p);
        const double t = j / (nw0 * Tp);
        const double bt = 1.0 / Tp - t;
        __syncthreads();  // the previous slice's reads of F and T are done
        for (int o = threadIdx.x; o < N8; o += blockDim.x) {
            const double2 c = __ldg(&gkp[o]);
            Tr[o] = (float)(c.y * exp((c.x > 0 ? -t : bt) * c.x));
        }
        __syncthreads();
        dct2_direct<H>(Tr, F, Tr, tabs);
        for (int o = threadIdx.x; o < N8; o += blockDim.x) {
            int l, m;
            oct_lm(o, l, m);
            out[o] = dct_z<H>(F, l, m);
        }
    }
}

// chi0(r, tau_j) = -2 G(r, tau_j) G(r, -tau_j) in FP64 from the FP32 G (kept in
// FP64 for the tau transforms), its DCT-I in FP32 -> chi0(q, tau_j) in FP64
// (k_chi0_slice32's stage, src/chi0.cpp:393-418, 497-517, 545-558)
template <int H>
__global__ void __launch_bounds__(kDctThreads, 1)
    k_chi0_slice_dct(const float *__restrict__ Grt, const float *__restrict__ tab, int nw0,
                     double *__restrict__ chirt, double *__restrict__ chiq, Bp b) {
    using P = DctPlan<H>;
    using SM = SliceDctSmem<H>;
    constexpr int N8 = P::N8;
    constexpr int PER = (N8 + kDctThreads - 1) / kDctThreads;
    extern __shared__ __align__(16) unsigned char smem[];
    float *tabs = reinterpret_cast<float *>(smem);
    float *F = reinterpret_cast<float *>(smem + SM::f_off);
    float *Tr = reinterpret_cast<float *>(smem + SM::t_off);
    load_dct_tables<H>(tabs, tab);
    const int nb = nw0 / 2 + 1;
    const long long items = (long long)nb * b.P;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int p = (int)(it / nb), j = (int)(it % nb);
        const float *G = at_point(Grt, b.arena, p);
        double *cr = at_point(chirt, b.arena, p);
        double *cq = at_point(chiq, b.arena, p);
        const long long nx = it + gridDim.x;
        if (nx < items) {
            const int pn = (int)(nx / nb), jn = (int)(nx % nb);
            const float *Gn = at_point(Grt, b.arena, pn);
            prefetch_l2_range(Gn + (size_t)jn * N8, (size_t)N8 * sizeof(float));
            prefetch_l2_range(Gn + (size_t)(nw0 - jn) * N8, (size_t)N8 * sizeof(float));
        }
        __syncthreads();  // the previous slice's reads of F are done
        float *gp = F;
        float *gm = F + SM::N8P;
        stage_frow32<N8>(gp, G + (size_t)j * N8);
        stage_frow32<N8>(gm, G + (size_t)(nw0 - j) * N8);
        cp_async_wait_all();
        __syncthreads();
        float v[PER];
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int o = threadIdx.x + i * kDctThreads;
            v[i] = 0.0f;
            if (o < N8) {
                const double a = gp[o];
                double c;
                if (j == 0)
                    c = (o == 0) ? -2.0 * a * (a + 1.0) : -2.0 * a * a;
                else if (j == nb - 1)
                    c = 2.0 * a * a;
                else
                    c = -2.0 * (-(double)gm[o]) * a;
                cr[bidx(j, o, nb)] = c;
                v[i] = (float)c;
            }
        }
        __syncthreads();  // the staged rows reach into T
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int o = threadIdx.x + i * kDctThreads;
            if (o < N8) Tr[o] = v[i];
        }
        __syncthreads();
        dct2_direct<H>(Tr, F, Tr, tabs);
        for (int o = threadIdx.x; o < N8; o += blockDim.x) {
            int l, m;
            oct_lm(o, l, m);
            cq[bidx(j, o, nb)] = dct_z<H>(F, l, m);
        }
    }
}

// V(q, iqn) in FP64 from chi0(q, iqn), its DCT-I over q in FP32 (k_vertex_q32's
// stage, src/chi.cpp:89-115); with a = Usp/2, b = Uch/2 one FP64 division per point
template <int H>
__global__ void __launch_bounds__(kDctThreads, 1)
    k_vertex_q_dct(const double *__restrict__ chiq, const float *__restrict__ tab, int nb, double normFact, double U,
                   const double *__restrict__ Usc, double *__restrict__ Vr, Bp b) {
    using P = DctPlan<H>;
    using SM = SliceDctSmem<H>;
    constexpr int NBK = P::NBK, N8 = P::N8;
    constexpr int PER = (N8 + kDctThreads - 1) / kDctThreads;
    extern __shared__ __align__(16) unsigned char smem[];
    float *tabs = reinterpret_cast<float *>(smem);
    float *F = reinterpret_cast<float *>(smem + SM::f_off);
    float *Tr = reinterpret_cast<float *>(smem + SM::t_off);
    load_dct_tables<H>(tabs, tab);
    const long long items = (long long)nb * b.P;
    for (long long it = blockIdx.x; it < items; it += gridDim.x) {
        const int p = (int)(it / nb), j = (int)(it % nb);
        const double *cq = at_point(chiq, b.arena, p);
        const double *us = at_point(Usc, b.arena, p);
        double *out = at_point(Vr, b.arena, p);
        const double nf = bpar_point(b, kPpNormFact, normFact, p);
        const double Up = bpar_point(b, kPpU, U, p);
        const long long nx = it + gridDim.x;
        if (nx < items) {
            const int pn = (int)(nx / nb), jn = (int)(nx % nb);
            prefetch_l2_blockrow(at_point(chiq, b.arena, pn), jn, nb, SM::N8P / 4);
        }
        const double Usp = us[0], Uch = us[1];
        __syncthreads();  // the previous slice's reads of F and T are done
        double *cs = reinterpret_cast<double *>(F);  // N8P doubles over F and the start of T
        stage_blockrow<NBK>(cs, cq, j, nb);
        cp_async_wait_all();
        __syncthreads();
        float v[PER];
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int o = threadIdx.x + i * kDctThreads;
            v[i] = 0.0f;
            if (o < N8) {
                const double c0 = cs[o];
                const double a = 0.5 * Usp, bb = 0.5 * Uch;
                const double ds = 1.0 - a * c0, dc = 1.0 + bb * c0;
                const double num = 3.0 * Usp * a * dc - Uch * bb * ds;
                v[i] = (float)(0.125 * nf * Up * c0 * c0 * num / (ds * dc));
            }
        }
        __syncthreads();  // the staged row overlaps T
#pragma unroll
        for (int i = 0; i < PER; ++i) {
            const int o = threadIdx.x + i * kDctThreads;
            if (o < N8) Tr[o] = v[i];
        }
        __syncthreads();
        dct2_direct<H>(Tr, F, Tr, tabs);
        for (int o = threadIdx.x; o < N8; o += blockDim.x) {
            int l, m;
            oct_lm(o, l, m);
            out[bidx(j, o, nb)] = dct_z<H>(F, l, m);
        }
    }
}

template <class K>
cudaError_t persistent_launch_config(K kernel, size_t sm, long long items, int *grid) {
    cudaError_t e = set_smem(kernel, sm);
    if (e != cudaSuccess) return e;
    const int ctas = resident_ctas(kernel, kDctThreads, sm);
    if (ctas <= 0) return cudaErrorInvalidConfiguration;
    *grid = (int)(items < ctas ? items : ctas);
    return cudaSuccess;
}

template <int H>
cudaError_t run_gslice_dct(const GridDev &g, float *Grt, double T, const Bp &b, cudaStream_t st) {
    int grid = 0;
    const size_t sm = SliceDctSmem<H>::bytes;
    cudaError_t e = persistent_launch_config(k_gslice_dct<H>, sm, (long long)(g.nw0 + 1) * b.P, &grid);
    if (e != cudaSuccess) return e;
    k_gslice_dct<H><<<grid, kDctThreads, sm, st>>>(g.gk, g.dct32, g.nw0, T, Grt, b);
    return launched();
}
template <int H>
cudaError_t run_chi0_slice_dct(const GridDev &g, const float *Grt, double *chirt, double *chiq, const Bp &b,
                               cudaStream_t st) {
    int grid = 0;
    const size_t sm = SliceDctSmem<H>::bytes;
    cudaError_t e = persistent_launch_config(k_chi0_slice_dct<H>, sm, (long long)g.nb * b.P, &grid);
    if (e != cudaSuccess) return e;
    k_chi0_slice_dct<H><<<grid, kDctThreads, sm, st>>>(Grt, g.dct32, g.nw0, chirt, chiq, b);
    return launched();
}
template <int H>
cudaError_t run_vertex_q_dct(const GridDev &g, const double *chiq, double *Vr, double U, const double *Usc, double T,
                             const Bp &b, cudaStream_t st) {
    int grid = 0;
    const size_t sm = SliceDctSmem<H>::bytes;
    cudaError_t e = persistent_launch_config(k_vertex_q_dct<H>, sm, (long long)g.nb * b.P, &grid);
    if (e != cudaSuccess) return e;
    const double normFact = T / ((double)g.nk0 * g.nk0);
    k_vertex_q_dct<H><<<grid, kDctThreads, sm, st>>>(chiq, g.dct32, g.nb, normFact, U, Usc, Vr, b);
    return launched();
}

template <int H>
cudaError_t run_sigma_slice_dct(const GridDev &g, const float *Grt, const double *V, double *sigt, const Bp &b,
                                cudaStream_t st) {
    const size_t sm = SigmaDctSmem<H>::bytes;
    cudaError_t e = set_smem(k_sigma_slice_dct<H>, sm);
    if (e != cudaSuccess) return e;
    const long long items = (long long)g.nb * b.P;
    int ctas = resident_ctas(k_sigma_slice_dct<H>, kDctThreads, sm);
    if (ctas <= 0) return cudaErrorInvalidConfiguration;
    const int grid = (int)(items < ctas ? items : ctas);
    k_sigma_slice_dct<H><<<grid, kDctThreads, sm, st>>>(Grt, V, g.dct32, g.tw_k, g.nw0, sigt, b);
    return launched();
}

}  // namespace

cudaError_t launch_gslice_dct(const GridDev &g, float *Grt, double mu0, double T, cudaStream_t st, const Bp &b) {
    if (!g.dct32) return cudaErrorInvalidValue;
    cudaError_t e = launch_gk_table(g, mu0, T, st, b);
    if (e != cudaSuccess) return e;
    switch (g.nbk) {
        case 33: return run_gslice_dct<16>(g, Grt, T, b, st);
        case 65: return run_gslice_dct<32>(g, Grt, T, b, st);
        case 129: return run_gslice_dct<64>(g, Grt, T, b, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_chi0_slice_dct(const GridDev &g, const float *Grt, double *chirt, double *chiq, cudaStream_t st,
                                  const Bp &b) {
    if (!g.dct32) return cudaErrorInvalidValue;
    switch (g.nbk) {
        case 33: return run_chi0_slice_dct<16>(g, Grt, chirt, chiq, b, st);
        case 65: return run_chi0_slice_dct<32>(g, Grt, chirt, chiq, b, st);
        case 129: return run_chi0_slice_dct<64>(g, Grt, chirt, chiq, b, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_vertex_q_dct(const GridDev &g, const double *chiq, double *Vr, double U, const double *Usc,
                                double T, cudaStream_t st, const Bp &b) {
    if (!g.dct32) return cudaErrorInvalidValue;
    switch (g.nbk) {
        case 33: return run_vertex_q_dct<16>(g, chiq, Vr, U, Usc, T, b, st);
        case 65: return run_vertex_q_dct<32>(g, chiq, Vr, U, Usc, T, b, st);
        case 129: return run_vertex_q_dct<64>(g, chiq, Vr, U, Usc, T, b, st);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_sigma_slice_dct(const GridDev &g, const float *Grt, const double *V, double *sigt,
                                   cudaStream_t st, const Bp &b) {
    if (!g.dct32) return cudaErrorInvalidValue;
    switch (g.nbk) {
        case 33: return run_sigma_slice_dct<16>(g, Grt, V, sigt, b, st);
        case 65: return run_sigma_slice_dct<32>(g, Grt, V, sigt, b, st);
        case 129: return run_sigma_slice_dct<64>(g, Grt, V, sigt, b, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace tpsc
