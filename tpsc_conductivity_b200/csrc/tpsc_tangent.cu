// tpsc_tangent.cu -- forward tangents of the chi0 stage (the differentiation
// form): directional derivatives of chi0(q, iqn) with respect to the band
// energies xi_k = eps_k - mu0, in FP64.
//
// The chi0 stage (src/chi0.cpp:279-718) is linear in G after its one product
// chi0(r, tau) = -2 G(r, tau) G(r, -tau), and G0(k, tau) depends on the
// parameters only through xi_k:
//   dG0(k, tau) / dxi = G0(k, tau) (beta f(xi) - tau),   f = Fermi function,
// so the tangent runs the same transforms on
//   dG(r, tau) = DCT-I[ G0 (beta f - tau) dxi / L^2 ],
//   dchi0(r, tau) = -2 [dG(tau) G(-tau) + G(tau) dG(-tau)],
// the tau -> iqn transform (linear, the primal kernel) and the tangent of the
// left end condition d/dtau chi0(q, 0).  The parameter directions (U, a shift
// of mu0, t') and the sum-rule roots' derivatives are assembled on the host
// (tpsc_engine.cpp, tpsc_sumrule_tangents).
#include <cuda_runtime.h>
#include <stdint.h>

#include "tpsc_device.cuh"

namespace tpsc {

namespace {

// the tangent of k_gslice: fd[o] = (beta f(xi_o), dxi_o); dGrt[j * n8 + o]
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_gslice_tan(const double2 *__restrict__ gk, const double2 *__restrict__ fd, const double2 *__restrict__ tw,
                 int n8, int nw0, double T, double *__restrict__ dGrt) {
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int j = blockIdx.x;
    const double t = j / (nw0 * T);
    const double bt = 1.0 / T - t;
    fill_octant<NBK>(S, n8, [&](int o) -> double {
        const double2 c = __ldg(&gk[o]);
        const double2 q = __ldg(&fd[o]);
        return c.y * exp((c.x > 0 ? -t : bt) * c.x) * (q.x - t) * q.y;
    });
    __syncthreads();
    dct2_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    double *out = dGrt + (size_t)j * n8;
    for (int o = threadIdx.x; o < n8; o += blockDim.x) {
        int l, m;
        oct_lm(o, l, m);
        out[o] = S[l * NBK + m];
    }
}

// the tangent of k_chi0_slice (the product rule on each of its three forms)
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_chi0_slice_tan(const double *__restrict__ Grt, const double *__restrict__ dGrt,
                     const double2 *__restrict__ tw, int n8, int nw0, double *__restrict__ dchiq) {
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int j = blockIdx.x;
    const int nb = nw0 / 2 + 1;
    const double *gp = Grt + (size_t)j * n8, *dgp = dGrt + (size_t)j * n8;
    const double *gm = Grt + (size_t)(nw0 - j) * n8, *dgm = dGrt + (size_t)(nw0 - j) * n8;
    fill_octant<NBK>(S, n8, [&](int o) -> double {
        const double a = gp[o], da = dgp[o];
        if (j == 0) return (o == 0) ? -2.0 * da * (2.0 * a + 1.0) : -4.0 * a * da;
        if (j == nb - 1) return 4.0 * a * da;
        return 2.0 * (dgm[o] * a + gm[o] * da);
    });
    __syncthreads();
    dct2_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    for (int o = threadIdx.x; o < n8; o += blockDim.x) {
        int l, m;
        oct_lm(o, l, m);
        dchiq[bidx(j, o, nb)] = S[l * NBK + m];
    }
}

// the tangent of k_chi0_boundary: d of d/dtau G(r, 0+) = DCT-I[-(dxi G0 + xi
// dG0)(k, 0+) / L^2], of d/dtau G(r, 0-) = (hopping or -mu0) - d/dtau G(r, 0+),
// and of d/dtau chi0(r, 0) by the product rule, then its DCT-I.  der[o] and
// dmu0 are the directions of the hopping table and of mu0.  One CTA.
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_chi0_boundary_tan(const double *__restrict__ ek, const double *__restrict__ er, const double *__restrict__ der,
                        const double2 *__restrict__ fd, const double2 *__restrict__ tw, const double *__restrict__ Grt,
                        const double *__restrict__ dGrt, const double *__restrict__ dG0p, int n8, double mu0,
                        double dmu0, double T, double nk02, double *__restrict__ d_dtau_chiqt0,
                        double *__restrict__ out_ddG0p, double *__restrict__ out_ddchir) {
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    for (int o = threadIdx.x; o < n8; o += blockDim.x) {
        int l, m;
        oct_lm(o, l, m);
        const double x = ek[o] - mu0;
        const double gkt = -1.0 / (exp(-x / T) + 1.0);
        const double2 q = fd[o];
        put_sym<NBK>(S, l, m, -(q.y * gkt + x * gkt * q.x * q.y) / nk02);
    }
    __syncthreads();
    dct2_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    constexpr int NR = (NBK * (NBK + 1) / 2 + kSliceThreads - 1) / kSliceThreads;
    double dc_[NR];
    int k = 0;
    for (int o = threadIdx.x; o < n8; o += blockDim.x, ++k) {
        int l, m;
        oct_lm(o, l, m);
        const double ddp = S[l * NBK + m];
        const double dp = dG0p[o];
        const double dm = ((o == 0) ? -mu0 : er[o]) - dp;
        const double ddm = ((o == 0) ? -dmu0 : der[o]) - ddp;
        const double g0 = Grt[o], dg0 = dGrt[o];
        dc_[k] = (o == 0) ? -2.0 * (ddp * (1.0 + g0) + dp * dg0 + ddm * g0 + dm * dg0)
                          : -2.0 * (ddp * g0 + dp * dg0 + ddm * g0 + dm * dg0);
        if (out_ddG0p) out_ddG0p[o] = ddp;
        if (out_ddchir) out_ddchir[o] = dc_[k];
    }
    __syncthreads();
    k = 0;
    for (int o = threadIdx.x; o < n8; o += blockDim.x, ++k) {
        int l, m;
        oct_lm(o, l, m);
        put_sym<NBK>(S, l, m, dc_[k]);
    }
    __syncthreads();
    dct2_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    for (int o = threadIdx.x; o < n8; o += blockDim.x) {
        int l, m;
        oct_lm(o, l, m);
        d_dtau_chiqt0[o] = S[l * NBK + m];
    }
}

template <int NBK>
struct RunChi0Tan {
    static cudaError_t run(const GridDev *g, const TangentBufs *t, double mu0, double dmu0, double T,
                           cudaStream_t st) {
        const size_t sm = SliceSmem<NBK>::bytes;
        cudaError_t e;
        if ((e = set_smem(k_gslice_tan<NBK>, sm)) != cudaSuccess) return e;
        if ((e = set_smem(k_chi0_slice_tan<NBK>, sm)) != cudaSuccess) return e;
        if ((e = set_smem(k_chi0_boundary_tan<NBK>, sm)) != cudaSuccess) return e;
        const double nk02 = (double)g->nk0 * g->nk0;
        k_gslice_tan<NBK><<<g->nw0 + 1, kSliceThreads, sm, st>>>(g->gk, t->fd, g->tw_k, g->n8, g->nw0, T, t->dGrt);
        if ((e = launched()) != cudaSuccess) return e;
        k_chi0_slice_tan<NBK><<<g->nb, kSliceThreads, sm, st>>>(t->Grt, t->dGrt, g->tw_k, g->n8, g->nw0, t->dchiq);
        if ((e = launched()) != cudaSuccess) return e;
        k_chi0_boundary_tan<NBK><<<1, kSliceThreads, sm, st>>>(g->ek, g->er, t->der, t->fd, g->tw_k, t->Grt, t->dGrt,
                                                               t->dG0p, g->n8, mu0, dmu0, T, nk02, t->ddq0,
                                                               t->ddG0p, t->ddchir);
        return launched();
    }
};

}  // namespace

cudaError_t launch_chi0_tangent(const GridDev &g, const TangentBufs &t, double mu0, double dmu0, double T,
                                cudaStream_t st) {
    return dispatch_nbk<RunChi0Tan>(g.nbk, &g, &t, mu0, dmu0, T, st);
}

}  // namespace tpsc
