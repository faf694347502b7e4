// tpsc_cond.cu -- current-current correlator chi_jj(iqn) with the
// Maki-Thompson vertex correction, and the diamagnetic term kx0, in FP64
// (cond_opt::calc_chijj_vertex_corr_all_optim, bubble + Maki-Thompson branch,
// src/cond_opt.cpp:2537-4286).
//
// The reference works on the K4 grid of interior kx points: l = 0..nbk-3
// stands for kx = (l+1) pi/(nbk-1), m = 0..nbk-1 for ky = m pi/(nbk-1); the
// current vertex d eps/d kx is odd in kx and even in ky, so the real-space
// transforms are DST-I (RODFT00) along kx and DCT-I (REDFT00) along ky.
// Three kernel families:
//  * cond slices: one CTA per (tau_j, h or f0).  h(r, tau) and f0(r, tau)
//    are built from eps_k, transformed, multiplied by 2 V(r, tau) and
//    transformed back (src/cond_opt.cpp:2696-2908, 3027-3112), in shared
//    memory; the result is written in a two-column-block layout (the two
//    columns of a pair contiguous along tau) for the tau kernel.
//  * cond boundary: four CTAs for the tau-derivative end conditions of the
//    two splines (src/cond_opt.cpp:2744-2887, 2910-3025).
//  * cond tau: a persistent kernel, one CTA per SM, looping over pairs of K4
//    columns.  Per pair: the two splines + pre-twiddled FFTs give
//    J(k, ikn) and J0(k, ikn); G(k, ikn) = T/(ikn - eps + mu - Sigma) with
//    its analytic tail; the two back-transforms to tau; the spline + FFT of
//    G J (Maki-Thompson moment) and of -G(tau) G(beta - tau) (bubble)
//    (src/cond_opt.cpp:3179-3849).  Sigma is read once per column.  Every
//    CTA accumulates its columns' contributions in its own row of a partial
//    array; a finish kernel adds the rows in a fixed order.
// Plus the kx = 0, pi line sums of kx0 (src/cond_opt.cpp:3993-4173).
#include <cuda_runtime.h>
#include <stdint.h>

#include "tpsc_device.cuh"

namespace tpsc {

namespace {


__device__ __forceinline__ double cabs2(double2 z) { return hypot(z.x, z.y); }

// principal square root
__device__ __forceinline__ double2 csqrt2(double2 z) {
    const double r = cabs2(z);
    if (r == 0.0) return make_double2(0.0, z.y);
    const double t = sqrt(0.5 * (r + fabs(z.x)));
    if (z.x >= 0.0) return make_double2(t, z.y / (2.0 * t));
    return make_double2(fabs(z.y) / (2.0 * t), copysign(t, z.y));
}


// z^2 + B z + C at x and its derivative
__device__ __forceinline__ void quad_eval(double2 x, double2 B, double2 C, double2 &y, double2 &p) {
    y = cadd(cadd(cmul(x, x), cmul(B, x)), C);
    p = cadd(cscale(x, 2.0), B);
}

// Roots of z^2 + B z + C: closed form, then Newton polish (tolerance 1e-16 on
// |p(x)|, at most 10 steps, halving back when a step makes |p| grow), a
// polished root kept only if it improved |p| (generique::find_roots_2pol,
// src/generique.cpp:1666-1727, with A = 1).
__device__ void roots_2pol(double2 B, double2 C, double2 &r0, double2 &r1) {
    const double2 R = csqrt2(csub(cmul(B, B), cscale(C, 4.0)));
    double2 root[2] = {cscale(csub(make_double2(-B.x, -B.y), R), 0.5), cscale(cadd(make_double2(-B.x, -B.y), R), 0.5)};
#pragma unroll 1
    for (int k = 0; k < 2; ++k) {
        double2 x = root[k], y, p;
        quad_eval(x, B, C, y, p);
        const double y0 = cabs2(y);
        for (int it = 0; it < 10 && cabs2(p) != 0.0 && cabs2(y) > 1.0e-16; ++it) {
            const double2 x2 = x;
            const double ay2 = cabs2(y);
            const double2 c = csub(y, cmul(p, x));
            x = cdiv(make_double2(-c.x, -c.y), p);
            quad_eval(x, B, C, y, p);
            if (ay2 < cabs2(y)) {
                x = cscale(cadd(x, x2), 0.5);
                quad_eval(x, B, C, y, p);
            }
        }
        if (cabs2(y) < y0) root[k] = x;
    }
    r0 = root[0];
    r1 = root[1];
}

// ---------------------------------------------------------------------------
// per-K4-point constants of the h and f0 slices (src/cond_opt.cpp:2696-2827):
// x = eps - mu0; with E(t) = exp(-x t) (x > 0) or exp(x (beta - t)) (x <= 0)
//   h(t)  = A E(t),  f0(t) = (A t + B) E(t)
//   x > 0:  A = dek/L^2 / (e^{-x/T} + 1),  B = -dek/L^2 e^{-x/T} / (T (e^{-x/T} + 1)^2)
//   x <= 0: A = dek/L^2 / (e^{x/T} + 1),   B = -dek/L^2 / (T (e^{x/T} + 1)^2)
// tab[4c..4c+2] = (x, A, B)
// ---------------------------------------------------------------------------
__global__ void k_cond_table(const double *__restrict__ ek, const double *__restrict__ dek, int K4, int nbk,
                             double mu0, double T, double nf, double *__restrict__ tab) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= K4) return;
    const int l = c / nbk, m = c % nbk;
    const double x = ek[oct_index(l + 1, m)] - mu0;
    const double d = nf * dek[c];
    double A, B;
    if (x > 0) {
        const double ep = exp(-x / T);
        A = d / (ep + 1.0);
        B = -d * ep / (T * (ep + 1.0) * (ep + 1.0));
    } else {
        const double en = exp(x / T);
        A = d / (en + 1.0);
        B = -d / (T * (en + 1.0) * (en + 1.0));
    }
    tab[4 * c] = x;
    tab[4 * c + 1] = A;
    tab[4 * c + 2] = B;
    tab[4 * c + 3] = 0.0;
}

// h V(r, tau_j) (blockIdx.y = 0) or f0 V(r, tau_j) (blockIdx.y = 1),
// j = blockIdx.x = 0..Nw0: the slice, its DST x DCT, times 2 V(r, tau_j)
// (V(r, beta - tau) for tau > beta/2; r = (l+1, m) folded into the octant),
// DST x DCT again.  The first transform at tau = 0 and beta is kept in
// `pre` for the boundary kernel.
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_cond_slice(const double *__restrict__ tab, const double *__restrict__ V, const double2 *__restrict__ tw,
                 int nw0, double T, int K4p, double *__restrict__ hV, double *__restrict__ f0V,
                 double *__restrict__ pre) {
    constexpr int K4 = (NBK - 2) * NBK;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int j = blockIdx.x, y = blockIdx.y;
    const int nb = nw0 / 2 + 1;
    const double t = j / (nw0 * T);
    const double bt = 1.0 / T - t;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const double2 xa = *reinterpret_cast<const double2 *>(tab + 4 * c);
        const double b = tab[4 * c + 2];
        const double E = exp(xa.x > 0 ? -xa.x * t : xa.x * bt);
        S[c] = (y == 0) ? xa.y * E : (xa.y * t + b) * E;  // row l, column m: c = l NBK + m
    }
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    const int jv = j < nb ? j : nw0 - j;
    const bool edge = (j == 0 || j == nw0);
    double *pe = pre + (size_t)(2 * y + (j == nw0 ? 1 : 0)) * K4p;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const int l = c / NBK, m = c % NBK;
        const double v = S[c];
        if (edge) pe[c] = v;
        S[c] = v * (2.0 * V[bidx(jv, oct_index(l + 1, m), nb)]);
    }
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    double *out = (y == 0) ? hV : f0V;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) out[bidx2(j, c, nw0 + 1)] = S[c];
}

// End conditions of the two splines (src/cond_opt.cpp:2744-2887, 2910-3025):
// kind 0: dhV(0), 1: dhV(beta), 2: df0V(0), 3: df0V(beta) =
//   DST x DCT[ 2 D V(r, 0) +- P fact d/dtau chi0(r, 0) ]
// with D the transformed tau-derivative of h (f0) at the end, P the
// transformed h (f0) there, + at tau = 0 and - at beta.
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_cond_boundary(const double *__restrict__ ek, const double *__restrict__ dek, const double *__restrict__ V,
                    const double *__restrict__ dchirt0, const double2 *__restrict__ tw, const double *__restrict__ pre,
                    int nw0, int K4p, double mu0, double T, double nf, double fact, double *__restrict__ dbound) {
    constexpr int K4 = (NBK - 2) * NBK;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int kind = blockIdx.x;
    const int nb = nw0 / 2 + 1;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const int l = c / NBK, m = c % NBK;
        const double x = ek[oct_index(l + 1, m)] - mu0;
        const double d = nf * dek[c];
        double v;
        if (x > 0) {
            const double ep = exp(-x / T), q = ep + 1.0;
            switch (kind) {
                case 0: v = -d * x / q; break;
                case 1: v = -d * x * ep / q; break;
                case 2: v = d * (x * ep / (T * q * q) + 1.0 / q); break;
                default: v = d * ep * ((-x) * (1.0 / (T * q) - ep / (T * q * q)) + 1.0 / q); break;
            }
        } else {
            const double en = exp(x / T), q = en + 1.0;
            switch (kind) {
                case 0: v = -d * x * en / q; break;
                case 1: v = -d * x / q; break;
                case 2: v = d * en * (x / (T * q * q) + 1.0 / q); break;
                default: v = d * ((-x) * (1.0 / (T * q) - 1.0 / (T * q * q)) + 1.0 / q); break;
            }
        }
        S[c] = v;
    }
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    const double sg = (kind & 1) ? -1.0 : 1.0;
    const double *pe = pre + (size_t)kind * K4p;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const int l = c / NBK, m = c % NBK;
        const int o = oct_index(l + 1, m);
        S[c] = 2.0 * S[c] * V[bidx(0, o, nb)] + sg * pe[c] * fact * dchirt0[o];
    }
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    for (int c = threadIdx.x; c < K4; c += blockDim.x) dbound[(size_t)kind * K4p + c] = S[c];
}

// ---------------------------------------------------------------------------
// the per-k tau kernel
// ---------------------------------------------------------------------------
template <int N>
struct CondTauSmem {
    // one FFT group (N/16 threads) up to N = 2048, so that every thread works
    // in the FFTs and two CTAs share an SM (the kernel needs ~240 registers
    // a thread, which holds a 256-thread CTA to one per SM); 256 beyond
    static constexpr int threads = N >= 4096 ? TauSmem<N>::threads : 128;
    static constexpr int min_blocks = N >= 4096 ? 1 : 2;
    static constexpr size_t r_bytes = ((size_t)2 * (N + 1) * sizeof(double) + 15) & ~(size_t)15;
    static constexpr size_t x_bytes = (size_t)padded_len(N) * sizeof(double2);
    static constexpr size_t tables_off = r_bytes + 2 * x_bytes;
    static constexpr size_t bytes = tables_off + 2 * sizeof(TwoLevelTw);
};

struct CondTauArgs {
    const double *hV, *f0V, *dbound;
    const double2 *S;
    const double *s2, *s3, *sinf;
    const double *ek, *dek, *d2ek;
    const int *bin;
    const double *spl_full, *spl_half;
    const double2 *tw, *ht;
    double *partial;
    int K4, K4p, nbk, pw;
    double mu, T, nf;
};

// per-column state of the pair being processed
struct ColState {
    int o, bin;
    double e, dk, d2, wt;
    double2 r1, r2, u1, u2, v1, v2;  // roots; a/den and b/den of each root
    bool big1, big2;
    double C1, C2, C3;               // tau moments of the J being built
    double q0;                       // Re sum_n G^2 J0 / T, all n
    double k0, dGp, dGm, dJ0, dJb;
    double Gt0, Jt0, Jraw0;
    double dchi, integ, V0, VN;
    double CJ1b, CJ3b;
};


// full Sigma(k, i k_n) at octant o, n >= 0
__device__ __forceinline__ double2 sigma_at(const CondTauArgs &a, int n, int o, int NO, double ik, double sinf) {
    const double2 Sv = a.S[bidx(n, o, NO)];
    double rS, iS;
    sigma_full(ik, sinf, a.s2[o], a.s3[o], Sv, rS, iS);
    return make_double2(rS, iS);
}

// analytic tails at tau: G0(tau) = Re(-u1 e1 - u2 e2), Jinf(tau) = Re(v1 j1 + v2 j2)
// (src/cond_opt.cpp:3574-3640)
__device__ __forceinline__ void tails(const ColState &q, double tau, double beta, double &g0, double &jinf) {
    const double2 e1 = q.big1 ? cexp2(cscale(q.r1, -tau)) : cexp2(cscale(q.r1, beta - tau));
    const double2 j1 = q.big1 ? cexp2(cscale(q.r1, tau - beta)) : cexp2(cscale(q.r1, tau));
    const double2 e2 = q.big2 ? cexp2(cscale(q.r2, -tau)) : cexp2(cscale(q.r2, beta - tau));
    const double2 j2 = q.big2 ? cexp2(cscale(q.r2, tau - beta)) : cexp2(cscale(q.r2, tau));
    g0 = -cmul(q.u1, e1).x - cmul(q.u2, e2).x;
    jinf = cmul(q.v1, j1).x + cmul(q.v2, j2).x;
}


template <int N>
__global__ void __launch_bounds__(CondTauSmem<N>::threads, CondTauSmem<N>::min_blocks) k_cond_tau(const CondTauArgs a) {
    constexpr int NJ = N + 1, NO = N / 2, NJ2 = NO + 1;
    constexpr int G = FftPlan<N>::G;
    extern __shared__ __align__(16) double R[];
    double2 *X1 = reinterpret_cast<double2 *>(reinterpret_cast<char *>(R) + CondTauSmem<N>::r_bytes);
    double2 *X2 = X1 + padded_len(N);
    TwoLevelTw *tw2 = reinterpret_cast<TwoLevelTw *>(reinterpret_cast<char *>(R) + CondTauSmem<N>::tables_off);
    const TwoLevelTw *ht2 = tw2 + 1;
    tau_tables(tw2, tw2 + 1, a.tw, a.ht, N);  // published by the first barrier of the pair loop
    __shared__ ColState cs[2];
    __shared__ double d0s[2], dNs[2], sums[8], sV[2], sM[2];
    const int tid = threadIdx.x, NT = blockDim.x;
    const double T = a.T, h = 1.0 / (N * T), ih = 1.0 / h, beta = 1.0 / T, pT = kPi * T;
    const double sinf = a.sinf[0], mu = a.mu, nf = a.nf;
    const int PWB = 2 * NJ2;
    double *part = a.partial + (size_t)blockIdx.x * a.pw;
    const int npairs = a.K4p / 2;

    // one spline + pre-twiddled FFT pass: R (two columns, NJ nodes, end slopes
    // d0s/dNs) -> X1 = FFT_{+}[exp(i pi j/N) 6 a_j] packed; sets C1, C2, C3
    auto moments_fft = [&]() {
        if (tid < 2) {
            ColState &q = cs[tid];
            q.C1 = -R[tid * NJ] - R[tid * NJ + N];
            q.C2 = d0s[tid] + dNs[tid];
        }
        spline_second_derivatives<2>(R, NJ, NJ, h, d0s, dNs, a.spl_full, a.spl_full + NJ);
        if (tid < 2) cs[tid].C3 = -(R[tid * NJ] + R[tid * NJ + N]);
        if (tid < G) {
            const double *Ma = R, *Mb = R + NJ;
            auto in = [&](int j) -> double2 {
                return cmul(tw_at(ht2, j), make_double2((Ma[j + 1] - Ma[j]) * ih, (Mb[j + 1] - Mb[j]) * ih));
            };
            group_fft_io<N, +1>(X1, tid, (const TwoLevelTw *)tw2, 0, in, ScratchIO{X1});
        }
        __syncthreads();
    };
    // J(i k_n), n >= 0, of column q from the split transform F
    auto jval = [&](const ColState &q, double2 F, double2 f, double ik) -> double2 {
        const double ik2 = ik * ik;
        const double2 w = cmul(f, F);
        return make_double2(-q.C2 * ik2 + w.x * ik2 * ik2, -q.C1 * ik + q.C3 * ik2 * ik + w.y * ik2 * ik2);
    };

#pragma unroll 1
    for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
        const int c0 = 2 * p;
        const bool two = c0 + 1 < a.K4;
        // ---- column constants
        if (tid < 2) {
            const int c = c0 + tid;
            const bool valid = c < a.K4;
            const int cc = valid ? c : c0;
            const int l = cc / a.nbk, m = cc % a.nbk;
            ColState &q = cs[tid];
            q.o = oct_index(l + 1, m);
            q.e = a.ek[q.o];
            q.dk = a.dek[cc];
            q.d2 = a.d2ek[cc];
            q.wt = valid ? ((m == 0 || m == a.nbk - 1) ? 2.0 : 4.0) : 0.0;
            q.bin = a.bin ? a.bin[cc] : 0;
            roots_2pol(make_double2(mu - q.e, 0.0), make_double2(-sinf, 0.0), q.r1, q.r2);
            d0s[tid] = valid ? a.dbound[2 * (size_t)a.K4p + c] : 0.0;  // df0V(0)
            dNs[tid] = valid ? a.dbound[3 * (size_t)a.K4p + c] : 0.0;  // df0V(beta)
        }
        // ---- f0 V: J0(i k_n) and sum_n G^2 J0 / T (src/cond_opt.cpp:3236-3308)
        stage_pair(R, a.f0V + (size_t)p * 2 * NJ, NJ, two);
        __syncthreads();
        moments_fft();
        {
            double acc[2] = {0.0, 0.0};
            for (int n = tid; n < NO; n += NT) {
                double2 F[2];
                split_real(X1[pidx(n)], X1[pidx(N - 1 - n)], F[0], F[1]);
                // the pre-twiddled split: F_b = (Z_n - conj Z_{N-1-n}) / (2i)
                const double kn = (2 * n + 1) * pT, ik = 1.0 / kn;
                const double2 e = tw_at(ht2, 2 * n + 1);
                const double2 f = make_double2(1.0 - e.x, -e.y);
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const ColState &s = cs[q];
                    const double2 J0 = jval(s, F[q], f, ik);
                    const double2 sg = sigma_at(a, n, s.o, NO, ik, sinf);
                    const double2 Gv = cdiv(make_double2(T, 0.0), make_double2(mu - s.e - sg.x, kn - sg.y));
                    X2[pidx(q == 0 ? n : N - 1 - n)] = Gv;
                    acc[q] += cmul(cmul(Gv, Gv), J0).x;
                }
            }
            block_sum<2>(acc, sums);
            if (tid < 2) cs[tid].q0 = 2.0 * sums[tid] / T;
        }
        // ---- h V: J(i k_n); G J minus tails; k0, dG/dtau, dJ/dtau sums
        // (src/cond_opt.cpp:3204-3407)
        if (tid < 2) {
            const int c = c0 + tid;
            const bool valid = c < a.K4;
            d0s[tid] = valid ? a.dbound[c] : 0.0;                   // dhV(0)
            dNs[tid] = valid ? a.dbound[(size_t)a.K4p + c] : 0.0;   // dhV(beta)
        }
        stage_pair(R, a.hV + (size_t)p * 2 * NJ, NJ, two);
        __syncthreads();
        moments_fft();
        {
            double acc[6] = {0, 0, 0, 0, 0, 0};
            for (int n = tid; n < NO; n += NT) {
                double2 F[2];
                split_real(X1[pidx(n)], X1[pidx(N - 1 - n)], F[0], F[1]);
                const double kn = (2 * n + 1) * pT, ik = 1.0 / kn;
                const double2 e = tw_at(ht2, 2 * n + 1);
                const double2 f = make_double2(1.0 - e.x, -e.y);
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    const ColState &s = cs[q];
                    const int slot = pidx(q == 0 ? n : N - 1 - n);
                    const double2 J = jval(s, F[q], f, ik);
                    const double2 Gv = X2[slot];
                    const double2 Gt = cdiv(make_double2(T, 0.0), make_double2(mu - s.e, kn + sinf * ik));
                    const double2 Gs = csub(Gv, Gt);
                    const double2 Js = csub(cmul(Gv, J), cmul(Gt, make_double2(0.0, -s.C1 * ik)));
                    acc[3 * q] += Gs.x;
                    acc[3 * q + 1] += kn * Gs.y;
                    acc[3 * q + 2] -= kn * Js.y;
                    X2[slot] = Gs;
                    X1[slot] = Js;
                }
            }
            block_sum<6>(acc, sums);
        }
        if (tid < 2) {
            ColState &q = cs[tid];
            const double k0s = 2.0 * sums[3 * tid], dGs = 2.0 * sums[3 * tid + 1], dJs = 2.0 * sums[3 * tid + 2];
            const double2 r1 = q.r1, r2 = q.r2;
            const double2 a1 = cdiv(r1, csub(r1, r2)), a2 = cdiv(r2, csub(r2, r1));
            const double2 b1 = cdiv(make_double2(q.C1, 0.0), csub(r1, r2)), b2 = make_double2(-b1.x, -b1.y);
            // src/cond_opt.cpp:3421-3467
            auto branch = [&](double2 r, double2 av, double2 bv, bool &big, double2 &u, double2 &v, double2 &fp,
                              double2 &fm, double2 &fj, double2 &fjb) {
                big = r.x > 0;
                const double2 ex = big ? cexp2(cscale(r, -1.0 / T)) : cexp2(cscale(r, 1.0 / T));
                const double2 den = make_double2(ex.x + 1.0, ex.y);
                const double2 rb = cmul(r, bv);
                if (big) {
                    fp = cdiv(av, den);
                    fm = cdiv(cmul(av, ex), den);
                    fj = cdiv(cmul(rb, ex), den);
                    fjb = cdiv(rb, den);
                } else {
                    fp = cdiv(cmul(av, ex), den);
                    fm = cdiv(av, den);
                    fj = cdiv(rb, den);
                    fjb = cdiv(cmul(rb, ex), den);
                }
                u = cdiv(av, den);
                v = cdiv(bv, den);
            };
            double2 f1p, f1m, fj1, fj1b, f2p, f2m, fj2, fj2b;
            branch(r1, a1, b1, q.big1, q.u1, q.v1, f1p, f1m, fj1, fj1b);
            branch(r2, a2, b2, q.big2, q.u2, q.v2, f2p, f2m, fj2, fj2b);
            q.k0 = k0s + (f1m.x + f2m.x);
            q.dGm = -dGs + (cmul(r1, f1m).x + cmul(r2, f2m).x);
            q.dGp = dGs + (cmul(r1, f1p).x + cmul(r2, f2p).x);
            q.dJb = -dJs + (fj1b.x + fj2b.x);
            q.dJ0 = dJs + (fj1.x + fj2.x);
        }
        __syncthreads();
        // ---- back to tau: G(tau) = sum_n G(ikn) e^{-ikn tau}, J(tau) = sum_n J(ikn) e^{+ikn tau}
        // (src/cond_opt.cpp:3545-3620); both real, so the pair packs as Re/Im
        if (tid < G) {
            auto inG = [&](int k) -> double2 {
                double2 A, B;
                if (k < NO) {
                    A = X2[pidx(k)];
                    B = X2[pidx(N - 1 - k)];
                } else {
                    A = cconj(X2[pidx(N - 1 - k)]);
                    B = cconj(X2[pidx(k)]);
                }
                return make_double2(A.x - B.y, A.y + B.x);
            };
            group_fft_io<N, -1, false, true>(X2, tid, (const TwoLevelTw *)tw2, 0, inG, ScratchIO{X2});
            auto inJ = [&](int k) -> double2 {
                double2 A, B;
                if (k < NO) {
                    A = X1[pidx(k)];
                    B = X1[pidx(N - 1 - k)];
                } else {
                    A = cconj(X1[pidx(N - 1 - k)]);
                    B = cconj(X1[pidx(k)]);
                }
                return make_double2(A.x - B.y, A.y + B.x);
            };
            group_fft_io<N, +1, false, true>(X1, tid, (const TwoLevelTw *)tw2, 0, inJ, ScratchIO{X1});
        }
        __syncthreads();
        // ---- G J(tau) into R; G(tau) kept in X2 for the bubble
        for (int j = tid; j < N; j += NT) {
            const double tau = j * h;
            const double2 ph = tw_at(ht2, j);
            const double2 g = cmul(cconj(ph), X2[pidx(j)]);
            const double2 jr = cmul(ph, X1[pidx(j)]);
            double g0a, jia, g0b, jib;
            tails(cs[0], tau, beta, g0a, jia);
            tails(cs[1], tau, beta, g0b, jib);
            const double Ga = g.x + g0a, Gb = g.y + g0b, Ja = jr.x + jia, Jb = jr.y + jib;
            R[j] = Ga * Ja;
            R[NJ + j] = Gb * Jb;
            X2[pidx(j)] = make_double2(Ga, Gb);
            if (j == 0) {
                cs[0].Gt0 = Ga;
                cs[1].Gt0 = Gb;
                cs[0].Jt0 = Ja;
                cs[1].Jt0 = Jb;
                cs[0].Jraw0 = jr.x;
                cs[1].Jraw0 = jr.y;
            }
        }
        __syncthreads();
        if (tid < 2) {
            ColState &q = cs[tid];
            double g0b, jinfb;
            tails(q, beta, beta, g0b, jinfb);
            const double Jbeta = -q.Jraw0 + jinfb;  // J(beta) = -sum_n J(ikn) + Jinf(beta)
            R[tid * NJ + N] = (-q.Gt0 - 1.0) * Jbeta;
            d0s[tid] = q.dGp * q.Jt0 + q.Gt0 * q.dJ0;
            dNs[tid] = q.dGm * Jbeta - (q.Gt0 + 1.0) * q.dJb;
            q.CJ1b = R[tid * NJ] - R[tid * NJ + N];
        }
        __syncthreads();
        // ---- Maki-Thompson moment J(iqn) from the G J spline (src/cond_opt.cpp:3622-3660, 3807)
        spline_second_derivatives<2>(R, NJ, NJ, h, d0s, dNs, a.spl_full, a.spl_full + NJ);
        if (tid < 2) cs[tid].CJ3b = R[tid * NJ] - R[tid * NJ + N];
        if (tid < G) {
            const double *Ma = R, *Mb = R + NJ;
            auto in = [&](int j) -> double2 {
                return make_double2((Ma[j + 1] - Ma[j]) * ih, (Mb[j + 1] - Mb[j]) * ih);
            };
            group_fft_io<N, -1>(X1, tid, (const TwoLevelTw *)tw2, 0, in, ScratchIO{X1});
        }
        __syncthreads();
        for (int n = 1 + tid; n <= NO; n += NT) {
            double2 F[2];
            split_real(X1[pidx(n)], X1[pidx(N - n)], F[0], F[1]);
            const double wq = 2 * n * pT, iw = 1.0 / wq, iw2 = iw * iw;
            const double2 e = tw_at(tw2, n);
            const double2 f = make_double2(1.0 - e.x, -e.y);
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const ColState &s = cs[q];
                const double imJ = -2.0 * s.CJ1b * iw + 2.0 * s.CJ3b * iw2 * iw + 2.0 * cmul(f, F[q]).y * iw2 * iw2;
                part[s.bin * PWB + NJ2 + n] -= nf * s.wt * s.dk * imJ * iw;
            }
        }
        __syncthreads();
        // ---- bubble -G(tau) G(beta - tau) on [0, beta/2] (src/cond_opt.cpp:3662-3700, 3784-3817)
        for (int j = tid; j <= NO; j += NT) {
            const double2 g = X2[pidx(j)];
            double ga, gb;
            if (j == 0) {
                ga = cs[0].Gt0 * (cs[0].Gt0 + 1.0);
                gb = cs[1].Gt0 * (cs[1].Gt0 + 1.0);
            } else {
                const double2 gm = X2[pidx(N - j)];
                ga = -g.x * gm.x;
                gb = -g.y * gm.y;
            }
            R[j] = ga;
            R[NJ2 + j] = gb;
        }
        if (tid < 2) {
            ColState &q = cs[tid];
            q.dchi = q.dGp * (q.Gt0 + 1.0) + q.Gt0 * q.dGm;
            d0s[tid] = q.dchi;
            dNs[tid] = 0.0;
        }
        __syncthreads();
        if (tid < 2) {
            cs[tid].V0 = R[tid * NJ2];
            cs[tid].VN = R[tid * NJ2 + NO];
        }
        column_sums<2>(R, NJ2, 0, NJ2, sV);
        spline_second_derivatives<2>(R, NJ2, NJ2, h, d0s, dNs, a.spl_half, a.spl_half + NJ2);
        column_sums<2>(R, NJ2, 0, NJ2, sM);
        if (tid < 2) {
            ColState &q = cs[tid];
            const double M0 = R[tid * NJ2], MN = R[tid * NJ2 + NO];
            q.integ = h * (sV[tid] - 0.5 * (q.V0 + q.VN)) - h * h * h / 24.0 * (2.0 * sM[tid] - M0 - MN);
        }
        if (tid < G) {
            const double *Ma = R, *Mb = R + NJ2;
            auto in = [&](int j) -> double2 {
                const bool lo = j < NO;
                const int jj = lo ? j : N - 1 - j;
                const double sg = lo ? 1.0 : -1.0;
                return make_double2(sg * (Ma[jj + 1] - Ma[jj]) * ih, sg * (Mb[jj + 1] - Mb[jj]) * ih);
            };
            group_fft_io<N, -1>(X1, tid, (const TwoLevelTw *)tw2, 0, in, ScratchIO{X1});
        }
        __syncthreads();
        for (int n = 1 + tid; n <= NO; n += NT) {
            double2 F[2];
            split_real(X1[pidx(n)], X1[pidx(N - n)], F[0], F[1]);
            const double wq = 2 * n * pT, iw = 1.0 / wq, iw2 = iw * iw;
            const double2 e = tw_at(tw2, n);
            const double2 f = make_double2(1.0 - e.x, -e.y);
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const ColState &s = cs[q];
                const double bub = -2.0 * s.dchi * iw2 + cmul(f, F[q]).x * iw2 * iw2;
                part[s.bin * PWB + n] -= 2.0 * s.wt * nf * s.dk * s.dk * bub;
            }
        }
        if (tid == 0) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const ColState &s = cs[q];
                part[s.bin * PWB] -= 2.0 * s.wt * nf * s.dk * s.dk * (2.0 * s.integ);
                part[s.bin * PWB + NJ2] -= nf * s.wt * s.dk * s.q0;
                part[a.pw - 1] -= 2.0 * s.wt * nf * s.d2 * s.k0;
            }
        }
        __syncthreads();
    }
}

// kx0 on the kx = 0 and kx = pi lines (src/cond_opt.cpp:3993-4173): one block
// per (line, m); lines[i] = -2 w nf d2eps/dkx2 [sum_n (G - Gtail) + tail roots]
__global__ void __launch_bounds__(256)
    k_cond_lines(const double2 *__restrict__ S, const double *__restrict__ s2, const double *__restrict__ s3,
                 const double *__restrict__ sinfp, const double *__restrict__ ek, const double *__restrict__ d2line,
                 int nbk, int nw0, double mu, double T, double nf, double *__restrict__ lines) {
    const int i = blockIdx.x;
    const int l = i < nbk ? 0 : nbk - 1, m = i % nbk;
    const int o = oct_index(l, m), NO = nw0 / 2;
    const double sinf = sinfp[0], e = ek[o], pT = kPi * T;
    double v[1] = {0.0};
    for (int n = threadIdx.x; n < NO; n += blockDim.x) {
        const double kn = (2 * n + 1) * pT, ik = 1.0 / kn;
        double rS, iS;
        sigma_full(ik, sinf, s2[o], s3[o], S[bidx(n, o, NO)], rS, iS);
        const double2 Gv = cdiv(make_double2(T, 0.0), make_double2(mu - e - rS, kn - iS));
        const double2 Gt = cdiv(make_double2(T, 0.0), make_double2(mu - e, kn + sinf * ik));
        v[0] += Gv.x - Gt.x;
    }
    __shared__ double tot[1];
    block_sum<1>(v, tot);
    if (threadIdx.x == 0) {
        double2 r1, r2;
        roots_2pol(make_double2(mu - e, 0.0), make_double2(-sinf, 0.0), r1, r2);
        const double2 a1 = cdiv(r1, csub(r1, r2)), a2 = cdiv(r2, csub(r2, r1));
        auto fm = [&](double2 r, double2 av) -> double2 {
            if (r.x > 0) {
                const double2 ex = cexp2(cscale(r, -1.0 / T));
                return cdiv(cmul(av, ex), make_double2(ex.x + 1.0, ex.y));
            }
            const double2 ex = cexp2(cscale(r, 1.0 / T));
            return cdiv(av, make_double2(ex.x + 1.0, ex.y));
        };
        const double kk = 2.0 * tot[0] + (fm(r1, a1).x + fm(r2, a2).x);
        const double w = (m == 0 || m == nbk - 1) ? 1.0 : 2.0;
        lines[i] = -2.0 * w * nf * d2line[i] * kk;
    }
}

// Sum the per-CTA rows in block order: out = [binned (nbins x 2 NB)],
// [totals chijj1 (NB), chijj2 (NB)], [kx0].  One thread per column of a bin
// row (i < 2 NB) plus one for kx0 (i = 2 NB).
__global__ void k_cond_finish(const double *__restrict__ partial, int nblk, int pw, int nbins, int PWB,
                              const double *__restrict__ lines, int nlines, double *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i > PWB) return;
    if (i == PWB) {
        KSum s;
        for (int b = 0; b < nblk; ++b) s.add(partial[(size_t)b * pw + pw - 1]);
        for (int k = 0; k < nlines; ++k) s.add(lines[k]);
        out[(size_t)nbins * PWB + PWB] = s.value();
        return;
    }
    KSum tot;
    for (int bin = 0; bin < nbins; ++bin) {
        // eight independent compensated sums over the rows b = r mod 8 (their
        // loads overlap), added in a fixed order: deterministic
        constexpr int NS = 8;
        KSum s8[NS];
        int b = 0;
        for (; b + NS <= nblk; b += NS) {
            double v[NS];
#pragma unroll
            for (int r = 0; r < NS; ++r) v[r] = partial[(size_t)(b + r) * pw + bin * PWB + i];
#pragma unroll
            for (int r = 0; r < NS; ++r) s8[r].add(v[r]);
        }
        for (; b < nblk; ++b) s8[b % NS].add(partial[(size_t)b * pw + bin * PWB + i]);
        KSum s;
        for (int r = 0; r < NS; ++r) {
            s.add(s8[r].s);
            s.add(s8[r].c);
        }
        const double v = s.value();
        out[(size_t)bin * PWB + i] = v;
        tot.add(v);
    }
    out[(size_t)nbins * PWB + i] = tot.value();
}

// ---------------------------------------------------------------------------
// batched continued-fraction Pade (Vidberg-Serene), one CTA per function:
// g_0(l) = y_l, g_m(l) = (g_{m-1}(m-1) - g_{m-1}(l)) / ((x_l - x_{m-1}) g_{m-1}(l)),
// a_m = g_m(m) (generique::pade_cont_frac_coef_rec, src/generique.cpp:1649-1663),
// computed in shared memory, one barrier per order m; then every thread
// evaluates the continued fraction at its energies with the recurrence of
// generique::pade (src/generique.cpp:1628-1646).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_pade_batch(const double2 *__restrict__ x, const double2 *__restrict__ y, int Nn, const double2 *__restrict__ z,
                 int Nz, double2 *__restrict__ out) {
    extern __shared__ __align__(16) double2 sp[];
    double2 *xs = sp, *g = sp + Nn;
    const int f = blockIdx.x;
    for (int l = threadIdx.x; l < Nn; l += blockDim.x) {
        xs[l] = x[(size_t)f * Nn + l];
        g[l] = y[(size_t)f * Nn + l];
    }
    __syncthreads();
    for (int m = 1; m < Nn; ++m) {
        const double2 gm = g[m - 1], xm = xs[m - 1];
        for (int l = m + threadIdx.x; l < Nn; l += blockDim.x)
            g[l] = cdiv(csub(gm, g[l]), cmul(csub(xs[l], xm), g[l]));
        __syncthreads();
    }
    for (int iz = threadIdx.x; iz < Nz; iz += blockDim.x) {
        const double2 zz = z[iz];
        double2 A = make_double2(1.0, 0.0);
        double2 B = cadd(make_double2(1.0, 0.0), cmul(csub(zz, xs[0]), g[1]));
        double2 q = cdiv(A, B);
        for (int j = 3; j <= Nn; ++j) {
            const double2 t = cmul(csub(zz, xs[j - 2]), g[j - 1]);
            A = cadd(make_double2(1.0, 0.0), cdiv(t, A));
            B = cadd(make_double2(1.0, 0.0), cdiv(t, B));
            q = cdiv(cmul(q, A), B);
        }
        out[(size_t)f * Nz + iz] = cmul(q, g[0]);
    }
}

// ---------------------------------------------------------------------------
// launch wrappers per compiled size
// ---------------------------------------------------------------------------
template <int NBK>
struct RunCondSlices {
    // ny = 2: the h and f0 slices and all four end conditions; ny = 1: h only
    static cudaError_t run(const GridDev *g, const CondDev *c, const double *V, const double *dchirt0, double mu0,
                           double T, double fact, int ny, bool f32, cudaStream_t st) {
        const size_t sm = SliceSmem<NBK>::bytes;
        cudaError_t e = set_smem(k_cond_slice<NBK>, sm);
        if (e != cudaSuccess) return e;
        if ((e = set_smem(k_cond_boundary<NBK>, sm)) != cudaSuccess) return e;
        const double nf = 1.0 / ((double)g->nk0 * g->nk0);
        k_cond_table<<<(c->K4 + 255) / 256, 256, 0, st>>>(g->ek, c->dek, c->K4, g->nbk, mu0, T, nf, c->tab);
        if ((e = launched()) != cudaSuccess) return e;
        if (f32) {
            if ((e = launch_cond_slice32(*g, *c, V, T, ny, st)) != cudaSuccess) return e;
        } else {
            k_cond_slice<NBK><<<dim3(g->nw0 + 1, ny), kSliceThreads, sm, st>>>(c->tab, V, g->tw_k, g->nw0, T,
                                                                                c->K4p, c->hV, c->f0V, c->pre);
            if ((e = launched()) != cudaSuccess) return e;
        }
        k_cond_boundary<NBK><<<2 * ny, kSliceThreads, sm, st>>>(g->ek, c->dek, V, dchirt0, g->tw_k, c->pre, g->nw0, c->K4p,
                                                            mu0, T, nf, fact, c->dbound);
        return launched();
    }
};

template <int N>
struct RunCondTau {
    static cudaError_t run(const GridDev *g, const CondDev *c, const double2 *S, const double *s2, const double *s3,
                           const double *sinf, double mu, double T, cudaStream_t st) {
        const size_t sm = CondTauSmem<N>::bytes;
        cudaError_t e = set_smem(k_cond_tau<N>, sm);
        if (e != cudaSuccess) return e;
        CondTauArgs a;
        a.hV = c->hV;
        a.f0V = c->f0V;
        a.dbound = c->dbound;
        a.S = S;
        a.s2 = s2;
        a.s3 = s3;
        a.sinf = sinf;
        a.ek = g->ek;
        a.dek = c->dek;
        a.d2ek = c->d2ek;
        a.bin = c->nbins > 1 ? c->bin : nullptr;
        a.spl_full = g->spl_full;
        a.spl_half = g->spl_half;
        a.tw = g->tw_w;
        a.ht = g->ht_w;
        a.partial = c->partial;
        a.K4 = c->K4;
        a.K4p = c->K4p;
        a.nbk = g->nbk;
        a.pw = c->pw;
        a.mu = mu;
        a.T = T;
        a.nf = 1.0 / ((double)g->nk0 * g->nk0);
        const size_t pbytes = (size_t)c->nblk * c->pw * sizeof(double);
        if ((e = cudaMemsetAsync(c->partial, 0, pbytes, st)) != cudaSuccess) return e;
        k_cond_tau<N><<<c->nblk, CondTauSmem<N>::threads, sm, st>>>(a);
        return launched();
    }
};

template <int N>
struct CondBlocks {
    static cudaError_t run(int *blocks) {
        cudaError_t e = set_smem(k_cond_tau<N>, CondTauSmem<N>::bytes);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0, per = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cond_tau<N>, CondTauSmem<N>::threads,
                                                          CondTauSmem<N>::bytes);
        if (e != cudaSuccess) return e;
        *blocks = sms * (per > 0 ? per : 1);
        return cudaSuccess;
    }
};

}  // namespace

cudaError_t cond_blocks(const GridDev &g, int *blocks) { return dispatch_nw<CondBlocks>(g.nw0, blocks); }

cudaError_t launch_cond_table(const GridDev &g, const CondDev &c, double mu0, double T, cudaStream_t st) {
    const double nf = 1.0 / ((double)g.nk0 * g.nk0);
    k_cond_table<<<(c.K4 + 255) / 256, 256, 0, st>>>(g.ek, c.dek, c.K4, g.nbk, mu0, T, nf, c.tab);
    return launched();
}

cudaError_t launch_cond_slices(const GridDev &g, const CondDev &c, const double *V, const double *dtau_chirt0,
                               double mu0, double T, double fact, cudaStream_t st) {
    return dispatch_nbk<RunCondSlices>(g.nbk, &g, &c, V, dtau_chirt0, mu0, T, fact, 2, false, st);
}

cudaError_t launch_cond_slices32(const GridDev &g, const CondDev &c, const double *V, const double *dtau_chirt0,
                                 double mu0, double T, double fact, cudaStream_t st) {
    return dispatch_nbk<RunCondSlices>(g.nbk, &g, &c, V, dtau_chirt0, mu0, T, fact, 2, true, st);
}

cudaError_t launch_cond_slices_h(const GridDev &g, const CondDev &c, const double *V, const double *dtau_chirt0,
                                 double mu0, double T, double fact, cudaStream_t st) {
    return dispatch_nbk<RunCondSlices>(g.nbk, &g, &c, V, dtau_chirt0, mu0, T, fact, 1, false, st);
}

cudaError_t launch_cond_tau(const GridDev &g, const CondDev &c, const double2 *S, const double *s2, const double *s3,
                            const double *sinf, double mu, double T, cudaStream_t st) {
    return dispatch_nw<RunCondTau>(g.nw0, &g, &c, S, s2, s3, sinf, mu, T, st);
}

cudaError_t launch_pade_batch(const double2 *x, const double2 *y, int nf, int Nn, const double2 *z, int Nz,
                              double2 *out, cudaStream_t st) {
    if (nf < 1 || Nn < 2 || Nn > kPadeBatchMax || Nz < 1) return cudaErrorInvalidValue;
    const size_t sm = (size_t)2 * Nn * sizeof(double2);
    cudaError_t e = set_smem(k_pade_batch, sm);
    if (e != cudaSuccess) return e;
    k_pade_batch<<<nf, 256, sm, st>>>(x, y, Nn, z, Nz, out);
    return launched();
}

cudaError_t launch_cond_finish(const GridDev &g, const CondDev &c, const double2 *S, const double *s2,
                               const double *s3, const double *sinf, double mu, double T, cudaStream_t st) {
    const double nf = 1.0 / ((double)g.nk0 * g.nk0);
    k_cond_lines<<<2 * g.nbk, 256, 0, st>>>(S, s2, s3, sinf, g.ek, c.d2line, g.nbk, g.nw0, mu, T, nf, c.lines);
    cudaError_t e = launched();
    if (e != cudaSuccess) return e;
    const int PWB = 2 * (g.nw0 / 2 + 1);
    k_cond_finish<<<(PWB + 1 + 255) / 256, 256, 0, st>>>(c.partial, c.nblk, c.pw, c.nbins, PWB, c.lines, 2 * g.nbk,
                                                          c.out);
    return launched();
}

}  // namespace tpsc
