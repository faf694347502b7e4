// tpsc_adjoint.cu -- the reverse pass (adjoint) of V -> Sigma -> mu -> chi_jj
// -> sigma(iq_n), in FP64 (the differentiation form; no counterpart in the
// reference, whose forward stages are src/chi.cpp:37-206 for V,
// src/green.cpp:1673-2025 for Sigma, src/green.cpp:3108-3259 for mu and
// src/cond_opt.cpp:2537-4286 for the bubble + Maki-Thompson chi_jj).
//
// Given a cotangent c_n on sigma(iq_n) = (-kx0 - chi_jj(iq_n)) / q_n, the
// kernels run the stages backward and leave, per CTA, partial sums of the
// loss derivative along the three parameter directions (U; a shift of mu0;
// t' at fixed density).  Everything upstream of V -- G(r, tau), chi0 and the
// sum-rule roots -- enters through the forward tangents of the chi0 stage
// (tpsc_tangent.cu): the backward pass contracts its adjoints of G(r, tau),
// chi0(q, iqn), chi0(r, tau) and the two tau-derivative end tables with
// those tangents, and the host adds the roots' sensitivities.
//
// Linear maps and their transposes:
//  * the octant 2D DCT-I A = P (C x C) E satisfies A^T = W A W^-1 with W the
//    full-zone multiplicity of an octant point (2 off the diagonal, times 2
//    for each index off the zone edges);
//  * DST-I is symmetric, DCT-I's transpose is w_e C w_e^-1 (w_e = 1 at the
//    ends, 2 inside), so the h-slice transform's transpose rescales the
//    ky columns;
//  * the clamped spline M = A^-1 R(V, d0, dN) has a symmetric A: the
//    adjoint solves the same system and applies R^T, which is the same
//    second difference with the end rows' slopes;
//  * the tau <-> i w_n FFTs transpose to FFTs of the opposite sign.
// The per-point nonlinear steps (G = T / (i k_n - eps + mu - Sigma), the
// roots of the G tail, the Fermi branches, the vertex's RPA factors) are
// differentiated by hand; every formula below was checked against central
// differences of the forward before it was written here.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tpsc_device.cuh"

namespace tpsc {

namespace {

__device__ __forceinline__ double fermi_fn(double r, double T) {
    if (r > 0) {
        const double e = exp(-r / T);
        return e / (1.0 + e);
    }
    return 1.0 / (exp(r / T) + 1.0);
}
// e^{-tau r} (1 - f(r)) and e^{r tau} f(r) without overflow
__device__ __forceinline__ double tail_g(double r, double tau, double beta) {
    return r > 0 ? exp(-tau * r) / (1.0 + exp(-beta * r)) : exp((beta - tau) * r) / (exp(beta * r) + 1.0);
}
__device__ __forceinline__ double tail_j(double r, double tau, double beta) {
    return r > 0 ? exp(r * (tau - beta)) / (exp(-beta * r) + 1.0) : exp(r * tau) / (exp(beta * r) + 1.0);
}
// the two real roots of z^2 + B z - sinf (sinf > 0), smaller first
__device__ __forceinline__ void real_roots(double B, double sinf, double &r1, double &r2) {
    const double disc = sqrt(B * B + 4.0 * sinf);
    const double q = -0.5 * (B + copysign(disc, B));
    const double ra = q, rb = q != 0.0 ? -sinf / q : 0.0;
    r1 = fmin(ra, rb);
    r2 = fmax(ra, rb);
}
__device__ __forceinline__ double edge_w(int i, int n) { return (i == 0 || i == n - 1) ? 1.0 : 2.0; }
// W of A^T = W A W^-1 for the octant DCT-I
__device__ __forceinline__ double oct_tw(int l, int m, int nbk) {
    return (l == m ? 1.0 : 2.0) * edge_w(l, nbk) * edge_w(m, nbk);
}

// adjoint of the spline's right-hand side: V_bar = R^T r (r = A^-1 M_bar)
__device__ __forceinline__ double spline_rT(const double *r, int i, int N, double a6) {
    if (i == 0) return a6 * (r[1] - r[0]);
    if (i == N) return a6 * (r[N - 1] - r[N]);
    return a6 * (r[i - 1] - 2.0 * r[i] + r[i + 1]);
}

// directions of the lattice tables along t' at K4 point (kx, ky)
__device__ __forceinline__ void tp_dirs(int l1, int m, int nbk, double &de, double &ddek, double &dd2) {
    const double kx = l1 * kPi / (nbk - 1), ky = m * kPi / (nbk - 1);
    const double cx = cos(kx), cy = cos(ky);
    de = -4.0 * cx * cy;
    ddek = 4.0 * sin(kx) * cy;
    dd2 = 4.0 * cx * cy;
}

}  // namespace

// ---------------------------------------------------------------------------
// the per-k tau kernel of chi_jj, backward: one K4 column per CTA iteration
// ---------------------------------------------------------------------------
template <int N>
struct CondBwdSmem {
    static constexpr int NJ = N + 1;
    static constexpr size_t x_bytes = (size_t)padded_len(N) * sizeof(double2);
    static constexpr size_t r_bytes = ((size_t)NJ * sizeof(double) + 15) & ~(size_t)15;
    static constexpr size_t gt_off = x_bytes;
    static constexpr size_t jt_off = gt_off + r_bytes;
    static constexpr size_t r_off = jt_off + r_bytes;
    static constexpr size_t q_off = r_off + r_bytes;
    static constexpr size_t tw_off = q_off + r_bytes;
    static constexpr size_t bytes = tw_off + 2 * sizeof(TwoLevelTw);
    static_assert(bytes <= 232448, "cond backward column does not fit");
    static_assert(x_bytes >= (size_t)(2 * N + 2) * sizeof(double), "X must hold the two spline adjoints");
};

struct CondBwdCol {
    int o, l, m;
    double e, dk, d2, wt;
    double C1, C2, C3;
    double k0s, dGs, dJs;
    double r[2], f[2], a[2], b[2];
    double k0, dGp, dGm, dJb, dJ0;
    double Gt0, Jt0, Jraw0, Jbeta, dchi, CJ1b, CJ3b;
    // adjoints
    double dkb, dchib, CJ1bb, CJ3bb, d0b2, dNb2;
    double Gt0bs, Jt0bs, dGpb, dGmb, dJ0b, dJbb, Jbetab;
    double k0sb, dGsb, dJsb, C1bs, mub, eb, sinfb;
};

// threads of the backward tau kernel: one FFT group (N/16) from N = 2048 on,
// so that every thread works in the FFTs and two CTAs share an SM up to 2048
template <int N>
constexpr int cond_bwd_threads() {
    return N >= 4096 ? 256 : 128;
}

template <int N>
__global__ void __launch_bounds__(cond_bwd_threads<N>(), N >= 4096 ? 1 : 2) k_cond_tau_bwd(const CondBwdArgs a) {
    constexpr int NJ = N + 1, NO = N / 2, NJ2 = NO + 1;
    constexpr int G = FftPlan<N>::G;
    using SM = CondBwdSmem<N>;
    extern __shared__ __align__(16) double smem[];
    char *base = reinterpret_cast<char *>(smem);
    double2 *X = reinterpret_cast<double2 *>(smem);
    double *Xd = smem;
    double *Gt = reinterpret_cast<double *>(base + SM::gt_off);
    double *Jt = reinterpret_cast<double *>(base + SM::jt_off);
    double *R = reinterpret_cast<double *>(base + SM::r_off);
    double *Q = reinterpret_cast<double *>(base + SM::q_off);
    TwoLevelTw *tw2 = reinterpret_cast<TwoLevelTw *>(base + SM::tw_off);
    const TwoLevelTw *ht2 = tw2 + 1;
    tau_tables(tw2, tw2 + 1, a.tw, a.ht, N);
    __shared__ CondBwdCol cs;
    __shared__ double sums[8], d0s[1], dNs[1], e0s[1], eNs[1];
    const int tid = threadIdx.x, NT = blockDim.x;
    const double T = a.T, h = 1.0 / (N * T), ih = 1.0 / h, beta = 1.0 / T, pT = kPi * T;
    const double a6 = 6.0 / (h * h), b6 = 6.0 / h;
    const double sinf = a.sinf[0], mu = a.mu, nf = a.nf;
    double2 *wsG = a.ws + (size_t)blockIdx.x * 2 * NO, *wsJ = wsG + NO;
    double acc_mu = 0.0, acc_sinf = 0.0, acc_tp = 0.0;  // thread 0

#pragma unroll 1
    for (int c = blockIdx.x; c < a.K4; c += gridDim.x) {
        // ---- column constants and the h V column
        if (tid == 0) {
            cs.l = c / a.nbk;
            cs.m = c % a.nbk;
            cs.o = oct_index(cs.l + 1, cs.m);
            cs.e = a.ek[cs.o];
            cs.dk = a.dek[c];
            cs.d2 = a.d2ek[c];
            cs.wt = (cs.m == 0 || cs.m == a.nbk - 1) ? 2.0 : 4.0;
            d0s[0] = a.dbound[c];
            dNs[0] = a.dbound[(size_t)a.K4p + c];
        }
        for (int j = tid; j < NJ; j += NT) R[j] = a.hV[bidx2(j, c, NJ)];
        __syncthreads();
        if (tid == 0) {
            cs.C1 = -R[0] - R[N];
            cs.C2 = d0s[0] + dNs[0];
        }
        spline_second_derivatives<1>(R, NJ, NJ, h, d0s, dNs, a.spl_full, a.spl_full + NJ);
        if (tid == 0) cs.C3 = -(R[0] + R[N]);
        if (tid < G) {
            auto in = [&](int j) -> double2 { return cscale(tw_at(ht2, j), (R[j + 1] - R[j]) * ih); };
            group_fft_io<N, +1>(X, tid, (const TwoLevelTw *)tw2, 0, in, ScratchIO{X});
        }
        __syncthreads();
        // ---- J(i k_n), G(i k_n), the tail-subtracted G and G J; packed for the tau transform
        {
            double acc[3] = {0.0, 0.0, 0.0};
            const double e = cs.e, C1 = cs.C1, C2 = cs.C2, C3 = cs.C3;
            const double s2 = a.s2[cs.o], s3 = a.s3[cs.o];
            for (int n = tid; n < NO; n += NT) {
                const double kn = (2 * n + 1) * pT, ik = 1.0 / kn, ik2 = ik * ik;
                const double2 ee = tw_at(ht2, 2 * n + 1);
                const double2 f = make_double2(1.0 - ee.x, -ee.y);
                const double2 fF = cmul(f, X[pidx(n)]);
                const double2 J =
                    make_double2(-C2 * ik2 + fF.x * ik2 * ik2, -C1 * ik + C3 * ik2 * ik + fF.y * ik2 * ik2);
                double rS, iS;
                sigma_full(ik, sinf, s2, s3, a.S[bidx(n, cs.o, NO)], rS, iS);
                const double2 Gv = cdiv(make_double2(T, 0.0), make_double2(mu - e - rS, kn - iS));
                const double2 Gl = cdiv(make_double2(T, 0.0), make_double2(mu - e, kn + sinf * ik));
                const double2 Gs = csub(Gv, Gl);
                const double2 Js = csub(cmul(Gv, J), cmul(Gl, make_double2(0.0, -C1 * ik)));
                wsG[n] = Gv;
                wsJ[n] = J;
                // Gs + i conj(Js) at n, conj(Gs) + i Js at N - 1 - n
                X[pidx(n)] = make_double2(Gs.x + Js.y, Gs.y + Js.x);
                X[pidx(N - 1 - n)] = make_double2(Gs.x - Js.y, -Gs.y + Js.x);
                acc[0] += Gs.x;
                acc[1] += kn * Gs.y;
                acc[2] -= kn * Js.y;
            }
            block_sum<3>(acc, sums);
        }
        if (tid == 0) {
            cs.k0s = 2.0 * sums[0];
            cs.dGs = 2.0 * sums[1];
            cs.dJs = 2.0 * sums[2];
            real_roots(mu - cs.e, sinf, cs.r[0], cs.r[1]);
            const double d = cs.r[0] - cs.r[1];
            cs.a[0] = cs.r[0] / d;
            cs.a[1] = -cs.r[1] / d;
            cs.b[0] = cs.C1 / d;
            cs.b[1] = -cs.C1 / d;
            double k0 = cs.k0s, dGm = -cs.dGs, dGp = cs.dGs, dJb = -cs.dJs, dJ0 = cs.dJs;
            for (int i = 0; i < 2; ++i) {
                const double f = fermi_fn(cs.r[i], T);
                cs.f[i] = f;
                k0 += cs.a[i] * f;
                dGm += cs.r[i] * cs.a[i] * f;
                dGp += cs.r[i] * cs.a[i] * (1.0 - f);
                dJb += cs.r[i] * cs.b[i] * (1.0 - f);
                dJ0 += cs.r[i] * cs.b[i] * f;
            }
            cs.k0 = k0;
            cs.dGm = dGm;
            cs.dGp = dGp;
            cs.dJb = dJb;
            cs.dJ0 = dJ0;
        }
        __syncthreads();
        // ---- back to tau: G(tau) + i J(tau) = conj(ht) FFT_-[Gs + i conj Js] plus the analytic tails
        if (tid < G) group_fft_io<N, -1, false, true>(X, tid, (const TwoLevelTw *)tw2, 0, ScratchIO{X}, ScratchIO{X});
        __syncthreads();
        for (int j = tid; j < N; j += NT) {
            const double tau = j * h;
            const double2 Z = cmul(cconj(tw_at(ht2, j)), X[pidx(j)]);
            const double g0t = -cs.a[0] * tail_g(cs.r[0], tau, beta) - cs.a[1] * tail_g(cs.r[1], tau, beta);
            const double jin = cs.b[0] * tail_j(cs.r[0], tau, beta) + cs.b[1] * tail_j(cs.r[1], tau, beta);
            Gt[j] = Z.x + g0t;
            Jt[j] = Z.y + jin;
            if (j == 0) cs.Jraw0 = Z.y;
        }
        __syncthreads();
        if (tid == 0) {
            cs.Gt0 = Gt[0];
            cs.Jt0 = Jt[0];
            cs.Jbeta = -cs.Jraw0 + cs.b[0] * tail_j(cs.r[0], beta, beta) + cs.b[1] * tail_j(cs.r[1], beta, beta);
            d0s[0] = cs.dGp * cs.Jt0 + cs.Gt0 * cs.dJ0;
            dNs[0] = cs.dGm * cs.Jbeta - (cs.Gt0 + 1.0) * cs.dJb;
            cs.dchi = cs.dGp * (cs.Gt0 + 1.0) + cs.Gt0 * cs.dGm;
            e0s[0] = cs.dchi;
            eNs[0] = 0.0;
            cs.CJ1b = cs.Gt0 * cs.Jt0 + (cs.Gt0 + 1.0) * cs.Jbeta;
            R[N] = (-cs.Gt0 - 1.0) * cs.Jbeta;
            Q[0] = cs.Gt0 * (cs.Gt0 + 1.0);
        }
        for (int j = tid; j < N; j += NT) R[j] = Gt[j] * Jt[j];
        for (int j = 1 + tid; j <= NO; j += NT) Q[j] = -Gt[j] * Gt[N - j];
        __syncthreads();
        spline_second_derivatives<1>(R, NJ, NJ, h, d0s, dNs, a.spl_full, a.spl_full + NJ);
        spline_second_derivatives<1>(Q, NJ2, NJ2, h, e0s, eNs, a.spl_half, a.spl_half + NJ2);
        if (tid == 0) cs.CJ3b = R[0] - R[N];
        // ---- the Maki-Thompson moment and the bubble: FFT_-[y2 + i fb]
        if (tid < G) {
            auto in = [&](int j) -> double2 {
                const double y2 = (R[j + 1] - R[j]) * ih;
                const double fb = j < NO ? (Q[j + 1] - Q[j]) * ih : -(Q[N - j] - Q[N - 1 - j]) * ih;
                return make_double2(y2, fb);
            };
            group_fft_io<N, -1>(X, tid, (const TwoLevelTw *)tw2, 0, in, ScratchIO{X});
        }
        __syncthreads();
        // ---- backward seeds at n = 1..NO; the cotangents of J0f and Fb parked in R, Q
        {
            double acc[4] = {0.0, 0.0, 0.0, 0.0};
            const double wt = cs.wt, dk = cs.dk;
            for (int n = 1 + tid; n <= NO; n += NT) {
                double2 J0f, Fb;
                split_real(X[pidx(n)], X[pidx(N - n)], J0f, Fb);
                const double wq = 2 * n * pT, iw = 1.0 / wq, iw2 = iw * iw, iw4 = iw2 * iw2;
                const double2 w = tw_at(tw2, n);
                const double2 zq = make_double2(1.0 - w.x, -w.y);
                const double imJ = -2.0 * cs.CJ1b * iw + 2.0 * cs.CJ3b * iw2 * iw + 2.0 * cmul(zq, J0f).y * iw4;
                const double bub = -2.0 * cs.dchi * iw2 + cmul(zq, Fb).x * iw4;
                const double cwn = a.cw[n];
                const double bubb = cwn * (-2.0 * wt * nf * dk * dk);
                const double imJb = cwn * (-nf * wt * dk * iw);
                acc[0] += cwn * (-4.0 * wt * nf * dk * bub) + cwn * (-nf * wt * imJ * iw);
                acc[1] += bubb * (-2.0 * iw2);
                acc[2] += imJb * (-2.0 * iw);
                acc[3] += imJb * (2.0 * iw2 * iw);
                // Fb_bar = bubb conj(zq) / wq^4, J0f_bar = imJb (2 / wq^4) i conj(zq)
                reinterpret_cast<double2 *>(Q)[n - 1] = cscale(cconj(zq), bubb * iw4);
                reinterpret_cast<double2 *>(R)[n - 1] = cscale(make_double2(zq.y, zq.x), 2.0 * imJb * iw4);
            }
            block_sum<4>(acc, sums);
        }
        if (tid == 0) {
            cs.dkb = sums[0];
            cs.dchib = sums[1];
            cs.CJ1bb = sums[2];
            cs.CJ3bb = sums[3];
        }
        // Hermitian parts, packed: P_k = Jh_k + i Fh_k
        for (int k = tid; k < N; k += NT) {
            double2 jh = make_double2(0.0, 0.0), fh = jh;
            const double2 *Jb = reinterpret_cast<const double2 *>(R);
            const double2 *Fbb = reinterpret_cast<const double2 *>(Q);
            if (k >= 1 && k < NO) {
                jh = cscale(Jb[k - 1], 0.5);
                fh = cscale(Fbb[k - 1], 0.5);
            } else if (k == NO) {
                jh = make_double2(Jb[NO - 1].x, 0.0);
                fh = make_double2(Fbb[NO - 1].x, 0.0);
            } else if (k > NO) {
                jh = cscale(cconj(Jb[N - k - 1]), 0.5);
                fh = cscale(cconj(Fbb[N - k - 1]), 0.5);
            }
            X[pidx(k)] = make_double2(jh.x - fh.y, jh.y + fh.x);
        }
        __syncthreads();
        if (tid < G) group_fft_io<N, +1, false, true>(X, tid, (const TwoLevelTw *)tw2, 0, ScratchIO{X}, ScratchIO{X});
        __syncthreads();
        // M_bar of the G J spline (R, NJ) and of the bubble spline (Q, NJ2)
        for (int i = tid; i <= N; i += NT) {
            const double ym = i >= 1 ? X[pidx(i - 1)].x : 0.0;
            const double y0 = i < N ? X[pidx(i)].x : 0.0;
            double v = ih * (ym - y0);
            if (i == 0) v += cs.CJ3bb;
            if (i == N) v -= cs.CJ3bb;
            R[i] = v;
        }
        for (int i = tid; i <= NO; i += NT) {
            auto y3 = [&](int k) -> double {
                if (k < 0 || k >= NO) return 0.0;
                return X[pidx(k)].y - X[pidx(N - 1 - k)].y;
            };
            Q[i] = ih * (y3(i - 1) - y3(i));
        }
        __syncthreads();
        spline_second_derivatives<1, true>(R, NJ, NJ, h, nullptr, nullptr, a.spl_full, a.spl_full + NJ);
        spline_second_derivatives<1, true>(Q, NJ2, NJ2, h, nullptr, nullptr, a.spl_half, a.spl_half + NJ2);
        // d L / d gj into Xd[0..N], d L / d GG into Xd[N+1 .. N+1+NO]
        for (int i = tid; i <= N; i += NT) {
            double v = spline_rT(R, i, N, a6);
            if (i == 0) v += cs.CJ1bb;
            if (i == N) v -= cs.CJ1bb;
            Xd[i] = v;
        }
        for (int i = tid; i <= NO; i += NT) Xd[N + 1 + i] = spline_rT(Q, i, NO, a6);
        __syncthreads();
        if (tid == 0) {
            cs.d0b2 = -b6 * R[0];
            cs.dNb2 = b6 * R[N];
            cs.dchib += -b6 * Q[0];
            const double gjbN = Xd[N], GGb0 = Xd[N + 1];
            const double dchib = cs.dchib, d0b = cs.d0b2, dNb = cs.dNb2;
            cs.Gt0bs = dchib * (cs.dGp + cs.dGm) + d0b * cs.dJ0 - dNb * cs.dJb - gjbN * cs.Jbeta +
                       GGb0 * (2.0 * cs.Gt0 + 1.0);
            cs.Jt0bs = d0b * cs.dGp;
            cs.dGpb = dchib * (cs.Gt0 + 1.0) + d0b * cs.Jt0;
            cs.dGmb = dchib * cs.Gt0 + dNb * cs.Jbeta;
            cs.dJ0b = d0b * cs.Gt0;
            cs.dJbb = -dNb * (cs.Gt0 + 1.0);
            cs.Jbetab = gjbN * (-cs.Gt0 - 1.0) + dNb * cs.dGm;
        }
        __syncthreads();
        // ---- d L / d G(tau), d L / d J(tau) (into R, Q) and the tails' parameters
        {
            double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // a1, a2, b1, b2, r1, r2
            for (int j = tid; j < N; j += NT) {
                const double gjb = Xd[j];
                double gtb = gjb * Jt[j], jtb = gjb * Gt[j];
                if (j >= 1) {
                    const double ggs = (j <= NO ? Xd[N + 1 + j] : 0.0) + (j >= NO ? Xd[N + 1 + N - j] : 0.0);
                    gtb -= ggs * Gt[N - j];
                } else {
                    gtb += cs.Gt0bs;
                    jtb += cs.Jt0bs;
                }
                R[j] = gtb;
                Q[j] = jtb;
                const double tau = j * h;
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                    const double g = tail_g(cs.r[i], tau, beta), jj = tail_j(cs.r[i], tau, beta);
                    acc[i] -= gtb * g;
                    acc[4 + i] += gtb * (-cs.a[i]) * g * (cs.f[i] / T - tau);
                    acc[2 + i] += jtb * jj;
                    acc[4 + i] += jtb * cs.b[i] * jj * (tau - (1.0 - cs.f[i]) / T);
                }
            }
            block_sum<6>(acc, sums);
        }
        if (tid == 0) {
            double ab[2] = {sums[0], sums[1]}, bb[2] = {sums[2], sums[3]}, rb[2] = {sums[4], sums[5]};
            const double k0b = a.kx0b * (-2.0 * cs.wt * nf * cs.d2);
            for (int i = 0; i < 2; ++i) {
                const double r = cs.r[i], f = cs.f[i], av = cs.a[i], bv = cs.b[i];
                const double jb = tail_j(r, beta, beta);
                bb[i] += cs.Jbetab * jb;
                rb[i] += cs.Jbetab * bv * jb * (beta - (1.0 - f) / T);
                const double fp = -f * (1.0 - f) / T;
                ab[i] += k0b * f + cs.dGmb * r * f + cs.dGpb * r * (1.0 - f);
                bb[i] += cs.dJbb * r * (1.0 - f) + cs.dJ0b * r * f;
                rb[i] += k0b * av * fp + cs.dGmb * av * (f + r * fp) + cs.dGpb * av * ((1.0 - f) - r * fp) +
                         cs.dJbb * bv * ((1.0 - f) - r * fp) + cs.dJ0b * bv * (f + r * fp);
            }
            const double r1 = cs.r[0], r2 = cs.r[1], d = r1 - r2, d2i = 1.0 / (d * d);
            rb[0] += ab[0] * (-r2 * d2i) + ab[1] * (r2 * d2i);
            rb[1] += ab[0] * (r1 * d2i) + ab[1] * (-r1 * d2i);
            cs.C1bs = (bb[0] - bb[1]) / d;
            const double db = -(bb[0] - bb[1]) * cs.C1 * d2i;
            rb[0] += db;
            rb[1] -= db;
            const double B = mu - cs.e;
            double Bb = 0.0, Cb = 0.0;
            for (int i = 0; i < 2; ++i) {
                Bb += rb[i] * (-cs.r[i] / (2.0 * cs.r[i] + B));
                Cb += rb[i] * (-1.0 / (2.0 * cs.r[i] + B));
            }
            cs.mub = Bb;
            cs.eb = -Bb;
            cs.sinfb = -Cb;
            cs.k0sb = k0b;
            cs.dGsb = cs.dGpb - cs.dGmb;
            cs.dJsb = cs.dJ0b - cs.dJbb;
        }
        __syncthreads();
        // ---- to frequency: FFT_+[ht (Gt_bar + i Jt_bar)]
        if (tid < G) {
            auto in = [&](int j) -> double2 { return cmul(tw_at(ht2, j), make_double2(R[j], Q[j])); };
            group_fft_io<N, +1>(X, tid, (const TwoLevelTw *)tw2, 0, in, ScratchIO{X});
        }
        __syncthreads();
        {
            double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // C1, C2, C3, mu, eps, sinf
            const double e = cs.e, C1 = cs.C1;
            double2 *Fbar = reinterpret_cast<double2 *>(R);
            double2 *sigc = a.sigc + (size_t)c * NO;
            for (int n = tid; n < NO; n += NT) {
                const double kn = (2 * n + 1) * pT, ik = 1.0 / kn, ik2 = ik * ik;
                double2 A, B;
                split_real(X[pidx(n)], X[pidx(N - 1 - n)], A, B);
                const double2 Gsb = make_double2(2.0 * A.x + 2.0 * cs.k0sb, 2.0 * A.y + 2.0 * kn * cs.dGsb);
                const double2 Jsb = make_double2(2.0 * B.x - 2.0 * cs.Jbetab, -2.0 * B.y - 2.0 * kn * cs.dJsb);
                const double2 Gv = wsG[n], J = wsJ[n];
                const double2 Gl = cdiv(make_double2(T, 0.0), make_double2(mu - e, kn + sinf * ik));
                const double2 Gvb = cadd(Gsb, cmul(Jsb, cconj(J)));
                const double2 Jb = cmul(Jsb, cconj(Gv));
                const double2 Glb = csub(make_double2(-Gsb.x, -Gsb.y), cmul(Jsb, make_double2(0.0, C1 * ik)));
                const double2 iGl = cmul(make_double2(0.0, ik), Gl);
                acc[0] += cmul(cconj(iGl), Jsb).x;
                acc[0] += -Jb.y * ik;
                acc[1] += -Jb.x * ik2;
                acc[2] += Jb.y * ik2 * ik;
                const double2 ee = tw_at(ht2, 2 * n + 1);
                const double2 f = make_double2(1.0 - ee.x, -ee.y);
                Fbar[n] = cscale(cmul(cconj(f), Jb), ik2 * ik2);
                const double2 gg = cscale(cmul(Gv, Gv), 1.0 / T);
                sigc[n] = cmul(Gvb, cconj(gg));
                const double rg = cmul(Gvb, cconj(gg)).x;
                acc[3] -= rg;
                acc[4] += rg;
                const double2 q = cscale(cmul(Gl, Gl), -1.0 / T);
                const double rq = cmul(Glb, cconj(q)).x;
                acc[3] += rq;
                acc[4] -= rq;
                acc[5] += cmul(Glb, cconj(cmul(q, make_double2(0.0, ik)))).x;
            }
            block_sum<6>(acc, sums);
        }
        for (int k = tid; k < N; k += NT)
            X[pidx(k)] = k < NO ? reinterpret_cast<const double2 *>(R)[k] : make_double2(0.0, 0.0);
        __syncthreads();
        if (tid < G) group_fft_io<N, -1, false, true>(X, tid, (const TwoLevelTw *)tw2, 0, ScratchIO{X}, ScratchIO{X});
        __syncthreads();
        {
            const double C3b = sums[2];
            for (int i = tid; i <= N; i += NT) {
                const double ym = i >= 1 ? cmul(cconj(tw_at(ht2, i - 1)), X[pidx(i - 1)]).x : 0.0;
                const double y0 = i < N ? cmul(cconj(tw_at(ht2, i)), X[pidx(i)]).x : 0.0;
                double v = ih * (ym - y0);
                if (i == 0) v -= C3b;
                if (i == N) v -= C3b;
                R[i] = v;
            }
        }
        __syncthreads();
        spline_second_derivatives<1, true>(R, NJ, NJ, h, nullptr, nullptr, a.spl_full, a.spl_full + NJ);
        {
            const double C1b = sums[0] + cs.C1bs;
            for (int i = tid; i <= N; i += NT) {
                double v = spline_rT(R, i, N, a6);
                if (i == 0 || i == N) v -= C1b;
                a.hVb[bidx2(i, c, NJ)] = v;
            }
        }
        if (tid == 0) {
            const double C2b = sums[1];
            a.dbb[c] = -b6 * R[0] + C2b;
            a.dbb[(size_t)a.K4p + c] = b6 * R[N] + C2b;
            acc_mu += cs.mub + sums[3];
            acc_sinf += cs.sinfb + sums[5];
            double de, ddek, dd2;
            tp_dirs(cs.l + 1, cs.m, a.nbk, de, ddek, dd2);
            const double d2b = a.kx0b * (-2.0 * cs.wt * nf * cs.k0);
            acc_tp += (cs.eb + sums[4]) * de + cs.dkb * ddek + d2b * dd2;
        }
        __syncthreads();
    }
    if (tid == 0) {
        double *row = a.part + (size_t)blockIdx.x * kAdjW;
        for (int k = 0; k < kAdjW; ++k) row[k] = 0.0;
        row[kAdjMu] = acc_mu;
        row[kAdjSinf] = acc_sinf;
        row[kAdjTh2] = acc_tp;
    }
}

// ---------------------------------------------------------------------------
// kx0 on the kx = 0, pi lines, backward: one block per line point
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_cond_lines_bwd(const double2 *__restrict__ S, const double *__restrict__ s2, const double *__restrict__ s3,
                     const double *__restrict__ sinfp, const double *__restrict__ ek, const double *__restrict__ d2line,
                     int nbk, int nw0, double mu, double T, double nf, double kx0b, double2 *__restrict__ sigl,
                     double *__restrict__ part) {
    const int i = blockIdx.x;
    const int l = i < nbk ? 0 : nbk - 1, m = i % nbk;
    const int o = oct_index(l, m), NO = nw0 / 2;
    const double sinf = sinfp[0], e = ek[o], pT = kPi * T;
    const double w = (m == 0 || m == nbk - 1) ? 1.0 : 2.0;
    const double kkb = kx0b * (-2.0 * w * nf * d2line[i]);
    __shared__ double tot[4];
    double v[4] = {0.0, 0.0, 0.0, 0.0};  // kk, mu, eps, sinf
    for (int n = threadIdx.x; n < NO; n += blockDim.x) {
        const double kn = (2 * n + 1) * pT, ik = 1.0 / kn;
        double rS, iS;
        sigma_full(ik, sinf, s2[o], s3[o], S[bidx(n, o, NO)], rS, iS);
        const double2 Gv = cdiv(make_double2(T, 0.0), make_double2(mu - e - rS, kn - iS));
        const double2 Gt = cdiv(make_double2(T, 0.0), make_double2(mu - e, kn + sinf * ik));
        v[0] += Gv.x - Gt.x;
        const double2 gg = cscale(cmul(Gv, Gv), 1.0 / T);
        const double2 Gvb = make_double2(2.0 * kkb, 0.0), Gtb = make_double2(-2.0 * kkb, 0.0);
        sigl[(size_t)i * NO + n] = cmul(Gvb, cconj(gg));
        const double rg = cmul(Gvb, cconj(gg)).x;
        v[1] -= rg;
        v[2] += rg;
        const double2 q = cscale(cmul(Gt, Gt), -1.0 / T);
        const double rq = cmul(Gtb, cconj(q)).x;
        v[1] += rq;
        v[2] -= rq;
        v[3] += cmul(Gtb, cconj(cmul(q, make_double2(0.0, ik)))).x;
    }
    block_sum<4>(v, tot);
    if (threadIdx.x == 0) {
        double r[2];
        real_roots(mu - e, sinf, r[0], r[1]);
        const double d = r[0] - r[1], d2i = 1.0 / (d * d);
        const double av[2] = {r[0] / d, -r[1] / d};
        double kk = 2.0 * tot[0], ab[2], rb[2];
        for (int q = 0; q < 2; ++q) {
            const double f = fermi_fn(r[q], T);
            kk += av[q] * f;
            ab[q] = kkb * f;
            rb[q] = kkb * av[q] * (-f * (1.0 - f) / T);
        }
        rb[0] += ab[0] * (-r[1] * d2i) + ab[1] * (r[1] * d2i);
        rb[1] += ab[0] * (r[0] * d2i) + ab[1] * (-r[0] * d2i);
        const double B = mu - e;
        double Bb = 0.0, Cb = 0.0;
        for (int q = 0; q < 2; ++q) {
            Bb += rb[q] * (-r[q] / (2.0 * r[q] + B));
            Cb += rb[q] * (-1.0 / (2.0 * r[q] + B));
        }
        const double mub = tot[1] + Bb, eb = tot[2] - Bb, sinfb = tot[3] - Cb;
        const double d2lb = kx0b * (-2.0 * w * nf * kk);
        const double kx = l * kPi / (nbk - 1), ky = m * kPi / (nbk - 1);
        const double cc = cos(kx) * cos(ky);
        double *row = part + (size_t)i * kAdjW;
        for (int k = 0; k < kAdjW; ++k) row[k] = 0.0;
        row[kAdjMu] = mub;
        row[kAdjSinf] = sinfb;
        row[kAdjTh2] = eb * (-4.0 * cc) + d2lb * (4.0 * cc);
    }
}

// ---------------------------------------------------------------------------
// the h slices of chi_jj, backward
// ---------------------------------------------------------------------------
namespace {
// x = eps - mu0 and A, E(t) of the h slice at K4 point c (k_cond_table):
// h(t) = A E(t), E = e^{-x t} (x > 0) or e^{x (beta - t)} (x <= 0)
struct HPoint {
    double x, A, base, dbase;
};
__device__ __forceinline__ HPoint h_point(const double *ek, const double *dek, int c, int nbk, double mu0, double T,
                                          double nf) {
    const int l = c / nbk, m = c % nbk;
    HPoint p;
    p.x = ek[oct_index(l + 1, m)] - mu0;
    const double f = fermi_fn(p.x, T);
    p.base = p.x > 0 ? 1.0 - f : f;
    p.dbase = (p.x > 0 ? 1.0 : -1.0) * f * (1.0 - f) / T;
    p.A = nf * dek[c] * p.base;
    return p;
}
__device__ __forceinline__ double h_E(double x, double t, double beta) {
    return x > 0 ? exp(-x * t) : exp(x * (beta - t));
}
__device__ __forceinline__ double h_dEdx(double x, double t, double beta) { return x > 0 ? -t : beta - t; }
}  // namespace

// kind = blockIdx.x (0: dhV(0), 1: dhV(beta)): u = T^T dbb_kind; V(0) and
// the end-value cotangents; D_kind's cotangent through its transform into
// the parameter directions.  tmp: [2][K4p] scratch for u.
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_cond_boundary_bwd(const double *__restrict__ ek, const double *__restrict__ dek, const double *__restrict__ V,
                        const double *__restrict__ dchirt0, const double *__restrict__ pre,
                        const double2 *__restrict__ tw, const double *__restrict__ dbb, int nw0, int K4p, double mu0,
                        double T, double nf, double fact, double dmu0_2, double *__restrict__ tmp,
                        double *__restrict__ vbk, double *__restrict__ preb, double *__restrict__ dchb,
                        double *__restrict__ part) {
    constexpr int K4 = (NBK - 2) * NBK;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int kind = blockIdx.x;
    const double sg = kind ? -1.0 : 1.0, beta = 1.0 / T, tE = kind ? beta : 0.0;
    const int nb = nw0 / 2 + 1;
    double *u = tmp + (size_t)kind * K4p;
    // u = T^T dbb
    for (int c = threadIdx.x; c < K4; c += blockDim.x) S[c] = dbb[(size_t)kind * K4p + c] / edge_w(c % NBK, NBK);
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    for (int c = threadIdx.x; c < K4; c += blockDim.x) u[c] = S[c] * edge_w(c % NBK, NBK);
    __syncthreads();
    // D = T v_kind, v = -x A E(tE)
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const HPoint p = h_point(ek, dek, c, NBK, mu0, T, nf);
        S[c] = -p.x * p.A * h_E(p.x, tE, beta);
    }
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    double f4b = 0.0;
    const double *pe = pre + (size_t)kind * K4p;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const int l = c / NBK, m = c % NBK;
        const int o = oct_index(l + 1, m);
        const double uc = u[c], v0 = V[bidx(0, o, nb)];
        vbk[(size_t)kind * K4p + c] = 2.0 * S[c] * uc;
        preb[(size_t)kind * K4p + c] = sg * fact * dchirt0[o] * uc;
        dchb[(size_t)kind * K4p + c] = sg * pe[c] * fact * uc;
        f4b += sg * pe[c] * dchirt0[o] * uc;
        S[c] = 2.0 * v0 * uc / edge_w(m, NBK);
    }
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    double th1 = 0.0, th2 = 0.0;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const int l = c / NBK, m = c % NBK;
        const double vb = S[c] * edge_w(m, NBK);
        const HPoint p = h_point(ek, dek, c, NBK, mu0, T, nf);
        const double E = h_E(p.x, tE, beta), dE = h_dEdx(p.x, tE, beta) * E;
        double de, ddek, dd2;
        tp_dirs(l + 1, m, NBK, de, ddek, dd2);
        // v = -x A E;  dv = -(dx A E + x dA E + x A dE),  dA = nf dk dbase dx + nf base ddek
        auto dv = [&](double dx, double dk_dir) {
            const double dA = nf * dek[c] * p.dbase * dx + nf * p.base * dk_dir;
            return -(dx * p.A * E + p.x * dA * E + p.x * p.A * dE * dx);
        };
        th1 += vb * dv(-1.0, 0.0);
        th2 += vb * dv(de - dmu0_2, ddek);
    }
    double v3[3] = {f4b, th1, th2};
    __shared__ double tot[3];
    block_sum<3>(v3, tot);
    if (threadIdx.x == 0) {
        double *row = part + (size_t)kind * kAdjW;
        for (int k = 0; k < kAdjW; ++k) row[k] = 0.0;
        row[kAdjFact4] = tot[0];
        row[kAdjTh1] = tot[1];
        row[kAdjTh2] = tot[2];
    }
}

// per-K4-point table of the h slices' backward: (x, A, dA/dx, dA/d dek,
// dx/dt', d dek/dt') with x = eps - mu0, A = nf dek (1 - f) or nf dek f
// (the branch of k_cond_table), the t' direction at fixed density
__global__ void k_hbwd_table(const double *__restrict__ ek, const double *__restrict__ dek, int K4, int nbk,
                             double mu0, double T, double nf, double dmu0_2, double *__restrict__ tab) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= K4) return;
    const HPoint p = h_point(ek, dek, c, nbk, mu0, T, nf);
    double de, ddek, dd2;
    tp_dirs(c / nbk + 1, c % nbk, nbk, de, ddek, dd2);
    double *t = tab + 8 * (size_t)c;
    t[0] = p.x;
    t[1] = p.A;
    t[2] = nf * dek[c] * p.dbase;
    t[3] = nf * p.base;
    t[4] = de - dmu0_2;
    t[5] = ddek;
    t[6] = 0.0;
    t[7] = 0.0;
}

// CTA jv = 0..Nw0/2 takes tau_j and tau_{Nw0 - j} (j = jv): u_j = T^T hVb(j);
// V-bar(jv) in the K4 layout (2 h_j u_j summed over the pair) -> vcond; the
// cotangent of h_j (2 V u_j, plus the boundary's at tau = 0, beta) through
// T^T into the parameter directions.  tmpU: [nb][K4p] scratch.
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_cond_slice_bwd(const double *__restrict__ htab, const double *__restrict__ V, const double *__restrict__ hVb,
                     const double *__restrict__ preb, const double2 *__restrict__ tw, int nw0, int K4p, double T,
                     double *__restrict__ tmpU, double *__restrict__ vcond, double *__restrict__ part) {
    constexpr int K4 = (NBK - 2) * NBK;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int jv = blockIdx.x, nb = nw0 / 2 + 1;
    const double beta = 1.0 / T;
    double *u = tmpU + (size_t)jv * K4p;
    double *vc = vcond + (size_t)jv * K4p;
    double th1 = 0.0, th2 = 0.0;
    const int nj = (jv == 0 || jv == nb - 1) ? (jv == 0 ? 2 : 1) : 2;
#pragma unroll 1
    for (int q = 0; q < nj; ++q) {
        const int j = q == 0 ? jv : nw0 - jv;
        const double t = j / (nw0 * T);
        // u = T^T hVb(j)
        for (int c = threadIdx.x; c < K4; c += blockDim.x) S[c] = hVb[bidx2(j, c, nw0 + 1)] / edge_w(c % NBK, NBK);
        __syncthreads();
        dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
        for (int c = threadIdx.x; c < K4; c += blockDim.x) u[c] = S[c] * edge_w(c % NBK, NBK);
        __syncthreads();
        // h_j = T (A E(t))
        for (int c = threadIdx.x; c < K4; c += blockDim.x) {
            const double2 xa = *reinterpret_cast<const double2 *>(htab + 8 * (size_t)c);
            S[c] = xa.y * h_E(xa.x, t, beta);
        }
        __syncthreads();
        dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
        for (int c = threadIdx.x; c < K4; c += blockDim.x) {
            const int l = c / NBK, m = c % NBK;
            const double uc = u[c];
            const double add = 2.0 * S[c] * uc;
            vc[c] = q == 0 ? add : vc[c] + add;
            double hb = 2.0 * V[bidx(jv, oct_index(l + 1, m), nb)] * uc;
            if (j == 0) hb += preb[c];
            if (j == nw0) hb += preb[(size_t)K4p + c];
            S[c] = hb / edge_w(m, NBK);
        }
        __syncthreads();
        dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
        for (int c = threadIdx.x; c < K4; c += blockDim.x) {
            const double s = S[c] * edge_w(c % NBK, NBK);
            const double *tc = htab + 8 * (size_t)c;
            const double2 xa = *reinterpret_cast<const double2 *>(tc);
            const double2 gb = *reinterpret_cast<const double2 *>(tc + 2);
            const double2 dd = *reinterpret_cast<const double2 *>(tc + 4);
            const double E = h_E(xa.x, t, beta), dEx = h_dEdx(xa.x, t, beta) * E;
            // d(A E) = (dA/dx E + A dE/dx) dx + dA/d dek E d dek
            const double gx = gb.x * E + xa.y * dEx;
            th1 += s * (-gx);
            th2 += s * (gx * dd.x + gb.y * E * dd.y);
        }
        __syncthreads();
    }
    double v2[2] = {th1, th2};
    __shared__ double tot[2];
    block_sum<2>(v2, tot);
    if (threadIdx.x == 0) {
        double *row = part + (size_t)jv * kAdjW;
        for (int k = 0; k < kAdjW; ++k) row[k] = 0.0;
        row[kAdjTh1] = tot[0];
        row[kAdjTh2] = tot[1];
    }
}

// ---------------------------------------------------------------------------
// Sigma-bar: gather of the K4 columns and lines, the implicit mu step
// (lam d traceDiffG / d Sigma, eps, mu0) and the map to (S, C2, C3, Sinf, S4).
// One block per octant point o.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
    k_sigbar(const double2 *__restrict__ sigc, const double2 *__restrict__ sigl, const double2 *__restrict__ S,
             const double *__restrict__ s2, const double *__restrict__ s3, const double *__restrict__ s4,
             const double *__restrict__ sinfp, const double *__restrict__ ek, const double *__restrict__ w16, int nbk,
             int nw0, double mu0, double mu, double lam, double T, double dmu0_2, double2 *__restrict__ Sb,
             double *__restrict__ s2b, double *__restrict__ s3b, double *__restrict__ part) {
    const int o = blockIdx.x, NO = nw0 / 2;
    int lo, mo;
    oct_lm(o, lo, mo);
    const int c1 = (lo >= 1 && lo <= nbk - 2) ? (lo - 1) * nbk + mo : -1;
    const int c2 = (mo >= 1 && mo <= nbk - 2 && mo != lo) ? (mo - 1) * nbk + lo : -1;
    const int i1 = mo == 0 ? lo : -1;
    const int i2 = lo == nbk - 1 ? nbk + mo : -1;
    const double e = ek[o], w = w16[o], sinf = sinfp[0], pT = kPi * T;
    const double kx = lo * kPi / (nbk - 1), ky = mo * kPi / (nbk - 1);
    const double de = -4.0 * cos(kx) * cos(ky);
    double v[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // s2b, s3b, s4b, sinfb, th1, th2
    auto mu_terms = [&](double wn, double rS, double iS, double2 &tb) {
        const double2 Gv = cdiv(make_double2(1.0, 0.0), make_double2(mu - e - rS, wn - iS));
        const double2 G0 = cdiv(make_double2(1.0, 0.0), make_double2(mu0 - e, wn));
        const double2 gg = cmul(Gv, Gv), g0 = cmul(G0, G0);
        tb = cscale(cconj(gg), lam * w);
        v[4] += lam * w * g0.x;
        v[5] += lam * w * ((gg.x - g0.x) * de + g0.x * dmu0_2);
    };
    for (int n = threadIdx.x; n < NO; n += blockDim.x) {
        const double wn = (2 * n + 1) * pT, iw = 1.0 / wn;
        double2 sf = make_double2(0.0, 0.0);
        if (c1 >= 0) sf = cadd(sf, sigc[(size_t)c1 * NO + n]);
        if (c2 >= 0) sf = cadd(sf, sigc[(size_t)c2 * NO + n]);
        if (i1 >= 0) sf = cadd(sf, sigl[(size_t)i1 * NO + n]);
        if (i2 >= 0) sf = cadd(sf, sigl[(size_t)i2 * NO + n]);
        double rS, iS;
        sigma_full(iw, sinf, s2[o], s3[o], S[bidx(n, o, NO)], rS, iS);
        double2 tb;
        mu_terms(wn, rS, iS, tb);
        sf = cadd(sf, tb);
        const double iw2 = iw * iw;
        Sb[(size_t)o * NO + n] = cscale(sf, iw2 * iw2);
        v[0] += -sf.x * iw2;
        v[1] += sf.y * iw2 * iw;
        v[3] += -sf.y * iw;
    }
    for (int n = NO + threadIdx.x; n <= nw0; n += blockDim.x) {
        const double wn = (2 * n + 1) * pT, iw = 1.0 / wn, iw2 = iw * iw;
        const double rS = -s2[o] * iw2 + s4[o] * iw2 * iw2;
        const double iS = -sinf * iw + s3[o] * iw2 * iw;
        double2 tb;
        mu_terms(wn, rS, iS, tb);
        v[0] += -tb.x * iw2;
        v[2] += tb.x * iw2 * iw2;
        v[1] += tb.y * iw2 * iw;
        v[3] += -tb.y * iw;
    }
    __shared__ double tot[6];
    block_sum<6>(v, tot);
    if (threadIdx.x == 0) {
        s2b[o] = tot[0];
        s3b[o] = tot[1];
        Sb[(size_t)o * NO + NO - 1].x += tot[2];
        double *row = part + (size_t)o * kAdjW;
        for (int k = 0; k < kAdjW; ++k) row[k] = 0.0;
        row[kAdjSinf] = tot[3];
        row[kAdjTh1] = tot[4];
        row[kAdjTh2] = tot[5];
    }
}

// ---------------------------------------------------------------------------
// Sigma's tau transform, backward: one octant column per CTA
// ---------------------------------------------------------------------------
template <int N>
struct SigTauBwdSmem {
    static constexpr size_t x_bytes = (size_t)padded_len(N) * sizeof(double2);
    static constexpr size_t r_bytes = ((size_t)(N + 1) * sizeof(double) + 15) & ~(size_t)15;
    static constexpr size_t tw_off = x_bytes + r_bytes;
    static constexpr size_t bytes = tw_off + 2 * sizeof(TwoLevelTw);
};

template <int N>
__global__ void __launch_bounds__(256, 2)
    k_sigma_tau_bwd(const double2 *__restrict__ Sb, const double *__restrict__ s2b, const double *__restrict__ s3b,
                    double sinfb, const double *__restrict__ spl, const double2 *__restrict__ tw,
                    const double2 *__restrict__ ht, double T, int n8, int n8p, double *__restrict__ stb,
                    double *__restrict__ dSb) {
    constexpr int NJ = N + 1, NO = N / 2, G = FftPlan<N>::G;
    using SM = SigTauBwdSmem<N>;
    extern __shared__ __align__(16) double smem[];
    char *base = reinterpret_cast<char *>(smem);
    double2 *X = reinterpret_cast<double2 *>(smem);
    double *R = reinterpret_cast<double *>(base + SM::x_bytes);
    TwoLevelTw *tw2 = reinterpret_cast<TwoLevelTw *>(base + SM::tw_off);
    const TwoLevelTw *ht2 = tw2 + 1;
    tau_tables(tw2, tw2 + 1, tw, ht, N);
    const int o = blockIdx.x, tid = threadIdx.x, NT = blockDim.x;
    const double h = 1.0 / (N * T), ih = 1.0 / h, a6 = 6.0 / (h * h), b6 = 6.0 / h;
    __syncthreads();
    for (int k = tid; k < N; k += NT) {
        double2 v = make_double2(0.0, 0.0);
        if (k < NO) {
            const double2 ee = tw_at(ht2, 2 * k + 1);
            v = cmul(Sb[(size_t)o * NO + k], make_double2(1.0 - ee.x, ee.y));
        }
        X[pidx(k)] = v;
    }
    __syncthreads();
    if (tid < G) group_fft_io<N, -1, false, true>(X, tid, (const TwoLevelTw *)tw2, 0, ScratchIO{X}, ScratchIO{X});
    __syncthreads();
    const double c3 = s3b[o];
    for (int i = tid; i <= N; i += NT) {
        const double ym = i >= 1 ? cmul(cconj(tw_at(ht2, i - 1)), X[pidx(i - 1)]).x : 0.0;
        const double y0 = i < N ? cmul(cconj(tw_at(ht2, i)), X[pidx(i)]).x : 0.0;
        double v = ih * (ym - y0);
        if (i == 0 || i == N) v -= c3;
        R[i] = v;
    }
    __syncthreads();
    spline_second_derivatives<1, true>(R, NJ, NJ, h, nullptr, nullptr, spl, spl + NJ);
    for (int i = tid; i <= N; i += NT) {
        double v = spline_rT(R, i, N, a6);
        if (o == 0 && (i == 0 || i == N)) v -= sinfb;
        stb[bidx(i, o, NJ)] = v;
    }
    if (tid == 0) {
        dSb[o] = -b6 * R[0] + s2b[o];
        dSb[(size_t)n8p + o] = b6 * R[N] + s2b[o];
    }
}

// ---------------------------------------------------------------------------
// Sigma's slices, backward: CTA jv takes tau_j, tau_{Nw0-j}; V-bar(jv) from
// them, the chi_jj slices (K4 layout) and, at jv = 0, the chi_jj boundary;
// G(r, tau)'s cotangent contracted with its two tangents.
// ---------------------------------------------------------------------------
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_sigma_slice_bwd(const double *__restrict__ stb, const double *__restrict__ Grt, const double *__restrict__ V,
                      const double *__restrict__ dGrt1, const double *__restrict__ dGrt2,
                      const double *__restrict__ vcond, const double *__restrict__ vbk, const double2 *__restrict__ tw,
                      int nw0, int K4p, double *__restrict__ Vb, double *__restrict__ part) {
    constexpr int n8 = NBK * (NBK + 1) / 2;
    constexpr int NR = (n8 + kSliceThreads - 1) / kSliceThreads;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int jv = blockIdx.x, nb = nw0 / 2 + 1;
    double vacc[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) vacc[k] = 0.0;
    double th1 = 0.0, th2 = 0.0;
    const int nj = jv == 0 ? 2 : (jv == nb - 1 ? 1 : 2);
#pragma unroll 1
    for (int q = 0; q < nj; ++q) {
        const int j = q == 0 ? jv : nw0 - jv;
        for (int o = threadIdx.x; o < n8; o += blockDim.x) {
            int l, m;
            oct_lm(o, l, m);
            put_sym<NBK>(S, l, m, stb[bidx(j, o, nw0 + 1)] / oct_tw(l, m, NBK));
        }
        __syncthreads();
        dct2_slice<NBK>(S, slice_scratch<NBK>(S), tws);
        int k = 0;
        const size_t rj = (size_t)j * n8;
        for (int o = threadIdx.x; o < n8; o += blockDim.x, ++k) {
            int l, m;
            oct_lm(o, l, m);
            const double u = S[l * NBK + m] * oct_tw(l, m, NBK);
            vacc[k] += Grt[rj + o] * u;
            const double gb = V[bidx(jv, o, nb)] * u;
            th1 += gb * dGrt1[rj + o];
            th2 += gb * dGrt2[rj + o];
        }
        __syncthreads();
    }
    int k = 0;
    const double *vc = vcond + (size_t)jv * K4p;
    for (int o = threadIdx.x; o < n8; o += blockDim.x, ++k) {
        int lo, mo;
        oct_lm(o, lo, mo);
        double v = vacc[k];
        if (lo >= 1 && lo <= NBK - 2) {
            const int c = (lo - 1) * NBK + mo;
            v += vc[c];
            if (jv == 0) v += vbk[c] + vbk[(size_t)K4p + c];
        }
        if (mo >= 1 && mo <= NBK - 2 && mo != lo) {
            const int c = (mo - 1) * NBK + lo;
            v += vc[c];
            if (jv == 0) v += vbk[c] + vbk[(size_t)K4p + c];
        }
        Vb[bidx(jv, o, nb)] = v;
    }
    double v2[2] = {th1, th2};
    __shared__ double tot[2];
    block_sum<2>(v2, tot);
    if (threadIdx.x == 0) {
        double *row = part + (size_t)jv * kAdjW;
        for (int i = 0; i < kAdjW; ++i) row[i] = 0.0;
        row[kAdjTh1] = tot[0];
        row[kAdjTh2] = tot[1];
    }
}

// Sigma's end conditions, backward (one CTA): u0 = A^T dSb(0), ub = A^T
// dSb(beta); V-bar(0) += ..., fact's cotangent, and the cotangents of
// d/dtau chi0(r, 0) (plus the chi_jj boundary's, K4 layout), d/dtau G(r, 0+),
// G(r, 0+), G(r, beta-) and the hopping table contracted with their tangents.
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_sigma_boundary_bwd(const double *__restrict__ dSb, const double *__restrict__ Grt, const double *__restrict__ V,
                         const double *__restrict__ dchirt0, const double *__restrict__ dG0p,
                         const double *__restrict__ er, const double *__restrict__ dchb,
                         const double *__restrict__ dGrt1, const double *__restrict__ dGrt2,
                         const double *__restrict__ ddG0p1, const double *__restrict__ ddG0p2,
                         const double *__restrict__ ddchir1, const double *__restrict__ ddchir2,
                         const double *__restrict__ der2, const double2 *__restrict__ tw, int nw0, int n8p, int K4p,
                         double mu0, double fact8, double dmu0_2, double *__restrict__ Vb, double *__restrict__ part) {
    constexpr int n8 = NBK * (NBK + 1) / 2;
    constexpr int NR = (n8 + kSliceThreads - 1) / kSliceThreads;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int nb = nw0 / 2 + 1;
    double u[2][NR];
#pragma unroll 1
    for (int side = 0; side < 2; ++side) {
        for (int o = threadIdx.x; o < n8; o += blockDim.x) {
            int l, m;
            oct_lm(o, l, m);
            put_sym<NBK>(S, l, m, dSb[(size_t)side * n8p + o] / oct_tw(l, m, NBK));
        }
        __syncthreads();
        dct2_slice<NBK>(S, slice_scratch<NBK>(S), tws);
        int k = 0;
        for (int o = threadIdx.x; o < n8; o += blockDim.x, ++k) {
            int l, m;
            oct_lm(o, l, m);
            u[side][k] = S[l * NBK + m] * oct_tw(l, m, NBK);
        }
        __syncthreads();
    }
    double f8b = 0.0, th1 = 0.0, th2 = 0.0;
    int k = 0;
    const double *g0 = Grt, *gN = Grt + (size_t)nw0 * n8;
    const double *d10 = dGrt1, *d1N = dGrt1 + (size_t)nw0 * n8;
    const double *d20 = dGrt2, *d2N = dGrt2 + (size_t)nw0 * n8;
    for (int o = threadIdx.x; o < n8; o += blockDim.x, ++k) {
        int lo, mo;
        oct_lm(o, lo, mo);
        const double u0 = u[0][k], ub = u[1][k];
        const double dc = dchirt0[o];
        f8b += dc * (g0[o] * u0 - gN[o] * ub);
        double dcb = fact8 * (g0[o] * u0 - gN[o] * ub);
        if (lo >= 1 && lo <= NBK - 2) {
            const int c = (lo - 1) * NBK + mo;
            dcb += dchb[c] + dchb[(size_t)K4p + c];
        }
        if (mo >= 1 && mo <= NBK - 2 && mo != lo) {
            const int c = (mo - 1) * NBK + lo;
            dcb += dchb[c] + dchb[(size_t)K4p + c];
        }
        const double g0b = fact8 * dc * u0, gNb = -fact8 * dc * ub;
        th1 += g0b * d10[o] + gNb * d1N[o];
        th2 += g0b * d20[o] + gNb * d2N[o];
        const double xi = (o == 0) ? -mu0 : er[o];
        const double v0 = V[bidx(0, o, nb)];
        Vb[bidx(0, o, nb)] += dG0p[o] * u0 + (-dG0p[o] + xi) * ub;
        const double dgb = v0 * (u0 - ub), xib = v0 * ub;
        th1 += dgb * ddG0p1[o] + dcb * ddchir1[o] + xib * (o == 0 ? -1.0 : 0.0);
        th2 += dgb * ddG0p2[o] + dcb * ddchir2[o] + xib * (o == 0 ? -dmu0_2 : der2[o]);
    }
    double v3[3] = {f8b, th1, th2};
    __shared__ double tot[3];
    block_sum<3>(v3, tot);
    if (threadIdx.x == 0) {
        for (int i = 0; i < kAdjW; ++i) part[i] = 0.0;
        part[kAdjFact8] = tot[0];
        part[kAdjTh1] = tot[1];
        part[kAdjTh2] = tot[2];
    }
}

// ---------------------------------------------------------------------------
// V's tau transform, backward: one octant column per CTA.  V(tau) = DCT-I_n
// [Vq-transform] + fact chi0(r, tau): fact's cotangent, chi0(r, tau)'s
// cotangent contracted with its two tangents (formed from G and its tangents
// as k_chi0_slice_tan does), and the column's transpose DCT-I in place.
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(256, 2)
    k_vertex_tau_bwd(double *__restrict__ Vb, const double *__restrict__ chirt, const double *__restrict__ Grt,
                     const double *__restrict__ dGrt1, const double *__restrict__ dGrt2, const double2 *__restrict__ tw,
                     double fact8, int n8, double *__restrict__ part) {
    constexpr int NJ = N / 2 + 1, NO = N / 2, G = FftPlan<N>::G;
    extern __shared__ __align__(16) double smem[];
    double2 *X = reinterpret_cast<double2 *>(smem);
    TwoLevelTw *tw2 = reinterpret_cast<TwoLevelTw *>(reinterpret_cast<char *>(smem) + padded_len(N) * sizeof(double2));
    __shared__ double col[NJ];
    tau_tables(tw2, tw2 + 1, tw, tw, N);
    const int o = blockIdx.x, tid = threadIdx.x, NT = blockDim.x;
    double v[3] = {0.0, 0.0, 0.0};  // fact8, th1, th2
    for (int j = tid; j < NJ; j += NT) {
        const double vb = Vb[bidx(j, o, NJ)];
        col[j] = vb;
        v[0] += vb * chirt[bidx(j, o, NJ)];
        const double a = Grt[(size_t)j * n8 + o];
        const double *dg[2] = {dGrt1, dGrt2};
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const double da = dg[p][(size_t)j * n8 + o];
            double dc;
            if (j == 0)
                dc = (o == 0) ? -2.0 * da * (2.0 * a + 1.0) : -4.0 * a * da;
            else if (j == NO)
                dc = 4.0 * a * da;
            else
                dc = 2.0 * (dg[p][(size_t)(N - j) * n8 + o] * a + Grt[(size_t)(N - j) * n8 + o] * da);
            v[1 + p] += fact8 * vb * dc;
        }
    }
    __syncthreads();
    if (tid < G) {
        auto in = [&](int j) -> double2 {
            const int jj = j < NJ ? j : N - j;
            return make_double2(col[jj] / edge_w(jj, NJ), 0.0);
        };
        group_fft_io<N, -1>(X, tid, (const TwoLevelTw *)tw2, 0, in, ScratchIO{X});
    }
    __syncthreads();
    for (int n = tid; n < NJ; n += NT) Vb[bidx(n, o, NJ)] = X[pidx(n)].x * edge_w(n, NJ);
    __shared__ double tot[3];
    block_sum<3>(v, tot);
    if (tid == 0) {
        double *row = part + (size_t)o * kAdjW;
        for (int i = 0; i < kAdjW; ++i) row[i] = 0.0;
        row[kAdjFact8] = tot[0];
        row[kAdjTh1] = tot[1];
        row[kAdjTh2] = tot[2];
    }
}

// V(q, iqn)'s slices, backward: one bosonic frequency per CTA; Vq-bar =
// A^T (transposed V-bar column), then the RPA factors' derivatives: chi0's
// cotangent contracted with its two tangents, and Usp, Uch, U.
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_vertex_q_bwd(const double *__restrict__ Vb, const double *__restrict__ chiq, const double *__restrict__ dchiq1,
                   const double *__restrict__ dchiq2, const double2 *__restrict__ tw, int nb, double normFact,
                   double U, double Usp, double Uch, double *__restrict__ part) {
    constexpr int n8 = NBK * (NBK + 1) / 2;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int n = blockIdx.x;
    for (int o = threadIdx.x; o < n8; o += blockDim.x) {
        int l, m;
        oct_lm(o, l, m);
        put_sym<NBK>(S, l, m, Vb[bidx(n, o, nb)] / oct_tw(l, m, NBK));
    }
    __syncthreads();
    dct2_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    const double nU = normFact * U;
    double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // th1, th2, Usp, Uch, U
    for (int o = threadIdx.x; o < n8; o += blockDim.x) {
        int l, m;
        oct_lm(o, l, m);
        const double qb = S[l * NBK + m] * oct_tw(l, m, NBK);
        const size_t ix = bidx(n, o, nb);
        const double c0 = chiq[ix];
        const double dsp = 1.0 - Usp * c0 / 2.0, dch = 1.0 + Uch * c0 / 2.0;
        const double csp = c0 / dsp, cch = c0 / dch;
        const double vq = nU * (3.0 * Usp * (csp - c0) + Uch * (cch - c0)) / 8.0;
        const double cb = qb * nU / 8.0 * (3.0 * Usp * (1.0 / (dsp * dsp) - 1.0) + Uch * (1.0 / (dch * dch) - 1.0));
        v[0] += cb * dchiq1[ix];
        v[1] += cb * dchiq2[ix];
        v[2] += qb * nU / 8.0 * (3.0 * (csp - c0) + 3.0 * Usp * c0 * c0 / (2.0 * dsp * dsp));
        v[3] += qb * nU / 8.0 * ((cch - c0) - Uch * c0 * c0 / (2.0 * dch * dch));
        v[4] += qb * vq / U;
    }
    __shared__ double tot[5];
    block_sum<5>(v, tot);
    if (threadIdx.x == 0) {
        double *row = part + (size_t)n * kAdjW;
        for (int i = 0; i < kAdjW; ++i) row[i] = 0.0;
        row[kAdjTh1] = tot[0];
        row[kAdjTh2] = tot[1];
        row[kAdjUsp] = tot[2];
        row[kAdjUch] = tot[3];
        row[kAdjU] = tot[4];
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
namespace {
template <int N>
struct RunCondTauBwd {
    static cudaError_t run(const CondBwdArgs *a, int nblk, cudaStream_t st) {
        const size_t sm = CondBwdSmem<N>::bytes;
        cudaError_t e = set_smem(k_cond_tau_bwd<N>, sm);
        if (e != cudaSuccess) return e;
        k_cond_tau_bwd<N><<<nblk, cond_bwd_threads<N>(), sm, st>>>(*a);
        return launched();
    }
};
template <int N>
struct CondBwdBlocks {
    static cudaError_t run(int *blocks) {
        const size_t sm = CondBwdSmem<N>::bytes;
        cudaError_t e = set_smem(k_cond_tau_bwd<N>, sm);
        if (e != cudaSuccess) return e;
        int dev = 0, sms = 0, per = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cond_tau_bwd<N>, cond_bwd_threads<N>(), sm)) !=
            cudaSuccess)
            return e;
        *blocks = sms * (per > 0 ? per : 1);
        return cudaSuccess;
    }
};
template <int NBK>
struct RunCondSliceBwd {
    static cudaError_t run(const GridDev *g, const CondDev *c, const AdjDev *a, const double *V,
                           const double *dchirt0, double mu0, double T, double fact4, double dmu0_2, cudaStream_t st) {
        const size_t sm = SliceSmem<NBK>::bytes;
        cudaError_t e = set_smem(k_cond_boundary_bwd<NBK>, sm);
        if (e != cudaSuccess) return e;
        if ((e = set_smem(k_cond_slice_bwd<NBK>, sm)) != cudaSuccess) return e;
        const double nf = 1.0 / ((double)g->nk0 * g->nk0);
        k_cond_boundary_bwd<NBK><<<2, kSliceThreads, sm, st>>>(g->ek, c->dek, V, dchirt0, c->pre, g->tw_k, a->dbb,
                                                                g->nw0, c->K4p, mu0, T, nf, fact4, dmu0_2, a->tmpB,
                                                                a->vbk, a->preb, a->dchb, a->part + a->row_cb * kAdjW);
        if ((e = launched()) != cudaSuccess) return e;
        k_hbwd_table<<<(c->K4 + 255) / 256, 256, 0, st>>>(g->ek, c->dek, c->K4, g->nbk, mu0, T, nf, dmu0_2, a->htab);
        if ((e = launched()) != cudaSuccess) return e;
        k_cond_slice_bwd<NBK><<<g->nb, kSliceThreads, sm, st>>>(a->htab, V, a->hVb, a->preb, g->tw_k, g->nw0, c->K4p,
                                                                 T, a->tmpU, a->vcond, a->part + a->row_cs * kAdjW);
        return launched();
    }
};
template <int N>
struct RunSigmaTauBwd {
    static cudaError_t run(const GridDev *g, const AdjDev *a, double sinfb, double T, cudaStream_t st) {
        const size_t sm = SigTauBwdSmem<N>::bytes;
        cudaError_t e = set_smem(k_sigma_tau_bwd<N>, sm);
        if (e != cudaSuccess) return e;
        k_sigma_tau_bwd<N><<<g->n8, 256, sm, st>>>(a->Sb, a->s2b, a->s3b, sinfb, g->spl_full, g->tw_w, g->ht_w, T,
                                                   g->n8, g->n8p, a->stb, a->dSb);
        return launched();
    }
};
template <int NBK>
struct RunSigmaSliceBwd {
    static cudaError_t run(const GridDev *g, const CondDev *c, const AdjDev *a, const double *Grt, const double *V,
                           const double *dchirt0, const double *dG0p, double mu0, double fact8, double dmu0_2,
                           cudaStream_t st) {
        const size_t sm = SliceSmem<NBK>::bytes;
        cudaError_t e = set_smem(k_sigma_slice_bwd<NBK>, sm);
        if (e != cudaSuccess) return e;
        if ((e = set_smem(k_sigma_boundary_bwd<NBK>, sm)) != cudaSuccess) return e;
        k_sigma_slice_bwd<NBK><<<g->nb, kSliceThreads, sm, st>>>(a->stb, Grt, V, a->dGrt[0], a->dGrt[1], a->vcond,
                                                                  a->vbk, g->tw_k, g->nw0, c->K4p, a->Vb,
                                                                  a->part + a->row_ss * kAdjW);
        if ((e = launched()) != cudaSuccess) return e;
        k_sigma_boundary_bwd<NBK><<<1, kSliceThreads, sm, st>>>(
            a->dSb, Grt, V, dchirt0, dG0p, g->er, a->dchb, a->dGrt[0], a->dGrt[1], a->ddG0p[0], a->ddG0p[1],
            a->ddchir[0], a->ddchir[1], a->der2, g->tw_k, g->nw0, g->n8p, c->K4p, mu0, fact8, dmu0_2, a->Vb,
            a->part + a->row_sb * kAdjW);
        return launched();
    }
};
template <int N>
struct RunVertexTauBwd {
    static cudaError_t run(const GridDev *g, const AdjDev *a, const double *chirt, const double *Grt, double fact8,
                           cudaStream_t st) {
        const size_t sm = (size_t)padded_len(N) * sizeof(double2) + 2 * sizeof(TwoLevelTw);
        cudaError_t e = set_smem(k_vertex_tau_bwd<N>, sm);
        if (e != cudaSuccess) return e;
        k_vertex_tau_bwd<N><<<g->n8, 256, sm, st>>>(a->Vb, chirt, Grt, a->dGrt[0], a->dGrt[1], g->tw_w, fact8, g->n8,
                                                    a->part + a->row_vt * kAdjW);
        return launched();
    }
};
template <int NBK>
struct RunVertexQBwd {
    static cudaError_t run(const GridDev *g, const AdjDev *a, const double *chiq, double U, double Usp, double Uch,
                           double T, cudaStream_t st) {
        const size_t sm = SliceSmem<NBK>::bytes;
        cudaError_t e = set_smem(k_vertex_q_bwd<NBK>, sm);
        if (e != cudaSuccess) return e;
        const double normFact = T / ((double)g->nk0 * g->nk0);
        k_vertex_q_bwd<NBK><<<g->nb, kSliceThreads, sm, st>>>(a->Vb, chiq, a->dchiq[0], a->dchiq[1], g->tw_k, g->nb,
                                                               normFact, U, Usp, Uch, a->part + a->row_vq * kAdjW);
        return launched();
    }
};
}  // namespace

cudaError_t cond_bwd_blocks(const GridDev &g, int *blocks) { return dispatch_nw<CondBwdBlocks>(g.nw0, blocks); }

cudaError_t launch_cond_tau_bwd(const GridDev &g, const CondBwdArgs &a, int nblk, cudaStream_t st) {
    return dispatch_nw<RunCondTauBwd>(g.nw0, &a, nblk, st);
}

cudaError_t launch_cond_lines_bwd(const GridDev &g, const CondDev &c, const AdjDev &a, const double2 *S,
                                  const double *s2, const double *s3, const double *sinf, double mu, double T,
                                  double kx0b, cudaStream_t st) {
    const double nf = 1.0 / ((double)g.nk0 * g.nk0);
    k_cond_lines_bwd<<<2 * g.nbk, 256, 0, st>>>(S, s2, s3, sinf, g.ek, c.d2line, g.nbk, g.nw0, mu, T, nf, kx0b,
                                                a.sigl, a.part + a.row_cl * kAdjW);
    return launched();
}

cudaError_t launch_cond_slices_bwd(const GridDev &g, const CondDev &c, const AdjDev &a, const double *V,
                                   const double *dchirt0, double mu0, double T, double fact4, double dmu0_2,
                                   cudaStream_t st) {
    return dispatch_nbk<RunCondSliceBwd>(g.nbk, &g, &c, &a, V, dchirt0, mu0, T, fact4, dmu0_2, st);
}

cudaError_t launch_sigbar(const GridDev &g, const CondDev &c, const AdjDev &a, const double2 *S, const double *s2,
                          const double *s3, const double *s4, const double *sinf, double mu0, double mu, double lam,
                          double T, double dmu0_2, cudaStream_t st) {
    (void)c;
    k_sigbar<<<g.n8, 256, 0, st>>>(a.sigc, a.sigl, S, s2, s3, s4, sinf, g.ek, g.w16, g.nbk, g.nw0, mu0, mu, lam, T,
                                   dmu0_2, a.Sb, a.s2b, a.s3b, a.part + a.row_sg * kAdjW);
    return launched();
}

cudaError_t launch_sigma_tau_bwd(const GridDev &g, const AdjDev &a, double sinfb, double T, cudaStream_t st) {
    return dispatch_nw<RunSigmaTauBwd>(g.nw0, &g, &a, sinfb, T, st);
}

cudaError_t launch_sigma_slices_bwd(const GridDev &g, const CondDev &c, const AdjDev &a, const double *Grt,
                                    const double *V, const double *dchirt0, const double *dG0p, double mu0,
                                    double fact8, double dmu0_2, cudaStream_t st) {
    return dispatch_nbk<RunSigmaSliceBwd>(g.nbk, &g, &c, &a, Grt, V, dchirt0, dG0p, mu0, fact8, dmu0_2, st);
}

cudaError_t launch_vertex_bwd(const GridDev &g, const AdjDev &a, const double *chirt, const double *chiq,
                              const double *Grt, double U, double Usp, double Uch, double T, cudaStream_t st) {
    const double fact8 = U * (3.0 * Usp + Uch) / 8.0;
    cudaError_t e = dispatch_nw<RunVertexTauBwd>(g.nw0, &g, &a, chirt, Grt, fact8, st);
    if (e != cudaSuccess) return e;
    return dispatch_nbk<RunVertexQBwd>(g.nbk, &g, &a, chiq, U, Usp, Uch, T, st);
}

}  // namespace tpsc
