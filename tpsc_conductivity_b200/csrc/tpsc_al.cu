// tpsc_al.cu -- the Aslamazov-Larkin vertex correction chijj3(iq_n) of the
// current-current correlator, FP64 (cond_opt::calc_chijj_vertex_corr_all_optim
// with chi3 = true, src/cond_opt.cpp:4292-6420).
//
// The correction is evaluated on the reference's non-uniform bosonic grid
// (src/cond_opt.cpp:5123-5155); every grid frequency q_n runs the same
// pipeline on the K4 grid of interior kx points (c = l nbk + m,
// k = ((l+1), m) pi/(nbk-1), r folded into the octant):
//   once per call (launch_al_setup):
//    * G(r, tau_j) in FP64 (k_gslice); the branch's G(r, -tau) is
//      -G(r, beta - tau), its tau-derivatives at 0 and beta follow from the
//      hopping table and d/dtau G(r, 0+);
//    * hG slices: h(k, tau) -> DST x DCT -> times G(r, -tau) -> DST x DCT
//      (src/cond_opt.cpp:5158-5248), and their end slopes;
//    * per column pair: clamped spline of hG over tau, FFT -> hG(q, i q_p)
//      and its 1/q^2 coefficient (src/cond_opt.cpp:5250-5330);
//   per grid frequency (launch_al_freq):
//    * k_al_hq: the difference quotient I_n(q, i q_m) of hG against chi0,
//      times the RPA vertices, minus its closed-form asymptote, FFT to tau,
//      plus the asymptote's closed form in tau (src/cond_opt.cpp:5351-5622);
//    * k_al_q2r: DST x DCT of Re and Im, q -> r (src/cond_opt.cpp:5628-5716);
//    * k_al_r2k: times G(r, -tau) for H(tau) and for the mirror
//      H2(tau) = H(beta - tau), DST x DCT back to k, and the four end slopes
//      (src/cond_opt.cpp:5718-5900, 5987-6180);
//    * k_al_tau: per k, the Re and Im splines of both, pre-twiddled FFTs to
//      fermionic frequencies, and the sum over k_m of
//      G(k, i k_m) G(k, i k_m + i q_n) (H - H2) (src/cond_opt.cpp:5906-5985,
//      6182-6398);
//    * k_al_finish: the per-k terms added in a fixed order, total and
//      angular bins.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tpsc_device.cuh"

namespace tpsc {

namespace {

// the AL branch's G(r, -tau_j) = DCT-I[G0(k, -tau_j)]/L^2 (src/cond_opt.cpp:4382-4410)
// from this library's G(r, tau): G(r, -tau) = -G(r, beta - tau), j = 0..Nw0
__device__ __forceinline__ double g_minus(const double *__restrict__ Grt, int nw0, int n8, int j, int o) {
    return -Grt[(size_t)(nw0 - j) * n8 + o];
}
// d/dtau G(r, -tau) at 0 (side 0) and beta (side 1) (src/cond_opt.cpp:4415-4446):
// DCT-I[(eps - mu0) n_F]/L^2 = er - mu0 delta_r0 - d/dtau G(r, 0+) at 0, and
// er - mu0 delta_r0 minus that at beta, i.e. d/dtau G(r, 0+)
__device__ __forceinline__ double dg_minus(const double *__restrict__ er, const double *__restrict__ dG0p, double mu0,
                                           int side, int o) {
    return side == 0 ? ((o == 0 ? -mu0 : er[o]) - dG0p[o]) : dG0p[o];
}

// complex helpers on double2
__device__ __forceinline__ double2 cneg(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ double2 cmuli(double2 a) { return make_double2(-a.y, a.x); }  // i a
__device__ __forceinline__ double2 crs(double a, double2 b) { return make_double2(a * b.x, a * b.y); }
__device__ __forceinline__ double2 cinv(double2 b) { return cdiv(make_double2(1.0, 0.0), b); }

// exp(-i pi m / N) for any m >= 0, from the table ht[m] = exp(+i pi m / N), m < N
__device__ __forceinline__ double2 half_twiddle_conj(const TwoLevelTw *ht2, int m, int N) {
    m %= 2 * N;
    const double2 h = tw_at(ht2, m < N ? m : m - N);
    return m < N ? make_double2(h.x, -h.y) : make_double2(-h.x, h.y);
}

// ---------------------------------------------------------------------------
// once per call
// ---------------------------------------------------------------------------

// h G(q, tau_j), j = blockIdx.x = 0..Nw0: h(k, tau_j) from the (eps - mu0, A)
// table (src/cond_opt.cpp:4304-4330), DST x DCT, times G(r, -tau_j), DST x DCT
// (src/cond_opt.cpp:5220-5248); h(r, 0) and h(r, beta) kept for the end slopes.
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_al_hg_slice(const double *__restrict__ tab, const double *__restrict__ Grt, const double2 *__restrict__ tw,
                  int nw0, int n8, double T, double *__restrict__ hGt, double *__restrict__ pre) {
    constexpr int K4 = (NBK - 2) * NBK;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int j = blockIdx.x;
    const double t = j / (nw0 * T);
    const double bt = 1.0 / T - t;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const double2 xa = *reinterpret_cast<const double2 *>(tab + 4 * c);
        S[c] = xa.y * exp(xa.x > 0 ? -xa.x * t : xa.x * bt);
    }
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const int l = c / NBK, m = c % NBK;
        const double v = S[c];
        if (j == 0) pre[c] = v;
        if (j == nw0) pre[K4 + c] = v;
        S[c] = v * g_minus(Grt, nw0, n8, j, oct_index(l + 1, m));
    }
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    for (int c = threadIdx.x; c < K4; c += blockDim.x) hGt[bidx2(j, c, nw0 + 1)] = S[c];
}

// End slopes of h G over tau (src/cond_opt.cpp:5158-5216): kind 0 (tau = 0),
// 1 (tau = beta): DST x DCT[ dh(r) G(r, -tau) + h(r) d/dtau G(r, -tau) ], with
// dh the transformed tau-derivative of h at that end (src/cond_opt.cpp:2744-2783).
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_al_hg_bound(const double *__restrict__ ek, const double *__restrict__ dek, const double *__restrict__ er,
                  const double *__restrict__ dG0p, const double *__restrict__ Grt, const double2 *__restrict__ tw,
                  const double *__restrict__ pre, int nw0, int n8, double mu0, double T, double nf,
                  double *__restrict__ dhG) {
    constexpr int K4 = (NBK - 2) * NBK;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int kind = blockIdx.x;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const int l = c / NBK, m = c % NBK;
        const double x = ek[oct_index(l + 1, m)] - mu0;
        const double d = nf * dek[c];
        double v;
        if (x > 0) {
            const double ep = exp(-x / T), q = ep + 1.0;
            v = kind == 0 ? -d * x / q : -d * x * ep / q;
        } else {
            const double en = exp(x / T), q = en + 1.0;
            v = kind == 0 ? -d * x * en / q : -d * x / q;
        }
        S[c] = v;
    }
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    const int jend = kind == 0 ? 0 : nw0;
    for (int c = threadIdx.x; c < K4; c += blockDim.x) {
        const int l = c / NBK, m = c % NBK;
        const int o = oct_index(l + 1, m);
        S[c] = S[c] * g_minus(Grt, nw0, n8, jend, o) + pre[kind * K4 + c] * dg_minus(er, dG0p, mu0, kind, o);
    }
    __syncthreads();
    dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
    for (int c = threadIdx.x; c < K4; c += blockDim.x) dhG[kind * K4 + c] = S[c];
}

// shared memory of the per-pair tau kernel: two staged columns, one FFT
// buffer, the two-level twiddle tables
template <int N>
struct AlHgTauSmem {
    static constexpr size_t r_bytes = ((size_t)2 * (N + 1) * sizeof(double) + 15) & ~(size_t)15;
    static constexpr size_t tables_off = r_bytes + (size_t)padded_len(N) * sizeof(double2);
    static constexpr size_t bytes = tables_off + 2 * sizeof(TwoLevelTw);
};

// h G(q, i q_p) from h G(q, tau), one column pair per CTA (src/cond_opt.cpp:5250-5330):
// clamped spline with the end slopes, F_p = sum_j 6 a_j exp(-2 pi i jp/N);
// p = 0: 2 x the spline's integral; 0 < p < N/2: 2 Re[(1 - exp(-2 pi i p/N)) F_p];
// then hg2 = 2 (dhG(0) - dhG(beta)), the coefficient of -1/q^2.
template <int N>
__global__ void __launch_bounds__(256, 1)
    k_al_hg_tau(const double *__restrict__ hGt, const double *__restrict__ dhG, const double *__restrict__ spl,
                const double2 *__restrict__ tw, const double2 *__restrict__ ht, double T, int K4,
                double *__restrict__ hgq) {
    constexpr int NJ = N + 1, NO = N / 2, G = FftPlan<N>::G;
    extern __shared__ __align__(16) double R[];
    double2 *X = reinterpret_cast<double2 *>(reinterpret_cast<char *>(R) + AlHgTauSmem<N>::r_bytes);
    TwoLevelTw *tw2 = reinterpret_cast<TwoLevelTw *>(reinterpret_cast<char *>(R) + AlHgTauSmem<N>::tables_off);
    __shared__ double d0s[2], dNs[2], sV[2], sM[2], V0[2], VN[2];
    const int tid = threadIdx.x;
    tau_tables(tw2, tw2 + 1, tw, ht, N);
    const int c0 = 2 * blockIdx.x;
    stage_pair(R, hGt + (size_t)blockIdx.x * 2 * NJ, NJ, c0 + 1 < K4);
    if (tid < 2) {
        const int c = c0 + tid;
        d0s[tid] = c < K4 ? dhG[c] : 0.0;
        dNs[tid] = c < K4 ? dhG[K4 + c] : 0.0;
    }
    __syncthreads();
    if (tid < 2) {
        V0[tid] = R[tid * NJ];
        VN[tid] = R[tid * NJ + N];
    }
    column_sums<2>(R, NJ, 0, NJ, sV);
    const double h = 1.0 / (N * T), ih = 1.0 / h;
    spline_second_derivatives<2>(R, NJ, NJ, h, d0s, dNs, spl, spl + NJ);
    column_sums<2>(R, NJ, 0, NJ, sM);
    if (tid < G) {
        const double *Ma = R, *Mb = R + NJ;
        auto in = [&](int j) -> double2 { return make_double2((Ma[j + 1] - Ma[j]) * ih, (Mb[j + 1] - Mb[j]) * ih); };
        group_fft_io<N, -1>(X, tid, (const TwoLevelTw *)tw2, 0, in, ScratchIO{X});
    }
    __syncthreads();
    for (int p = tid; p < NO; p += blockDim.x) {
        double2 F[2];
        if (p > 0) split_real(X[pidx(p)], X[pidx(N - p)], F[0], F[1]);
        const double2 w = tw_at(tw2, p);
        const double2 f = make_double2(1.0 - w.x, -w.y);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int c = c0 + q;
            if (c >= K4) continue;
            double v;
            if (p == 0) {
                const double M0 = R[q * NJ], MN = R[q * NJ + N];
                v = 2.0 * (h * (sV[q] - 0.5 * (V0[q] + VN[q])) - h * h * h / 24.0 * (2.0 * sM[q] - M0 - MN));
            } else {
                v = 2.0 * (f.x * F[q].x - f.y * F[q].y);
            }
            hgq[(size_t)c * (NO + 1) + p] = v;
        }
    }
    if (tid < 2 && c0 + tid < K4) hgq[(size_t)(c0 + tid) * (NO + 1) + NO] = 2.0 * (d0s[tid] - dNs[tid]);
}

// ---------------------------------------------------------------------------
// per grid frequency q_nn
// ---------------------------------------------------------------------------
struct AlHqArgs {
    const double *chiq;            // chi0(q, i q_p), p <= NO, column blocks
    const double *cinf, *cinf2;    // [n8] its 1/q^2, 1/q^4 tail coefficients
    const double *hgq;             // [K4 (NO+1)]
    const double2 *tw, *ht;        // [N] FFT twiddles, half-step twiddles
    double2 *HQ, *dHQ;
    int K4, nbk, nn;
    double T, Usp, Uch;
};

// per-column constants of k_al_hq
struct HqCol {
    int o;
    const double *hq;
    double ci, ci2, hg2;
    double2 zsp0, zsp1, dsp0, dsp1;  // spin poles +-i sqrt(Usp ci/2) and their denominators
    double zch0, zch1, dch0, dch1;   // charge poles +-sqrt(Uch ci/2) and denominators
    double dt0;                      // d/dtau of the FFT part at 0 (src/cond_opt.cpp:5539-5546)
};

// I_n(q, i q_m) -> H(q, tau) for one column pair per CTA (src/cond_opt.cpp:5351-5622):
//   m in [0, NO - nc): p1 = m, p2 = m + nn; m in [NO - nc, N): p1 = m - N, p2 = p1 + nn;
//   I = (3 Usp chisp(p1) + Uch chich(p1)) (hG(p1) - hG(p2)) / (chi0(p1) - chi0(p2)),
//   with (4 D(m-1) - D(m-2))/3 for the quotient D where p1 = p2 (nn even);
//   ft_m = T (I - Hinf(q_m)), H(q, tau_j) = FFT_{-}[ft]_j + Hinf(tau_j), closed form.
template <int N>
__global__ void __launch_bounds__(256, 1) k_al_hq(const AlHqArgs a) {
    constexpr int NO = N / 2, G = FftPlan<N>::G;
    extern __shared__ __align__(16) double2 X[];
    TwoLevelTw *tw2 = reinterpret_cast<TwoLevelTw *>(X + padded_len(N));
    __shared__ HqCol col[2];
    __shared__ double sums[2];
    const int tid = threadIdx.x, NT = blockDim.x;
    const int c0 = 2 * blockIdx.x;
    const double T = a.T, Usp = a.Usp, Uch = a.Uch, tp = 2.0 * kPi * T;
    const int nn = a.nn, nc = nn / 2, NB = NO + 1;
    tau_tables(tw2, tw2 + 1, a.tw, a.ht, N);  // published by the barrier below
    if (tid < 2) {
        const int c = min(c0 + tid, a.K4 - 1);
        const int l = c / a.nbk, m = c % a.nbk;
        HqCol &q = col[tid];
        q.o = oct_index(l + 1, m);
        q.hq = a.hgq + (size_t)c * (NO + 1);
        q.ci = a.cinf[q.o];
        q.ci2 = a.cinf2[q.o];
        q.hg2 = q.hq[NO];
        const double s = sqrt(Usp * q.ci / 2.0);
        q.zsp0 = make_double2(0.0, s);
        q.zsp1 = make_double2(-0.0, -s);
        q.dsp0 = cmul(csub(cexp2(cscale(q.zsp0, -1.0 / T)), make_double2(1.0, 0.0)), csub(q.zsp0, q.zsp1));
        q.dsp1 = cmul(csub(cexp2(cscale(q.zsp1, -1.0 / T)), make_double2(1.0, 0.0)), csub(q.zsp1, q.zsp0));
        q.zch0 = sqrt(Uch * q.ci / 2.0);
        q.zch1 = -q.zch0;
        q.dch0 = (exp(-q.zch0 / T) - 1.0) * (q.zch0 - q.zch1);
        q.dch1 = (1.0 - exp(q.zch1 / T)) * (q.zch1 - q.zch0);
    }
    __syncthreads();
    auto chi0_at = [&](const HqCol &q, int p) -> double {
        p = abs(p);
        if (p <= NO) return a.chiq[bidx(p, q.o, NB)];
        const double wn = tp * p;
        return q.ci / (wn * wn) + q.ci2 / (wn * wn * wn * wn);
    };
    auto hg_at = [&](const HqCol &q, int p) -> double {
        p = abs(p);
        if (p == 0) return q.hq[0];
        const double wn = tp * p;
        return -q.hg2 / (wn * wn) + q.hq[p < NO ? p : NO - 1] / (wn * wn * wn * wn);
    };
    auto quot = [&](const HqCol &q, int p1, int p2) -> double {
        return (hg_at(q, p1) - hg_at(q, p2)) / (chi0_at(q, p1) - chi0_at(q, p2));
    };
    // ---- the quotient minus its asymptote, packed as Re/Im of one FFT
    double acc[2] = {0.0, 0.0};
    for (int m = tid; m < N; m += NT) {
        const bool first = m < NO - nc;
        const int p1 = first ? m : m - N, p2 = p1 + nn;
        const double wn = tp * (first ? m : m - N);
        double ft[2];
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            const HqCol &q = col[k];
            const double ch = chi0_at(q, p1);
            const double pre = 3 * Usp * (ch / (1.0 - Usp * ch / 2)) + Uch * (ch / (1.0 + Uch * ch / 2));
            double D;
            if (!first && (nn % 2) == 0 && m - N == -(nn / 2))
                D = (4 * quot(q, p1 - 1, p2 - 1) - quot(q, p1 - 2, p2 - 2)) / 3.0;
            else
                D = quot(q, p1, p2);
            const double cq = -q.ci;
            const double hinf =
                q.hg2 * (3.0 * Usp * (1.0 / (-wn * wn - Usp * cq / 2.0)) + Uch * (1.0 / (-wn * wn + Uch * cq / 2.0)));
            ft[k] = T * (pre * D - hinf);
            acc[k] += wn * ft[k];
        }
        X[pidx(m)] = make_double2(ft[0], ft[1]);
    }
    block_sum<2>(acc, sums);
    if (tid < 2) col[tid].dt0 = -sums[tid];
    if (tid < G) group_fft<N, -1>(X, tid, (const TwoLevelTw *)tw2, 0);
    __syncthreads();
    // ---- back in tau: the FFT part plus the asymptote's closed form
    for (int j = tid; j <= N; j += NT) {
        const int k = j % N;
        double2 F[2];
        split_real(X[pidx(k)], X[pidx((N - k) % N)], F[0], F[1]);
        const double t = j / (N * T);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const HqCol &s = col[q];
            const int c = c0 + q;
            if (c >= a.K4) continue;
            double2 tsp;
            double tch;
            if (j < N) {
                tsp = cadd(cdiv(cexp2(cscale(s.zsp0, -t)), s.dsp0), cdiv(cexp2(cscale(s.zsp1, -t)), s.dsp1));
                tch = exp(-s.zch0 * t) / s.dch0 + exp(s.zch1 * (1.0 / T - t)) / s.dch1;
            } else {
                const double2 one = make_double2(1.0, 0.0);
                tsp = cadd(cinv(cmul(csub(one, cexp2(cscale(s.zsp0, 1.0 / T))), csub(s.zsp0, s.zsp1))),
                           cinv(cmul(csub(one, cexp2(cscale(s.zsp1, 1.0 / T))), csub(s.zsp1, s.zsp0))));
                const double e0 = exp(-s.zch0 / T);
                tch = e0 / ((e0 - 1.0) * (s.zch0 - s.zch1)) + 1.0 / ((1.0 - exp(s.zch1 / T)) * (s.zch1 - s.zch0));
            }
            const double2 hinf = crs(s.hg2, cadd(crs(3.0 * Usp, tsp), make_double2(Uch * tch, 0.0)));
            a.HQ[(size_t)j * a.K4 + c] = cadd(F[q], hinf);
        }
    }
    // the end slopes: i dt0 plus the asymptote's tau-derivative at 0 and beta
    if (tid < 2 && c0 + tid < a.K4) {
        const HqCol &s = col[tid];
        const int c = c0 + tid;
        const double2 e0 = cexp2(cscale(s.zsp0, -1.0 / T)), e1 = cexp2(cscale(s.zsp1, -1.0 / T));
        double2 tsp = csub(cneg(cdiv(s.zsp0, s.dsp0)), cdiv(s.zsp1, s.dsp1));
        const double x1 = exp(s.zch1 / T);
        double tch = -s.zch0 / s.dch0 - s.zch1 * x1 / s.dch1;
        double2 dinf = crs(s.hg2, cadd(crs(3.0 * Usp, tsp), make_double2(Uch * tch, 0.0)));
        a.dHQ[c] = cadd(make_double2(0.0, s.dt0), dinf);
        tsp = csub(cneg(cdiv(cmul(s.zsp0, e0), s.dsp0)), cdiv(cmul(s.zsp1, e1), s.dsp1));
        const double x0 = exp(-s.zch0 / T);
        tch = -s.zch0 * x0 / s.dch0 - s.zch1 / s.dch1;
        dinf = crs(s.hg2, cadd(crs(3.0 * Usp, tsp), make_double2(Uch * tch, 0.0)));
        a.dHQ[a.K4 + c] = cadd(make_double2(0.0, s.dt0), dinf);
    }
}

// H(q, tau_j) -> H(r, tau_j) = DST x DCT[nf H] of the real and imaginary parts
// (src/cond_opt.cpp:5628-5716); blocks Nw0 + 1 and Nw0 + 2 transform the two
// end slopes.
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_al_q2r(const double2 *__restrict__ HQ, const double2 *__restrict__ dHQ, const double2 *__restrict__ tw,
             int nw0, double nf, double2 *__restrict__ HR, double2 *__restrict__ dHR) {
    constexpr int K4 = (NBK - 2) * NBK;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int b = blockIdx.x, NJ = nw0 + 1;
    const double2 *src = b < NJ ? HQ + (size_t)b * K4 : dHQ + (size_t)(b - NJ) * K4;
    double *dst = reinterpret_cast<double *>(b < NJ ? HR + (size_t)b * K4 : dHR + (size_t)(b - NJ) * K4);
#pragma unroll 1
    for (int part = 0; part < 2; ++part) {
        for (int c = threadIdx.x; c < K4; c += blockDim.x) S[c] = nf * (part == 0 ? src[c].x : src[c].y);
        __syncthreads();
        dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
        for (int c = threadIdx.x; c < K4; c += blockDim.x) dst[2 * c + part] = S[c];
        __syncthreads();
    }
}

// H(r, tau_j) G(r, -tau_j) and H2(r, tau_j) G(r, -tau_j), H2(r, tau) = H(r, beta - tau),
// -> DST x DCT to k, real and imaginary parts (src/cond_opt.cpp:5845-5900, 6125-6180),
// into the two-column-block layouts of HK and H2K.  Blocks Nw0 + 1 + k, k < 4,
// transform the end slopes (src/cond_opt.cpp:5729-5843, 6004-6123):
//   k = 0: H(r, 0) dG(0) + dH(r, 0) G(r, 0);   k = 1: H(r, beta) dG(beta) + dH(r, beta) G(r, -beta);
//   k = 2, 3: the same for H2, whose end values are H(r, beta), H(r, 0) and
//   whose end slopes are -dH(r, beta), -dH(r, 0).
template <int NBK>
__global__ void __launch_bounds__(kSliceThreads, 1)
    k_al_r2k(const double2 *__restrict__ HR, const double2 *__restrict__ dHR, const double *__restrict__ Grt,
             const double *__restrict__ er, const double *__restrict__ dG0p, const double2 *__restrict__ tw, int nw0,
             int n8, double mu0, double2 *__restrict__ HK, double2 *__restrict__ H2K, double2 *__restrict__ dHK) {
    constexpr int K4 = (NBK - 2) * NBK;
    extern __shared__ __align__(16) double S[];
    const auto *tws = slice_twiddles<NBK>(S, tw);
    const int b = blockIdx.x, NJ = nw0 + 1;
    const int npass = b < NJ ? 4 : 2;
#pragma unroll 1
    for (int pass = 0; pass < npass; ++pass) {
        const int part = pass & 1;
        for (int c = threadIdx.x; c < K4; c += blockDim.x) {
            const int l = c / NBK, m = c % NBK;
            const int o = oct_index(l + 1, m);
            const double *hr = reinterpret_cast<const double *>(HR);
            const double *dr = reinterpret_cast<const double *>(dHR);
            double v;
            if (b < NJ) {
                const int row = pass < 2 ? b : nw0 - b;
                v = hr[2 * ((size_t)row * K4 + c) + part] * g_minus(Grt, nw0, n8, b, o);
            } else {
                const int k = b - NJ;
                const int side = k & 1;                                        // 0: tau = 0, 1: beta
                const int row = (k == 0 || k == 3) ? 0 : nw0;                  // H at 0 / beta
                const int sl = (k == 0) ? 0 : (k == 1) ? 1 : (k == 2) ? 1 : 0;  // which dH
                const double sg = k < 2 ? 1.0 : -1.0;
                v = hr[2 * ((size_t)row * K4 + c) + part] * dg_minus(er, dG0p, mu0, side, o) +
                    sg * dr[2 * ((size_t)sl * K4 + c) + part] * g_minus(Grt, nw0, n8, side == 0 ? 0 : nw0, o);
            }
            S[c] = v;
        }
        __syncthreads();
        dst_dct_slice<NBK>(S, slice_scratch<NBK>(S), tws);
        for (int c = threadIdx.x; c < K4; c += blockDim.x) {
            double *dst;
            if (b < NJ)
                dst = reinterpret_cast<double *>((pass < 2 ? HK : H2K) + bidx2(b, c, NJ));
            else
                dst = reinterpret_cast<double *>(dHK + (size_t)(b - NJ) * K4 + c);
            dst[part] = S[c];
        }
        __syncthreads();
    }
}

struct AlTauArgs {
    const double2 *HK, *H2K, *dHK;
    const double2 *S;
    const double *s2, *s3, *sinf;
    const double *ek, *dek;
    const double *spl;
    const double2 *tw, *ht;
    double *colv;
    int K4, nbk, nn;
    double T, mu, U, nf;
};

// shared memory of k_al_tau: the Re/Im columns being splined, the two
// transforms (H, H2), the twiddle tables
template <int N>
struct AlTauSmem {
    static constexpr size_t r_bytes = ((size_t)2 * (N + 1) * sizeof(double) + 15) & ~(size_t)15;
    static constexpr size_t x_bytes = (size_t)padded_len(N) * sizeof(double2);
    static constexpr size_t tables_off = r_bytes + 2 * x_bytes;
    static constexpr size_t bytes = tables_off + 2 * sizeof(TwoLevelTw);
};

// One k point per CTA: for H and H2 the Re and Im splines over tau with their
// end slopes, F_j = sum_l exp(-i pi l/N) 6 (a_l^Re + i a_l^Im) exp(-2 pi i lj/N)
// (src/cond_opt.cpp:5906-5985, 6187-6251), the fermionic values
//   H(i w) = -i C1/w - C2/w^2 + i C3/w^3 + (1 - exp(-i (2f+1) pi/N)) F/w^4
// (H at k_m + q_nn, H2 at k_m), and the term
//   -i U T nf wt dek sum_m G(k, i k_m) G(k, i k_m + i q_nn) (H - H2) / (2 q_nn)
// (src/cond_opt.cpp:6253-6398); its real part -> colv[c].
template <int N>
__global__ void __launch_bounds__(256, 1) k_al_tau(const AlTauArgs a) {
    constexpr int NJ = N + 1, NO = N / 2, G = FftPlan<N>::G;
    extern __shared__ __align__(16) double R[];
    double2 *X1 = reinterpret_cast<double2 *>(reinterpret_cast<char *>(R) + AlTauSmem<N>::r_bytes);
    double2 *X2 = X1 + padded_len(N);
    TwoLevelTw *tw2 = reinterpret_cast<TwoLevelTw *>(reinterpret_cast<char *>(R) + AlTauSmem<N>::tables_off);
    const TwoLevelTw *ht2 = tw2 + 1;
    __shared__ double d0s[2], dNs[2];
    __shared__ double2 cw[2], dsum[2], d2sum[2];
    __shared__ double sums[2];
    const int tid = threadIdx.x, NT = blockDim.x;
    const int c = blockIdx.x;
    const double T = a.T, h = 1.0 / (N * T), ih = 1.0 / h, pT = kPi * T;
    tau_tables(tw2, tw2 + 1, a.tw, a.ht, N);
#pragma unroll 1
    for (int which = 0; which < 2; ++which) {
        const double2 *src = (which == 0 ? a.HK : a.H2K);
        for (int j = tid; j < NJ; j += NT) {
            const double2 v = src[bidx2(j, c, NJ)];
            R[j] = v.x;
            R[NJ + j] = v.y;
        }
        if (tid < 2) {
            const double2 s0 = a.dHK[(size_t)(2 * which) * a.K4 + c], s1 = a.dHK[(size_t)(2 * which + 1) * a.K4 + c];
            d0s[tid] = tid == 0 ? s0.x : s0.y;
            dNs[tid] = tid == 0 ? s1.x : s1.y;
        }
        __syncthreads();
        if (tid == 0) {
            cw[which] = make_double2(R[0] + R[N], R[NJ] + R[NJ + N]);
            dsum[which] = make_double2(d0s[0] + dNs[0], d0s[1] + dNs[1]);
        }
        spline_second_derivatives<2>(R, NJ, NJ, h, d0s, dNs, a.spl, a.spl + NJ);
        if (tid == 0) d2sum[which] = make_double2(R[0] + R[N], R[NJ] + R[NJ + N]);
        double2 *X = which == 0 ? X1 : X2;
        if (tid < G) {
            const double *Mr = R, *Mi = R + NJ;
            auto in = [&](int j) -> double2 {
                const double2 e = tw_at(ht2, j);
                return cmul(make_double2(e.x, -e.y), make_double2((Mr[j + 1] - Mr[j]) * ih, (Mi[j + 1] - Mi[j]) * ih));
            };
            group_fft_io<N, -1>(X, tid, (const TwoLevelTw *)tw2, 0, in, ScratchIO{X});
        }
        __syncthreads();
    }
    // ---- the sum over k_m
    const int l = c / a.nbk, m = c % a.nbk;
    const int o = oct_index(l + 1, m);
    const int nn = a.nn, nc = nn / 2;
    const double e = a.ek[o], mu = a.mu, sinf = a.sinf[0], C2 = a.s2[o], C3 = a.s3[o];
    auto green = [&](int f) -> double2 {
        const double kn = (2 * f + 1) * pT;
        double sr = -C2 / (kn * kn), si = -sinf / kn + C3 / (kn * kn * kn);
        const int n = f >= 0 ? f : -f - 1;
        if (n < NO) {
            const double2 Sv = a.S[bidx(n, o, NO)];
            const double k4 = kn * kn * kn * kn;
            sr += Sv.x / k4;
            si += (f >= 0 ? Sv.y : -Sv.y) / k4;
        }
        return cinv(make_double2(-e + mu - sr, kn - si));
    };
    auto hval = [&](double2 cwv, double2 ds, double2 d2s, double w, bool has, double2 Fv, int ph) -> double2 {
        const double w2 = w * w, w3 = w2 * w, w4 = w2 * w2;
        double2 v = cadd(csub(cmuli(cscale(cwv, -1.0 / w)), cscale(ds, 1.0 / w2)), cmuli(cscale(d2s, 1.0 / w3)));
        if (has) {
            const double2 ex = half_twiddle_conj(ht2, ph, N);
            v = cadd(v, cscale(cmul(make_double2(1.0 - ex.x, -ex.y), Fv), 1.0 / w4));
        }
        return v;
    };
    double acc[2] = {0.0, 0.0};
    for (int j = tid; j < N; j += NT) {
        const bool first = j < NO - nc;
        const int f1 = first ? j : j - N;
        const double w1 = (2 * (f1 + nn) + 1) * pT;
        int idx = -1;
        if (first)
            idx = j + nn < N ? j + nn : -1;
        else if (j + nn - N < 0)
            idx = j + nn;
        else if (j + nn - N < N)
            idx = j + nn - N;
        const double2 v1 =
            hval(cw[0], dsum[0], d2sum[0], w1, idx >= 0, idx >= 0 ? X1[pidx(idx)] : make_double2(0, 0), 2 * (j + nn) + 1);
        const double w2 = (2 * f1 + 1) * pT;
        const double2 v2 = hval(cw[1], dsum[1], d2sum[1], w2, true, X2[pidx(j)], 2 * j + 1);
        const double2 t = cmul(cmul(green(f1), green(f1 + nn)), csub(v1, v2));
        acc[0] += t.x;
        acc[1] += t.y;
    }
    block_sum<2>(acc, sums);
    if (tid == 0) {
        const double qn = 2.0 * nn * kPi * T;
        const double wt = (m == 0 || m == a.nbk - 1) ? 2.0 : 4.0;
        // Re[-i K acc] = K Im(acc)
        a.colv[c] = a.U * T * a.nf * wt * a.dek[c] * sums[1] / (2.0 * qn);
    }
}

// out[row (1 + nbins) + 0] = sum_c colv[c], then per bin b the sum over the
// points of bin b; each warp adds one value in a fixed order (lane-strided
// compensated sums, shuffle tree).
__global__ void k_al_finish(const double *__restrict__ colv, const int *__restrict__ bin, int K4, int nbins,
                            double *__restrict__ out) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int v = warp; v <= nbins; v += blockDim.x >> 5) {
        KSum s;
        for (int c = lane; c < K4; c += 32)
            if (v == 0 || (bin ? bin[c] : 0) == v - 1) s.add(colv[c]);
        double x = s.value();
        for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
        if (lane == 0) out[v] = x;
    }
}

// ---------------------------------------------------------------------------
// launch wrappers
// ---------------------------------------------------------------------------
template <int NBK>
struct RunAlHg {
    static cudaError_t run(const GridDev *g, const CondDev *c, const AlDev *a, const double *dG0p, double mu0,
                           double T, cudaStream_t st) {
        const size_t sm = SliceSmem<NBK>::bytes;
        cudaError_t e = set_smem(k_al_hg_slice<NBK>, sm);
        if (e != cudaSuccess) return e;
        if ((e = set_smem(k_al_hg_bound<NBK>, sm)) != cudaSuccess) return e;
        const double nf = 1.0 / ((double)g->nk0 * g->nk0);
        k_al_hg_slice<NBK><<<g->nw0 + 1, kSliceThreads, sm, st>>>(c->tab, a->Grt, g->tw_k, g->nw0, g->n8, T, a->hGt,
                                                                   a->pre);
        if ((e = launched()) != cudaSuccess) return e;
        k_al_hg_bound<NBK><<<2, kSliceThreads, sm, st>>>(g->ek, c->dek, g->er, dG0p, a->Grt, g->tw_k, a->pre, g->nw0,
                                                          g->n8, mu0, T, nf, a->dhG);
        return launched();
    }
};

template <int N>
struct RunAlHgTau {
    static cudaError_t run(const GridDev *g, const AlDev *a, double T, cudaStream_t st) {
        const size_t sm = AlHgTauSmem<N>::bytes;
        cudaError_t e = set_smem(k_al_hg_tau<N>, sm);
        if (e != cudaSuccess) return e;
        k_al_hg_tau<N><<<a->K4p / 2, 256, sm, st>>>(a->hGt, a->dhG, g->spl_full, g->tw_w, g->ht_w, T, a->K4, a->hgq);
        return launched();
    }
};

template <int N>
struct RunAlHq {
    static cudaError_t run(const AlHqArgs *args, int npairs, cudaStream_t st) {
        const size_t sm = (size_t)padded_len(N) * sizeof(double2) + 2 * sizeof(TwoLevelTw);
        cudaError_t e = set_smem(k_al_hq<N>, sm);
        if (e != cudaSuccess) return e;
        k_al_hq<N><<<npairs, 256, sm, st>>>(*args);
        return launched();
    }
};

template <int NBK>
struct RunAlSlices {
    static cudaError_t run(const GridDev *g, const AlDev *a, const double *dG0p, double mu0, cudaStream_t st) {
        const size_t sm = SliceSmem<NBK>::bytes;
        cudaError_t e = set_smem(k_al_q2r<NBK>, sm);
        if (e != cudaSuccess) return e;
        if ((e = set_smem(k_al_r2k<NBK>, sm)) != cudaSuccess) return e;
        const double nf = 1.0 / ((double)g->nk0 * g->nk0);
        k_al_q2r<NBK><<<g->nw0 + 3, kSliceThreads, sm, st>>>(a->HQ, a->dHQ, g->tw_k, g->nw0, nf, a->HR, a->dHR);
        if ((e = launched()) != cudaSuccess) return e;
        k_al_r2k<NBK><<<g->nw0 + 5, kSliceThreads, sm, st>>>(a->HR, a->dHR, a->Grt, g->er, dG0p, g->tw_k, g->nw0,
                                                              g->n8, mu0, a->HK, a->H2K, a->dHK);
        return launched();
    }
};

template <int N>
struct RunAlTau {
    static cudaError_t run(const AlTauArgs *args, cudaStream_t st) {
        const size_t sm = AlTauSmem<N>::bytes;
        cudaError_t e = set_smem(k_al_tau<N>, sm);
        if (e != cudaSuccess) return e;
        k_al_tau<N><<<args->K4, 256, sm, st>>>(*args);
        return launched();
    }
};

}  // namespace

cudaError_t launch_al_setup(const GridDev &g, const CondDev &c, const AlDev &a, const double *dG0p, double mu0,
                            double T, cudaStream_t st) {
    cudaError_t e = launch_gslice(g, a.Grt, mu0, T, st);
    if (e != cudaSuccess) return e;
    if ((e = dispatch_nbk<RunAlHg>(g.nbk, &g, &c, &a, dG0p, mu0, T, st)) != cudaSuccess) return e;
    return dispatch_nw<RunAlHgTau>(g.nw0, &g, &a, T, st);
}

cudaError_t launch_al_freq(const GridDev &g, const CondDev &c, const AlDev &a, const double *chiq, const double *cinf,
                           const double *cinf2, const double2 *S, const double *s2, const double *s3,
                           const double *sinf, const double *dG0p, int nn, int row, double U, double Usp, double Uch,
                           double mu, double mu0, double T, cudaStream_t st) {
    AlHqArgs h;
    h.chiq = chiq;
    h.cinf = cinf;
    h.cinf2 = cinf2;
    h.hgq = a.hgq;
    h.tw = g.tw_w;
    h.ht = g.ht_w;
    h.HQ = a.HQ;
    h.dHQ = a.dHQ;
    h.K4 = a.K4;
    h.nbk = g.nbk;
    h.nn = nn;
    h.T = T;
    h.Usp = Usp;
    h.Uch = Uch;
    cudaError_t e = dispatch_nw<RunAlHq>(g.nw0, &h, a.K4p / 2, st);
    if (e != cudaSuccess) return e;
    if ((e = dispatch_nbk<RunAlSlices>(g.nbk, &g, &a, dG0p, mu0, st)) != cudaSuccess) return e;
    AlTauArgs t;
    t.HK = a.HK;
    t.H2K = a.H2K;
    t.dHK = a.dHK;
    t.S = S;
    t.s2 = s2;
    t.s3 = s3;
    t.sinf = sinf;
    t.ek = g.ek;
    t.dek = c.dek;
    t.spl = g.spl_full;
    t.tw = g.tw_w;
    t.ht = g.ht_w;
    t.colv = a.colv;
    t.K4 = a.K4;
    t.nbk = g.nbk;
    t.nn = nn;
    t.T = T;
    t.mu = mu;
    t.U = U;
    t.nf = 1.0 / ((double)g.nk0 * g.nk0);
    if ((e = dispatch_nw<RunAlTau>(g.nw0, &t, st)) != cudaSuccess) return e;
    k_al_finish<<<1, 32 * (a.nbins + 1 < 32 ? a.nbins + 1 : 32), 0, st>>>(a.colv, a.nbins > 1 ? c.bin : nullptr, a.K4,
                                                                          a.nbins, a.out + (size_t)row * (1 + a.nbins));
    return launched();
}

}  // namespace tpsc
