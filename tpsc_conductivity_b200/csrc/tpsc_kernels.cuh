// tpsc_kernels.cuh -- launchers of the sm_100a kernels of the TPSC hot path.
// Host-side declarations shared by tpsc_kernels.cu and tpsc_engine.cpp.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

namespace tpsc {

// Device tables of one lattice / frequency grid.
struct GridDev {
    int nk0 = 0;        // lattice side L
    int nbk = 0;        // quadrant side L/2 + 1
    int n8 = 0;         // octant size nbk (nbk + 1) / 2
    int n8p = 0;        // n8 rounded up to a multiple of 4 (column blocks)
    int nw0 = 0;        // Nw0: fermionic frequencies (+ and -)
    int nb = 0;         // Nw0/2 + 1: bosonic n >= 0 == tau nodes on [0, beta/2]
    double *ek = nullptr;          // [n8] eps_k on the octant
    double2 *gk = nullptr;         // [n8] (eps_k - mu0, G0 prefactor) for the G(r, tau) slices
    double *er = nullptr;          // [n8] real-space hopping table
    double *w16 = nullptr;         // [n8p] octant weight: 16 halved on edges and diagonal, 0 on padding
    double *tailq = nullptr;       // [kTailQ] sum-rule tail power sums Q_k = sum_n qn^-2k (T dependent)
    double *tailP = nullptr;       // [kTailP] P_p = sum over the fermionic tail n = Nw0/2..Nw0 of w_n^-p
    double2 *tw_k = nullptr;       // [L]   exp(-2 pi i m / L)
    float4 *tw_k32 = nullptr;      // [L]   the same as (cos, sin) rounded to float, then the float remainders
    float *dct32 = nullptr;        // [(nk0 + 1)(nk0/4 + 4)] folded DCT-I tables of the direct slice plan (nk0 >= 64)
    float *dct_tc = nullptr;       // A-operand tables of the tensor slice plan (nk0 = 256)
    double2 *tw_w = nullptr;       // [Nw0] exp(-2 pi i m / Nw0)
    double2 *ht_w = nullptr;       // [Nw0] exp(+i pi m / Nw0)
    double *spl_half = nullptr;    // [2 nb]       spline LU tables, nb nodes
    double *spl_full = nullptr;    // [2 (Nw0+1)]  spline LU tables, Nw0+1 nodes
};

// Column-block layout of the (tau or frequency) x octant arrays: element
// (j, o) of an array with NJ rows sits at ((o / 4) NJ + j) 4 + o % 4, so the
// four columns of a block are contiguous along j (32-byte granules).
__host__ __device__ inline size_t bidx(int j, int o, int NJ) {
    return ((size_t)(o >> 2) * NJ + j) * 4 + (o & 3);
}

// The clamped-spline system's Thomas pivots converge to 2 + sqrt(3): from this
// row on (up to the last row) the pivot tables hold one constant, which the
// spline sweeps use instead of loading the entry (the host checks the tables
// where it builds them)
constexpr int kSplinePivotConst = 32;

constexpr int kMaxBlocks = 4096;
constexpr int kTailP = 41;  // P_p for p < kTailP: the find_mu tail series uses p <= kMuMomP + 28
constexpr int kTailQ = 20;  // Q_k for k < kTailQ (the series uses k <= 18)  // >= column blocks of the largest grid (2097)
struct Reduce {
    double *partial = nullptr;   // [4 * kMaxBlocks]
    double *result = nullptr;    // [8]
    unsigned *ticket = nullptr;  // arrival counter of the last-block finish (0 between launches)
};

// ---- one launch over the points of a shape group (the batched sweep) -------
// Every point of a group keeps its arrays at the same offsets inside its own
// arena of `arena` bytes, point p's at p * arena from point 0's; a batched
// launch passes point 0's pointers, P = gridDim.z and the arena, and each
// block works on point p = blockIdx.z (at() below).  The shape tables
// (twiddles, spline pivots, octant weights) are shared.  The point's scalars
// are pp[slot] in its arena (pp non-null): they replace the launch's
// by-value arguments.  Bp{} (P = 1, arena 0, pp null) is a plain launch.
constexpr int kPP = 16;
enum PpSlot {
    kPpT = 0,       // temperature
    kPpMu0,         // mu0 (written on the device by the batched density root)
    kPpU,           // U
    kPpN,           // density n
    kPpNsr,         // nsr of the sum rules
    kPpNormFact,    // T / L^2
    kPpJc,          // first frequency of the find_mu series
    kPpWc,          // w_jc
    kPpMu0Fixed,    // 1: mu0 = 0 (half filling with t' = t'' = 0), no root search
};
struct Bp {
    int P = 1;
    long long arena = 0;       // bytes between consecutive points' arrays
    const double *pp = nullptr;  // point 0's scalars [kPP]
};

// ---- launchers (all asynchronous on `st`) ---------------------------------
cudaError_t launch_density(const GridDev &g, double mu, double n, double T, Reduce r, cudaStream_t st);

// per-octant (eps - mu0, G0 prefactor) into g.gk
cudaError_t launch_gk_table(const GridDev &g, double mu0, double T, cudaStream_t st, const Bp &b = Bp{});
cudaError_t launch_gslice(const GridDev &g, double *Grt, double mu0, double T, cudaStream_t st);
cudaError_t launch_chi0_boundary(const GridDev &g, const double *Grt, double mu0, double T,
                                 double *dG0p, double *dtau_chirt0, double *dtau_chiqt0, cudaStream_t st);
cudaError_t launch_chi0_boundary(const GridDev &g, const float *Grt, double mu0, double T,
                                 double *dG0p, double *dtau_chirt0, double *dtau_chiqt0, cudaStream_t st,
                                 const Bp &b = Bp{});
// the mixed-precision form's FP32 slice transforms (tpsc_mixed.cu)
cudaError_t launch_gslice32(const GridDev &g, float *Grt, double mu0, double T, cudaStream_t st, const Bp &b = Bp{});
cudaError_t launch_chi0_slice32(const GridDev &g, const float *Grt, double *chirt, double *chiq, cudaStream_t st,
                                const Bp &b = Bp{});
// Usc: the device pair (Usp, Uch) -- the sum-rule root search leaves it there
cudaError_t launch_vertex_q32(const GridDev &g, const double *chiq, double *Vr, double U, const double *Usc, double T,
                              cudaStream_t st, const Bp &b = Bp{});
cudaError_t launch_chi0_slice(const GridDev &g, const double *Grt, double *chirt, double *chiq, cudaStream_t st);
cudaError_t launch_chi0_tau(const GridDev &g, double *chiq, const double *dtau_chiqt0, double *chi0_inf,
                            double *chi0_inf2, double T, cudaStream_t st, const Bp &b = Bp{});

// mu0 by safeguarded Newton in one block -> r.result[0] (iterations in r.result[1])
cudaError_t launch_mu0_newton(const GridDev &g, double n, double T, Reduce r, cudaStream_t st, const Bp &b = Bp{});
// chi0max, qmax -> r.result[0..2]
cudaError_t launch_chi0max(const GridDev &g, const double *chiq, Reduce r, cudaStream_t st, const Bp &b = Bp{});

// sum-rule trace and its U derivative -> r.result[0..1]; stored frequencies
// j < jdir term by term (jdir = -1: all)
cudaError_t launch_sumrule(const GridDev &g, const double *chiq, const double *chi0_inf, const double *chi0_inf2,
                           double Uv, double sign, double T, Reduce r, cudaStream_t st, int jdir = -1,
                           int tail = 1);
// Matsubara-tail moments sum_q w S_(k+2) -> r.result[0..kMomP), max tail |chi| ->
// r.result[kMomP + 1] (r.partial must hold (2 kMomP + 2) kMaxBlocks doubles)
cudaError_t launch_tail_moments(const GridDev &g, const double *chi0_inf, const double *chi0_inf2, double T,
                                Reduce r, cudaStream_t st, const Bp &b = Bp{});
// per-frequency moments sum_q w f chi^(k+2), k < kMomP -> mom [nb][kMomP]; max_q |chi| -> cmax [nb]
constexpr int kMomP = 8;
constexpr double kMomSeriesMax = 0.004;  // |h chi| bound of the series terms: 0.004^8 < 1e-19
constexpr double kMomMuRange = 0.35;     // |mu - mu0| the find_mu series is built to cover
constexpr int kMuMomP = 12;              // terms of the find_mu series
constexpr double kMuSeriesMax = 0.03;    // |mu - mu0| / |z| bound of its terms: 0.03^12 < 1e-18
cudaError_t launch_chi0_moments(const GridDev &g, const double *chiq, double *mom, double *cmax, cudaStream_t st,
                                const Bp &b = Bp{});
// Forward tangents of the chi0 stage (tpsc_tangent.cu): buffers of one
// direction.  fd[o] = (beta f(xi_o), dxi_o); der[o] the direction of the
// hopping table; Grt the FP64 G(r, tau) and dG0p the primal d/dtau G(r, 0+).
struct TangentBufs {
    const double *Grt = nullptr, *dG0p = nullptr, *der = nullptr;
    const double2 *fd = nullptr;
    double *dGrt = nullptr;  // [(Nw0+1) n8]  dG(r, tau)
    double *dchiq = nullptr; // blocked nb    dchi0(q, tau) -> dchi0(q, iqn) after launch_chi0_tau
    double *ddq0 = nullptr;  // [n8]          d of d/dtau chi0(q, 0)
    double *ddG0p = nullptr; // [n8] or null  d of d/dtau G(r, 0+)
    double *ddchir = nullptr; // [n8] or null d of d/dtau chi0(r, 0)
};
// dG(r, tau), dchi0(q, tau_j) and d(d/dtau chi0(q, 0)) for the direction in t
// (mu0 the primal chemical potential, dmu0 its direction)
cudaError_t launch_chi0_tangent(const GridDev &g, const TangentBufs &t, double mu0, double dmu0, double T,
                                cudaStream_t st);
// the directional derivative of the full sum-rule trace (k_sumrule with
// every frequency and the tail term by term) at U = Uv in the direction
// (dchiq, dchi0_inf, dchi0_inf2) -> r.result[0]
cudaError_t launch_sumrule_tan(const GridDev &g, const double *chiq, const double *dchiq, const double *chi0_inf,
                               const double *chi0_inf2, const double *dchi0_inf, const double *dchi0_inf2, double Uv,
                               double sign, double T, Reduce r, cudaStream_t st);
// sums of mom over the frequencies >= j (double-double, rounded once),
// j = 0..nb -> mom_suf [(nb + 1)][kMomP]; suffix maxima of cmax -> cmax_suf
// [nb + 1]; the tail moments and tail maximum of launch_tail_moments' result
// -> tailm [kMomP + 1].  One launch, no host round trip.
cudaError_t launch_moment_suffix(const GridDev &g, const double *mom, const double *cmax, const double *tail_result,
                                 double *mom_suf, double *cmax_suf, double *tailm, cudaStream_t st,
                                 const Bp &b = Bp{});
cudaError_t launch_trace_chi0(const GridDev &g, const double *chiq, const double *chi0_inf,
                              const double *chi0_inf2, double T, Reduce r, cudaStream_t st);

// Usc: the device pair (Usp, Uch); fact = U (3 Usp + Uch) / 8 is formed in the kernels
cudaError_t launch_vertex_q(const GridDev &g, const double *chiq, double *Vr, double U, const double *Usc, double T,
                            cudaStream_t st);
cudaError_t launch_vertex_tau(const GridDev &g, double *Vr, const double *chirt, double U, const double *Usc,
                              cudaStream_t st, const Bp &b = Bp{});

cudaError_t launch_sigma_boundary(const GridDev &g, const double *Grt, const double *V, const double *dtau_chirt0,
                                  const double *dG0p, double mu0, double U, const double *Usc, double *dS,
                                  cudaStream_t st);
cudaError_t launch_sigma_boundary(const GridDev &g, const float *Grt, const double *V, const double *dtau_chirt0,
                                  const double *dG0p, double mu0, double U, const double *Usc, double *dS,
                                  cudaStream_t st, const Bp &b = Bp{});
cudaError_t launch_sigma_slice(const GridDev &g, const double *Grt, const double *V, double *sigt, cudaStream_t st);
// the mixed form's Sigma slices: FP32 transform, local term in FP64 (tpsc_mixed.cu)
cudaError_t launch_sigma_slice32(const GridDev &g, const float *Grt, const double *V, double *sigt, cudaStream_t st,
                                 const Bp &b = Bp{});
cudaError_t launch_sigma_tau(const GridDev &g, const double *sigt, const double *dS, double2 *S, double *s2,
                             double *s3, double *s4, double *sinf, double T, cudaStream_t st, const Bp &b = Bp{});

// Tr(G - G0) at pmu and its pmu derivative -> r.result[0..1]; jdir = -1: all
// frequencies (stored and tail), else stored j < jdir only
cudaError_t launch_trace_diff_G(const GridDev &g, const double2 *S, const double *s2, const double *s3,
                                const double *s4, const double *sinf, double mu0, double pmu, double T, Reduce r,
                                cudaStream_t st, int jdir = -1);
cudaError_t launch_trace_self_G(const GridDev &g, const double2 *S, const double *s2, const double *s3,
                                const double *sinf, double mu0, double T, Reduce r, cudaStream_t st);
cudaError_t launch_trace_self_G2(const GridDev &g, const double2 *S, const double *s2, const double *s3,
                                 const double *sinf, double mu, double T, Reduce r, cudaStream_t st);

// ---- the Newton form's root searches on the device (tpsc_roots.cu) ----------
constexpr int kRootMaxBlocks = 1024;
constexpr int kRootVals = 3;  // per-block partials of an evaluation: value and two derivatives
struct RootScratch {
    double *partial = nullptr;  // [2 kRootVals kRootMaxBlocks]: two parities
    unsigned *bar = nullptr;    // [8]: arrivals, generation, error flag of the sum-rule search (0..2)
                                //      and of the mu search (4..6)
    double *out = nullptr;      // [8] results
    int max_blocks = 0;         // cap on the cooperative grid (0: two blocks per SM)
    // Zero the search's barrier words before its launch.  The barrier leaves
    // them zero after every launch that did not time out, so the host clears
    // these once it has read a zero error flag after the last launch.
    bool reset_sr = true, reset_mu = true;
};
// The Newton form's Sigma pass: Tr Sigma G0 (green::traceSelfG) and the
// find_mu series moments around mu0 over the frequencies n >= jc and the tail
// -> r.result[0..1] = (trace, asymptotic correction), r.result[2 + 2m],
// r.result[3 + 2m] = Re, Im sum w (i w_n - eps + mu0 - Sigma)^-(m+1), m < kMuMomP,
// r.result[2 + 2 kMuMomP] = sum w Re 1/(i w_n - eps + mu0).  r.partial must
// hold (2 kMuMomP + 3) kMaxBlocks doubles.
constexpr int kSigmaMomNV = 2 * kMuMomP + 3;
cudaError_t launch_sigma_moments(const GridDev &g, const double2 *S, const double *s2, const double *s3,
                                 const double *s4, const double *sinf, double mu0, double T, int jc, Reduce r,
                                 cudaStream_t st, const Bp &b = Bp{});
// mu by safeguarded Newton from mu0 (the series of the moments `mom` while
// |mu - mu0| <= kMuSeriesMax (wc - 2 |Sigma_inf| / wc), wc = w_jc, the full
// sum beyond), then Tr Sigma G at mu; one cooperative launch -> rs.out =
// {mu, evals, ok, Tr Sigma G}
cudaError_t launch_mu_roots(const GridDev &g, const double2 *S, const double *s2, const double *s3, const double *s4,
                            const double *sinf, const double *mom, double mu0, double T, int jc, double wc,
                            RootScratch rs, cudaStream_t st, const Bp &b = Bp{});
// Usp then Uch by safeguarded Newton with the moment series, one cooperative
// launch -> rs.out = {Usp, Uch, evals_sp, evals_ch, ok_sp, ok_ch}.  With
// chi0max (device), the spin interval ends at 2 / chi0max[0] - hi_off and
// hi_sp is not used.
cudaError_t launch_sumrule_roots(const GridDev &g, const double *chiq, const double *chi0_inf, const double *chi0_inf2,
                                 const double *mom_suf, const double *cmax_suf, const double *tailm, double T,
                                 double n, double nsr, double U, double hi_sp, RootScratch rs, cudaStream_t st,
                                 const double *chi0max = nullptr, double hi_off = 0.0, const Bp &b = Bp{});

// ---- real-frequency continuation (Pade / Lagrange) and local G ---------------
cudaError_t launch_pade_sigma(const GridDev &g, const double2 *S, const double *s2, const double *s3,
                              const double *sinf, const int *nidx, int Nn, const double2 *z, int Nz, int mode,
                              double mu, double T, double2 *out_sig, double *out_A, cudaStream_t st);
cudaError_t launch_gwn_local(const GridDev &g, const double2 *S, const double *s2, const double *s3,
                             const double *sinf, double mu, double T, double2 *out, cudaStream_t st);

// ---- current-current correlator (bubble + Maki-Thompson) and kx0 -----------
// K4 = (nbk - 2) nbk interior-kx points, c = l nbk + m for kx = (l+1) pi/(nbk-1),
// ky = m pi/(nbk-1).
struct CondDev {
    int K4 = 0;             // interior-kx points
    int K4p = 0;            // K4 rounded up to even (column pairs)
    int nbins = 1;          // angular bins of the k-resolved sums (N_theta_k)
    int nblk = 0;           // CTAs of the persistent tau kernel
    int pw = 0;             // partial row width: nbins 2 (Nw0/2+1) + 1
    double *dek = nullptr;     // [K4]  d eps/d kx
    double *d2ek = nullptr;    // [K4]  d2 eps/d kx2
    double *d2line = nullptr;  // [2 nbk] d2 eps/d kx2 on kx = 0, then kx = pi
    int *bin = nullptr;        // [K4]  angular bin of each point
    double *tab = nullptr;     // [4 K4] (eps - mu0, A, B, 0) of the h, f0 slices
    double *hV = nullptr;      // [K4p (Nw0+1)] h V(r, tau), two-column blocks
    double *f0V = nullptr;     // [K4p (Nw0+1)] f0 V(r, tau), two-column blocks
    double *pre = nullptr;     // [4 K4p] transformed h, f0 at tau = 0, beta
    double *dbound = nullptr;  // [4 K4p] dhV(0), dhV(beta), df0V(0), df0V(beta)
    double *partial = nullptr; // [nblk pw] per-CTA sums
    double *lines = nullptr;   // [2 nbk] kx0 terms of the kx = 0, pi lines
    double *out = nullptr;     // [nbins 2 NB] binned, [2 NB] totals, kx0 (NB = Nw0/2+1)
};

cudaError_t cond_blocks(const GridDev &g, int *blocks);
// the (eps - mu0, A, B) table of the h and f0 slices into c.tab
cudaError_t launch_cond_table(const GridDev &g, const CondDev &c, double mu0, double T, cudaStream_t st);
// table + h V, f0 V slices + end conditions (fact = U (3 Usp + Uch)/4)
cudaError_t launch_cond_slices(const GridDev &g, const CondDev &c, const double *V, const double *dtau_chirt0,
                               double mu0, double T, double fact, cudaStream_t st);
// the mixed form's slices: both transforms of the h and f0 slices in FP32
// (tpsc_mixed.cu), the table and the end conditions in FP64
cudaError_t launch_cond_slices32(const GridDev &g, const CondDev &c, const double *V, const double *dtau_chirt0,
                                 double mu0, double T, double fact, cudaStream_t st);
// the FP32 slice kernel alone (after the table), ny = 2: h and f0, 1: h
cudaError_t launch_cond_slice32(const GridDev &g, const CondDev &c, const double *V, double T, int ny,
                                cudaStream_t st);
// the h slices and their two end conditions only (the reverse pass's forward values)
cudaError_t launch_cond_slices_h(const GridDev &g, const CondDev &c, const double *V, const double *dtau_chirt0,
                                 double mu0, double T, double fact, cudaStream_t st);
// per-k pairs -> c.partial (zeroed first)
cudaError_t launch_cond_tau(const GridDev &g, const CondDev &c, const double2 *S, const double *s2, const double *s3,
                            const double *sinf, double mu, double T, cudaStream_t st);
// kx = 0, pi lines and the ordered sum of the partial rows -> c.out
cudaError_t launch_cond_finish(const GridDev &g, const CondDev &c, const double2 *S, const double *s2,
                               const double *s3, const double *sinf, double mu, double T, cudaStream_t st);

// ---- the reverse pass of V -> Sigma -> mu -> chi_jj -> sigma(iq_n) (tpsc_adjoint.cu)
// Every backward kernel leaves per-CTA rows of kAdjW partial sums: the loss
// derivative along mu, Sigma_inf, the mu0-shift and t' directions (through
// the tangents), and along fact4 = U(3Usp+Uch)/4, fact8 = U(3Usp+Uch)/8,
// Usp, Uch and U held fixed elsewhere.  The host adds the rows in order.
constexpr int kAdjW = 12;
enum AdjSlot { kAdjMu = 0, kAdjSinf, kAdjTh1, kAdjTh2, kAdjFact4, kAdjFact8, kAdjUsp, kAdjUch, kAdjU };
struct AdjDev {
    // forward tangents of the chi0 stage along the mu0 shift [0] and t' [1]
    double *dGrt[2] = {nullptr, nullptr};   // [(Nw0+1) n8]
    double *dchiq[2] = {nullptr, nullptr};  // blocked nb: dchi0(q, iqn)
    double *ddG0p[2] = {nullptr, nullptr};  // [n8] d of d/dtau G(r, 0+)
    double *ddchir[2] = {nullptr, nullptr}; // [n8] d of d/dtau chi0(r, 0)
    double *der2 = nullptr;                 // [n8] the hopping table's direction along t'
    double *cw = nullptr;                   // [Nw0/2 + 1] d L / d chi_jj(iq_n)
    double2 *ws = nullptr;                  // [nblk 2 (Nw0/2)] per-CTA G(ik_n), J(ik_n)
    double *hVb = nullptr;                  // [K4p (Nw0+1)] two-column blocks: d L / d hV
    double *dbb = nullptr;                  // [2 K4p] d L / d dhV(0), dhV(beta)
    double2 *sigc = nullptr;                // [K4 (Nw0/2)] d L / d Sigma per K4 column
    double2 *sigl = nullptr;                // [2 nbk (Nw0/2)] the same on the kx = 0, pi lines
    double *tmpB = nullptr, *vbk = nullptr, *preb = nullptr, *dchb = nullptr;  // [2 K4p] each
    double *tmpU = nullptr, *vcond = nullptr;                                  // [nb K4p] each
    double *htab = nullptr;                 // [8 K4] the h slices' point table of the reverse pass
    double2 *Sb = nullptr;                  // [n8 (Nw0/2)] d L / d S, column-major
    double *s2b = nullptr, *s3b = nullptr;  // [n8]
    double *stb = nullptr;                  // blocked Nw0+1: d L / d Sigma(k, tau)
    double *dSb = nullptr;                  // [2 n8p]
    double *Vb = nullptr;                   // blocked nb: d L / d V(r, tau), then d L / d V(r, iqn)
    double *part = nullptr;                 // [rows kAdjW]
    int nblk = 0;
    int row_ct = 0, row_cl = 0, row_cb = 0, row_cs = 0, row_sg = 0, row_ss = 0, row_sb = 0, row_vt = 0, row_vq = 0;
    int rows = 0;
};
struct CondBwdArgs {
    const double *hV = nullptr, *dbound = nullptr;
    const double2 *S = nullptr;
    const double *s2 = nullptr, *s3 = nullptr, *sinf = nullptr;
    const double *ek = nullptr, *dek = nullptr, *d2ek = nullptr;
    const double *spl_full = nullptr, *spl_half = nullptr;
    const double2 *tw = nullptr, *ht = nullptr;
    const double *cw = nullptr;
    double kx0b = 0.0;
    double2 *ws = nullptr;
    double *hVb = nullptr, *dbb = nullptr;
    double2 *sigc = nullptr;
    double *part = nullptr;
    int K4 = 0, K4p = 0, nbk = 0;
    double mu = 0.0, T = 0.0, nf = 0.0;
};
cudaError_t cond_bwd_blocks(const GridDev &g, int *blocks);
cudaError_t launch_cond_tau_bwd(const GridDev &g, const CondBwdArgs &a, int nblk, cudaStream_t st);
cudaError_t launch_cond_lines_bwd(const GridDev &g, const CondDev &c, const AdjDev &a, const double2 *S,
                                  const double *s2, const double *s3, const double *sinf, double mu, double T,
                                  double kx0b, cudaStream_t st);
// the chi_jj boundary (two CTAs) and h slices (one CTA per tau pair) backward
cudaError_t launch_cond_slices_bwd(const GridDev &g, const CondDev &c, const AdjDev &a, const double *V,
                                   const double *dchirt0, double mu0, double T, double fact4, double dmu0_2,
                                   cudaStream_t st);
// lam = -(d L / d mu) / (d traceDiffG / d mu)
cudaError_t launch_sigbar(const GridDev &g, const CondDev &c, const AdjDev &a, const double2 *S, const double *s2,
                          const double *s3, const double *s4, const double *sinf, double mu0, double mu, double lam,
                          double T, double dmu0_2, cudaStream_t st);
cudaError_t launch_sigma_tau_bwd(const GridDev &g, const AdjDev &a, double sinfb, double T, cudaStream_t st);
cudaError_t launch_sigma_slices_bwd(const GridDev &g, const CondDev &c, const AdjDev &a, const double *Grt,
                                    const double *V, const double *dchirt0, const double *dG0p, double mu0,
                                    double fact8, double dmu0_2, cudaStream_t st);
cudaError_t launch_vertex_bwd(const GridDev &g, const AdjDev &a, const double *chirt, const double *chiq,
                              const double *Grt, double U, double Usp, double Uch, double T, cudaStream_t st);

// ---- Aslamazov-Larkin correction chijj3 on the non-uniform iqn grid --------
// (tpsc_al.cu).  Arrays on the K4 grid of the correlator; NJ = Nw0 + 1 tau
// nodes, NO = Nw0 / 2.
struct AlDev {
    int K4 = 0, K4p = 0;        // as CondDev
    int nrows = 0;              // rows of out (grid frequencies)
    int nbins = 1;              // angular bins
    double *Grt = nullptr;      // [NJ n8]   FP64 G(r, tau_j) (the G(r, -tau) of the AL branch by symmetry)
    double *hGt = nullptr;      // [K4p NJ]  h G(q, tau), two-column blocks
    double *pre = nullptr;      // [2 K4]    h(r, 0), h(r, beta)
    double *dhG = nullptr;      // [2 K4]    d/dtau h G(q) at 0, beta
    double *hgq = nullptr;      // [K4 (NO+1)] h G(q, i q_p), p < NO, then its 1/q^2 coefficient hg2
    double2 *HQ = nullptr;      // [NJ K4]   H(q, tau_j) of the current frequency
    double2 *dHQ = nullptr;     // [2 K4]    d/dtau H(q) at 0, beta
    double2 *HR = nullptr;      // [NJ K4]   H(r, tau_j)
    double2 *dHR = nullptr;     // [2 K4]
    double2 *HK = nullptr;      // [K4p NJ]  G H(k, tau), two-column blocks
    double2 *H2K = nullptr;     // [K4p NJ]  G H2(k, tau), H2(r, tau) = H(r, beta - tau)
    double2 *dHK = nullptr;     // [4 K4]    end slopes: H at 0, beta; H2 at 0, beta
    double *colv = nullptr;     // [K4]      per-point term of the current frequency
    double *out = nullptr;      // [nrows (1 + nbins)] chijj3, then its angular bins
};
// once per call: G(r, tau) in FP64, h G(q, tau), its end slopes and h G(q, i q_p)
// (c.tab, c.dek must be current)
cudaError_t launch_al_setup(const GridDev &g, const CondDev &c, const AlDev &a, const double *dG0p, double mu0,
                            double T, cudaStream_t st);
// one grid frequency q_nn -> row `row` of a.out
cudaError_t launch_al_freq(const GridDev &g, const CondDev &c, const AlDev &a, const double *chiq, const double *cinf,
                           const double *cinf2, const double2 *S, const double *s2, const double *s3,
                           const double *sinf, const double *dG0p, int nn, int row, double U, double Usp, double Uch,
                           double mu, double mu0, double T, cudaStream_t st);

// The root searches' bounded grid barrier on its own, in a cooperative launch
// of their grid (returned in *blocks): block `withhold` never arrives
// (negative: all do).  words [4], zeroed here: barrier, generation, error
// flag, blocks that left the barrier with the error.
cudaError_t launch_barrier_probe(unsigned *words, int withhold, int *blocks, cudaStream_t st);

// Batched continued-fraction Pade of nf functions sampled at Nn points
// (x, y: [nf][Nn]) evaluated at Nz shared points: out [nf][Nz].
constexpr int kPadeBatchMax = 4096;
cudaError_t launch_pade_batch(const double2 *x, const double2 *y, int nf, int Nn, const double2 *z, int Nz,
                              double2 *out, cudaStream_t st);

// ---- layout conversion for the getters ------------------------------------
// blocked (NJ rows) -> reference layout [j][o], j < nrows
cudaError_t launch_unblock(const double *src, double *dst, int NJ, int nrows, int n8, cudaStream_t st);
cudaError_t launch_unblock_c(const double2 *src, double2 *dst, int NJ, int nrows, int n8, cudaStream_t st);
// the full Sigma(k, i w_n), n < Nw0/2, in FP32, [n][o]
cudaError_t launch_sigma_full32(const GridDev &g, const double2 *S, const double *s2, const double *s3,
                                const double *sinf, double T, float2 *dst, cudaStream_t st);
// row j of a blocked (NJ rows) array -> dst[o], o < n8
cudaError_t launch_take_row(const double *src, int NJ, int j, int n8, double *dst, cudaStream_t st);
// reference layout [j][o], j < nrows -> blocked (NJ rows): the setters
cudaError_t launch_block(const double *src, double *dst, int NJ, int nrows, int n8, cudaStream_t st);
cudaError_t launch_block_c(const double2 *src, double2 *dst, int NJ, int nrows, int n8, cudaStream_t st);

// ---- gathers done by the SMs instead of a copy engine -----------------------
// Up to kGatherPieces ranges of 4-byte words, each copied to a word offset of
// dst.  With dst in mapped pinned host memory this is the solve's scalar
// readback: no copy engine is involved, so it is not queued behind a large
// device-to-host copy running on another stream (tpsc_get_self_async).
constexpr int kGatherPieces = 8;
struct GatherPieces {
    const unsigned *src[kGatherPieces] = {};
    long long words[kGatherPieces] = {};
    long long dst[kGatherPieces] = {};
    int n = 0;
};
cudaError_t launch_gather(const GatherPieces &p, unsigned *dst, int blocks, cudaStream_t st);
// up to four host values stored to dst[0..n) in stream order (no copy engine)
cudaError_t launch_store(double *dst, const double *v, int n, cudaStream_t st);

// tiling of the tau transforms (chi0, V, Sigma) per N, process-wide: 0 one
// column pair per CTA (the default), 1 four columns per CTA; the version
// counts the changes
constexpr int kTauChi0 = 0, kTauVertex = 1, kTauSigma = 2;
int tau_tile(int kind, int n);
void set_tau_tile(int kind, int n, int tile);
long long tau_tiles_version();
// adds one to the version above (a plan changed: captured graphs are stale)
void bump_plans_version();

// plan of the mixed form's FP32 slice transforms per kind and lattice,
// process-wide: kSliceFft the packed radix-16 FFTs (tpsc_fft.cuh),
// kSliceDirect the folded matrix DCT-I (tpsc_dct.cuh; nbk 33, 65, 129)
constexpr int kSliceG = 0, kSliceChi0 = 1, kSliceVertex = 2, kSliceSigma = 3;
constexpr int kSliceFft = 0, kSliceDirect = 1, kSliceTensor = 2;
int slice_plan(int kind, int nbk);
void set_slice_plan(int kind, int nbk, int plan);
bool slice_plan_supported(int kind, int plan, int nbk);
// the table of the direct plan for a quadrant side nbk (empty where it does not apply)
void dct_table(int nbk, std::vector<float> &out);
// the tensor plan (tpsc_tcdct.cu): the Sigma and V slices of the 256 x 256 lattice
void dct_tc_table(int nbk, std::vector<float> &out);
cudaError_t launch_sigma_slice_tc(const GridDev &g, const float *Grt, const double *V, double *sigt,
                                  cudaStream_t st, const Bp &b = Bp{});
cudaError_t launch_vertex_q_tc(const GridDev &g, const double *chiq, double *Vr, double U, const double *Usc,
                               double T, cudaStream_t st, const Bp &b = Bp{});
// the tensor plan's error word (nonzero after a bounded wait ran out); 0 on success
int tensor_plan_errors(unsigned *out, bool clear);
cudaError_t launch_sigma_slice_dct(const GridDev &g, const float *Grt, const double *V, double *sigt,
                                   cudaStream_t st, const Bp &b = Bp{});
cudaError_t launch_gslice_dct(const GridDev &g, float *Grt, double mu0, double T, cudaStream_t st,
                              const Bp &b = Bp{});
cudaError_t launch_chi0_slice_dct(const GridDev &g, const float *Grt, double *chirt, double *chiq, cudaStream_t st,
                                  const Bp &b = Bp{});
cudaError_t launch_vertex_q_dct(const GridDev &g, const double *chiq, double *Vr, double U, const double *Usc,
                                double T, cudaStream_t st, const Bp &b = Bp{});

// kernels launched by the library so far
long long launches_total();
// kernels launched (or captured) by the calling host thread so far
long long launches_thread();
// adds n to the library's count (kernels replayed by a CUDA graph; negative
// to take back the kernels that a stream capture only recorded)
void add_launches(long long n);

// the FFT lengths the build instantiates
bool supported_grid(int nk0, int nw0);

}  // namespace tpsc
