/*
 * tpsc_b200.h -- C ABI of the B200 (sm_100a) TPSC engine.
 *
 * The reference (dbergeron1/TPSC_conductivity) has no FFI: its interface is a
 * chain of C++ classes (hamiltonien -> green0 -> chi0 -> chi -> green ->
 * cond_opt) whose methods run OpenMP loops over FFTW and LAPACK.  Each entry
 * point below replaces one of those methods (cited as path:line in the
 * reference checkout) and is what a drop-in of those classes binds.
 *
 * Conventions
 *  - plain C types only; every call returns a tpsc_status (0 = OK);
 *  - one context owns one CUDA stream and all device arrays of its grids; a
 *    context is not thread-safe (the reference's objects are not either);
 *  - host output buffers use the reference's layouts: octant index
 *    o = m + l(l+1)/2 (m <= l < nbk = nk0/2+1), frequency-major arrays
 *    [j * N8 + o], complex numbers as interleaved (re, im) doubles;
 *  - "the current grid" is the (nk0, Nw0) of the last tpsc_chi0 call, as
 *    chi0::calc_chiqw_FFT_spline re-grids the reference object (set_grid,
 *    src/green0.h:44).
 */
#ifndef TPSC_B200_H
#define TPSC_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct tpsc_ctx tpsc_ctx;

enum tpsc_status {
    TPSC_OK = 0,
    TPSC_ERR_ARG = 1,        /* bad argument or unsupported size */
    TPSC_ERR_CUDA = 2,       /* CUDA runtime error (message in tpsc_last_error) */
    TPSC_ERR_OOM = 3,        /* device allocation failed */
    TPSC_ERR_NO_ROOT = 4,    /* root search failed (find_zero returned false) */
    TPSC_ERR_STATE = 5,      /* a prerequisite stage has not run */
    TPSC_ERR_NONFINITE = 6   /* non-finite result */
};

/* Scalar results, index into tpsc_get_scalars(). */
enum tpsc_scalar {
    TPSC_S_MU0 = 0,        /* green0::mu0 (src/green0.cpp:240-262) */
    TPSC_S_CHI0MAX,        /* chi0::chi0max (src/chi0.cpp:703-717) */
    TPSC_S_QMAX0,          /* chi0::qmax[0] */
    TPSC_S_QMAX1,          /* chi0::qmax[1] */
    TPSC_S_USP,            /* chi::Usp */
    TPSC_S_UCH,            /* chi::Uch */
    TPSC_S_DBLOCC,         /* chi::dblOcc ansatz (src/chi.cpp:370-371) */
    TPSC_S_DIFRELSP,       /* half grid vs full grid (src/chi.cpp:308-309) */
    TPSC_S_DIFRELCH,
    TPSC_S_SIGMA_INF,      /* green::Sigma_inf */
    TPSC_S_MU,             /* green::mu */
    TPSC_S_TR_SG,          /* traceSelfG raw sum (src/green.cpp:3088) */
    TPSC_S_TR_SG_ASYMP,    /* traceSelfG with asymptotic correction (:3089) */
    TPSC_S_TR_SG2,         /* traceSelfG2 (src/green.cpp:2979) */
    TPSC_S_DBLOCC_SG2,     /* double occupancy from Tr Sigma G (:2980) */
    TPSC_S_TR_CHI0,        /* traceChi0 raw (src/chi0.cpp:1578) */
    TPSC_S_TR_CHI0_CORR,   /* traceChi0 extrapolated (src/chi0.cpp:1580) */
    TPSC_S_EVALS_SP,       /* sum-rule evaluations spent on Usp */
    TPSC_S_EVALS_CH,       /* ... on Uch */
    TPSC_S_EVALS_MU,       /* Tr(G-G0) evaluations spent on mu */
    TPSC_S_COUNT
};

/* How a solve computes (tpsc_set_form); the flags combine.
 *  TPSC_FORM_REFERENCE (0): FP64 throughout and the reference's find_zero
 *    control flow for mu0, Usp, Uch and mu (src/generique.cpp:604-1234) --
 *    the FP64 drop-in, same roots and the same number of function
 *    evaluations as the reference;
 *  TPSC_FORM_NEWTON (1): safeguarded Newton steps inside the reference's
 *    search intervals, with the derivative from the same device pass as the
 *    value (d trace/dU of the sum rules, d Tr(G-G0)/d mu, dn/d mu0); the
 *    high frequencies of the sum rules and of Tr(G-G0) enter as power series
 *    from moments computed once per search (truncation below 1e-19 of the
 *    leading term).  Same roots to ~1e-14, several times fewer passes;
 *  TPSC_FORM_MIXED (2): the G(r, tau), chi0(q, tau) and V(q) slice transforms
 *    in FP32 with compensated twiddles (G stored in FP32); Sigma's
 *    transforms, every tau transform, the sum rules, traces, roots and the
 *    continuation in FP64.  Sigma within ~1e-6 of the FP64 forms.
 * Neither NEWTON nor MIXED has a counterpart in the reference. */
enum tpsc_form { TPSC_FORM_REFERENCE = 0, TPSC_FORM_NEWTON = 1, TPSC_FORM_MIXED = 2 };

/* Create a context on CUDA device `device`.  Returns NULL and sets *status on
 * failure (no CUDA device, driver error). */
tpsc_ctx *tpsc_create(int device, int *status);
void tpsc_destroy(tpsc_ctx *ctx);
/* Last error message of the context (static storage if ctx is NULL). */
const char *tpsc_last_error(const tpsc_ctx *ctx);

/* Model of the green(nk0, Nw0, n, T, eta, {tp, tpp, t3, U}) constructor
 * (src/green.h:26, src/hamiltonien.cpp:13-30, src/green0.cpp:13-23):
 * lattice side nk0 (power of two, 8..256), Nw0 total fermionic frequencies
 * (power of two, 16..4096), density n in (0,2), temperature T > 0.
 * Computes eps_k and mu0 of the finite lattice on the device. */
int tpsc_set_model(tpsc_ctx *ctx, int nk0, int Nw0, double n, double T, double tp, double tpp, double t3,
                   double U);

/* Root-search form of the following solves (enum tpsc_form); default
 * TPSC_FORM_REFERENCE. */
int tpsc_set_form(tpsc_ctx *ctx, int form);

/* The sum rules' nsr (src/chi.cpp:18-19: n, or 2 - n for n > 1), which
 * tpsc_set_model derives from the density; this value holds instead until the
 * next tpsc_set_model.  The reference sets nsr once, in the chi constructor,
 * so a chi object whose density changes (set_density, chi::calc_corr_length
 * src/chi.cpp:931-981) keeps its constructor's nsr. */
int tpsc_set_nsr(tpsc_ctx *ctx, double nsr);

/* CUDA graphs for Newton-form solves (no counterpart in the reference, whose
 * solve runs on the host).  A Newton-form tpsc_solve queues its launches with
 * no host round trip, so the whole solve from the chi0 stage to the final
 * readback can run as one captured graph.  mode 0: direct launches; 1
 * (default): a solve whose launches repeat those of the previous solve
 * (same grid, form, model and mu0) is captured and replayed from then on;
 * 2: every solve is captured (after the grid's first direct solve in that
 * form), the executable graph updated in place for the new arguments.  A
 * capture that fails leaves the context on direct launches. */
int tpsc_set_graph_mode(tpsc_ctx *ctx, int mode);

/* Tilings of the three tau transforms (chi0, V, Sigma), process-wide per
 * Nw0: tile 0 one column pair per CTA (two CTAs per SM, the default), 1 four
 * columns per CTA.  tpsc_tune_tau_tiles times both on the current grid after
 * a solve (reps runs each) and keeps the faster of each; ms (may be NULL)
 * receives the mean times, ms[2 kind + tile].  The transforms run in place,
 * so the next solve recomputes the grid's stages.  tpsc_set_tau_tile sets
 * one tiling (kind 0 chi0, 1 V, 2 Sigma). */
int tpsc_tune_tau_tiles(tpsc_ctx *ctx, int reps, double ms[6]);
/* The same tuner over the FFT plan as well: tile 2 = one column pair per CTA
 * with radix-8 FFT passes (twice the threads in the FFT; Nw0 <= 2048), timed
 * beside tiles 0 and 1; ms[3 kind + plan] (0 where plan 2 does not apply). */
int tpsc_tune_tau_plans(tpsc_ctx *ctx, int reps, double ms[9]);
int tpsc_set_tau_tile(int kind, int nw0, int tile);

/* Plan of the mixed form's FP32 slice transforms (2D DCT-I of symmetric
 * slices; the reference runs them as FFTW REDFT00 x REDFT00 plans,
 * src/chi0.cpp:462-517, src/chi.cpp:89-115, src/green.cpp:1830-1885),
 * process-wide per slice kind (0 G(r, tau), 1 chi0, 2 V, 3 Sigma) and
 * lattice side nk0: plan 0 packed radix-16 FFTs of the even extension,
 * 1 folded matrix DCT-I on the FP32 pipe (nk0 64, 128, 256), 2 the same on
 * the tensor cores (below).  Graphs captured
 * with another plan are captured again.  tpsc_get_slice_plan returns the
 * plan in use (the library's default until one is set), or -TPSC_ERR_ARG. */
int tpsc_set_slice_plan(int kind, int nk0, int plan);
int tpsc_get_slice_plan(int kind, int nk0);
/* Plan 2 (nk0 256, kinds 2 and 3) runs the V or Sigma slice's folded matrix
 * DCT-I on the tcgen05 tensor cores (3xTF32, FP32 accumulation in tensor
 * memory).  Its
 * kernels wait on the tensor cores with a 2 s bound; a wait that runs out
 * sets a process-wide error word (the results of that launch are not valid,
 * the context stays usable).  tpsc_tensor_plan_errors reads the word of the
 * current device into *word and clears it when clear != 0. */
int tpsc_tensor_plan_errors(unsigned *word, int clear);
/* The autotuner over the slice plans: after a mixed-form solve, times every
 * plan each slice kind supports on the current grid (reps launches each),
 * keeps the fastest per kind (process-wide, for this nk0) and leaves the
 * grid to be recomputed by the next solve.  ms (may be NULL) receives the
 * mean times, ms[3 kind + plan], 0 where a plan does not apply. */
int tpsc_tune_slice_plans(tpsc_ctx *ctx, int reps, double ms[12]);

/* out = {captures, replays, kernels in the current graph, 1 if a capture
 * failed and graphs are off}. */
int tpsc_graph_stats(tpsc_ctx *ctx, long long out[4]);

/* chi0::calc_chiqw_FFT_spline(nq0, nw0) (src/chi0.cpp:279-718): switches the
 * current grid to (nq0, nw0) -- re-deriving eps_k and mu0 as set_grid does --
 * and computes chi0(q, iqn), n = 0..nw0/2, with its tail coefficients. */
int tpsc_chi0(tpsc_ctx *ctx, int nq0, int nw0);

/* chi0::traceChi0 (src/chi0.cpp:1498-1584): out[0] raw trace, out[1]
 * extrapolated trace; both compare to n - n^2/2. */
int tpsc_trace_chi0(tpsc_ctx *ctx, double out[2]);

/* chi::traceDiffChispChi0 (channel 0) / traceDiffChichChi0 (channel 1)
 * (src/chi.cpp:738-830) at vertex Uv; *dtrace = d trace / d Uv. */
int tpsc_trace_diff_chi(tpsc_ctx *ctx, int channel, double Uv, double *trace, double *dtrace);

/* chi::find_Usp_Uch(nq0, nw0, Usc) (src/chi.cpp:846-876): chi0 on the grid,
 * then the spin and charge sum-rule roots; Usc = {Usp, Uch}. */
int tpsc_find_Usp_Uch_grid(tpsc_ctx *ctx, int nq0, int nw0, double Usc[2]);

/* chi::find_Usp_Uch() (src/chi.cpp:210-371): half grid, then full grid,
 * difRel diagnostics and the double occupancy ansatz. */
int tpsc_find_Usp_Uch(tpsc_ctx *ctx);

/* Differentiation form, forward half beyond the Newton steps (no counterpart
 * in the reference): the sensitivities of the sum-rule roots and the double
 * occupancy on the current grid, after its chi0 and roots (tpsc_chi0 +
 * tpsc_find_Usp_Uch_grid, or a solve), by forward tangents of
 * chi0 -> sum rules (FP64, tpsc_tangent.cu) and the implicit derivatives of
 * R_sp(Usp) = 0, R_ch(Uch) = 0:
 *   out[3 p + k] = d{Usp, Uch, D}_k / d{U, mu, t'}_p,
 * with mu a shift of the non-interacting chemical potential mu0 at fixed n
 * (tpsc_set_mu_shift) and t' at fixed n (mu0 follows the density). */
int tpsc_sumrule_tangents(tpsc_ctx *ctx, double out[9]);
/* The backward pair: grad[p] = sum_k cot[k] d{Usp, Uch, D}_k / d{U, mu, t'}_p. */
int tpsc_sumrule_vjp(tpsc_ctx *ctx, const double cot[3], double grad[3]);
/* Shift of the non-interacting chemical potential: mu0 = (density root) +
 * dmu on every grid from the next stage on (default 0). */
int tpsc_set_mu_shift(tpsc_ctx *ctx, double dmu);

/* chi::sp_corr_length (src/chi.cpp:420-718) on the current grid after its
 * chi0 and Usp: the Fermi velocity at the hot spots of the non-interacting
 * Fermi surface (green0::find_FS with 10001 lines, src/green0.cpp:626-676)
 * and the spin correlation lengths from chi_sp(q, 0) = chi0/(1 - Usp chi0/2):
 * out = {vF, xi_y, xi_x, xiAs_y, xiAs_x, xi0_y, xi0_x} -- half-maximum
 * lengths along y and x, asymptotic (Ornstein-Zernike) lengths, and xi0. */
int tpsc_sp_corr_length(tpsc_ctx *ctx, double out[7]);
/* The same with the Fermi surface (and so vF and xi0) of mu_fs instead of the
 * current mu0: the reference computes its Fermi surface once, in the green0
 * constructor (src/green0.cpp:35), so after set_density / set_tem
 * (chi::calc_corr_length, src/chi.cpp:931-981) it keeps the constructor's. */
int tpsc_sp_corr_length_fs(tpsc_ctx *ctx, double mu_fs, double out[7]);

/* chi::calc_chirt (src/chi.cpp:37-170): V(r, tau) on tau in [0, beta/2]. */
int tpsc_vertex(tpsc_ctx *ctx);

/* green::calc_Self_FFT_spline, stages after calc_chirt (src/green.cpp:1741-2025):
 * Sigma(k, i w_n) = Sigma_inf/z + C2/z^2 + C3/z^3 + S/z^4, z = i w_n. */
int tpsc_self_energy(tpsc_ctx *ctx);

/* green::traceSelfG (src/green.cpp:3001-3104). */
int tpsc_trace_self_G(tpsc_ctx *ctx, double out[2]);

/* green::traceDiffG (src/green.cpp:3108-3182): Tr(G - G0) at chemical potential
 * mu; *dtrace (may be NULL) = d Tr(G - G0) / d mu from the same pass. */
int tpsc_trace_diff_G(tpsc_ctx *ctx, double mu, double *trace, double *dtrace);

/* green::find_mu (src/green.cpp:3185-3282): mu from Tr(G - G0) = 0, then traceSelfG2. */
int tpsc_find_mu(tpsc_ctx *ctx);

/* One full TPSC solve on the model's grid: chi0 -> Usp, Uch -> V -> Sigma ->
 * traceSelfG -> mu -> traceSelfG2, i.e. green::calc_Self_FFT_spline +
 * traceSelfG + find_mu (src/tpsc_main.cpp:71-75) without the half-grid
 * Usp/Uch pre-pass (which only feeds the difRel diagnostics) and without
 * file output. */
int tpsc_solve(tpsc_ctx *ctx);

/* ---- results ------------------------------------------------------------ */
/* n doubles of the scalar table (enum tpsc_scalar order). */
int tpsc_get_scalars(tpsc_ctx *ctx, double *out, int n);
/* grid of the context: dims = {nk0, Nw0, nbk, N8}. */
int tpsc_get_dims(tpsc_ctx *ctx, int dims[4]);
/* eps_k on the quadrant, ek[m + l*nbk] (src/hamiltonien.cpp:358-375). */
int tpsc_get_ek(tpsc_ctx *ctx, double *ek);
/* chiqw_array [ (Nw0/2+1) * N8 ] (any pointer may be NULL). */
int tpsc_get_chi0(tpsc_ctx *ctx, double *chiqw, double *chi0_inf, double *chi0_inf2, double *dtau_chirt0);
/* vertex_rt_array [ (Nw0/2+1) * N8 ]. */
int tpsc_get_vertex(tpsc_ctx *ctx, double *vertex_rt);
/* Self_kw_array [ (Nw0/2) * N8 ] complex (interleaved), Sigma_inf2/3/4 [N8]. */
int tpsc_get_self(tpsc_ctx *ctx, double *self_kw, double *sigma_inf2, double *sigma_inf3, double *sigma_inf4);

/* The arrays of tpsc_get_self without waiting for them (no counterpart in
 * the reference): the self-energy is snapshotted on the device, in the
 * getter's layout, on the context stream, and the snapshot is copied to the
 * host on a separate copy stream, so that the next stages -- the next solve
 * included -- run while the copy is in flight.  Two snapshots alternate; a
 * snapshot is reused only after its previous copy has finished.  The copies
 * overlap other work only for page-locked (pinned) host buffers.  The host
 * buffers may be read only after tpsc_wait_copies(ctx, 0). */
int tpsc_get_self_async(tpsc_ctx *ctx, double *self_kw, double *sigma_inf2, double *sigma_inf3, double *sigma_inf4);
/* The full self-energy Sigma(k, i w_n) = Sigma_inf/z + C2/z^2 + C3/z^3 +
 * S/z^4, z = i (2n+1) pi T, n < Nw0/2, formed in FP64 on the device, rounded
 * to FP32 and copied out the same way ([Nw0/2][N8] complex float, interleaved
 * re, im); no counterpart in the reference.  Half the bytes of S over the
 * host link, for the mixed-precision form, whose bound (1e-6 of Sigma) it
 * keeps: each element moves by at most 6e-8 of itself.  (S itself cannot be
 * rounded: at low n its 1/z^4 term cancels against the others.) */
int tpsc_get_sigma32_async(tpsc_ctx *ctx, float *sigma_kw);
/* Waits for the copies of tpsc_get_self_async (join_stream = 0), or, with
 * join_stream = 1, makes the context stream wait for them without blocking
 * the host (work and events queued on the stream afterwards follow them). */
int tpsc_wait_copies(tpsc_ctx *ctx, int join_stream);

/* ---- real-frequency continuation (needs tpsc_find_mu) -------------------- */
/* Sigma(k, z) and A(k, z) = -Im 1/(z - eps_k + mu - Sigma(k, z)) / pi for every
 * octant k at the Nz complex energies z (interleaved re, im), from Sigma
 * sampled at z_j = i (2 n_idx[j] + 1) pi T, j < Nn (2 <= Nn <= 32), read at
 * the stored frequency j as green::MDC does (src/green.cpp:986-993).
 * mode 0: Vidberg-Serene continued-fraction Pade (generique::
 * pade_cont_frac_coef_rec and pade, src/generique.cpp:1605-1663);
 * mode 1: Lagrange polynomial through the Nn samples (src/green.cpp:887-897).
 * out_sigma [N8][Nz] complex (may be NULL), out_A [N8][Nz]. */
int tpsc_pade_sigma(tpsc_ctx *ctx, const int *n_idx, int Nn, const double *z, int Nz, int mode,
                    double *out_sigma, double *out_A);

/* green::Gwn_local (src/green.cpp:209-266): local G(i w_n), n < Nw0/2,
 * out [Nw0/2] complex interleaved. */
int tpsc_gwn_local(tpsc_ctx *ctx, double *out);

/* ---- current-current correlator (needs tpsc_find_mu) -------------------- */
/* cond_opt::calc_chijj_vertex_corr_all_optim(false, mmin, n_theta, NULL, 0),
 * the bubble + Maki-Thompson branch (src/cond_opt.cpp:2537-4286), on the
 * context's solve: chi_jj1(iq_n) (bubble) and chi_jj2(iq_n) (Maki-Thompson
 * vertex correction), n = 0..Nw0/2, the diamagnetic term kx0, and both
 * chi_jj resolved into n_theta >= 1 bins of the angle
 * theta_k = atan((L/2 - m)/(L/2 - kx index)) (N_theta_k of the reference).
 * Needs nk0 >= 8. */
int tpsc_chijj(tpsc_ctx *ctx, int n_theta);
/* Results of the last tpsc_chijj (any pointer may be NULL): chijj1, chijj2
 * [Nw0/2+1]; kx0 [1]; chijj1_k, chijj2_k [(Nw0/2+1) * n_theta] in the
 * reference's layout p + j * n_theta. */
int tpsc_get_chijj(tpsc_ctx *ctx, double *chijj1, double *chijj2, double *kx0, double *chijj1_k,
                   double *chijj2_k);

/* The Aslamazov-Larkin vertex correction chijj3(iq_n) -- the chi3 = true
 * branch of cond_opt::calc_chijj_vertex_corr_all_optim
 * (src/cond_opt.cpp:4292-6529) -- on the current grid after the self-energy
 * and mu, in FP64.  It is computed on the reference's non-uniform bosonic
 * grid of mmin (src/cond_opt.cpp:5123-5155): every n up to (Nw0/2)/2^mmin,
 * then mmin blocks of (Nw0/2)/2^(mmin+1) points whose spacing doubles; the
 * entry n = 0 is not computed and stays 0, as in the reference.  n_theta >= 1
 * angle bins as in tpsc_chijj; 0 <= mmin <= 24.  Each grid frequency costs
 * about one and a half tpsc_chijj. */
int tpsc_chijj3(tpsc_ctx *ctx, int mmin, int n_theta);
/* Results of the last tpsc_chijj3: *n_freq = N, the grid size; then, where the
 * pointer is not NULL (cap >= N is required for those), ind_freq [N] the
 * bosonic indices n of the grid, chijj3 [N] and chijj3_k [N * n_theta] in the
 * layout p + j * n_theta (row j for grid entry j). */
int tpsc_get_chijj3(tpsc_ctx *ctx, int cap, int *n_freq, int *ind_freq, double *chijj3, double *chijj3_k);

/* Optical conductivity on the bosonic Matsubara axis from the last tpsc_chijj
 * (no counterpart in the reference, which stops at chi_jj and kx0):
 * sigma(iq_n) = (-kx0 - chi_jj(iq_n)) / q_n, q_n = 2 pi n T, n = 1..nq, with
 * chi_jj = chijj1 + chijj2 (sigma, with vertex correction) and chi_jj =
 * chijj1 (sigma_bubble).  nq <= Nw0/2; either pointer may be NULL. */
int tpsc_sigma_iqn(tpsc_ctx *ctx, int nq, double *sigma, double *sigma_bubble);
/* Sensitivities of sigma(iq_n), n = 1..nq (with vertex correction, one angle
 * bin), and of the double occupancy D to {U, mu, t'} by central differences of
 * full FP64 Newton-form device solves with the steps h[3] (no counterpart in
 * the reference): dsigma[p * nq + n - 1] = d sigma(iq_n) / d theta_p, dD[p]
 * (may be NULL).  mu is the shift of mu0 at fixed n (tpsc_set_mu_shift), t'
 * moves at fixed n.  Six solves + tpsc_chijj, then the model, mu shift and
 * form are restored and the base point solved again.  The forward tangents
 * of the sum-rule stage (tpsc_sumrule_tangents) give dD exactly; the reverse
 * pass tpsc_sigma_iqn_bwd gives the sigma derivatives exactly and is checked
 * against this. */
int tpsc_sigma_iqn_fd(tpsc_ctx *ctx, int nq, const double h[3], double *dsigma, double dD[3]);
/* The backward pair of tpsc_sigma_iqn (no counterpart in the reference): for
 * the cotangent cot[n - 1] on sigma(iq_n), n = 1..nq (with vertex correction,
 * one angle bin), grad[p] = sum_n cot[n-1] d sigma(iq_n) / d theta_p,
 * theta = {U, mu, t'} as in tpsc_sigma_iqn_fd, by one reverse pass through
 * chi_jj, mu (an implicit root), Sigma and V in FP64 on the device, chained
 * with the forward tangents of chi0 and of the sum-rule roots
 * (tpsc_sumrule_tangents, which it runs).  dD (may be NULL) = d D / d theta.
 * Needs the self-energy and mu of the current grid (a solve); the point is
 * not re-solved. */
int tpsc_sigma_iqn_bwd(tpsc_ctx *ctx, int nq, const double *cot, double grad[3], double dD[3]);
/* Continued-fraction Pade continuation of sigma(iq_n), n = 1..Nn, and of
 * sigma_bubble to z = w + i eta for the Nw real frequencies w:
 * out [2][Nw] complex interleaved (sigma, then sigma_bubble). */
int tpsc_sigma_pade(tpsc_ctx *ctx, int Nn, const double *w, int Nw, double eta, double *out);
/* Batched continued-fraction Pade (the recursion of
 * generique::pade_cont_frac_coef_rec and generique::pade,
 * src/generique.cpp:1628-1663): nf functions sampled at x[f][j] with values
 * y[f][j] (j < Nn, 2 <= Nn <= 4096, complex interleaved) evaluated at the Nz
 * complex points z: out [nf][Nz] complex interleaved. */
int tpsc_pade_batch(tpsc_ctx *ctx, int nf, int Nn, const double *x, const double *y, int Nz, const double *z,
                    double *out);

/* Many points at once, by shape (no counterpart in the reference, which
 * solves one model at a time): the rows params[i] = {nk0, Nw0, n, T, tp, tpp,
 * t3, U} are grouped by (nk0, Nw0), and each group (up to 128 points) is
 * solved by ONE launch per stage of the Newton-form mixed-precision solve
 * over all its points -- every point's arrays in its own arena, its scalars
 * read on the device -- captured as one CUDA graph per group shape and size
 * and replayed on later calls.  results: npts rows of TPSC_S_COUNT scalars
 * (those of tpsc_solve in that form); status[i] per point (a failing point
 * gets NaN or its partial scalars and does not stop the others).  *ms (may
 * be NULL): host wall time of the solves, device idle at both ends.  The
 * context's own model and grids are not changed. */
int tpsc_solve_points(tpsc_ctx *ctx, int npts, const double *params, double *results, int *status, double *ms);
/* Streams tpsc_solve_points spreads its groups over (1..4, default 2), the
 * largest first onto the least loaded; each group's cooperative root searches
 * then take 2 blocks per SM / n. */
int tpsc_set_group_streams(tpsc_ctx *ctx, int n);

/* Device time of the last tpsc_solve per stage in ms:
 * {chi0, sum rules, vertex, self energy, traces + mu}, then of the last
 * tpsc_chijj: {h V / f0 V slices + end conditions, per-k tau kernel,
 * kx lines + final sums}; n <= 8. */
int tpsc_stage_times(tpsc_ctx *ctx, double *ms, int n);

/* ---- instrumentation (no counterpart in the reference) ------------------ */
/* The context's CUDA stream (a cudaStream_t), so callers can record timing
 * events on the stream the kernels run on. */
int tpsc_get_stream(tpsc_ctx *ctx, void **stream);

/* Re-launch the kernel(s) of one stage on the current grid's state,
 * asynchronously on the context stream (for timing and profiling):
 *  0 G(r,tau) slices   1 chi0 slices   2 chi0 tau transform
 *  3 V q-slices        4 V tau transform   5 Sigma slices
 *  6 Sigma tau transform  7 one spin sum-rule evaluation at Usp
 *  8 one Tr(G-G0) evaluation at mu   9 stages 1 and 2 back to back
 *  10 one Newton-form sum-rule evaluation at Usp (stored frequencies below
 *     the series cut)   11 one Newton-form Tr(G-G0) evaluation at mu
 *  12 the Newton-form sum-rule moments (per frequency, tail, suffix sums)
 *  13 the device Usp/Uch root search   14 the Sigma moment pass (Tr Sigma G0
 *     and the find_mu series)   15 stage 14 followed by the device mu search.
 * Requires a completed tpsc_solve.  Stages 2 and 4 transform in place and
 * expect stage 1 (resp. 3) to have run just before; launching the stages in
 * increasing order leaves the state as the solve left it. */
int tpsc_run_kernel(tpsc_ctx *ctx, int which);

/* Algorithmic HBM bytes of one launch of tpsc_run_kernel(which) on the current
 * grid: every distinct input read once plus every output written once. */
int tpsc_kernel_bytes(tpsc_ctx *ctx, int which, double *bytes);

/* Instrumentation: the device's FMA throughput (bits 64 or 32), TFLOP/s, by
 * a kernel of independent FMA chains on every SM -- the arithmetic ceiling of
 * the transform kernels' roofline beside the HBM copy bandwidth. */
int tpsc_fma_peak(int bits, double *tflops);
/* Check of the bounded grid barrier of the device root searches (no
 * counterpart in the reference): their barrier in a cooperative launch of
 * their grid (*blocks), where block `withhold` never arrives (negative: every
 * block does).  Every other block's wait then runs out after about a second,
 * sets the error flag and leaves, so the kernel ends and the context stays
 * usable.  *err_flag: the flag after the launch; *timed_out: blocks that left
 * with it; *ms: the kernel's time.  Returns TPSC_OK when the launch itself
 * ran (the flag reports the barrier). */
int tpsc_barrier_probe(tpsc_ctx *ctx, int withhold, int *err_flag, int *timed_out, int *blocks, double *ms);

/* Number of CUDA kernels the library has launched (all contexts) since it was
 * loaded. */
int tpsc_launch_count(tpsc_ctx *ctx, long long *count);

/* ---- allocation-free sum rule (no counterpart in the reference) ----------
 * The spin (channel 0) or charge (channel 1) sum-rule trace and its U
 * derivative, as tpsc_trace_diff_chi computes them, for callers that cannot
 * allocate device memory at the point of the call: code running inside a
 * memory pool or arena that owns the device memory, callbacks from a
 * framework that forbids allocation on its hot path, solver loops that must
 * not call cudaMalloc/cudaFree because they synchronise the device.  It
 * needs no context and allocates nothing: the caller passes device pointers
 * to chi0(q, iqn) in the reference's layout ([(Nw0/2+1) * N8], octant index
 * m + l(l+1)/2), chi0_inf and chi0_inf2 ([N8]) and out (2 doubles: trace,
 * d trace/dU), and the work runs asynchronously on `stream` (a cudaStream_t,
 * NULL for the default stream) of the current device.
 *
 * Its per-block partial sums live in a fixed device array of the library
 * (about 33 KB), which every GPU that loads the library holds until the
 * process exits.  That array bounds the lattice: nk0 up to 256 (N8 up to
 * 8385); larger lattices return TPSC_ERR_ARG.  The first call on each device
 * looks up the array's address with that device current; make that first
 * call before any stream capture.  All calls on a device share the array and
 * it keeps the last call's contents; calls whose work overlaps on the GPU
 * race on it, so order them (one stream, or events).  The address is looked
 * up once per device and kept for the life of the process: after a device
 * reset (cudaDeviceReset) the library's device image may load elsewhere, so
 * a process that resets a device must not call this entry point again. */
int tpsc_sumrule_noalloc(const double *chiqw, const double *chi0_inf, const double *chi0_inf2, int nk0, int Nw0,
                         double T, int channel, double Uv, double *out, void *stream);

/* ---------------------------------------------------------------------------
 * Batched sweep (no counterpart in the reference, which solves one parameter
 * point per run; tpsc_batch.cpp): many independent solves with uneven
 * lattices and Matsubara cutoffs on one GPU.  A batch owns nstreams solver
 * contexts (own streams, scratch and per-shape grid cache, kept across
 * calls) driven by one host thread each; the points of a call run largest
 * first (nk0^2 Nw0), each on the next free context, so that small solves
 * overlap on the GPU.  Not thread-safe: one call at a time per batch.
 * ------------------------------------------------------------------------- */
typedef struct tpsc_batch tpsc_batch;
/* 1 <= nstreams <= 32; NULL and *status set on failure. */
tpsc_batch *tpsc_batch_create(int device, int nstreams, int *status);
void tpsc_batch_destroy(tpsc_batch *b);
const char *tpsc_batch_last_error(const tpsc_batch *b);
int tpsc_batch_streams(const tpsc_batch *b, int *nstreams);
/* tpsc_set_graph_mode of every context of the batch (default 1); with 2,
 * each Newton-form point runs as one graph launch, the graph of its grid
 * updated in place for the point's model; with 3, a Newton + mixed sweep runs
 * by shape groups, one launch per stage over every point of a group, one
 * graph launch per group (tpsc_solve_points on the first context). */
int tpsc_batch_set_graph_mode(tpsc_batch *b, int mode);
/* params: npts rows {nk0, Nw0, n, T, tp, tpp, t3, U} (row-major doubles);
 * form: enum tpsc_form; results: npts rows of TPSC_S_COUNT scalars in the
 * tpsc_get_scalars order (NaN for a failed point); status[i]: point i's
 * status -- a failing point does not stop the others; ms (may be NULL): wall
 * time of the call from a device-idle start to a device-idle end.  Returns
 * TPSC_OK, or the status of the first failing point. */
int tpsc_batch_solve(tpsc_batch *b, int form, int npts, const double *params, double *results, int *status,
                     double *ms);
/* The tuner: one untimed pass of the sample (allocating every shape on
 * max_streams contexts), the tau transforms' tiling of every shape
 * (tpsc_tune_tau_tiles on its first good point), then the sample timed on 1,
 * 2, 4, ... <= max_streams contexts; later tpsc_batch_solve calls use the
 * fastest count.  ms (may be NULL) receives each count's time,
 * floor(log2(max_streams)) + 1 entries. */
int tpsc_batch_tune(tpsc_batch *b, int form, int npts, const double *params, int max_streams, double *ms);
/* The parameter-sweep workload: npts rows in the tpsc_batch_solve layout
 * from std::mt19937_64(seed), drawn per point in this order: nk0 uniform in
 * {32, 64, 128, 256}, U ~ U[1, 6], n ~ U[0.7, 1], log T ~ U[ln 0.03, ln 0.5],
 * t' ~ U[-0.3, 0]; t'' = t3 = 0 and Nw0 = 2 nextpow2(ceil(40 / (pi T))). */
int tpsc_sweep_points(int npts, unsigned long long seed, double *params);
/* chi::calc_corr_length (src/chi.cpp:931-981) on the batch's contexts: the
 * (n, T) grid dens[0]..dens[1] (nD points) x Temp[0]..Temp[1] (nT points),
 * point i = l nT + j at n = dens[0] + l dn, T = Temp[0] + j dT; per point the
 * two-grid find_Usp_Uch and sp_corr_length.  rows: nD nT rows of 19 values in
 * the corrLgth line's order {n, T, mu0, vF, Usp, difRelsp, Uch, difRelch,
 * dblOcc, xi_x, xi_y, xiAs_x, xiAs_y, xi0_x, xi0_y, nbq, qmax0, qmax1,
 * chi0max} -- the reference prints 0 in the two error columns (their
 * assignment is commented out, src/chi.cpp:361-362); here they are the
 * half-to-full-grid differences.  nsr > 0 fixes the sum rules' nsr for every
 * point (0: each point's own), mu_fs the Fermi surface's mu (NaN: each
 * point's mu0); the reference's own scan keeps both from its constructor.
 * A failing point has status != 0 and a row of NaN; returns the first
 * failure's status. */
int tpsc_batch_corr_length(tpsc_batch *b, int form, int nk0, int Nw0, double tp, double tpp, double t3, double U,
                           const double *dens, int nD, const double *Temp, int nT, double nsr, double mu_fs,
                           double *rows, int *status, double *ms);

/* ---- warm start from saved results ---------------------------------------
 * tpsc_set_self <- green::load_Self_bin / load_Self (src/green.cpp:1517-1541,
 * 1637-1670): self_kw [Nw0/2][N8] complex (the Self_kw_array layout) becomes
 * the current grid's S; sigma_inf2/3/4 [N8] and sigma_inf (one double)
 * replace the device's only when not NULL, as the reference's loaders leave
 * them.  find_mu, the traces and chi_jj then run on it. */
int tpsc_set_self(tpsc_ctx *ctx, const double *self_kw, const double *sigma_inf2, const double *sigma_inf3,
                  const double *sigma_inf4, const double *sigma_inf);
/* tpsc_set_chi0 <- chi0::loadChi0 (src/chi0.cpp:99-154): chiqw
 * [Nw0/2 + 1][N8] becomes the current grid's chi0(q, iqn); chi0max and qmax
 * are found again (TPSC_S_CHI0MAX, _QMAX0/1); the tail coefficients and
 * chi0(r, tau) stay those of the last chi0 stage. */
int tpsc_set_chi0(tpsc_ctx *ctx, const double *chiqw);
/* ---- the infinite lattice (spot checks of the finite-lattice results) ----
 * green0::find_mu_inf_syst (src/green0.cpp:265-287): mu0 of the infinite
 * lattice at the model's n and T; chi0::chiqw (src/chi0.cpp:211-276): chi0(q,
 * i w_n) of the infinite lattice at npts points qw[p] = (qx, qy, w_n) for the
 * chemical potential mu.  The reference integrates adaptively; here the
 * integrands, analytic and periodic at T > 0, are summed on L x L grids of
 * the zone (the trapezoid rule, exponentially convergent), L doubled from 128
 * until two sums agree to 1e-13; L_used (may be NULL) is the last L.  With
 * L > 0, tpsc_chi0_infinite sums that lattice only: chi0::chiqw_discret
 * (src/chi0.cpp:1587-1612) at nq0 = L. */
int tpsc_mu0_infinite(tpsc_ctx *ctx, double *mu, int *L_used);
int tpsc_chi0_infinite(tpsc_ctx *ctx, double mu, int npts, const double *qw, int L, double *out, int *L_used);
/* Sigma(k, tau_j) [N8], 0 <= j <= Nw0, of the last Sigma stage: the spline
 * nodes of green::calc_Self_FFT_spline (src/green.cpp:1872-1950). */
int tpsc_get_sigma_tau(tpsc_ctx *ctx, int j, double *out);

/* ---- the reference's on-disk formats (host only; no context) -------------
 * Names: the reference's sprintf formats, written into out[cap]. */
enum tpsc_file_kind {
    TPSC_FILE_CHI0_BIN = 0,   /* chi0_<tp>_<tpp>_<t3>_<n>_<T>_<nk0>_<nbw>.dat (src/chi0.cpp:63) */
    TPSC_FILE_SELF_BIN = 1,   /* self_bin_<U>_..._<nk0>_<nbw>.dat (src/green.cpp:1507) */
    TPSC_FILE_SELF_ASCII = 2, /* self_tpsc_<U>_..._<nk0>_<nbw>.dat (src/green.cpp:1557) */
    TPSC_FILE_GREEN = 3       /* Green_<U>_..._<nk0>_<nbw>_<l>_<m>.dat (src/green.cpp:1606) */
};
int tpsc_file_name(int kind, char *out, int cap, double U, double tp, double tpp, double t3, double n, double T,
                   int nk0, int nbw, int l, int m);
/* chi0::save_chi / loadChi0 (src/chi0.cpp:61-154): int nbq, int nwmax, then
 * nwmax + 1 frames of N8 = nbq (nbq + 1) / 2 doubles.  The reader returns the
 * header and, when chiqw is not NULL, the frames (cap doubles available). */
int tpsc_write_chi0_bin(const char *path, int nbq, int nwmax, const double *chiqw);
int tpsc_read_chi0_bin(const char *path, int *nbq, int *nwmax, double *chiqw, long long cap);
/* green::save_Self_bin / load_Self_bin (src/green.cpp:1496-1541): nbw/2 + 1
 * frames of N8 complex.  The first nbw/2 are S; the last is what the
 * reference's Sigma stage leaves there, (Sigma(k, beta/2), 0) -- pass it as
 * last [N8] complex (tpsc_get_sigma_tau(ctx, nbw/2, ...)), or NULL for zeros.
 * The reader fills all nbw/2 + 1 frames. */
int tpsc_write_self_bin(const char *path, int nbk, int nbw, const double *self_kw, const double *last);
int tpsc_read_self_bin(const char *path, int nbk, int nbw, double *self_kw);
/* green::save_Self / load_Self (src/green.cpp:1544-1574, 1637-1670): ascii,
 * "n l m Re Im" per line; nfreq frames (0 or > nbw/2: all nbw/2). */
int tpsc_write_self_ascii(const char *path, int nbk, int nbw, int nfreq, const double *self_kw);
int tpsc_read_self_ascii(const char *path, int nbk, int nbw, double *self_kw);
/* green::save_Green (src/green.cpp:1577-1633) at one k: G(i w_n) =
 * 1 / (z - ek_mu - Sigma(z)), Sigma = sigma_inf/z + s2/z^2 + s3/z^3 + S/z^4,
 * S read at self_col[2 stride j] (complex stride), n < nbw/2. */
int tpsc_write_green_ascii(const char *path, int nbw, double T, double ek_mu, double sigma_inf, double s2, double s3,
                           const double *self_col, long long stride);

#ifdef __cplusplus
}
#endif

#endif /* TPSC_B200_H */
