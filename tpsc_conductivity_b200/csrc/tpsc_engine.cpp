// tpsc_engine.cpp -- host side of the C ABI (include/tpsc_b200.h).
//
// Owns the device arrays of each (nk0, Nw0) grid, builds the lattice and FFT
// tables, sequences the kernels of tpsc_kernels.cu on one CUDA stream and
// runs the root searches of the reference (generique::find_zero) with every
// function evaluation a device reduction.  Only scalars cross PCIe during a
// solve.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <initializer_list>
#include <limits>
#include <map>
#include <string>
#include <utility>
#include <vector>

#include "../../include/tpsc_b200.h"
#include "tpsc_host.h"
#include "tpsc_kernels.cuh"

using namespace tpsc;

namespace {

const double PI = std::acos(-1.0);
const double EPS = std::numeric_limits<double>::epsilon();

// ---------------------------------------------------------------------------
// Root search with the control flow of generique::find_zero: bracketing
// inverse-quadratic interpolation with secant and bisection fallbacks, tol
// 1e-16 and 20 iterations (src/generique.cpp:604-913); with lims, the bounded
// variant: tol 1e-15, 12 iterations, eps = 2 machine epsilons
// (src/generique.cpp:917-1234).  The evaluator returns false on a device
// error, which aborts the search.
// ---------------------------------------------------------------------------
template <typename F>
bool find_zero(F &&func, const double init[3], double *root, const double *lims, int *nev, bool *dev_err) {
    double tol, eps;
    int itmax;
    if (!lims) {
        tol = 1.0e-16;
        eps = 10.0 * EPS;
        itmax = 20;
    } else {
        tol = 1.0e-15;
        eps = 2.0 * EPS;
        itmax = 12;
    }
    *nev = 0;
    *dev_err = false;
    auto f = [&](double x, double &y) -> bool {
        ++*nev;
        if (!func(x, y)) {
            *dev_err = true;
            return false;
        }
        return true;
    };
    int nbiter = 0;
    const double dytol = 0.01;
    double x0 = init[0], xmin = init[1], xmax = init[2];
    double ymin, ymax;
    if (!f(xmin, ymin) || !f(xmax, ymax)) return false;
    double x[3] = {x0, xmin, xmax}, y[3] = {0.0, ymin, ymax};
    if (std::fabs(ymin) < tol) {
        *root = xmin;
        return true;
    }
    if (std::fabs(ymax) < tol) {
        *root = xmax;
        return true;
    }
    if (ymin * ymax > 0) {
        if (!f(x[0], y[0])) return false;
        if (std::fabs(y[0]) < tol) {
            *root = x[0];
            return true;
        }
        if (y[0] * y[2] < 0) {
            const double xt = x[0];
            x[0] = (x[0] + x[2]) / 2;
            x[1] = xt;
            y[1] = y[0];
        } else {
            double ytmp = y[0], xtmp = x[0], xtmp1, ytmp1;
            if (std::fabs(y[1]) < std::fabs(ytmp)) ytmp = y[1], xtmp = x[1];
            if (std::fabs(y[2]) < std::fabs(ytmp)) ytmp = y[2], xtmp = x[2];
            xtmp1 = xtmp + 10 * eps;
            if (!f(xtmp1, ytmp1)) return false;
            xtmp1 = xtmp - ytmp * ((xtmp1 - xtmp) / (ytmp1 - ytmp));
            if (!f(xtmp1, ytmp1)) return false;
            nbiter++;
            while (std::fabs(ytmp1) > tol && nbiter < itmax && ytmp1 * ytmp > 0 && std::isfinite(xtmp1)) {
                xtmp = xtmp1;
                ytmp = ytmp1;
                xtmp1 = xtmp + 10 * eps;
                if (!f(xtmp1, ytmp1)) return false;
                xtmp1 = xtmp - ytmp * ((xtmp1 - xtmp) / (ytmp1 - ytmp));
                if (!f(xtmp1, ytmp1)) return false;
                nbiter++;
            }
            if (std::fabs(ytmp1) < tol) {
                *root = xtmp1;
                return true;
            }
            if (ytmp1 * ytmp < 0) {
                x[0] = (xtmp + xtmp1) / 2;
                x[1] = xtmp;
                y[1] = ytmp;
                x[2] = xtmp1;
                y[2] = ytmp1;
            }
            if (nbiter >= itmax) return false;
            if (!std::isfinite(xtmp1)) return false;
        }
    }
    if (lims) {
        if (x[1] < lims[0] || x[1] > lims[1] || x[2] < lims[0] || x[2] > lims[1]) return false;
    }
    if (std::fabs(xmax - xmin) < eps) {
        *root = xmin;
        return true;
    }
    if (!f(x[0], y[0])) return false;
    if (std::fabs(y[0]) < tol) {
        *root = x[0];
        return true;
    }
    int ind1, ind2, ind3, indm = 0, indp = 0, indfar, indmid;
    auto classify = [&]() {
        if (y[0] * y[1] > 0)
            ind1 = 0, ind2 = 1;
        else if (y[0] * y[2] > 0)
            ind1 = 0, ind2 = 2;
        else
            ind1 = 1, ind2 = 2;
        ind3 = 3 - ind1 - ind2;
        if (x[ind3] > x[ind1]) {
            if (x[ind1] > x[ind2])
                indfar = ind2, indmid = ind1;
            else
                indfar = ind1, indmid = ind2;
            indm = indmid, indp = ind3;
        } else {
            if (x[ind1] < x[ind2])
                indfar = ind2, indmid = ind1;
            else
                indfar = ind1, indmid = ind2;
            indm = ind3, indp = indmid;
        }
    };
    classify();
    x[indfar] = -y[indmid] * (x[ind3] - x[indmid]) / (y[ind3] - y[indmid]) + x[indmid];
    if (!f(x[indfar], y[indfar])) return false;
    double dy = y[indfar], dyprec;
    double a = 0.0, b = 0.0, c = 0.0;
    while (std::fabs(dy) > tol && nbiter < itmax) {
        classify();
        const double denom = -x[0] * x[0] * x[2] + x[0] * x[0] * x[1] - x[0] * x[1] * x[1] + x[0] * x[2] * x[2] -
                             x[2] * x[2] * x[1] + x[2] * x[1] * x[1];
        if (std::fabs(denom) > 0.0) {
            a = (x[0] * y[2] - x[0] * y[1] + x[2] * y[1] - y[2] * x[1] - y[0] * x[2] + y[0] * x[1]) / denom;
            b = -(-y[2] * x[1] * x[1] + x[1] * x[1] * y[0] - x[2] * x[2] * y[0] - y[1] * x[0] * x[0] +
                  y[2] * x[0] * x[0] + y[1] * x[2] * x[2]) /
                denom;
            c = (y[2] * x[0] * x[0] * x[1] - y[1] * x[0] * x[0] * x[2] - x[1] * x[1] * x[0] * y[2] +
                 x[2] * x[2] * x[0] * y[1] + x[1] * x[1] * y[0] * x[2] - x[2] * x[2] * y[0] * x[1]) /
                denom;
        }
        if ((b * b - 4.0 * a * c) > 0.0 && std::fabs(denom) > 0.0) {
            const double sq = std::sqrt(b * b - 4.0 * a * c);
            const double xp = (-b + sq) / (2 * a), xm = (-b - sq) / (2 * a);
            if (xp > x[indm] && xp < x[indp])
                x[indfar] = xp;
            else if (xm > x[indm] && xm < x[indp])
                x[indfar] = xm;
            else if (std::fabs(y[ind3] - y[indmid]) > tol)
                x[indfar] = -y[indmid] * (x[ind3] - x[indmid]) / (y[ind3] - y[indmid]) + x[indmid];
            else {
                *root = x[indmid];
                return true;
            }
        } else {
            if (std::fabs(y[ind3] - y[indmid]) > tol)
                x[indfar] = -y[indmid] * (x[ind3] - x[indmid]) / (y[ind3] - y[indmid]) + x[indmid];
            else {
                *root = x[indmid];
                return true;
            }
        }
        if (!f(x[indfar], y[indfar])) return false;
        dyprec = std::fabs(dy);
        dy = y[indfar];
        if (std::fabs(dyprec - std::fabs(dy)) < dytol * dyprec || dyprec < std::fabs(dy)) {
            x[indfar] = (x[ind3] + x[indmid]) / 2.0;
            if (!f(x[indfar], y[indfar])) return false;
            dy = y[indfar];
        }
        nbiter++;
    }
    int best = 0;
    *root = x[0];
    if (std::fabs(y[1]) < std::fabs(y[best])) {
        *root = x[1];
        best = 1;
    }
    if (std::fabs(y[2]) < std::fabs(y[best])) *root = x[2];
    return true;
}

// ---------------------------------------------------------------------------
// Safeguarded Newton root search for the Newton form: f returns the value and
// the derivative (from the same device pass).  [lo, hi] is the reference's
// search interval; it shrinks to the side of each evaluation that the
// derivative's sign and the value's sign rule out, and a Newton step that
// leaves it is replaced by the midpoint.  Converged when |f| is below tol,
// when the step is below 1e-14 relative, or when the step stops shrinking
// (at most half the previous one) while already below 1e-10 relative: f is
// then at its rounding-noise floor and further steps only dither.
// ---------------------------------------------------------------------------
template <typename F>
bool newton_root(F &&func, double x0, double lo, double hi, double tol, double *root, int *nev, bool *dev_err) {
    *nev = 0;
    *dev_err = false;
    // the start must lie strictly inside the interval (the spin sum rule has
    // its pole at the upper end: U/2 can lie beyond it)
    double x = (x0 > lo && x0 < hi) ? x0 : 0.5 * (lo + hi), prev_step = 0.0;
    for (int it = 0; it < 60; ++it) {
        double y, dy;
        ++*nev;
        if (!func(x, y, dy)) {
            *dev_err = true;
            return false;
        }
        if (!std::isfinite(y) || !std::isfinite(dy)) return false;
        if (std::fabs(y) < tol) {
            *root = x;
            return true;
        }
        // the root lies on the side where f changes sign
        if ((y > 0) == (dy > 0))
            hi = std::min(hi, x);
        else
            lo = std::max(lo, x);
        const double scale = std::max(1.0, std::fabs(x));
        double xn = (dy != 0.0) ? x - y / dy : 0.5 * (lo + hi);
        // convergence is judged on the Newton step itself, before the bracket
        // safeguard: at the root the step rounds to (or next to) x, which may
        // coincide with the bracket end just moved to x
        if (dy != 0.0 && std::fabs(xn - x) <= 1e-14 * scale) {
            *root = xn;
            return true;
        }
        if (!(xn >= lo && xn <= hi)) xn = 0.5 * (lo + hi);
        const double step = std::fabs(xn - x);
        if (it >= 2 && step < 1e-10 * scale && step > 0.5 * prev_step) {
            *root = xn;
            return true;
        }
        prev_step = step;
        x = xn;
    }
    return false;
}

// ---------------------------------------------------------------------------
// one (nk0, Nw0) grid: tables and arrays
// ---------------------------------------------------------------------------
// What a Newton-form solve's launches take beyond the grid's buffers: the
// key of a captured solve graph (tpsc_set_graph_mode)
struct SolveKey {
    int form = -1, cap = -1;
    long long model_id = -1;
    double mu0 = 0.0, nsr = -1.0;
    long long tiles = -1;  // tau_tiles_version(): the tau transforms' tiling
    bool rsr = true, rmu = true;
    bool operator==(const SolveKey &o) const {
        return form == o.form && cap == o.cap && model_id == o.model_id && mu0 == o.mu0 && nsr == o.nsr &&
               tiles == o.tiles && rsr == o.rsr && rmu == o.rmu;
    }
};

struct Grid {
    GridDev d;
    cudaStream_t st = nullptr;    // the owning context's stream: every fill and upload is ordered on it
    std::vector<double> ek_host;  // [nbk * nbk], ek[m + l*nbk]
    double mu0 = 0.0;
    double *Grt = nullptr;        // [(Nw0+1) * n8]      G(r, tau_j)
    float *Grt32 = nullptr;       // [(Nw0+1) * n8]      G(r, tau_j) in FP32 (mixed form; allocated on first use)
    double *chirt = nullptr;      // blocked nb          chi0(r, tau_j)
    double *chiq = nullptr;       // blocked nb          chi0(q, tau_j) -> chi0(q, iqn)
    double *dG0p = nullptr, *dchirt0 = nullptr, *dchiqt0 = nullptr;  // [n8]
    double *cinf = nullptr, *cinf2 = nullptr;                        // [n8]
    double *V = nullptr;          // blocked nb          V(r, iqn) -> V(r, tau_j)
    double *dS = nullptr;         // [2 n8p]             Sigma'(k, 0), Sigma'(k, beta)
    double *sigt = nullptr;       // blocked Nw0+1       Sigma(k, tau_j)
    double2 *S = nullptr;         // blocked Nw0/2       coefficient of 1/z^4
    double *s2 = nullptr, *s3 = nullptr, *s4 = nullptr, *sinf = nullptr;
    bool have_chi0 = false, have_V = false, have_S = false;
    bool have_U = false;  // Usp, Uch found from this grid's chi0
    bool g_mixed = false;         // G(r, tau) of the last chi0 stage is Grt32
    long long model_id = -1;      // the model (tpsc_set_model call) the eps_k tables and mu0 belong to
    // Newton form: moments of chi0 for the high-frequency sum-rule series
    double *mom = nullptr, *cmax = nullptr;  // device [nb][kMomP], [nb]
    bool have_mom = false;
    bool have_mom_host = false;              // the host copies below are current
    std::vector<double> mom_suf;             // [(nb + 1) kMomP] sums over frequencies >= j
    std::vector<double> cmax_suf;            // [nb + 1] max |chi| over frequencies >= j
    double tail_mom[kMomP] = {0};            // the same moments of the Matsubara tail n > Nw0/2
    double tail_max = 0.0;                   // max |chi| over the tail
    double *d_mom_suf = nullptr, *d_cmax_suf = nullptr, *d_tailm = nullptr;  // on the device
    // forward tangents (tpsc_sumrule_tangents; allocated on first use)
    // (the two directions' dG(r, tau), dchi0(q, iqn) and end tables are kept
    // in adj for the reverse pass)
    double *t_ddq0 = nullptr, *t_dcinf = nullptr, *t_dcinf2 = nullptr;
    double *t_der = nullptr;
    double2 *t_fd = nullptr;
    double t_dmu0_tp = 0.0;   // d mu0 / d t' at fixed density of the last tangents
    // the reverse pass of sigma(iq_n) (tpsc_sigma_iqn_bwd; allocated on first use)
    AdjDev adj;
    bool adj_alloc = false;
    double tailq_T = -1.0;         // temperature the tail power sums were built for
    double tailq_host[kTailQ] = {0};
    double tailP_host[kTailP] = {0};
    std::vector<void *> allocs;
    unsigned warm_forms = 0;  // bit f: a direct (uncaptured) Newton solve in form f ran on this grid
    // the Newton-form solve on this grid as an executable CUDA graph, the key
    // it was captured with and the kernels in it
    cudaGraphExec_t graph_exec = nullptr;
    SolveKey graph_key;
    long long graph_kernels = 0;
    // current-current correlator: device state (allocated on first use) and
    // the last result, [n_theta 2 NB] binned, [2 NB] totals, kx0
    CondDev cond;
    bool cond_alloc = false;
    size_t cond_part_cap = 0, cond_out_cap = 0;  // doubles in cond.partial, cond.out
    std::vector<double> cond_host;
    int cond_bins = 0;                            // n_theta of cond_host (0: none yet)
    // Aslamazov-Larkin correction: device state (allocated on first use) and
    // the last result, [N (1 + n_theta)] on the grid al_ind
    AlDev al;
    bool al_alloc = false;
    size_t al_out_cap = 0;                        // doubles in al.out
    std::vector<double> al_host;
    std::vector<int> al_ind;
    int al_bins = 0;                              // n_theta of al_host (0: none yet)
};

// The points of one shape (nk0, Nw0) of a batched sweep, solved together:
// every point's arrays live in its own arena (see Bp), point p's at
// base + p * arena, and each stage of the Newton-form mixed solve is one
// launch over all of them.  The group's solve -- upload of the points' tables
// and scalars, the launches, the readback -- is one CUDA graph, replayed
// while the group's point count stays the same.
struct Group {
    int nk0 = 0, nw0 = 0, cap = 0;  // cap: points the arenas are allocated for
    GridDev d;                      // the shape's tables; ek, er, gk, tailq, tailP of point 0
    char *base = nullptr;           // cap * arena bytes
    long long arena = 0;
    size_t in_bytes = 0;            // the per-point inputs at arena offset 0: ek, er, tailq, tailP, scalars
    size_t res_off = 0;             // the results block: kGroupRes doubles
    double *pp = nullptr;           // point 0's scalars [kPP]
    float *Grt32 = nullptr;
    double *chirt = nullptr, *chiq = nullptr, *V = nullptr, *sigt = nullptr, *dS = nullptr;
    double *dG0p = nullptr, *dchirt0 = nullptr, *dchiqt0 = nullptr, *cinf = nullptr, *cinf2 = nullptr;
    double2 *S = nullptr;
    double *s2 = nullptr, *s3 = nullptr, *s4 = nullptr, *sinf = nullptr;
    double *mom = nullptr, *cmax = nullptr, *msuf = nullptr, *csuf = nullptr, *tailm = nullptr;
    double *dres = nullptr, *mu_out = nullptr;
    Reduce red, redm, mu0r;
    RootScratch roots;
    char *h_in = nullptr;    // pinned, cap * in_bytes
    double *h_res = nullptr; // pinned, cap * kGroupRes
    cudaGraphExec_t gexec = nullptr;
    int gexec_P = 0;
    long long gexec_tiles = -1;  // tau_tiles_version() the graph was captured with
};
// results block of a point (doubles): [0, 3) chi0max, qmax; [8, 14) the
// sum-rule roots; [16, 20) the root searches' barrier words; [20, 24) the mu
// search; [28] Sigma_inf; [32, 64) the moment sums (Tr Sigma G0 at 32, 33)
constexpr int kGroupRes = 64;

}  // namespace

struct tpsc_ctx {
    int device = 0;
    int form = TPSC_FORM_REFERENCE;
    cudaStream_t st = nullptr;
    cudaStream_t st2 = nullptr;   // side stream: the single-CTA boundary transforms, overlapped with the slices
    cudaEvent_t evf[4] = {};      // fork / join events of the side stream
    Reduce red;
    Reduce redm;              // moment sums: partial [(2 kMomP + 1) kMaxBlocks], result [32]
    RootScratch roots;        // the device root searches' state
    // device results the later stages read without a host round trip:
    // [0..5] Usp, Uch, evals_sp, evals_ch, ok_sp, ok_ch (the vertex reads [0..1])
    double *dres = nullptr;
    double *h_res = nullptr;  // pinned and mapped, 32 doubles
    unsigned *h_res_dev = nullptr;  // its device address: the readback kernel writes there
    // model
    bool have_model = false;
    long long model_id = 0;   // incremented by every tpsc_set_model
    int nk0 = 0, Nw0 = 0;
    double n = 0, T = 0, tp = 0, tpp = 0, t3 = 0, U = 0, nsr = 0;
    double Usp = 0, Uch = 0;
    double mu_shift = 0;  // added to the density root mu0 (tpsc_set_mu_shift)
    std::map<std::pair<int, int>, Grid *> grids;
    Grid *cur = nullptr;
    double scal[TPSC_S_COUNT] = {0};
    double stage_ms[8] = {0};
    cudaEvent_t ev[6] = {};
    void *stage = nullptr;
    size_t stage_bytes = 0;
    // tpsc_get_self_async: two device snapshots of Sigma, copied out on cst
    cudaStream_t cst = nullptr;
    cudaEvent_t snap_ev[2] = {}, copy_ev[2] = {};
    void *snap[2] = {nullptr, nullptr};
    size_t snap_bytes[2] = {0, 0};
    int snap_next = 0;
    bool copies_pending = false;
    // Newton-form solves as CUDA graphs (tpsc_set_graph_mode; the executable
    // graphs live in the grids)
    int graph_mode = 1;       // 0 off, 1 replay a repeated solve, 2 capture every solve
    bool graph_off = false;   // a capture failed: direct launches from then on
    bool capturing = false;
    const void *seen_grid = nullptr;
    SolveKey seen_key;        // of the last direct solve
    long long graph_kernels = 0;  // in the graph of the last captured or replayed solve
    long long graph_replays = 0, graph_captures = 0;
    std::map<std::pair<int, int>, Group *> groups;  // tpsc_solve_points' shape groups
    int group_streams = 2;                          // streams the groups are spread over (1..4)
    cudaStream_t gst[2] = {nullptr, nullptr};       // the third and fourth (st, st2 are the first two)
    std::string err;
};

namespace {

std::string g_static_err;

int fail(tpsc_ctx *c, int code, const std::string &msg) {
    if (c)
        c->err = msg;
    else
        g_static_err = msg;
    return code;
}

int cuda_fail(tpsc_ctx *c, cudaError_t e, const char *where) {
    return fail(c, e == cudaErrorMemoryAllocation ? TPSC_ERR_OOM : TPSC_ERR_CUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                  \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call);  \
    } while (0)

template <typename T>
cudaError_t dalloc(Grid *g, T **p, size_t count) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) + 16);
    if (e != cudaSuccess) return e;
    g->allocs.push_back(q);
    *p = static_cast<T *>(q);
    // on the context's (non-blocking) stream, so that the kernels queued there
    // after it see the zeros: a legacy-stream memset is not ordered with them
    return cudaMemsetAsync(q, 0, count * sizeof(T) + 16, g->st);
}

void free_group(Group *q) {
    if (q->gexec) cudaGraphExecDestroy(q->gexec);
    if (q->base) cudaFree(q->base);
    if (q->h_in) cudaFreeHost(q->h_in);
    if (q->h_res) cudaFreeHost(q->h_res);
    delete q;
}

void free_grid(Grid *g) {
    if (g->graph_exec) cudaGraphExecDestroy(g->graph_exec);
    for (void *p : g->allocs) cudaFree(p);
    if (g->cond.partial) cudaFree(g->cond.partial);
    if (g->cond.out) cudaFree(g->cond.out);
    if (g->al.out) cudaFree(g->al.out);
    delete g;
}

// eps_k = -2(cx + cy) - 4 t' cx cy - 2 t''(c2x + c2y) - 4 t3 (c2x cy + c2y cx) on
// k = l pi/(nbk-1) (hamiltonien::calc_ek / dispk, src/hamiltonien.cpp:358-375, 428-431)
double dispk(double kx, double ky, double tp, double tpp, double t3) {
    return -2.0 * (std::cos(kx) + std::cos(ky)) - 4.0 * tp * std::cos(kx) * std::cos(ky) -
           2.0 * tpp * (std::cos(2 * kx) + std::cos(2 * ky)) -
           4 * t3 * (std::cos(2 * kx) * std::cos(ky) + std::cos(2 * ky) * std::cos(kx));
}

// d eps/d kx and d2 eps/d kx2 (hamiltonien::grad_ek direction 0 and
// Hessian_ek (0, 0), src/hamiltonien.cpp:134-155)
double grad_ek_x(double kx, double ky, double tp, double tpp, double t3) {
    return 2.0 * std::sin(kx) + 4.0 * tp * std::sin(kx) * std::cos(ky) + 4.0 * tpp * std::sin(2 * kx) +
           4 * t3 * (2.0 * std::sin(2 * kx) * std::cos(ky) + std::cos(2 * ky) * std::sin(kx));
}
double hessian_ek_xx(double kx, double ky, double tp, double tpp, double t3) {
    return 2.0 * std::cos(kx) + 4.0 * tp * std::cos(kx) * std::cos(ky) + 8.0 * tpp * std::cos(2 * kx) +
           4 * t3 * (4.0 * std::cos(2 * kx) * std::cos(ky) + std::cos(2 * ky) * std::cos(kx));
}

// Thomas-algorithm tables of the clamped-spline system with NJ nodes:
// invp[i] = 1/pivot_i, cp[i] = superdiagonal / pivot (cp[NJ-1] = 0).
bool spline_tables(int NJ, std::vector<double> &out) {
    out.assign(2 * NJ, 0.0);
    const int N = NJ - 1;
    long double cpv = 0.0L;
    for (int i = 0; i <= N; ++i) {
        long double p;
        if (i == 0)
            p = 2.0L;
        else if (i < N)
            p = 4.0L - cpv;
        else
            p = 2.0L - cpv;
        out[i] = (double)(1.0L / p);
        cpv = (i < N) ? 1.0L / p : 0.0L;
        out[NJ + i] = (double)cpv;
    }
    // the device sweeps take rows kSplinePivotConst..N-1 as one constant: the
    // pivots converge to 2 + sqrt(3) within ~15 rows, so this always holds
    for (int i = kSplinePivotConst; i < N; ++i)
        if (out[i] != out[kSplinePivotConst] || out[NJ + i] != out[kSplinePivotConst]) return false;
    return true;
}

void twiddles(int N, long double sign, long double scale, std::vector<double2> &out) {
    out.resize(N);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < N; ++m) {
        const long double a = sign * scale * pi * m / N;
        out[m] = make_double2((double)cosl(a), (double)sinl(a));
    }
}

// FP32 twiddles exp(-2 pi i m / N) as (cos_hi, sin_hi, cos_lo, sin_lo):
// hi = float(x), lo = float(x - hi), from long double
void twiddles32(int N, std::vector<float4> &out) {
    out.resize(N);
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int m = 0; m < N; ++m) {
        const long double a = -2.0L * pi * m / N;
        const long double c = cosl(a), s = sinl(a);
        const float ch = (float)c, sh = (float)s;
        out[m] = make_float4(ch, sh, (float)(c - ch), (float)(s - sh));
    }
}

template <typename T>
cudaError_t upload(Grid *g, T **dst, const std::vector<T> &src) {
    cudaError_t e = dalloc(g, dst, src.size());
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, g->st);
}

int build_grid(tpsc_ctx *ctx, int nk0, int nw0, Grid **out) {
    auto key = std::make_pair(nk0, nw0);
    auto it = ctx->grids.find(key);
    if (it != ctx->grids.end()) {
        *out = it->second;
        return TPSC_OK;
    }
    if (!supported_grid(nk0, nw0))
        return fail(ctx, TPSC_ERR_ARG, "unsupported grid nk0=" + std::to_string(nk0) +
                                           " Nw0=" + std::to_string(nw0) +
                                           " (nk0 in {8,16,32,64,128,256}, Nw0 power of two in [16, 4096])");
    Grid *g = new Grid;
    g->st = ctx->st;
    GridDev &d = g->d;
    d.nk0 = nk0;
    d.nbk = nk0 / 2 + 1;
    d.n8 = d.nbk * (d.nbk + 1) / 2;
    d.n8p = (d.n8 + 3) & ~3;
    d.nw0 = nw0;
    d.nb = nw0 / 2 + 1;
    std::vector<double> w16(d.n8p, 0.0);
    for (int l = 0; l < d.nbk; ++l)
        for (int m = 0; m <= l; ++m) {
            // multiplicity of octant point (l, m): 16 halved on the l edges, the m
            // edges and the diagonal (src/chi.cpp:755-759)
            int w = 16;
            if (l == 0 || l == d.nbk - 1) w /= 2;
            if (m == 0 || m == d.nbk - 1) w /= 2;
            if (m == l) w /= 2;
            w16[m + l * (l + 1) / 2] = w;
        }
    std::vector<double2> twk, tww, htw;
    std::vector<float4> twk32;
    twiddles32(nk0, twk32);
    twiddles(nk0, -2.0L, 1.0L, twk);
    twiddles(nw0, -2.0L, 1.0L, tww);
    twiddles(nw0, 1.0L, 1.0L, htw);
    std::vector<double> sh, sf;
    if (!spline_tables(d.nb, sh) || !spline_tables(nw0 + 1, sf)) {
        delete g;
        return fail(ctx, TPSC_ERR_ARG, "spline pivot tables are not constant from the interior row on");
    }
    cudaError_t e = cudaSuccess;
    const size_t n8 = d.n8, n8p = d.n8p, nb = d.nb, nw = nw0;
#define A(x)                                       \
    if (e == cudaSuccess) {                        \
        e = (x);                                   \
    }
    A(upload(g, &d.w16, w16));
    A(upload(g, &d.tw_k, twk));
    A(upload(g, &d.tw_k32, twk32));
    std::vector<float> dct;
    dct_table(d.nbk, dct);
    if (!dct.empty()) A(upload(g, &d.dct32, dct));
    dct_tc_table(d.nbk, dct);
    if (!dct.empty()) A(upload(g, &d.dct_tc, dct));
    A(upload(g, &d.tw_w, tww));
    A(upload(g, &d.ht_w, htw));
    A(upload(g, &d.spl_half, sh));
    A(upload(g, &d.spl_full, sf));
    A(dalloc(g, &d.ek, n8));
    A(dalloc(g, &d.gk, n8));
    A(dalloc(g, &d.tailq, (size_t)kTailQ));
    A(dalloc(g, &d.tailP, (size_t)kTailP));
    A(dalloc(g, &d.er, n8));
    A(dalloc(g, &g->Grt, (nw + 1) * n8));
    A(dalloc(g, &g->chirt, nb * n8p));
    A(dalloc(g, &g->chiq, nb * n8p));
    A(dalloc(g, &g->dG0p, n8));
    A(dalloc(g, &g->dchirt0, n8));
    A(dalloc(g, &g->dchiqt0, n8));
    A(dalloc(g, &g->cinf, n8));
    A(dalloc(g, &g->cinf2, n8));
    A(dalloc(g, &g->V, nb * n8p));
    A(dalloc(g, &g->dS, 2 * n8p));
    A(dalloc(g, &g->sigt, (nw + 1) * n8p));
    A(dalloc(g, &g->S, (nw / 2) * n8p));
    A(dalloc(g, &g->s2, n8));
    A(dalloc(g, &g->s3, n8));
    A(dalloc(g, &g->s4, n8));
    A(dalloc(g, &g->sinf, 1));
    A(dalloc(g, &g->mom, nb * kMomP));
    A(dalloc(g, &g->cmax, nb));
    A(dalloc(g, &g->d_mom_suf, (nb + 1) * kMomP));
    A(dalloc(g, &g->d_cmax_suf, nb + 1));
    A(dalloc(g, &g->d_tailm, (size_t)kMomP + 1));
#undef A
    // the host tables above are released on return
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    if (e != cudaSuccess) {
        free_grid(g);
        return cuda_fail(ctx, e, "grid allocation");
    }
    ctx->grids[key] = g;
    *out = g;
    return TPSC_OK;
}

// Small device ranges (bytes a multiple of 4) copied into ctx->h_res at the
// given double offsets by one kernel on ctx->st, then a wait on ctx->st.  The
// kernel writes the mapped pinned buffer directly, so the readback takes no
// copy engine and never waits behind a Sigma copy-out queued on ctx->cst.
struct Piece {
    const void *src;
    size_t bytes;
    int at;  // offset in ctx->h_res, doubles
};
int queue_read_back(tpsc_ctx *ctx, std::initializer_list<Piece> pieces) {
    GatherPieces p;
    for (const Piece &q : pieces) {
        p.src[p.n] = static_cast<const unsigned *>(q.src);
        p.words[p.n] = (long long)(q.bytes / sizeof(unsigned));
        p.dst[p.n] = 2LL * q.at;
        ++p.n;
    }
    CK(launch_gather(p, ctx->h_res_dev, 1, ctx->st));
    return TPSC_OK;
}
int read_back(tpsc_ctx *ctx, std::initializer_list<Piece> pieces) {
    int rc = queue_read_back(ctx, pieces);
    if (rc) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return TPSC_OK;
}

// device scalar readback after a reduction launched on ctx->st
int read_result(tpsc_ctx *ctx, int count, double *out, const double *src = nullptr) {
    int rc = read_back(ctx, {{src ? src : ctx->red.result, count * sizeof(double), 0}});
    if (rc) return rc;
    for (int i = 0; i < count; ++i) out[i] = ctx->h_res[i];
    return TPSC_OK;
}

// eps_k tables of the grid for the current model, then mu0 by the density
// root of green0::find_mu (src/green0.cpp:240-262)
// power sums Q_k = sum_{n = Nw0/2+1}^{Nw0} qn^(-2k), qn = 2 pi n T, for the
// sum-rule tail series (smallest terms first, long double), and
// P_p = sum_{t=0}^{Nw0/2} w^-p, w = (Nw0 + 2t + 1) pi T: the fermionic tail of
// the find_mu moments (largest t first, long double)
void tail_power_sums(int nw0, double T, double tailq[kTailQ], double tailP[kTailP]) {
    std::vector<long double> acc(kTailQ, 0.0L);
    const int nwmax = nw0 / 2;
    for (int j = 2 * nwmax; j > nwmax; --j) {
        const long double wn = 2.0L * 3.141592653589793238462643383279502884L * j * (long double)T;
        const long double x = 1.0L / (wn * wn);
        long double xp = x;
        for (int k = 1; k < kTailQ; ++k, xp *= x) acc[k] += xp;
    }
    for (int k = 0; k < kTailQ; ++k) tailq[k] = (double)acc[k];
    std::vector<long double> pw(kTailP, 0.0L);
    const int NO = nw0 / 2;
    for (int t = NO; t >= 0; --t) {
        const long double x =
            1.0L / ((2.0L * (NO + t) + 1.0L) * 3.141592653589793238462643383279502884L * (long double)T);
        long double xp = 1.0L;
        for (int k = 0; k < kTailP; ++k, xp *= x) pw[k] += xp;
    }
    for (int k = 0; k < kTailP; ++k) tailP[k] = (double)pw[k];
}

// eps_k on the octant of the nbk x nbk quadrant (dispk from tables of cos(k)
// and cos(2k): the same values and expression as the reference's, one pair
// of cosines per index instead of ten per point); full = the quadrant, or null
void octant_eps(int nbk, double tp, double tpp, double t3, double *eo, std::vector<double> *full) {
    std::vector<double> c1(nbk), c2(nbk);
    for (int l = 0; l < nbk; ++l) {
        const double k = l * PI / (nbk - 1);
        c1[l] = std::cos(k);
        c2[l] = std::cos(2 * k);
    }
    if (full) full->assign((size_t)nbk * nbk, 0.0);
    for (int l = 0; l < nbk; ++l)
        for (int m = 0; m < nbk; ++m) {
            const double e = -2.0 * (c1[l] + c1[m]) - 4.0 * tp * c1[l] * c1[m] - 2.0 * tpp * (c2[l] + c2[m]) -
                             4 * t3 * (c2[l] * c1[m] + c2[m] * c1[l]);
            if (full) (*full)[m + (size_t)l * nbk] = e;
            if (m <= l) eo[m + (size_t)l * (l + 1) / 2] = e;
        }
}

int grid_set_model(tpsc_ctx *ctx, Grid *g) {
    GridDev &d = g->d;
    std::vector<double> eo(d.n8), er(d.n8, 0.0);
    octant_eps(d.nbk, ctx->tp, ctx->tpp, ctx->t3, eo.data(), &g->ek_host);
    er[1] = -1;
    er[2] = -ctx->tp;
    er[3] = -ctx->tpp;
    er[4] = -ctx->t3;
    CK(cudaMemcpyAsync(d.ek, eo.data(), d.n8 * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(d.er, er.data(), d.n8 * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    if (g->tailq_T != ctx->T) {
        tail_power_sums(d.nw0, ctx->T, g->tailq_host, g->tailP_host);
        CK(cudaMemcpyAsync(d.tailq, g->tailq_host, kTailQ * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(d.tailP, g->tailP_host, kTailP * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
        g->tailq_T = ctx->T;
    }
    CK(cudaStreamSynchronize(ctx->st));
    g->have_chi0 = g->have_V = g->have_S = false;
    if (ctx->n == 1.0 && ctx->tp == 0 && ctx->tpp == 0) {
        g->mu0 = 0.0 + ctx->mu_shift;
        return TPSC_OK;
    }
    int rc = TPSC_OK;
    if (ctx->form & TPSC_FORM_NEWTON) {
        CK(launch_mu0_newton(d, ctx->n, ctx->T, ctx->red, ctx->st));
        double r[2];
        if ((rc = read_result(ctx, 2, r))) return rc;
        if (!std::isfinite(r[0]) || r[1] >= 200) return fail(ctx, TPSC_ERR_NO_ROOT, "mu0 not found");
        g->mu0 = r[0] + ctx->mu_shift;
        return TPSC_OK;
    }
    auto dens = [&](double mu, double &y) -> bool {
        cudaError_t e = launch_density(d, mu, ctx->n, ctx->T, ctx->red, ctx->st);
        if (e != cudaSuccess) {
            rc = cuda_fail(ctx, e, "launch_density");
            return false;
        }
        rc = read_result(ctx, 1, &y);
        return rc == TPSC_OK;
    };
    const double init[3] = {0.0, -8.0, 8.0};
    double root = 0;
    int nev;
    bool derr;
    if (!find_zero(dens, init, &root, nullptr, &nev, &derr)) {
        if (derr) return rc;
        return fail(ctx, TPSC_ERR_NO_ROOT, "mu0 not found");
    }
    g->mu0 = root + ctx->mu_shift;
    return TPSC_OK;
}

// Make (nk0, nw0) the current grid with the model's eps_k tables and mu0;
// those are computed once per model and grid, as the reference computes them
// once in its constructors (src/hamiltonien.cpp:328-394, src/green0.cpp:18-23),
// not by every solve.
int switch_grid(tpsc_ctx *ctx, int nk0, int nw0) {
    Grid *g = nullptr;
    int rc = build_grid(ctx, nk0, nw0, &g);
    if (rc) return rc;
    if (g->model_id != ctx->model_id) {
        rc = grid_set_model(ctx, g);
        if (rc) return rc;
        g->model_id = ctx->model_id;
    }
    g->have_chi0 = g->have_V = g->have_S = g->have_mom = g->have_U = false;
    ctx->cur = g;
    ctx->scal[TPSC_S_MU0] = g->mu0;
    return TPSC_OK;
}

int need_model(tpsc_ctx *ctx) {
    if (!ctx) return fail(nullptr, TPSC_ERR_ARG, "null context");
    if (!ctx->have_model) return fail(ctx, TPSC_ERR_STATE, "tpsc_set_model has not been called");
    return TPSC_OK;
}

bool mixed(const tpsc_ctx *ctx) { return (ctx->form & TPSC_FORM_MIXED) != 0; }

// The side stream st2 takes over after everything queued on st so far
// (fork), and st waits for what st2 queued (join).
int fork_side(tpsc_ctx *ctx, int k) {
    CK(cudaEventRecord(ctx->evf[2 * k], ctx->st));
    CK(cudaStreamWaitEvent(ctx->st2, ctx->evf[2 * k], 0));
    return TPSC_OK;
}
int join_side(tpsc_ctx *ctx, int k) {
    CK(cudaEventRecord(ctx->evf[2 * k + 1], ctx->st2));
    CK(cudaStreamWaitEvent(ctx->st, ctx->evf[2 * k + 1], 0));
    return TPSC_OK;
}

// ---- results read back from the device, checked and stored in ctx->scal ----
// r = (chi0max, qmax0, qmax1)
int set_chi0max(tpsc_ctx *ctx, const double *r) {
    ctx->scal[TPSC_S_CHI0MAX] = r[0];
    ctx->scal[TPSC_S_QMAX0] = r[1];
    ctx->scal[TPSC_S_QMAX1] = r[2];
    if (!std::isfinite(r[0]) || r[0] <= 0.0) return fail(ctx, TPSC_ERR_NONFINITE, "chi0(q, 0) has no positive maximum");
    return TPSC_OK;
}
// r = (Usp, Uch, evals_sp, evals_ch, ok_sp, ok_ch) of the device search, err its barrier flag
int set_roots(tpsc_ctx *ctx, const double *r, unsigned err) {
    if (err) return fail(ctx, TPSC_ERR_CUDA, "device root search: grid barrier timed out");
    if (r[4] != 1.0) return fail(ctx, TPSC_ERR_NO_ROOT, "Usp not found");
    if (r[5] != 1.0) return fail(ctx, TPSC_ERR_NO_ROOT, "Uch not found");
    ctx->Usp = r[0];
    ctx->Uch = r[1];
    ctx->scal[TPSC_S_EVALS_SP] = r[2];
    ctx->scal[TPSC_S_EVALS_CH] = r[3];
    ctx->scal[TPSC_S_USP] = ctx->Usp;
    ctx->scal[TPSC_S_UCH] = ctx->Uch;
    return TPSC_OK;
}
// r = (Tr Sigma G0, its asymptotic part, mu, evals, ok, Tr Sigma G at mu, -, Sigma_inf)
// of the Newton-form mu search, err its barrier flag
int set_mu(tpsc_ctx *ctx, const double *r, int err) {
    if (err) return fail(ctx, TPSC_ERR_CUDA, "device mu search: grid barrier timed out");
    ctx->scal[TPSC_S_SIGMA_INF] = r[7];
    ctx->scal[TPSC_S_TR_SG] = r[0];
    ctx->scal[TPSC_S_TR_SG_ASYMP] = r[0] + r[1];
    if (r[4] != 1.0) return fail(ctx, TPSC_ERR_NO_ROOT, "mu not found");
    ctx->scal[TPSC_S_MU] = r[2];
    ctx->scal[TPSC_S_EVALS_MU] = r[3];
    ctx->scal[TPSC_S_TR_SG2] = r[5];
    ctx->scal[TPSC_S_DBLOCC_SG2] = (r[5] + ctx->U * ctx->n * ctx->n / 4.0) / ctx->U;
    return TPSC_OK;
}

// read: take chi0max back now and check it; a Newton-form solve leaves that
// to its one readback at the end (the root search reads the device value)
int run_chi0(tpsc_ctx *ctx, bool read = true) {
    Grid *g = ctx->cur;
    const GridDev &d = g->d;
    int rc;
    // the chi0 boundary (one CTA: G(r, 0) -> d/dtau chi0) runs beside the
    // chi0 slices; both need only G(r, tau)
    if (mixed(ctx)) {
        if (!g->Grt32) CK(dalloc(g, &g->Grt32, (size_t)(d.nw0 + 1) * d.n8));
        CK(launch_gslice32(d, g->Grt32, g->mu0, ctx->T, ctx->st));
        if ((rc = fork_side(ctx, 0))) return rc;
        CK(launch_chi0_boundary(d, (const float *)g->Grt32, g->mu0, ctx->T, g->dG0p, g->dchirt0, g->dchiqt0,
                                ctx->st2));
        CK(launch_chi0_slice32(d, g->Grt32, g->chirt, g->chiq, ctx->st));
    } else {
        CK(launch_gslice(d, g->Grt, g->mu0, ctx->T, ctx->st));
        if ((rc = fork_side(ctx, 0))) return rc;
        CK(launch_chi0_boundary(d, (const double *)g->Grt, g->mu0, ctx->T, g->dG0p, g->dchirt0, g->dchiqt0,
                                ctx->st2));
        CK(launch_chi0_slice(d, g->Grt, g->chirt, g->chiq, ctx->st));
    }
    if ((rc = join_side(ctx, 0))) return rc;
    g->g_mixed = mixed(ctx);
    CK(launch_chi0_tau(d, g->chiq, g->dchiqt0, g->cinf, g->cinf2, ctx->T, ctx->st));
    CK(launch_chi0max(d, g->chiq, ctx->red, ctx->st));
    g->have_chi0 = true;
    g->have_V = g->have_S = g->have_mom = g->have_U = false;
    if (!read) return TPSC_OK;
    double r[3];
    rc = read_result(ctx, 3, r);
    if (rc) return rc;
    return set_chi0max(ctx, r);
}

// Per-frequency moments of chi0, their sums over the frequencies >= j and the
// tail moments, for the high-frequency series of the Newton-form sum rule:
// formed on the device (tpsc_kernels.cu), queued on the stream without a host
// round trip.
int ensure_moments(tpsc_ctx *ctx, Grid *g) {
    if (g->have_mom) return TPSC_OK;
    const GridDev &d = g->d;
    CK(launch_chi0_moments(d, g->chiq, g->mom, g->cmax, ctx->st));
    CK(launch_tail_moments(d, g->cinf, g->cinf2, ctx->T, ctx->redm, ctx->st));
    CK(launch_moment_suffix(d, g->mom, g->cmax, ctx->redm.result, g->d_mom_suf, g->d_cmax_suf, g->d_tailm,
                            ctx->st));
    g->have_mom = true;
    g->have_mom_host = false;
    return TPSC_OK;
}

// Host copies of the suffix sums and tail values, for the host-side series
// of sumrule().
int ensure_moments_host(tpsc_ctx *ctx, Grid *g) {
    int rc = ensure_moments(ctx, g);
    if (rc || g->have_mom_host) return rc;
    const int nb = g->d.nb;
    g->mom_suf.resize((size_t)(nb + 1) * kMomP);
    g->cmax_suf.resize(nb + 1);
    double tl[kMomP + 1];
    CK(cudaMemcpyAsync(g->mom_suf.data(), g->d_mom_suf, g->mom_suf.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->st));
    CK(cudaMemcpyAsync(g->cmax_suf.data(), g->d_cmax_suf, g->cmax_suf.size() * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(tl, g->d_tailm, sizeof(tl), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int k = 0; k < kMomP; ++k) g->tail_mom[k] = tl[k];
    g->tail_max = tl[kMomP];
    g->have_mom_host = true;
    return TPSC_OK;
}

// First stored frequency from which |U/2 chi| < kMomSeriesMax for every q, and
// whether the Matsubara tail needs the term-by-term sum (tail = 1).
void series_cut(const Grid *g, double Uv, int *jdir, int *tail) {
    const double ah = std::fabs(Uv) / 2.0;
    int j = 0;
    while (j < g->d.nb && ah * g->cmax_suf[j] >= kMomSeriesMax) ++j;
    *jdir = j;
    *tail = (ah * g->tail_max < kMomSeriesMax) ? 0 : 1;
}

// Sum-rule trace and its derivative in U (the reference's traceDiffChispChi0 /
// traceDiffChichChi0, src/chi.cpp:738-830).  The Newton form sums the stored
// frequencies j < jdir term by term and the rest as the series
//   sum_{q, j >= jdir} w [chi/(1 + h chi) - chi] = sum_{m=1}^{kMomP} (-h)^m M_{m+1}(jdir),
// h = -+ U/2, where jdir is the first frequency from which |h chi| < kMomSeriesMax
// for every q (truncation below (kMomSeriesMax)^kMomP relative).
int sumrule(tpsc_ctx *ctx, int channel, double Uv, double *tr, double *dtr) {
    Grid *g = ctx->cur;
    const GridDev &d = g->d;
    const double sgn = channel == 0 ? -1.0 : 1.0;
    const bool series = (ctx->form & TPSC_FORM_NEWTON) != 0;
    int jdir = d.nb, tail = 1;
    if (series) {
        int rc = ensure_moments_host(ctx, g);
        if (rc) return rc;
        series_cut(g, Uv, &jdir, &tail);
    }
    CK(launch_sumrule(d, g->chiq, g->cinf, g->cinf2, Uv, sgn, ctx->T, ctx->red, ctx->st, jdir, tail));
    double r[2];
    int rc = read_result(ctx, 2, r);
    if (rc) return rc;
    if (series && (jdir < d.nb || !tail)) {
        long double M[kMomP];
        for (int k = 0; k < kMomP; ++k)
            M[k] = (jdir < d.nb ? g->mom_suf[(size_t)jdir * kMomP + k] : 0.0L) + (tail ? 0.0L : g->tail_mom[k]);
        const long double h = sgn * Uv / 2.0;
        long double S = 0.0L, dS = 0.0L, hm1 = 1.0L;  // hm1 = (-h)^(m-1)
        for (int m = 1; m <= kMomP; ++m) {
            S += -h * hm1 * M[m - 1];
            dS += -m * hm1 * M[m - 1];
            hm1 *= -h;
        }
        const long double scale = (long double)ctx->T / (4.0L * (d.nbk - 1) * (d.nbk - 1));
        r[0] += (double)(scale * S);
        r[1] += (double)(scale * 0.5L * sgn * dS);
    }
    *tr = r[0];
    if (dtr) *dtr = r[1];
    return TPSC_OK;
}

// chi::find_Usp_Uch(nq0, nw0, Usc) on the current grid after chi0 (src/chi.cpp:850-876)
// read: take the roots back now; a Newton-form solve defers that to its one
// readback at the end, the interval's end then coming from the device chi0max
int roots_Usp_Uch(tpsc_ctx *ctx, double Usc[2], bool read = true) {
    const double n = ctx->n, U = ctx->U, nsr = ctx->nsr;
    const bool newton = (ctx->form & TPSC_FORM_NEWTON) != 0;
    int rc = TPSC_OK;
    if (newton) {
        // both roots in one cooperative launch (tpsc_roots.cu), into ctx->dres
        Grid *g = ctx->cur;
        if ((rc = ensure_moments(ctx, g))) return rc;
        RootScratch rs = ctx->roots;
        rs.out = ctx->dres;
        if (read)
            CK(launch_sumrule_roots(g->d, g->chiq, g->cinf, g->cinf2, g->d_mom_suf, g->d_cmax_suf, g->d_tailm,
                                    ctx->T, n, nsr, U, 2.0 / ctx->scal[TPSC_S_CHI0MAX] - 2 * EPS, rs, ctx->st));
        else
            CK(launch_sumrule_roots(g->d, g->chiq, g->cinf, g->cinf2, g->d_mom_suf, g->d_cmax_suf, g->d_tailm,
                                    ctx->T, n, nsr, U, 0.0, rs, ctx->st, ctx->red.result, 2 * EPS));
        ctx->roots.reset_sr = true;
        ctx->cur->have_U = true;
        if (!read) return TPSC_OK;
        // the results and the barrier's error flag in one readback
        if ((rc = read_back(ctx, {{ctx->dres, 6 * sizeof(double), 0}, {ctx->roots.bar + 2, sizeof(unsigned), 6}})))
            return rc;
        unsigned err;
        std::memcpy(&err, ctx->h_res + 6, sizeof(unsigned));
        ctx->roots.reset_sr = err != 0;
        if ((rc = set_roots(ctx, ctx->h_res, err))) return rc;
        Usc[0] = ctx->Usp;
        Usc[1] = ctx->Uch;
        return TPSC_OK;
    }
    // R_sp(Us) = trace + n - n^2/2 - nsr + Us nsr^2/(2U)  (chi::sum_rule_sp, src/chi.cpp:833-836)
    auto rsp = [&](double Us, double &y, double &dy) -> bool {
        double tr, dtr;
        rc = sumrule(ctx, 0, Us, &tr, &dtr);
        if (rc) return false;
        y = tr + n - n * n / 2.0 - nsr + Us * nsr * nsr / (2.0 * U);
        dy = dtr + nsr * nsr / (2.0 * U);
        return true;
    };
    auto rsp1 = [&](double Us, double &y) -> bool {
        double dy;
        return rsp(Us, y, dy);
    };
    const double init_sp[3] = {U / 2.0, 0.0, 2.0 / ctx->scal[TPSC_S_CHI0MAX] - 2 * EPS};
    int nev;
    bool derr, ok;
    double root = 0;
    ok = newton ? newton_root(rsp, init_sp[0], init_sp[1], init_sp[2], 1e-16, &root, &nev, &derr)
                : find_zero(rsp1, init_sp, &root, nullptr, &nev, &derr);
    if (!ok) {
        if (derr) return rc;
        return fail(ctx, TPSC_ERR_NO_ROOT, "Usp not found");
    }
    ctx->scal[TPSC_S_EVALS_SP] = nev;
    Usc[0] = root;
    ctx->Usp = root;
    // R_ch(Uc) = trace + n - n^2/2 - (nsr + Usp nsr^2/(2U) - nsr^2)  (src/chi.cpp:840-843)
    auto rch = [&](double Uc, double &y, double &dy) -> bool {
        double tr, dtr;
        rc = sumrule(ctx, 1, Uc, &tr, &dtr);
        if (rc) return false;
        y = tr + n - n * n / 2.0 - (nsr + ctx->Usp * nsr * nsr / (2.0 * U) - nsr * nsr);
        dy = dtr;
        return true;
    };
    auto rch1 = [&](double Uc, double &y) -> bool {
        double dy;
        return rch(Uc, y, dy);
    };
    const double init_ch[3] = {0.0, 0.0, 1000.0 * U};
    // the Newton form starts the charge search at U (the interval's lower end
    // is not an interior point)
    ok = newton ? newton_root(rch, U, init_ch[1], init_ch[2], 1e-16, &root, &nev, &derr)
                : find_zero(rch1, init_ch, &root, nullptr, &nev, &derr);
    if (!ok) {
        if (derr) return rc;
        return fail(ctx, TPSC_ERR_NO_ROOT, "Uch not found");
    }
    ctx->scal[TPSC_S_EVALS_CH] = nev;
    Usc[1] = root;
    ctx->Uch = root;
    ctx->scal[TPSC_S_USP] = ctx->Usp;
    ctx->scal[TPSC_S_UCH] = ctx->Uch;
    ctx->cur->have_U = true;
    // where the vertex and Sigma kernels read them
    CK(launch_store(ctx->dres, Usc, 2, ctx->st));
    return TPSC_OK;
}

void set_dblocc(tpsc_ctx *ctx) {
    const double nsr = ctx->nsr;
    double D = ctx->Usp / ctx->U * nsr * nsr / 4.0;
    if (ctx->n > 1.0) D += 1.0 - nsr;
    ctx->scal[TPSC_S_DBLOCC] = D;
}

int run_vertex(tpsc_ctx *ctx) {
    Grid *g = ctx->cur;
    if (!g || !g->have_chi0) return fail(ctx, TPSC_ERR_STATE, "chi0 has not been computed on the current grid");
    // Usp, Uch from ctx->dres, where the root search left them
    if (mixed(ctx))
        CK(launch_vertex_q32(g->d, g->chiq, g->V, ctx->U, ctx->dres, ctx->T, ctx->st));
    else
        CK(launch_vertex_q(g->d, g->chiq, g->V, ctx->U, ctx->dres, ctx->T, ctx->st));
    CK(launch_vertex_tau(g->d, g->V, g->chirt, ctx->U, ctx->dres, ctx->st));
    g->have_V = true;
    return TPSC_OK;
}

// settle: read Sigma_inf back now; a Newton-form solve leaves it to the
// readback of the mu search that follows
int run_self(tpsc_ctx *ctx, bool settle = true) {
    Grid *g = ctx->cur;
    if (!g || !g->have_V) return fail(ctx, TPSC_ERR_STATE, "the vertex V(r, tau) has not been computed");
    const GridDev &d = g->d;
    // G(r, tau) as the chi0 stage left it (FP32 in the mixed form); the two
    // boundary CTAs run beside the Sigma slices
    int rc = fork_side(ctx, 1);
    if (rc) return rc;
    if (g->g_mixed) {
        CK(launch_sigma_boundary(d, (const float *)g->Grt32, g->V, g->dchirt0, g->dG0p, g->mu0, ctx->U, ctx->dres,
                                 g->dS, ctx->st2));
        CK(launch_sigma_slice32(d, g->Grt32, g->V, g->sigt, ctx->st));
    } else {
        CK(launch_sigma_boundary(d, (const double *)g->Grt, g->V, g->dchirt0, g->dG0p, g->mu0, ctx->U, ctx->dres,
                                 g->dS, ctx->st2));
        CK(launch_sigma_slice(d, (const double *)g->Grt, g->V, g->sigt, ctx->st));
    }
    if ((rc = join_side(ctx, 1))) return rc;
    CK(launch_sigma_tau(d, g->sigt, g->dS, g->S, g->s2, g->s3, g->s4, g->sinf, ctx->T, ctx->st));
    g->have_S = true;
    if (!settle) return TPSC_OK;
    if ((rc = read_back(ctx, {{g->sinf, sizeof(double), 0}}))) return rc;
    ctx->scal[TPSC_S_SIGMA_INF] = ctx->h_res[0];
    return TPSC_OK;
}

int trace_self_G(tpsc_ctx *ctx, double out[2]) {
    Grid *g = ctx->cur;
    if (!g || !g->have_S) return fail(ctx, TPSC_ERR_STATE, "the self-energy has not been computed");
    CK(launch_trace_self_G(g->d, g->S, g->s2, g->s3, g->sinf, g->mu0, ctx->T, ctx->red, ctx->st));
    double r[2];
    int rc = read_result(ctx, 2, r);
    if (rc) return rc;
    out[0] = r[0];
    out[1] = r[0] + r[1];
    ctx->scal[TPSC_S_TR_SG] = out[0];
    ctx->scal[TPSC_S_TR_SG_ASYMP] = out[1];
    return TPSC_OK;
}

int trace_diff_G(tpsc_ctx *ctx, double pmu, double *tr, double *dtr = nullptr) {
    Grid *g = ctx->cur;
    CK(launch_trace_diff_G(g->d, g->S, g->s2, g->s3, g->s4, g->sinf, g->mu0, pmu, ctx->T, ctx->red, ctx->st));
    double r[2];
    int rc = read_result(ctx, 2, r);
    if (rc) return rc;
    *tr = r[0];
    if (dtr) *dtr = r[1];
    return TPSC_OK;
}

// The find_mu series covers the frequencies from jc = first n with
// w_n >= kMomMuRange / kMuSeriesMax (capped at Nw0/2: then only the tail);
// w_jc is returned for the root search, which takes the series while
// |mu - mu0| <= kMuSeriesMax |z|_min with |z|_min = w_jc - 2 Sigma_inf / w_jc
// (|z| >= w_n - |Im Sigma| on the series set).
void mu_series_cut(int nw0, double T, int *jc_out, double *wc_out) {
    const int NO = nw0 / 2;
    const double pt = PI * T;
    int jc = (int)std::ceil((kMomMuRange / kMuSeriesMax / pt - 1.0) / 2.0);
    jc = std::max(0, std::min(jc, NO));
    *wc_out = (2 * jc + 1) * pt;
    *jc_out = jc;
}
void mu_series_cut(const tpsc_ctx *ctx, int *jc_out, double *wc_out) {
    mu_series_cut(ctx->cur->d.nw0, ctx->T, jc_out, wc_out);
}

// The Newton form of traceSelfG + find_mu + traceSelfG2: one pass over Sigma
// for Tr Sigma G0 and the series moments (k_sigma_moments), then the Newton
// search and Tr Sigma G at mu in one cooperative launch (k_mu_roots), one
// readback for all of it.
int queue_mu_newton(tpsc_ctx *ctx) {
    Grid *g = ctx->cur;
    const GridDev &d = g->d;
    int jc;
    double wc;
    mu_series_cut(ctx, &jc, &wc);
    CK(launch_sigma_moments(d, g->S, g->s2, g->s3, g->s4, g->sinf, g->mu0, ctx->T, jc, ctx->redm, ctx->st));
    CK(launch_mu_roots(d, g->S, g->s2, g->s3, g->s4, g->sinf, ctx->redm.result, g->mu0, ctx->T, jc, wc, ctx->roots,
                       ctx->st));
    ctx->roots.reset_mu = true;
    return TPSC_OK;
}

int self_traces_and_mu_newton(tpsc_ctx *ctx) {
    int rc = queue_mu_newton(ctx);
    if (rc) return rc;
    if ((rc = read_back(ctx, {{ctx->redm.result, 2 * sizeof(double), 0},
                              {ctx->roots.out, 4 * sizeof(double), 2},
                              {ctx->roots.bar + 6, sizeof(int), 6},
                              {ctx->cur->sinf, sizeof(double), 7}})))
        return rc;
    int err;
    std::memcpy(&err, ctx->h_res + 6, sizeof(int));
    ctx->roots.reset_mu = err != 0;
    return set_mu(ctx, ctx->h_res, err);
}

// stage times from ctx->ev[0..5] and the finiteness check of the scalars
int finish_solve(tpsc_ctx *ctx) {
    CK(cudaEventSynchronize(ctx->ev[5]));
    for (int i = 0; i < 5; ++i) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->ev[i], ctx->ev[i + 1]));
        ctx->stage_ms[i] = ms;
    }
    for (int i = 0; i < TPSC_S_COUNT; ++i)
        if (!std::isfinite(ctx->scal[i])) return fail(ctx, TPSC_ERR_NONFINITE, "non-finite scalar result");
    return TPSC_OK;
}

// stage boundary i of a solve (ctx->ev[i]); an event record node of the graph
// while the solve is being captured
int mark(tpsc_ctx *ctx, int i) {
    CK(cudaEventRecordWithFlags(ctx->ev[i], ctx->st, ctx->capturing ? cudaEventRecordExternal : cudaEventRecordDefault));
    return TPSC_OK;
}

// The Newton-form solve from the chi0 stage on, queued on ctx->st without a
// host round trip (the roots, the vertex and Sigma read their inputs on the
// device), ending in the gather of everything the host checks into ctx->h_res;
// newton_finish waits for it and checks chi0max, the sum-rule roots, the mu
// search and their barrier flags in stage order.
int newton_queue(tpsc_ctx *ctx) {
    double Usc[2];
    int rc;
    if ((rc = mark(ctx, 0))) return rc;
    if ((rc = run_chi0(ctx, false))) return rc;
    if ((rc = mark(ctx, 1))) return rc;
    if ((rc = roots_Usp_Uch(ctx, Usc, false))) return rc;
    if ((rc = mark(ctx, 2))) return rc;
    if ((rc = run_vertex(ctx))) return rc;
    if ((rc = mark(ctx, 3))) return rc;
    if ((rc = run_self(ctx, false))) return rc;
    if ((rc = mark(ctx, 4))) return rc;
    if ((rc = queue_mu_newton(ctx))) return rc;
    if ((rc = mark(ctx, 5))) return rc;
    // h_res: [0..2] chi0max, qmax; [3..8] the sum-rule roots; [9] their flag;
    // [10..11] the Sigma traces; [12..15] the mu search; [16] its flag; [17] Sigma_inf
    return queue_read_back(ctx, {{ctx->red.result, 3 * sizeof(double), 0},
                                 {ctx->dres, 6 * sizeof(double), 3},
                                 {ctx->roots.bar + 2, sizeof(unsigned), 9},
                                 {ctx->redm.result, 2 * sizeof(double), 10},
                                 {ctx->roots.out, 4 * sizeof(double), 12},
                                 {ctx->roots.bar + 6, sizeof(int), 16},
                                 {ctx->cur->sinf, sizeof(double), 17}});
}

int newton_finish(tpsc_ctx *ctx) {
    CK(cudaStreamSynchronize(ctx->st));
    int rc;
    const double *h = ctx->h_res;
    if ((rc = set_chi0max(ctx, h))) return rc;
    unsigned err_sr;
    std::memcpy(&err_sr, h + 9, sizeof(unsigned));
    int err_mu;
    std::memcpy(&err_mu, h + 16, sizeof(int));
    ctx->roots.reset_sr = err_sr != 0;
    ctx->roots.reset_mu = err_mu != 0;
    if ((rc = set_roots(ctx, h + 3, err_sr))) return rc;
    set_dblocc(ctx);
    double r[8];
    for (int i = 0; i < 6; ++i) r[i] = h[10 + i];
    r[6] = 0.0;
    r[7] = h[17];
    return set_mu(ctx, r, err_mu);
}

// the host state newton_queue leaves behind (a replayed graph only launches)
void newton_state(tpsc_ctx *ctx) {
    Grid *g = ctx->cur;
    g->g_mixed = mixed(ctx);
    g->have_chi0 = g->have_mom = g->have_U = g->have_V = g->have_S = true;
    g->have_mom_host = false;
    ctx->roots.reset_sr = ctx->roots.reset_mu = true;
}

// The Newton-form solve on the current grid, queued directly or as a CUDA
// graph (ctx->graph_mode): a solve whose key (grid, form, model, mu0, the
// root searches' barrier state and grid cap: everything its launches take)
// equals the captured one replays the executable graph; in mode 1 a key seen
// twice in a row is captured, in mode 2 every key after the grid's first
// direct solve in that form (so that the kernels' one-time attribute calls
// happen outside a capture); a new capture updates the executable graph in
// place when its topology allows.  A capture that fails turns graphs off for
// the context and the solve runs as direct launches.
int newton_solve(tpsc_ctx *ctx) {
    Grid *g = ctx->cur;
    const GridDev &d = g->d;
    if (mixed(ctx) && !g->Grt32) CK(dalloc(g, &g->Grt32, (size_t)(d.nw0 + 1) * d.n8));
    SolveKey key;
    key.form = ctx->form;
    key.cap = ctx->roots.max_blocks;
    key.model_id = ctx->model_id;
    key.mu0 = g->mu0;
    key.nsr = ctx->nsr;
    key.tiles = tau_tiles_version();
    key.rsr = ctx->roots.reset_sr;
    key.rmu = ctx->roots.reset_mu;
    const unsigned fbit = 1u << (ctx->form & 3);
    const bool graphs = ctx->graph_mode > 0 && !ctx->graph_off && (g->warm_forms & fbit);
    int rc = TPSC_OK;
    if (graphs && g->graph_exec && key == g->graph_key) {
        CK(cudaGraphLaunch(g->graph_exec, ctx->st));
        add_launches(g->graph_kernels);
        ctx->graph_kernels = g->graph_kernels;
        ++ctx->graph_replays;
        newton_state(ctx);
        return newton_finish(ctx);
    }
    if (graphs && (ctx->graph_mode == 2 || (key == ctx->seen_key && ctx->seen_grid == g))) {
        const long long k0 = launches_thread();
        CK(cudaStreamBeginCapture(ctx->st, cudaStreamCaptureModeThreadLocal));
        ctx->capturing = true;
        rc = newton_queue(ctx);
        ctx->capturing = false;
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(ctx->st, &graph);
        const long long nk = launches_thread() - k0;
        add_launches(-nk);
        if (rc == TPSC_OK && e == cudaSuccess && graph) {
            if (g->graph_exec) {
                cudaGraphExecUpdateResultInfo info;
                if (cudaGraphExecUpdate(g->graph_exec, graph, &info) != cudaSuccess) {
                    cudaGetLastError();
                    cudaGraphExecDestroy(g->graph_exec);
                    g->graph_exec = nullptr;
                }
            }
            if (!g->graph_exec) e = cudaGraphInstantiate(&g->graph_exec, graph, 0);
        }
        if (graph) cudaGraphDestroy(graph);
        if (rc == TPSC_OK && e == cudaSuccess && g->graph_exec) {
            g->graph_key = key;
            g->graph_kernels = ctx->graph_kernels = nk;
            ++ctx->graph_captures;
            CK(cudaGraphLaunch(g->graph_exec, ctx->st));
            add_launches(nk);
            return newton_finish(ctx);
        }
        // the capture failed: the same launches, directly, from now on
        cudaGetLastError();
        if (g->graph_exec) cudaGraphExecDestroy(g->graph_exec);
        g->graph_exec = nullptr;
        ctx->graph_off = true;
        ctx->err.clear();
    }
    ctx->seen_key = key;
    ctx->seen_grid = g;
    if ((rc = newton_queue(ctx))) return rc;
    g->warm_forms |= fbit;
    return newton_finish(ctx);
}

int find_mu(tpsc_ctx *ctx) {
    Grid *g = ctx->cur;
    if (!g || !g->have_S) return fail(ctx, TPSC_ERR_STATE, "the self-energy has not been computed");
    if (ctx->form & TPSC_FORM_NEWTON) return self_traces_and_mu_newton(ctx);
    int rc = TPSC_OK;
    auto f = [&](double m, double &y) -> bool {
        rc = trace_diff_G(ctx, m, &y);
        return rc == TPSC_OK;
    };
    const double init[3] = {0.0, -10.0, 10.0}, lims[2] = {-20.0, 20.0};
    double root = 0;
    int nev;
    bool derr;
    if (!find_zero(f, init, &root, lims, &nev, &derr)) {
        if (derr) return rc;
        return fail(ctx, TPSC_ERR_NO_ROOT, "mu not found");
    }
    ctx->scal[TPSC_S_EVALS_MU] = nev;
    ctx->scal[TPSC_S_MU] = root;
    // traceSelfG2 at the new mu (src/green.cpp:3281)
    CK(launch_trace_self_G2(g->d, g->S, g->s2, g->s3, g->sinf, root, ctx->T, ctx->red, ctx->st));
    double r;
    rc = read_result(ctx, 1, &r);
    if (rc) return rc;
    ctx->scal[TPSC_S_TR_SG2] = r;
    ctx->scal[TPSC_S_DBLOCC_SG2] = (r + ctx->U * ctx->n * ctx->n / 4.0) / ctx->U;
    return TPSC_OK;
}

// Device state of the correlator on grid g for n_theta bins: the K4 arrays
// once, the per-CTA partial rows and the output when n_theta grows, and the
// eps-derivative tables (model dependent) and angle bins on every call.
int ensure_cond(tpsc_ctx *ctx, Grid *g, int nbins) {
    CondDev &c = g->cond;
    const GridDev &d = g->d;
    const int nbk = d.nbk;
    if (!g->cond_alloc) {
        c.K4 = (nbk - 2) * nbk;
        c.K4p = (c.K4 + 1) & ~1;
        int nblk = 0;
        CK(cond_blocks(d, &nblk));
        c.nblk = std::max(1, std::min(nblk, c.K4p / 2));
        const size_t K4 = c.K4, K4p = c.K4p, NJ = d.nw0 + 1;
        cudaError_t e = cudaSuccess;
#define A(x)                \
    if (e == cudaSuccess) { \
        e = (x);            \
    }
        A(dalloc(g, &c.dek, K4));
        A(dalloc(g, &c.d2ek, K4));
        A(dalloc(g, &c.d2line, (size_t)2 * nbk));
        A(dalloc(g, &c.bin, K4));
        A(dalloc(g, &c.tab, 4 * K4));
        A(dalloc(g, &c.hV, K4p * NJ));
        A(dalloc(g, &c.f0V, K4p * NJ));
        A(dalloc(g, &c.pre, 4 * K4p));
        A(dalloc(g, &c.dbound, 4 * K4p));
        A(dalloc(g, &c.lines, (size_t)2 * nbk));
#undef A
        if (e != cudaSuccess) return cuda_fail(ctx, e, "conductivity allocation");
        g->cond_alloc = true;
    }
    const int NB = d.nw0 / 2 + 1;
    c.nbins = nbins;
    c.pw = nbins * 2 * NB + 1;
    const size_t need_part = (size_t)c.nblk * c.pw, need_out = (size_t)nbins * 2 * NB + 2 * NB + 1;
    if (need_part > g->cond_part_cap) {
        if (c.partial) cudaFree(c.partial);
        c.partial = nullptr;
        g->cond_part_cap = 0;
        CK(cudaMalloc(&c.partial, need_part * sizeof(double)));
        g->cond_part_cap = need_part;
    }
    if (need_out > g->cond_out_cap) {
        if (c.out) cudaFree(c.out);
        c.out = nullptr;
        g->cond_out_cap = 0;
        CK(cudaMalloc(&c.out, need_out * sizeof(double)));
        g->cond_out_cap = need_out;
    }
    // tables on k = (l+1, m) pi/(nbk-1) (src/cond_opt.cpp:2588-2611) and on
    // the kx = 0, pi lines; the angle bin theta_k = atan((L/2 - m)/(L/2 - l - 1)),
    // floor(theta_k / (pi / (2 n_theta))) (src/cond_opt.cpp:3174, 3790-3793)
    std::vector<double> dek(c.K4), d2(c.K4), d2l(2 * nbk);
    std::vector<int> bins(c.K4, 0);
    const int nk0 = d.nk0;
    const double Dtheta = PI / (2.0 * nbins);
    for (int l = 0; l < nbk - 2; ++l) {
        const double kx = (l + 1) * PI / (nbk - 1);
        for (int m = 0; m < nbk; ++m) {
            const double ky = m * PI / (nbk - 1);
            dek[m + l * nbk] = grad_ek_x(kx, ky, ctx->tp, ctx->tpp, ctx->t3);
            d2[m + l * nbk] = hessian_ek_xx(kx, ky, ctx->tp, ctx->tpp, ctx->t3);
            if (nbins > 1) {
                const double th = std::atan((1.0 * (nk0 / 2 - m)) / (nk0 / 2 - l - 1));
                bins[m + l * nbk] = std::min(nbins - 1, std::max(0, (int)std::floor(th / Dtheta)));
            }
        }
    }
    for (int side = 0; side < 2; ++side) {
        const double kx = side == 0 ? 0.0 : (nbk - 1) * PI / (nbk - 1);
        for (int m = 0; m < nbk; ++m)
            d2l[side * nbk + m] = hessian_ek_xx(kx, m * PI / (nbk - 1), ctx->tp, ctx->tpp, ctx->t3);
    }
    CK(cudaMemcpyAsync(c.dek, dek.data(), c.K4 * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(c.d2ek, d2.data(), c.K4 * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(c.d2line, d2l.data(), 2 * nbk * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(c.bin, bins.data(), c.K4 * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    // the host vectors are released when this function returns
    CK(cudaStreamSynchronize(ctx->st));
    return TPSC_OK;
}

// cond_opt::calc_chijj_vertex_corr_all_optim, bubble + Maki-Thompson branch,
// on the current grid after Sigma and mu (src/cond_opt.cpp:2537-4286)
int run_cond(tpsc_ctx *ctx, int nbins) {
    Grid *g = ctx->cur;
    int rc = ensure_cond(ctx, g, nbins);
    if (rc) return rc;
    const GridDev &d = g->d;
    const CondDev &c = g->cond;
    const double mu = ctx->scal[TPSC_S_MU];
    const double fact = ctx->U * (3.0 * ctx->Usp + ctx->Uch) / 4.0;  // TPSC_fact (src/cond_opt.cpp:2892)
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    if (ctx->form & TPSC_FORM_MIXED)
        CK(launch_cond_slices32(d, c, g->V, g->dchirt0, g->mu0, ctx->T, fact, ctx->st));
    else
        CK(launch_cond_slices(d, c, g->V, g->dchirt0, g->mu0, ctx->T, fact, ctx->st));
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    CK(launch_cond_tau(d, c, g->S, g->s2, g->s3, g->sinf, mu, ctx->T, ctx->st));
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    CK(launch_cond_finish(d, c, g->S, g->s2, g->s3, g->sinf, mu, ctx->T, ctx->st));
    CK(cudaEventRecord(ctx->ev[3], ctx->st));
    const int NB = d.nw0 / 2 + 1;
    g->cond_host.assign((size_t)nbins * 2 * NB + 2 * NB + 1, 0.0);
    CK(cudaMemcpyAsync(g->cond_host.data(), c.out, g->cond_host.size() * sizeof(double), cudaMemcpyDeviceToHost,
                       ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    for (int i = 0; i < 3; ++i) {
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->ev[i], ctx->ev[i + 1]));
        ctx->stage_ms[5 + i] = ms;
    }
    g->cond_bins = nbins;
    for (double v : g->cond_host)
        if (!std::isfinite(v)) return fail(ctx, TPSC_ERR_NONFINITE, "non-finite chi_jj");
    return TPSC_OK;
}

// The non-uniform bosonic grid of the AL correction (src/cond_opt.cpp:5123-5155):
// every n up to (N0-1)/2^mmin, then mmin blocks of (N0-1)/2^(mmin+1) points
// whose spacing doubles from block to block (N0 = Nw0/2 + 1).
std::vector<int> al_frequencies(int nw0, int mmin) {
    const int n0 = nw0 / 2;
    const int jf = n0 >> mmin, nj = n0 >> (mmin + 1);
    std::vector<int> ind;
    for (int j = 0; j <= jf; ++j) ind.push_back(j);
    int n = jf, d = 1;
    for (int b = 0; b < mmin; ++b) {
        d *= 2;
        for (int j = 0; j < nj; ++j) ind.push_back(n += d);
    }
    return ind;
}

// cond_opt::calc_chijj_vertex_corr_all_optim, Aslamazov-Larkin branch
// (chi3 = true), on the current grid after Sigma and mu
// (src/cond_opt.cpp:4292-6529): one setup, then the per-frequency pipeline
// for every grid frequency n >= 1 (entry 0 stays 0, as in the reference)
int run_al(tpsc_ctx *ctx, int mmin, int nbins) {
    Grid *g = ctx->cur;
    int rc = ensure_cond(ctx, g, nbins);  // the K4 tables and the angle bins
    if (rc) return rc;
    const GridDev &d = g->d;
    const CondDev &c = g->cond;
    AlDev &a = g->al;
    const std::vector<int> ind = al_frequencies(d.nw0, mmin);
    const int N = (int)ind.size();
    if (!g->al_alloc) {
        a.K4 = c.K4;
        a.K4p = c.K4p;
        const size_t K4 = a.K4, K4p = a.K4p, NJ = d.nw0 + 1, NO = d.nw0 / 2;
        cudaError_t e = cudaSuccess;
#define A(x)                \
    if (e == cudaSuccess) { \
        e = (x);            \
    }
        A(dalloc(g, &a.Grt, NJ * d.n8));
        A(dalloc(g, &a.hGt, K4p * NJ));
        A(dalloc(g, &a.pre, 2 * K4));
        A(dalloc(g, &a.dhG, 2 * K4));
        A(dalloc(g, &a.hgq, K4 * (NO + 1)));
        A(dalloc(g, &a.HQ, NJ * K4));
        A(dalloc(g, &a.dHQ, 2 * K4));
        A(dalloc(g, &a.HR, NJ * K4));
        A(dalloc(g, &a.dHR, 2 * K4));
        A(dalloc(g, &a.HK, K4p * NJ));
        A(dalloc(g, &a.H2K, K4p * NJ));
        A(dalloc(g, &a.dHK, 4 * K4));
        A(dalloc(g, &a.colv, K4));
#undef A
        if (e != cudaSuccess) return cuda_fail(ctx, e, "Aslamazov-Larkin allocation");
        g->al_alloc = true;
    }
    a.nbins = nbins;
    a.nrows = N;
    const size_t need_out = (size_t)N * (1 + nbins);
    if (need_out > g->al_out_cap) {
        if (a.out) cudaFree(a.out);
        a.out = nullptr;
        g->al_out_cap = 0;
        CK(cudaMalloc(&a.out, need_out * sizeof(double)));
        g->al_out_cap = need_out;
    }
    CK(cudaMemsetAsync(a.out, 0, need_out * sizeof(double), ctx->st));
    const double mu = ctx->scal[TPSC_S_MU];
    CK(launch_cond_table(d, c, g->mu0, ctx->T, ctx->st));
    CK(launch_al_setup(d, c, a, g->dG0p, g->mu0, ctx->T, ctx->st));
    for (int n = 1; n < N; ++n)
        CK(launch_al_freq(d, c, a, g->chiq, g->cinf, g->cinf2, g->S, g->s2, g->s3, g->sinf, g->dG0p, ind[n], n,
                          ctx->U, ctx->Usp, ctx->Uch, mu, g->mu0, ctx->T, ctx->st));
    g->al_host.assign(need_out, 0.0);
    CK(cudaMemcpyAsync(g->al_host.data(), a.out, need_out * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    g->al_ind = ind;
    g->al_bins = nbins;
    for (double v : g->al_host)
        if (!std::isfinite(v)) return fail(ctx, TPSC_ERR_NONFINITE, "non-finite chijj3");
    return TPSC_OK;
}

int ensure_stage(tpsc_ctx *ctx, size_t bytes) {
    if (ctx->stage_bytes >= bytes) return TPSC_OK;
    if (ctx->stage) cudaFree(ctx->stage);
    ctx->stage = nullptr;
    ctx->stage_bytes = 0;
    CK(cudaMalloc(&ctx->stage, bytes));
    ctx->stage_bytes = bytes;
    return TPSC_OK;
}

int copy_out(tpsc_ctx *ctx, void *host, const void *dev, size_t bytes) {
    CK(cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ctx->st));
    return TPSC_OK;
}

}  // namespace

namespace tpsc {
int static_fail(int code, const std::string &msg) { return fail(nullptr, code, msg); }
}  // namespace tpsc

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

tpsc_ctx *tpsc_create(int device, int *status) {
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        g_static_err = std::string("no CUDA device: ") + cudaGetErrorString(e);
        if (status) *status = TPSC_ERR_CUDA;
        return nullptr;
    }
    if (device < 0 || device >= ndev) {
        g_static_err = "device index out of range";
        if (status) *status = TPSC_ERR_ARG;
        return nullptr;
    }
    tpsc_ctx *ctx = new tpsc_ctx;
    ctx->device = device;
    auto bad = [&](cudaError_t er) {
        g_static_err = cudaGetErrorString(er);
        if (status) *status = TPSC_ERR_CUDA;
        tpsc_destroy(ctx);
        return (tpsc_ctx *)nullptr;
    };
    if ((e = cudaSetDevice(device)) != cudaSuccess) return bad(e);
    if ((e = cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking)) != cudaSuccess) return bad(e);
    if ((e = cudaStreamCreateWithFlags(&ctx->st2, cudaStreamNonBlocking)) != cudaSuccess) return bad(e);
    for (auto &ev : ctx->evf)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return bad(e);
    if ((e = cudaMalloc(&ctx->red.partial, 4 * kMaxBlocks * sizeof(double))) != cudaSuccess) return bad(e);
    if ((e = cudaMalloc(&ctx->red.result, 8 * sizeof(double))) != cudaSuccess) return bad(e);
    if ((e = cudaMalloc(&ctx->red.ticket, sizeof(unsigned))) != cudaSuccess) return bad(e);
    if ((e = cudaMemsetAsync(ctx->red.ticket, 0, sizeof(unsigned), ctx->st)) != cudaSuccess) return bad(e);
    if ((e = cudaMalloc(&ctx->redm.partial, (size_t)std::max(2 * kMomP + 2, kSigmaMomNV) * kMaxBlocks *
                                                 sizeof(double))) != cudaSuccess)
        return bad(e);
    if ((e = cudaMalloc(&ctx->redm.result, 32 * sizeof(double))) != cudaSuccess) return bad(e);
    if ((e = cudaMalloc(&ctx->roots.partial, 2 * kRootVals * kRootMaxBlocks * sizeof(double))) != cudaSuccess)
        return bad(e);
    if ((e = cudaMalloc(&ctx->roots.bar, 8 * sizeof(unsigned))) != cudaSuccess) return bad(e);
    if ((e = cudaMemsetAsync(ctx->roots.bar, 0, 8 * sizeof(unsigned), ctx->st)) != cudaSuccess) return bad(e);
    ctx->roots.reset_sr = ctx->roots.reset_mu = false;
    if ((e = cudaMalloc(&ctx->dres, 16 * sizeof(double))) != cudaSuccess) return bad(e);
    if ((e = cudaMemsetAsync(ctx->dres, 0, 16 * sizeof(double), ctx->st)) != cudaSuccess) return bad(e);
    if ((e = cudaMalloc(&ctx->roots.out, 8 * sizeof(double))) != cudaSuccess) return bad(e);
    if ((e = cudaHostAlloc(&ctx->h_res, 32 * sizeof(double), cudaHostAllocMapped)) != cudaSuccess) return bad(e);
    if ((e = cudaHostGetDevicePointer(&ctx->h_res_dev, ctx->h_res, 0)) != cudaSuccess) return bad(e);
    for (auto &ev : ctx->ev)
        if ((e = cudaEventCreate(&ev)) != cudaSuccess) return bad(e);
    if (status) *status = TPSC_OK;
    return ctx;
}

void tpsc_destroy(tpsc_ctx *ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->st) cudaStreamSynchronize(ctx->st);
    for (auto &kv : ctx->grids) free_grid(kv.second);
    for (auto &kv : ctx->groups) free_group(kv.second);
    for (cudaStream_t s : ctx->gst)
        if (s) cudaStreamDestroy(s);
    if (ctx->red.partial) cudaFree(ctx->red.partial);
    if (ctx->red.result) cudaFree(ctx->red.result);
    if (ctx->red.ticket) cudaFree(ctx->red.ticket);
    if (ctx->redm.partial) cudaFree(ctx->redm.partial);
    if (ctx->redm.result) cudaFree(ctx->redm.result);
    if (ctx->roots.partial) cudaFree(ctx->roots.partial);
    if (ctx->roots.bar) cudaFree(ctx->roots.bar);
    if (ctx->roots.out) cudaFree(ctx->roots.out);
    if (ctx->dres) cudaFree(ctx->dres);
    if (ctx->h_res) cudaFreeHost(ctx->h_res);
    if (ctx->stage) cudaFree(ctx->stage);
    if (ctx->cst) cudaStreamSynchronize(ctx->cst);
    for (int k = 0; k < 2; ++k) {
        if (ctx->snap[k]) cudaFree(ctx->snap[k]);
        if (ctx->snap_ev[k]) cudaEventDestroy(ctx->snap_ev[k]);
        if (ctx->copy_ev[k]) cudaEventDestroy(ctx->copy_ev[k]);
    }
    if (ctx->cst) cudaStreamDestroy(ctx->cst);
    for (auto &ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    for (auto &ev : ctx->evf)
        if (ev) cudaEventDestroy(ev);
    if (ctx->st2) cudaStreamDestroy(ctx->st2);
    if (ctx->st) cudaStreamDestroy(ctx->st);
    delete ctx;
}

const char *tpsc_last_error(const tpsc_ctx *ctx) { return ctx ? ctx->err.c_str() : g_static_err.c_str(); }

int tpsc_set_model(tpsc_ctx *ctx, int nk0, int Nw0, double n, double T, double tp, double tpp, double t3,
                   double U) {
    if (!ctx) return fail(nullptr, TPSC_ERR_ARG, "null context");
    if (!(n > 0.0 && n < 2.0) || !(T > 0.0) || !std::isfinite(U) || !(U > 0.0) || !std::isfinite(tp) ||
        !std::isfinite(tpp) || !std::isfinite(t3))
        return fail(ctx, TPSC_ERR_ARG, "need 0 < n < 2, T > 0, U > 0 and finite hoppings");
    if (!supported_grid(nk0, Nw0))
        return fail(ctx, TPSC_ERR_ARG, "unsupported grid nk0=" + std::to_string(nk0) + " Nw0=" + std::to_string(Nw0));
    cudaSetDevice(ctx->device);
    ctx->nk0 = nk0;
    ctx->Nw0 = Nw0;
    ctx->n = n;
    ctx->T = T;
    ctx->tp = tp;
    ctx->tpp = tpp;
    ctx->t3 = t3;
    ctx->U = U;
    ctx->nsr = n > 1.0 ? 2.0 - n : n;  // src/chi.cpp:18-19
    ctx->Usp = ctx->Uch = 0.0;
    for (double &s : ctx->scal) s = 0.0;
    for (auto &kv : ctx->grids)
        kv.second->have_chi0 = kv.second->have_V = kv.second->have_S = kv.second->have_U = false;
    ctx->have_model = true;
    ++ctx->model_id;
    return switch_grid(ctx, nk0, Nw0);
}

int tpsc_chi0(tpsc_ctx *ctx, int nq0, int nw0) {
    int rc = need_model(ctx);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    rc = switch_grid(ctx, nq0, nw0);
    if (rc) return rc;
    return run_chi0(ctx);
}

int tpsc_trace_chi0(tpsc_ctx *ctx, double out[2]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g->have_chi0) return fail(ctx, TPSC_ERR_STATE, "chi0 has not been computed");
    CK(launch_trace_chi0(g->d, g->chiq, g->cinf, g->cinf2, ctx->T, ctx->red, ctx->st));
    double r[2];
    rc = read_result(ctx, 2, r);
    if (rc) return rc;
    const double tr1 = r[0], tr = r[0] + r[1];
    const double N1 = g->d.nb;
    out[0] = tr;
    out[1] = tr + N1 * (tr1 - tr) / (N1 - 2.0 * (g->d.nb - 1));  // src/chi0.cpp:1580
    ctx->scal[TPSC_S_TR_CHI0] = out[0];
    ctx->scal[TPSC_S_TR_CHI0_CORR] = out[1];
    return TPSC_OK;
}

int tpsc_trace_diff_chi(tpsc_ctx *ctx, int channel, double Uv, double *trace, double *dtrace) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!ctx->cur->have_chi0) return fail(ctx, TPSC_ERR_STATE, "chi0 has not been computed");
    if (channel != 0 && channel != 1) return fail(ctx, TPSC_ERR_ARG, "channel must be 0 (spin) or 1 (charge)");
    return sumrule(ctx, channel, Uv, trace, dtrace);
}

int tpsc_find_Usp_Uch_grid(tpsc_ctx *ctx, int nq0, int nw0, double Usc[2]) {
    int rc = tpsc_chi0(ctx, nq0, nw0);
    if (rc) return rc;
    return roots_Usp_Uch(ctx, Usc);
}

// ---------------------------------------------------------------------------
// forward tangents of chi0 -> sum rules -> Usp, Uch, D
// ---------------------------------------------------------------------------

// the nsr of the sum rules (chi::nsr, src/chi.cpp:18-19): n or 2 - n from
// the density of tpsc_set_model, or this value until the next tpsc_set_model
// (the reference sets it once, in the chi constructor)
int tpsc_set_nsr(tpsc_ctx *ctx, double nsr) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!(nsr > 0.0 && nsr <= 1.0)) return fail(ctx, TPSC_ERR_ARG, "need 0 < nsr <= 1");
    if (nsr != ctx->nsr)
        for (auto &kv : ctx->grids) kv.second->have_U = kv.second->have_V = kv.second->have_S = false;
    ctx->nsr = nsr;
    return TPSC_OK;
}

int tpsc_set_mu_shift(tpsc_ctx *ctx, double dmu) {
    if (!ctx || !std::isfinite(dmu)) return fail(ctx, TPSC_ERR_ARG, "bad mu shift");
    if (dmu != ctx->mu_shift) {
        ctx->mu_shift = dmu;
        ++ctx->model_id;  // every grid re-derives mu0
    }
    return TPSC_OK;
}

int tpsc_sumrule_tangents(tpsc_ctx *ctx, double out[9]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!out) return fail(ctx, TPSC_ERR_ARG, "null output");
    Grid *g = ctx->cur;
    if (!g || !g->have_chi0 || !g->have_U)
        return fail(ctx, TPSC_ERR_STATE, "chi0 and the sum-rule roots have not been computed on the current grid");
    cudaSetDevice(ctx->device);
    const GridDev &d = g->d;
    const size_t n8 = d.n8, n8p = d.n8p, nb = d.nb, nw = d.nw0;
    if (!g->adj.dGrt[0]) {
        cudaError_t e = cudaSuccess;
#define A(x)                                       \
    if (e == cudaSuccess) {                        \
        e = (x);                                   \
    }
        for (int q = 0; q < 2; ++q) {
            A(dalloc(g, &g->adj.dGrt[q], (nw + 1) * n8));
            A(dalloc(g, &g->adj.dchiq[q], nb * n8p));
            A(dalloc(g, &g->adj.ddG0p[q], n8));
            A(dalloc(g, &g->adj.ddchir[q], n8));
        }
        A(dalloc(g, &g->adj.der2, n8));
        A(dalloc(g, &g->t_ddq0, n8));
        A(dalloc(g, &g->t_dcinf, n8));
        A(dalloc(g, &g->t_dcinf2, n8));
        A(dalloc(g, &g->t_der, n8));
        A(dalloc(g, &g->t_fd, n8));
#undef A
        if (e != cudaSuccess) return cuda_fail(ctx, e, "tangent buffers");
    }
    const double T = ctx->T, beta = 1.0 / T, mu0 = g->mu0, U = ctx->U, n = ctx->n, nsr = ctx->nsr;
    const double Usp = ctx->Usp, Uch = ctx->Uch;
    // the primal FP64 G(r, tau) (the mixed form keeps only its FP32 copy)
    CK(launch_gslice(d, g->Grt, mu0, T, ctx->st));
    // per octant point: xi, beta f(xi), d eps/d t' and the density weight
    const int nbk = d.nbk;
    std::vector<double> xi(n8), bf(n8), deps(n8), wf(n8);
    double sw = 0.0, swd = 0.0;
    for (int l = 0; l < nbk; ++l)
        for (int m = 0; m <= l; ++m) {
            const size_t o = m + (size_t)l * (l + 1) / 2;
            const double kx = l * PI / (nbk - 1), ky = m * PI / (nbk - 1);
            xi[o] = g->ek_host[m + (size_t)l * nbk] - mu0;
            const double z = xi[o] / T;
            const double f = z > 0 ? std::exp(-z) / (1.0 + std::exp(-z)) : 1.0 / (1.0 + std::exp(z));
            bf[o] = beta * f;
            deps[o] = -4.0 * std::cos(kx) * std::cos(ky);
            // the density's weight (k_density) times df/dxi = -beta f (1 - f)
            double w = 8;
            if (l == 0 || l == nbk - 1) w /= 2;
            if (m == 0 || m == nbk - 1) w /= 2;
            if (m == l) w /= 2;
            wf[o] = w * (-beta * f * (1.0 - f));
            sw += wf[o];
            swd += wf[o] * deps[o];
        }
    // t' moves mu0 so that the density stays n (the reference's finite-lattice
    // mu0, src/green0.cpp:182-262); the half-filled symmetric point keeps 0,
    // which is also the density root there
    const double dmu0_dtp = sw != 0.0 ? swd / sw : 0.0;
    g->t_dmu0_tp = dmu0_dtp;
    // d R / d theta at fixed (Usp, Uch) from the chi0 tangent, theta = mu, t'
    double dRsp[3] = {0, 0, 0}, dRch[3] = {0, 0, 0};
    for (int p = 1; p < 3; ++p) {
        std::vector<double2> fd(n8);
        std::vector<double> der(n8, 0.0);
        double dmu0;
        if (p == 1) {  // a shift of mu0: dxi = -1
            for (size_t o = 0; o < n8; ++o) fd[o] = make_double2(bf[o], -1.0);
            dmu0 = 1.0;
        } else {  // t': deps - dmu0/dt'; the hopping table er[2] = -t'
            for (size_t o = 0; o < n8; ++o) fd[o] = make_double2(bf[o], deps[o] - dmu0_dtp);
            if (n8 > 2) der[2] = -1.0;
            dmu0 = dmu0_dtp;
        }
        CK(cudaMemcpyAsync(g->t_fd, fd.data(), n8 * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
        CK(cudaMemcpyAsync(g->t_der, der.data(), n8 * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
        if (p == 2)
            CK(cudaMemcpyAsync(g->adj.der2, der.data(), n8 * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
        double *dchiq = g->adj.dchiq[p - 1];
        TangentBufs tb;
        tb.Grt = g->Grt;
        tb.dG0p = g->dG0p;
        tb.der = g->t_der;
        tb.fd = g->t_fd;
        tb.dGrt = g->adj.dGrt[p - 1];
        tb.dchiq = dchiq;
        tb.ddq0 = g->t_ddq0;
        tb.ddG0p = g->adj.ddG0p[p - 1];
        tb.ddchir = g->adj.ddchir[p - 1];
        CK(launch_chi0_tangent(d, tb, mu0, dmu0, T, ctx->st));
        CK(launch_chi0_tau(d, dchiq, g->t_ddq0, g->t_dcinf, g->t_dcinf2, T, ctx->st));
        CK(launch_sumrule_tan(d, g->chiq, dchiq, g->cinf, g->cinf2, g->t_dcinf, g->t_dcinf2, Usp, -1.0, T,
                              ctx->red, ctx->st));
        if ((rc = read_result(ctx, 1, &dRsp[p]))) return rc;
        CK(launch_sumrule_tan(d, g->chiq, dchiq, g->cinf, g->cinf2, g->t_dcinf, g->t_dcinf2, Uch, 1.0, T,
                              ctx->red, ctx->st));
        if ((rc = read_result(ctx, 1, &dRch[p]))) return rc;
    }
    // the roots' own derivatives (the Newton derivative of each sum rule)
    double tr, dtr_sp, dtr_ch;
    if ((rc = sumrule(ctx, 0, Usp, &tr, &dtr_sp))) return rc;
    if ((rc = sumrule(ctx, 1, Uch, &tr, &dtr_ch))) return rc;
    // R_sp = tr_sp + n - n^2/2 - nsr + Us nsr^2/(2U),
    // R_ch = tr_ch + n - n^2/2 - (nsr + Usp nsr^2/(2U) - nsr^2)  (src/chi.cpp:833-843)
    const double q2 = nsr * nsr;
    const double dRsp_dUs = dtr_sp + q2 / (2.0 * U), dRch_dUc = dtr_ch, dRch_dUsp = -q2 / (2.0 * U);
    dRsp[0] = -Usp * q2 / (2.0 * U * U);
    dRch[0] = Usp * q2 / (2.0 * U * U);
    for (int p = 0; p < 3; ++p) {
        const double dUsp = -dRsp[p] / dRsp_dUs;
        const double dUch = -(dRch[p] + dRch_dUsp * dUsp) / dRch_dUc;
        // D = Usp nsr^2/(4U) (+ 1 - nsr for n > 1)  (src/chi.cpp:370-371)
        const double dD = q2 / (4.0 * U) * dUsp - (p == 0 ? Usp * q2 / (4.0 * U * U) : 0.0);
        out[3 * p] = dUsp;
        out[3 * p + 1] = dUch;
        out[3 * p + 2] = dD;
    }
    (void)n;
    for (int i = 0; i < 9; ++i)
        if (!std::isfinite(out[i])) return fail(ctx, TPSC_ERR_NONFINITE, "non-finite sensitivity");
    return TPSC_OK;
}

int tpsc_sumrule_vjp(tpsc_ctx *ctx, const double cot[3], double grad[3]) {
    if (!ctx || !cot || !grad) return fail(ctx, TPSC_ERR_ARG, "null argument");
    double J[9];
    int rc = tpsc_sumrule_tangents(ctx, J);
    if (rc) return rc;
    for (int p = 0; p < 3; ++p) grad[p] = cot[0] * J[3 * p] + cot[1] * J[3 * p + 1] + cot[2] * J[3 * p + 2];
    return TPSC_OK;
}

// ---------------------------------------------------------------------------
// spin correlation length: host post-processing of chi0(q, 0) and Usp
// ---------------------------------------------------------------------------

// green0::find_FS(nk) (src/green0.cpp:626-676): on each line kx - ky = kx0,
// kx0 = j pi/(nk - 1), the root kx in [kx0, pi] of eps(kx, kx - kx0) - mu0 by
// the bounded find_zero from {(kx0 + pi)/2, kx0, pi}; the first line without
// a root ends the search and the later points stay (-1, -1).
void find_fs(const tpsc_ctx *ctx, double mu0, int nk, std::vector<double> &fs) {
    fs.assign(2 * (size_t)nk, -1.0);
    for (int j = 0; j < nk; ++j) {
        const double kx0 = j * PI / (nk - 1);
        const double init[3] = {0.5 * (kx0 + PI), kx0, PI}, lims[2] = {kx0, PI};
        auto f = [&](double kx, double &y) -> bool {
            y = dispk(kx, kx - kx0, ctx->tp, ctx->tpp, ctx->t3) - mu0;
            return true;
        };
        double root = 0.0;
        int nev;
        bool derr;
        if (!find_zero(f, init, &root, lims, &nev, &derr)) break;
        fs[2 * (size_t)j] = root;
        fs[2 * (size_t)j + 1] = root - kx0;
    }
}

// chi::vF_hot_spots (src/chi.cpp:420-447): the first pair of consecutive
// Fermi-surface points across kx + ky = pi (or the last pair), |grad eps| at
// their midpoint (hamiltonien::grad_ek, src/hamiltonien.cpp:125-131).
double vf_hot_spots(const tpsc_ctx *ctx, const std::vector<double> &fs, int nk) {
    double kx1 = fs[0], ky1 = fs[1], kx2 = fs[2], ky2 = fs[3];
    int j = 1;
    while ((kx1 + ky1 - PI) * (kx2 + ky2 - PI) > 0 && j < nk - 1) {
        ++j;
        kx1 = kx2;
        ky1 = ky2;
        kx2 = fs[2 * (size_t)j];
        ky2 = fs[2 * (size_t)j + 1];
    }
    const double kx = (kx1 + kx2) / 2, ky = (ky1 + ky2) / 2;
    const double tp = ctx->tp, tpp = ctx->tpp, t3 = ctx->t3;
    const double gx = 2.0 * std::sin(kx) + 4.0 * tp * std::sin(kx) * std::cos(ky) + 4.0 * tpp * std::sin(2 * kx) +
                      4 * t3 * (2.0 * std::sin(2 * kx) * std::cos(ky) + std::cos(2 * ky) * std::sin(kx));
    const double gy = 2.0 * std::sin(ky) + 4.0 * tp * std::cos(kx) * std::sin(ky) + 4.0 * tpp * std::sin(2 * ky) +
                      4 * t3 * (std::cos(2 * kx) * std::sin(ky) + 2.0 * std::sin(2 * ky) * std::cos(kx));
    return std::sqrt(gx * gx + gy * gy);
}

int tpsc_sp_corr_length(tpsc_ctx *ctx, double out[7]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    return tpsc_sp_corr_length_fs(ctx, ctx->cur->mu0, out);
}

int tpsc_sp_corr_length_fs(tpsc_ctx *ctx, double mu_fs, double out[7]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!out) return fail(ctx, TPSC_ERR_ARG, "null output");
    Grid *g = ctx->cur;
    if (!g || !g->have_chi0 || !g->have_U)
        return fail(ctx, TPSC_ERR_STATE, "chi0 and Usp have not been computed on the current grid");
    cudaSetDevice(ctx->device);
    const GridDev &d = g->d;
    const int nbq = d.nbk;
    // chi0(q, 0): row j = 0 of the column-block layout, 4 columns per block
    std::vector<double> a((size_t)d.n8p);
    CK(cudaMemcpy2DAsync(a.data(), 4 * sizeof(double), g->chiq, (size_t)d.nb * 4 * sizeof(double),
                         4 * sizeof(double), d.n8p / 4, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    const int nkfs = 10001;
    std::vector<double> fs;
    find_fs(ctx, mu_fs, nkfs, fs);
    const double vF = vf_hot_spots(ctx, fs, nkfs);
    // chi::sp_corr_length (src/chi.cpp:450-718): half maximum of
    // chi_sp(q, 0) = chi0/(1 - Usp chi0/2) around qmax along y and x, and the
    // asymptotic (Ornstein-Zernike) lengths from the second difference of chi0
    const double Usp = ctx->Usp, chi0max = ctx->scal[TPSC_S_CHI0MAX];
    const int qx = (int)ctx->scal[TPSC_S_QMAX0], qy = (int)ctx->scal[TPSC_S_QMAX1];
    auto csp = [&](size_t i) { return a[i] / (1.0 - Usp * a[i] / 2.0); };
    auto oi = [](int x, int y) { return (size_t)y + ((size_t)x * (x + 1)) / 2; };
    const double dq = PI / (nbq - 1), half = chi0max / (1.0 - Usp * chi0max / 2.0) / 2.0;
    int l = qx, m = 0;
    const size_t base = ((size_t)l * (l + 1)) / 2;
    double cur = csp(base), prev = cur;
    while (cur < half && m <= qy) {
        ++m;
        prev = cur;
        cur = csp(base + m);
    }
    double q0 = (m - 1) * dq;
    double qHM = dq * (half - prev) / (cur - prev) + q0;
    const double xi_y = 1.0 / (qy * dq - qHM);
    double xi_x = xi_y;
    m = qy;
    l = m;
    cur = csp(oi(l, m));
    if (cur < half) {
        while (cur < half && l <= qx) {
            ++l;
            prev = cur;
            cur = csp(oi(l, m));
        }
        q0 = (l - 1) * dq;
        qHM = dq * (half - prev) / (cur - prev) + q0;
        xi_x = 1.0 / (qx * dq - qHM);
    }
    const double fac = (double)(nbq - 1) * (nbq - 1) / (PI * PI);
    double xi0_x, xi0_y, xiAs_x, xiAs_y;
    if (qx == nbq - 1 && qy == nbq - 1) {
        const double dchi2 = 2.0 * (a[base + nbq - 2] - chi0max) * fac;
        xi0_x = std::sqrt(-0.5 * dchi2 / chi0max);
        xiAs_x = xi0_x * std::sqrt(Usp / (2.0 / chi0max - Usp));
        xi0_y = xi0_x;
        xiAs_y = xiAs_x;
    } else {
        int x = qx, y = qy - 1;
        if (y < 0) y = qy + 1;
        const double cl = a[oi(x, y)];
        y = qy;
        const double cm = a[oi(x, y)];
        y = qy + 1;
        if (y > x) {
            x = qy + 1;
            y = qx;
        }
        const double cr = a[oi(x, y)];
        double dchi2 = (cr - 2 * cm + cl) * fac;
        xi0_y = std::sqrt(-0.5 * dchi2 / chi0max);
        xiAs_y = xi0_y * std::sqrt(Usp / (2.0 / chi0max - Usp));
        x = qx - 1;
        y = qy;
        if (y > x) {
            x = qy;
            y = qx - 1;
            if (y < 0) y = qx + 1;
        }
        const double dl = a[oi(x, y)];
        x = qx;
        y = qy;
        const double dm = a[oi(x, y)];
        x = qx + 1;
        if (x > nbq - 1) x = qx - 1;
        const double dr = a[oi(x, y)];
        dchi2 = (dr - 2 * dm + dl) * fac;
        xi0_x = std::sqrt(-0.5 * dchi2 / chi0max);
        xiAs_x = xi0_x * std::sqrt(Usp / (2.0 / chi0max - Usp));
    }
    const double r[7] = {vF, xi_y, xi_x, xiAs_y, xiAs_x, xi0_y, xi0_x};
    for (int i = 0; i < 7; ++i) out[i] = r[i];
    return TPSC_OK;
}

int tpsc_find_Usp_Uch(tpsc_ctx *ctx) {
    int rc = need_model(ctx);
    if (rc) return rc;
    double Us_half[2], Us_full[2];
    // src/chi.cpp:285-306: (nbq-1, nwmax) then twice that
    rc = tpsc_find_Usp_Uch_grid(ctx, ctx->nk0 / 2, ctx->Nw0 / 2, Us_half);
    if (rc) return rc;
    rc = tpsc_find_Usp_Uch_grid(ctx, ctx->nk0, ctx->Nw0, Us_full);
    if (rc) return rc;
    ctx->scal[TPSC_S_DIFRELSP] = std::fabs((Us_full[0] - Us_half[0]) / Us_full[0]);
    ctx->scal[TPSC_S_DIFRELCH] = std::fabs((Us_full[1] - Us_half[1]) / Us_full[1]);
    set_dblocc(ctx);
    return TPSC_OK;
}

int tpsc_vertex(tpsc_ctx *ctx) {
    int rc = need_model(ctx);
    if (rc) return rc;
    return run_vertex(ctx);
}

int tpsc_self_energy(tpsc_ctx *ctx) {
    int rc = need_model(ctx);
    if (rc) return rc;
    return run_self(ctx);
}

int tpsc_trace_self_G(tpsc_ctx *ctx, double out[2]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    return trace_self_G(ctx, out);
}

int tpsc_trace_diff_G(tpsc_ctx *ctx, double mu, double *trace, double *dtrace) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!ctx->cur->have_S) return fail(ctx, TPSC_ERR_STATE, "the self-energy has not been computed");
    return trace_diff_G(ctx, mu, trace, dtrace);
}

int tpsc_find_mu(tpsc_ctx *ctx) {
    int rc = need_model(ctx);
    if (rc) return rc;
    return find_mu(ctx);
}

int tpsc_solve(tpsc_ctx *ctx) {
    int rc = need_model(ctx);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    if (ctx->form & TPSC_FORM_NEWTON) {
        // no host round trip from the chi0 stage to the one readback at the end
        if ((rc = switch_grid(ctx, ctx->nk0, ctx->Nw0))) return rc;
        if ((rc = newton_solve(ctx))) return rc;
        return finish_solve(ctx);
    }
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    rc = switch_grid(ctx, ctx->nk0, ctx->Nw0);
    if (rc) return rc;
    rc = run_chi0(ctx);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    double Usc[2];
    rc = roots_Usp_Uch(ctx, Usc);
    if (rc) return rc;
    set_dblocc(ctx);
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    rc = run_vertex(ctx);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev[3], ctx->st));
    rc = run_self(ctx, !(ctx->form & TPSC_FORM_NEWTON));
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev[4], ctx->st));
    // the Newton form computes traceSelfG in the same Sigma pass as the find_mu moments
    if (!(ctx->form & TPSC_FORM_NEWTON)) {
        double tsg[2];
        rc = trace_self_G(ctx, tsg);
        if (rc) return rc;
    }
    rc = find_mu(ctx);
    if (rc) return rc;
    CK(cudaEventRecord(ctx->ev[5], ctx->st));
    return finish_solve(ctx);
}

namespace {
// ---------------------------------------------------------------------------
// many points of one shape at once: one launch per stage (tpsc_solve_points)
// ---------------------------------------------------------------------------
constexpr int kGroupMax = 128;  // points per group launch (the root searches' grid is shared out)

// the group of shape (nk0, nw0) with arenas for at least P points
int group_alloc(tpsc_ctx *ctx, int nk0, int nw0, int P, Group **out) {
    const auto key = std::make_pair(nk0, nw0);
    auto it = ctx->groups.find(key);
    if (it != ctx->groups.end()) {
        if (it->second->cap >= P) {
            *out = it->second;
            return TPSC_OK;
        }
        CK(cudaStreamSynchronize(ctx->st));
        free_group(it->second);
        ctx->groups.erase(it);
    }
    Grid *g = nullptr;
    int rc = build_grid(ctx, nk0, nw0, &g);  // the shape tables
    if (rc) return rc;
    Group *q = new Group;
    q->nk0 = nk0;
    q->nw0 = nw0;
    q->cap = P;
    q->d = g->d;
    const GridDev &d = q->d;
    const size_t n8 = d.n8, n8p = d.n8p, nb = d.nb, nw = nw0, NO = nw0 / 2;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) & ~(size_t)255;
        return o;
    };
    const size_t o_ek = take(n8 * 8), o_er = take(n8 * 8), o_tq = take(kTailQ * 8), o_tp = take(kTailP * 8),
                 o_pp = take(kPP * 8);
    q->in_bytes = off;
    q->res_off = take(kGroupRes * 8);
    const size_t o_gk = take(n8 * 16), o_grt = take((nw + 1) * n8 * 4), o_chirt = take(nb * n8p * 8),
                 o_chiq = take(nb * n8p * 8), o_V = take(nb * n8p * 8), o_dG0p = take(n8 * 8),
                 o_dchirt0 = take(n8 * 8), o_dchiqt0 = take(n8 * 8), o_cinf = take(n8 * 8), o_cinf2 = take(n8 * 8),
                 o_dS = take(2 * n8p * 8), o_sigt = take((nw + 1) * n8p * 8), o_S = take(NO * n8p * 16),
                 o_s2 = take(n8 * 8), o_s3 = take(n8 * 8), o_s4 = take(n8 * 8), o_mom = take(nb * kMomP * 8),
                 o_cmax = take(nb * 8), o_msuf = take((nb + 1) * kMomP * 8), o_csuf = take((nb + 1) * 8),
                 o_tailm = take((kMomP + 1) * 8), o_redp = take(4 * kMaxBlocks * 8), o_redt = take(16),
                 o_redmp = take((size_t)std::max(2 * kMomP + 2, kSigmaMomNV) * kMaxBlocks * 8),
                 o_redmt = take(16), o_rootp = take(2 * kRootVals * kRootMaxBlocks * 8);
    q->arena = (long long)off;
    cudaError_t e = cudaMalloc(&q->base, (size_t)P * off);
    if (e == cudaSuccess) e = cudaMemsetAsync(q->base, 0, (size_t)P * off, ctx->st);
    if (e == cudaSuccess) e = cudaHostAlloc(&q->h_in, (size_t)P * q->in_bytes, cudaHostAllocDefault);
    if (e == cudaSuccess) e = cudaHostAlloc(&q->h_res, (size_t)P * kGroupRes * sizeof(double), cudaHostAllocDefault);
    if (e != cudaSuccess) {
        free_group(q);
        return cuda_fail(ctx, e, "group allocation");
    }
    char *b0 = q->base;
    auto P0 = [&](size_t o) { return b0 + o; };
    q->d.ek = reinterpret_cast<double *>(P0(o_ek));
    q->d.er = reinterpret_cast<double *>(P0(o_er));
    q->d.tailq = reinterpret_cast<double *>(P0(o_tq));
    q->d.tailP = reinterpret_cast<double *>(P0(o_tp));
    q->d.gk = reinterpret_cast<double2 *>(P0(o_gk));
    q->pp = reinterpret_cast<double *>(P0(o_pp));
    double *res = reinterpret_cast<double *>(P0(q->res_off));
    q->red.result = res;                  // [0, 8)
    q->dres = res + 8;                    // [8, 16)
    q->roots.bar = reinterpret_cast<unsigned *>(res + 16);  // [16, 20): 8 words
    q->mu_out = res + 20;                 // [20, 28)
    q->sinf = res + 28;                   // [28]
    q->redm.result = res + 32;            // [32, 64)
    q->Grt32 = reinterpret_cast<float *>(P0(o_grt));
    q->chirt = reinterpret_cast<double *>(P0(o_chirt));
    q->chiq = reinterpret_cast<double *>(P0(o_chiq));
    q->V = reinterpret_cast<double *>(P0(o_V));
    q->dG0p = reinterpret_cast<double *>(P0(o_dG0p));
    q->dchirt0 = reinterpret_cast<double *>(P0(o_dchirt0));
    q->dchiqt0 = reinterpret_cast<double *>(P0(o_dchiqt0));
    q->cinf = reinterpret_cast<double *>(P0(o_cinf));
    q->cinf2 = reinterpret_cast<double *>(P0(o_cinf2));
    q->dS = reinterpret_cast<double *>(P0(o_dS));
    q->sigt = reinterpret_cast<double *>(P0(o_sigt));
    q->S = reinterpret_cast<double2 *>(P0(o_S));
    q->s2 = reinterpret_cast<double *>(P0(o_s2));
    q->s3 = reinterpret_cast<double *>(P0(o_s3));
    q->s4 = reinterpret_cast<double *>(P0(o_s4));
    q->mom = reinterpret_cast<double *>(P0(o_mom));
    q->cmax = reinterpret_cast<double *>(P0(o_cmax));
    q->msuf = reinterpret_cast<double *>(P0(o_msuf));
    q->csuf = reinterpret_cast<double *>(P0(o_csuf));
    q->tailm = reinterpret_cast<double *>(P0(o_tailm));
    q->red.partial = reinterpret_cast<double *>(P0(o_redp));
    q->red.ticket = reinterpret_cast<unsigned *>(P0(o_redt));
    q->redm.partial = reinterpret_cast<double *>(P0(o_redmp));
    q->redm.ticket = reinterpret_cast<unsigned *>(P0(o_redmt));
    q->roots.partial = reinterpret_cast<double *>(P0(o_rootp));
    // the density root's result in the scalars' spare slots 10, 11
    q->mu0r.result = q->pp + 10;
    ctx->groups[key] = q;
    *out = q;
    return TPSC_OK;
}

// the input block of one point (params row nk0, Nw0, n, T, t', t'', t3, U):
// eps_k on the octant, the hopping table, the tail power sums, the scalars
void group_point_inputs(const Group *q, const double *p, char *dst) {
    const GridDev &d = q->d;
    const double n = p[2], T = p[3], tp = p[4], tpp = p[5], t3 = p[6], U = p[7];
    size_t off = 0;
    auto next = [&](size_t bytes) {
        double *r = reinterpret_cast<double *>(dst + off);
        off += (bytes + 255) & ~(size_t)255;
        return r;
    };
    double *ek = next((size_t)d.n8 * 8), *er = next((size_t)d.n8 * 8), *tq = next(kTailQ * 8),
           *tpw = next(kTailP * 8), *pp = next(kPP * 8);
    octant_eps(d.nbk, tp, tpp, t3, ek, nullptr);
    std::fill(er, er + d.n8, 0.0);
    er[1] = -1;
    er[2] = -tp;
    er[3] = -tpp;
    er[4] = -t3;
    tail_power_sums(q->nw0, T, tq, tpw);
    std::fill(pp, pp + kPP, 0.0);
    pp[kPpT] = T;
    pp[kPpU] = U;
    pp[kPpN] = n;
    pp[kPpNsr] = n > 1.0 ? 2.0 - n : n;  // src/chi.cpp:18-19
    pp[kPpNormFact] = T / ((double)q->nk0 * q->nk0);
    int jc;
    double wc;
    mu_series_cut(q->nw0, T, &jc, &wc);
    pp[kPpJc] = jc;
    pp[kPpWc] = wc;
    // the reference's shortcut for mu0 (green0::find_mu): half filling without t', t''
    pp[kPpMu0Fixed] = (n == 1.0 && tp == 0 && tpp == 0) ? 1.0 : 0.0;
}

// the Newton-form mixed solve of the group's first P points, queued on
// ctx->st: inputs up, one launch per stage over the P points, results down
int group_queue(tpsc_ctx *ctx, Group *q, int P, cudaStream_t st, int root_cap) {
    const GridDev &d = q->d;
    Bp b;
    b.P = P;
    b.arena = q->arena;
    b.pp = q->pp;
    CK(cudaMemcpy2DAsync(q->base, (size_t)q->arena, q->h_in, q->in_bytes, q->in_bytes, P, cudaMemcpyHostToDevice,
                         st));
    CK(launch_mu0_newton(d, 0.0, 0.0, q->mu0r, st, b));
    CK(launch_gslice32(d, q->Grt32, 0.0, 0.0, st, b));
    CK(launch_chi0_boundary(d, (const float *)q->Grt32, 0.0, 0.0, q->dG0p, q->dchirt0, q->dchiqt0, st, b));
    CK(launch_chi0_slice32(d, q->Grt32, q->chirt, q->chiq, st, b));
    CK(launch_chi0_tau(d, q->chiq, q->dchiqt0, q->cinf, q->cinf2, 0.0, st, b));
    CK(launch_chi0max(d, q->chiq, q->red, st, b));
    CK(launch_chi0_moments(d, q->chiq, q->mom, q->cmax, st, b));
    CK(launch_tail_moments(d, q->cinf, q->cinf2, 0.0, q->redm, st, b));
    CK(launch_moment_suffix(d, q->mom, q->cmax, q->redm.result, q->msuf, q->csuf, q->tailm, st, b));
    RootScratch rs = q->roots;
    rs.max_blocks = root_cap;
    rs.reset_sr = rs.reset_mu = true;
    rs.out = q->dres;
    CK(launch_sumrule_roots(d, q->chiq, q->cinf, q->cinf2, q->msuf, q->csuf, q->tailm, 0.0, 0.0, 0.0, 0.0, 0.0, rs,
                            st, q->red.result, 2 * EPS, b));
    CK(launch_vertex_q32(d, q->chiq, q->V, 0.0, q->dres, 0.0, st, b));
    CK(launch_vertex_tau(d, q->V, q->chirt, 0.0, q->dres, st, b));
    CK(launch_sigma_boundary(d, (const float *)q->Grt32, q->V, q->dchirt0, q->dG0p, 0.0, 0.0, q->dres, q->dS, st,
                             b));
    CK(launch_sigma_slice32(d, q->Grt32, q->V, q->sigt, st, b));
    CK(launch_sigma_tau(d, q->sigt, q->dS, q->S, q->s2, q->s3, q->s4, q->sinf, 0.0, st, b));
    CK(launch_sigma_moments(d, q->S, q->s2, q->s3, q->s4, q->sinf, 0.0, 0.0, 0, q->redm, st, b));
    rs.out = q->mu_out;
    CK(launch_mu_roots(d, q->S, q->s2, q->s3, q->s4, q->sinf, q->redm.result, 0.0, 0.0, 0, 0.0, rs, st, b));
    // the results block and the scalars (mu0 and its search) of every point
    CK(cudaMemcpy2DAsync(q->h_res, kGroupRes * sizeof(double), q->base + q->res_off, (size_t)q->arena,
                         kGroupRes * sizeof(double), P, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpy2DAsync(q->h_in + (q->in_bytes - ((kPP * 8 + 255) & ~(size_t)255)), q->in_bytes, q->pp,
                         (size_t)q->arena, kPP * sizeof(double), P, cudaMemcpyDeviceToHost, st));
    return TPSC_OK;
}

// the group's solve as one graph launch: captured on the first call after a
// direct one (the kernels' one-time attribute calls happen outside a
// capture), replayed while P stays the same
int group_run(tpsc_ctx *ctx, Group *q, int P, cudaStream_t st, int root_cap) {
    if (q->gexec_tiles != tau_tiles_version()) {
        // the tau transforms' plans changed: launch directly, then capture again
        q->gexec_P = 0;
        q->gexec_tiles = tau_tiles_version();
    }
    if (q->gexec && q->gexec_P == P) {
        CK(cudaGraphLaunch(q->gexec, st));
        return TPSC_OK;
    }
    if (q->gexec_P != -P) {
        // first call with this P: direct launches
        int rc = group_queue(ctx, q, P, st, root_cap);
        if (rc) return rc;
        q->gexec_P = -P;
        return TPSC_OK;
    }
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = group_queue(ctx, q, P, st, root_cap);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess) return cuda_fail(ctx, e, "group capture");
    if (q->gexec) cudaGraphExecDestroy(q->gexec);
    q->gexec = nullptr;
    e = cudaGraphInstantiate(&q->gexec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "group graph instantiation");
    q->gexec_P = P;
    CK(cudaGraphLaunch(q->gexec, st));
    return TPSC_OK;
}

// the scalars of point p of the group (the Newton-form solve's checks and
// results, as newton_finish and switch_grid leave them) -> out; its status
int group_point_result(const Group *q, int p, const double *prm, double *out, std::string &msg) {
    const double *r = q->h_res + (size_t)p * kGroupRes;
    const double *pp = reinterpret_cast<const double *>(q->h_in + (size_t)p * q->in_bytes +
                                                        (q->in_bytes - ((kPP * 8 + 255) & ~(size_t)255)));
    const double n = prm[2], U = prm[7], nsr = n > 1.0 ? 2.0 - n : n;
    for (int k = 0; k < TPSC_S_COUNT; ++k) out[k] = 0.0;
    out[TPSC_S_MU0] = pp[kPpMu0];
    if (!std::isfinite(pp[kPpMu0]) || pp[11] >= 200) {
        msg = "mu0 not found";
        return TPSC_ERR_NO_ROOT;
    }
    out[TPSC_S_CHI0MAX] = r[0];
    out[TPSC_S_QMAX0] = r[1];
    out[TPSC_S_QMAX1] = r[2];
    if (!std::isfinite(r[0]) || r[0] <= 0.0) {
        msg = "chi0(q, 0) has no positive maximum";
        return TPSC_ERR_NONFINITE;
    }
    unsigned bar[8];
    std::memcpy(bar, r + 16, sizeof(bar));
    if (bar[2]) {
        msg = "device root search: grid barrier timed out";
        return TPSC_ERR_CUDA;
    }
    if (r[12] != 1.0 || r[13] != 1.0) {
        msg = r[12] != 1.0 ? "Usp not found" : "Uch not found";
        return TPSC_ERR_NO_ROOT;
    }
    out[TPSC_S_USP] = r[8];
    out[TPSC_S_UCH] = r[9];
    out[TPSC_S_EVALS_SP] = r[10];
    out[TPSC_S_EVALS_CH] = r[11];
    double D = r[8] / U * nsr * nsr / 4.0;  // src/chi.cpp:370-371
    if (n > 1.0) D += 1.0 - nsr;
    out[TPSC_S_DBLOCC] = D;
    if (bar[6]) {
        msg = "device mu search: grid barrier timed out";
        return TPSC_ERR_CUDA;
    }
    out[TPSC_S_SIGMA_INF] = r[28];
    out[TPSC_S_TR_SG] = r[32];
    out[TPSC_S_TR_SG_ASYMP] = r[32] + r[33];
    if (r[22] != 1.0) {
        msg = "mu not found";
        return TPSC_ERR_NO_ROOT;
    }
    out[TPSC_S_MU] = r[20];
    out[TPSC_S_EVALS_MU] = r[21];
    out[TPSC_S_TR_SG2] = r[23];
    out[TPSC_S_DBLOCC_SG2] = (r[23] + U * n * n / 4.0) / U;
    for (int k = 0; k < TPSC_S_COUNT; ++k)
        if (!std::isfinite(out[k])) {
            msg = "non-finite scalar result";
            return TPSC_ERR_NONFINITE;
        }
    return TPSC_OK;
}
}  // namespace

int tpsc_solve_points(tpsc_ctx *ctx, int npts, const double *params, double *results, int *status, double *ms) {
    if (!ctx) return fail(nullptr, TPSC_ERR_ARG, "null context");
    if (npts < 0 || (npts > 0 && (!params || !results || !status))) return fail(ctx, TPSC_ERR_ARG, "bad arguments");
    cudaSetDevice(ctx->device);
    // valid points by shape, in input order
    std::map<std::pair<int, int>, std::vector<int>> shapes;
    for (int i = 0; i < npts; ++i) {
        const double *p = params + (size_t)i * 8;
        double *out = results + (size_t)i * TPSC_S_COUNT;
        for (int k = 0; k < TPSC_S_COUNT; ++k) out[k] = NAN;
        const bool ok = p[0] == std::floor(p[0]) && p[1] == std::floor(p[1]) && p[0] >= 8 && p[0] <= 256 &&
                        p[1] >= 16 && p[1] <= 4096 && supported_grid((int)p[0], (int)p[1]) && p[2] > 0.0 &&
                        p[2] < 2.0 && p[3] > 0.0 && p[7] > 0.0 && std::isfinite(p[7]) && std::isfinite(p[4]) &&
                        std::isfinite(p[5]) && std::isfinite(p[6]);
        status[i] = ok ? TPSC_OK : TPSC_ERR_ARG;
        if (ok) shapes[std::make_pair((int)p[0], (int)p[1])].push_back(i);
    }
    // the groups' arenas first (allocation waits for the device)
    for (auto &kv : shapes) {
        Group *q = nullptr;
        const int P = (int)std::min<size_t>(kGroupMax, kv.second.size());
        int rc = group_alloc(ctx, kv.first.first, kv.first.second, P, &q);
        if (rc) return rc;
    }
    CK(cudaStreamSynchronize(ctx->st));
    const auto t0 = std::chrono::steady_clock::now();
    std::string first_msg;
    // every group queued without a wait (the host builds the next group's
    // tables while the device runs the previous ones), largest first, on two
    // streams by least queued work (a group's root searches then take half
    // of the resident grid, so that both streams' fit on the GPU together); a
    // shape with more than kGroupMax points waits for its previous chunk
    // before its staging buffers are refilled
    struct Chunk {
        Group *q;
        size_t c0;
        int P;
        const std::vector<int> *idx;
    };
    std::vector<Chunk> done;
    std::vector<std::pair<double, const std::pair<const std::pair<int, int>, std::vector<int>> *>> order;
    for (auto &kv : shapes)
        order.push_back({-(double)kv.first.first * kv.first.first * kv.first.second * kv.second.size(), &kv});
    std::sort(order.begin(), order.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    const int ns = ctx->group_streams;
    for (int k = 0; k + 2 < ns; ++k)
        if (!ctx->gst[k]) CK(cudaStreamCreateWithFlags(&ctx->gst[k], cudaStreamNonBlocking));
    cudaStream_t streams[4] = {ctx->st, ctx->st2, ctx->gst[0], ctx->gst[1]};
    double load[4] = {0.0, 0.0, 0.0, 0.0};
    int dev_sms = 0;
    CK(cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, ctx->device));
    const int root_cap = std::max(8, 2 * dev_sms / ns);  // two blocks per SM, shared out
    auto collect = [&](const Chunk &ch) {
        for (int k = 0; k < ch.P; ++k) {
            const int i = (*ch.idx)[ch.c0 + k];
            std::string msg;
            status[i] = group_point_result(ch.q, k, params + (size_t)i * 8, results + (size_t)i * TPSC_S_COUNT, msg);
            if (status[i] && first_msg.empty()) first_msg = "point " + std::to_string(i) + ": " + msg;
        }
    };
    for (const auto &o : order) {
        const std::vector<int> &idx = o.second->second;
        Group *q = ctx->groups[o.second->first];
        int s = 0;
        for (int k = 1; k < ns; ++k)
            if (load[k] < load[s]) s = k;
        load[s] += -o.first;
        for (size_t c0 = 0; c0 < idx.size(); c0 += kGroupMax) {
            const int P = (int)std::min<size_t>(kGroupMax, idx.size() - c0);
            if (c0 > 0) {
                CK(cudaStreamSynchronize(streams[s]));
                collect(done.back());
                done.pop_back();
            }
            for (int k = 0; k < P; ++k)
                group_point_inputs(q, params + (size_t)idx[c0 + k] * 8, q->h_in + (size_t)k * q->in_bytes);
            int rc = group_run(ctx, q, P, streams[s], root_cap);
            if (rc) return rc;
            done.push_back({q, c0, P, &idx});
        }
    }
    for (int k = 0; k < ns; ++k) CK(cudaStreamSynchronize(streams[k]));
    for (const Chunk &ch : done) collect(ch);
    const auto t1 = std::chrono::steady_clock::now();
    if (ms) *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    ctx->err = first_msg;
    return TPSC_OK;
}

int tpsc_set_group_streams(tpsc_ctx *ctx, int n) {
    if (!ctx) return fail(nullptr, TPSC_ERR_ARG, "null context");
    if (n < 1 || n > 4) return fail(ctx, TPSC_ERR_ARG, "need 1 <= n <= 4");
    if (n != ctx->group_streams)
        for (auto &kv : ctx->groups) kv.second->gexec_P = 0;  // the root grids' cap changes: capture again
    ctx->group_streams = n;
    return TPSC_OK;
}

int tpsc_get_scalars(tpsc_ctx *ctx, double *out, int n) {
    if (!ctx || !out || n < 0) return fail(ctx, TPSC_ERR_ARG, "bad arguments");
    for (int i = 0; i < n && i < TPSC_S_COUNT; ++i) out[i] = ctx->scal[i];
    return TPSC_OK;
}

int tpsc_get_dims(tpsc_ctx *ctx, int dims[4]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    const GridDev &d = ctx->cur->d;
    dims[0] = d.nk0;
    dims[1] = d.nw0;
    dims[2] = d.nbk;
    dims[3] = d.n8;
    return TPSC_OK;
}

int tpsc_get_ek(tpsc_ctx *ctx, double *ek) {
    int rc = need_model(ctx);
    if (rc) return rc;
    std::memcpy(ek, ctx->cur->ek_host.data(), ctx->cur->ek_host.size() * sizeof(double));
    return TPSC_OK;
}

int tpsc_get_chi0(tpsc_ctx *ctx, double *chiqw, double *chi0_inf, double *chi0_inf2, double *dtau_chirt0) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g->have_chi0) return fail(ctx, TPSC_ERR_STATE, "chi0 has not been computed");
    const GridDev &d = g->d;
    if (chiqw) {
        const size_t bytes = (size_t)d.nb * d.n8 * sizeof(double);
        if ((rc = ensure_stage(ctx, bytes))) return rc;
        CK(launch_unblock(g->chiq, (double *)ctx->stage, d.nb, d.nb, d.n8, ctx->st));
        if ((rc = copy_out(ctx, chiqw, ctx->stage, bytes))) return rc;
    }
    if (chi0_inf && (rc = copy_out(ctx, chi0_inf, g->cinf, d.n8 * sizeof(double)))) return rc;
    if (chi0_inf2 && (rc = copy_out(ctx, chi0_inf2, g->cinf2, d.n8 * sizeof(double)))) return rc;
    if (dtau_chirt0 && (rc = copy_out(ctx, dtau_chirt0, g->dchirt0, d.n8 * sizeof(double)))) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return TPSC_OK;
}

int tpsc_get_vertex(tpsc_ctx *ctx, double *vertex_rt) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g->have_V) return fail(ctx, TPSC_ERR_STATE, "the vertex has not been computed");
    const GridDev &d = g->d;
    const size_t bytes = (size_t)d.nb * d.n8 * sizeof(double);
    if ((rc = ensure_stage(ctx, bytes))) return rc;
    CK(launch_unblock(g->V, (double *)ctx->stage, d.nb, d.nb, d.n8, ctx->st));
    if ((rc = copy_out(ctx, vertex_rt, ctx->stage, bytes))) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return TPSC_OK;
}

int tpsc_get_self(tpsc_ctx *ctx, double *self_kw, double *s2, double *s3, double *s4) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g->have_S) return fail(ctx, TPSC_ERR_STATE, "the self-energy has not been computed");
    const GridDev &d = g->d;
    if (self_kw) {
        const size_t bytes = (size_t)(d.nw0 / 2) * d.n8 * sizeof(double2);
        if ((rc = ensure_stage(ctx, bytes))) return rc;
        CK(launch_unblock_c(g->S, (double2 *)ctx->stage, d.nw0 / 2, d.nw0 / 2, d.n8, ctx->st));
        if ((rc = copy_out(ctx, self_kw, ctx->stage, bytes))) return rc;
    }
    if (s2 && (rc = copy_out(ctx, s2, g->s2, d.n8 * sizeof(double)))) return rc;
    if (s3 && (rc = copy_out(ctx, s3, g->s3, d.n8 * sizeof(double)))) return rc;
    if (s4 && (rc = copy_out(ctx, s4, g->s4, d.n8 * sizeof(double)))) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return TPSC_OK;
}

// Sigma(k, tau_j) of the last Sigma stage, j <= Nw0 (the spline nodes of
// green::calc_Self_FFT_spline, src/green.cpp:1872-1885, 1936-1950)
int tpsc_get_sigma_tau(tpsc_ctx *ctx, int j, double *out) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    const GridDev &d = g->d;
    if (!out || j < 0 || j > d.nw0) return fail(ctx, TPSC_ERR_ARG, "need 0 <= j <= Nw0 and an output array");
    if (!g->have_S) return fail(ctx, TPSC_ERR_STATE, "the self-energy has not been computed");
    cudaSetDevice(ctx->device);
    const size_t bytes = (size_t)d.n8 * sizeof(double);
    if ((rc = ensure_stage(ctx, bytes))) return rc;
    CK(launch_take_row(g->sigt, d.nw0 + 1, j, d.n8, (double *)ctx->stage, ctx->st));
    if ((rc = copy_out(ctx, out, ctx->stage, bytes))) return rc;
    CK(cudaStreamSynchronize(ctx->st));
    return TPSC_OK;
}

// The tiling of the three tau transforms for the current grid's Nw0, picked
// by timing: each transform runs in both tilings (one column pair per CTA,
// four columns per CTA) reps times on this grid's buffers after one warm-up,
// and the faster stays (process-wide).  ms[2 kind + tile] receives the mean
// times (kind 0 chi0, 1 V, 2 Sigma).  The transforms run in place, so the
// grid's stage results are stale afterwards: the next solve recomputes them.
int tpsc_tune_tau_tiles(tpsc_ctx *ctx, int reps, double ms[6]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g || !g->have_S) return fail(ctx, TPSC_ERR_STATE, "tune after a solve on the current grid");
    if (reps < 1 || reps > 100) return fail(ctx, TPSC_ERR_ARG, "need 1 <= reps <= 100");
    cudaSetDevice(ctx->device);
    const GridDev &d = g->d;
    cudaEvent_t a = ctx->ev[0], b = ctx->ev[1];
    for (int kind = 0; kind < 3; ++kind) {
        double best = 0.0;
        int pick = 0;
        for (int tile = 0; tile < 2; ++tile) {
            set_tau_tile(kind, d.nw0, tile);
            auto run = [&]() -> cudaError_t {
                if (kind == kTauChi0) return launch_chi0_tau(d, g->chiq, g->dchiqt0, g->cinf, g->cinf2, ctx->T, ctx->st);
                if (kind == kTauVertex) return launch_vertex_tau(d, g->V, g->chirt, ctx->U, ctx->dres, ctx->st);
                return launch_sigma_tau(d, g->sigt, g->dS, g->S, g->s2, g->s3, g->s4, g->sinf, ctx->T, ctx->st);
            };
            CK(run());
            CK(cudaEventRecord(a, ctx->st));
            for (int r = 0; r < reps; ++r) CK(run());
            CK(cudaEventRecord(b, ctx->st));
            CK(cudaEventSynchronize(b));
            float t = 0;
            CK(cudaEventElapsedTime(&t, a, b));
            const double mean = t / reps;
            if (ms) ms[2 * kind + tile] = mean;
            if (tile == 0 || mean < best) {
                best = mean;
                pick = tile;
            }
        }
        set_tau_tile(kind, d.nw0, pick);
    }
    g->have_chi0 = g->have_V = g->have_S = g->have_mom = g->have_U = false;
    return TPSC_OK;
}

// The FFT plan and tiling of the three tau transforms for the current grid's
// Nw0: one column pair per CTA with radix-16 passes (0), four columns per CTA
// (1), one pair per CTA with radix-8 passes (2, Nw0 <= 2048: twice the
// threads in the FFT, one more pass) -- each timed as in
// tpsc_tune_tau_tiles, the fastest kept; ms[3 kind + plan] (plan 2 is 0
// where it does not apply).
int tpsc_tune_tau_plans(tpsc_ctx *ctx, int reps, double ms[9]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g || !g->have_S) return fail(ctx, TPSC_ERR_STATE, "tune after a solve on the current grid");
    if (reps < 1 || reps > 100) return fail(ctx, TPSC_ERR_ARG, "need 1 <= reps <= 100");
    cudaSetDevice(ctx->device);
    const GridDev &d = g->d;
    cudaEvent_t a = ctx->ev[0], b = ctx->ev[1];
    const int nplans = d.nw0 <= 2048 ? 3 : 2;
    for (int kind = 0; kind < 3; ++kind) {
        double best = 0.0;
        int pick = 0;
        for (int plan = 0; plan < 3; ++plan) {
            if (ms) ms[3 * kind + plan] = 0.0;
            if (plan >= nplans) continue;
            set_tau_tile(kind, d.nw0, plan);
            auto run = [&]() -> cudaError_t {
                if (kind == kTauChi0) return launch_chi0_tau(d, g->chiq, g->dchiqt0, g->cinf, g->cinf2, ctx->T, ctx->st);
                if (kind == kTauVertex) return launch_vertex_tau(d, g->V, g->chirt, ctx->U, ctx->dres, ctx->st);
                return launch_sigma_tau(d, g->sigt, g->dS, g->S, g->s2, g->s3, g->s4, g->sinf, ctx->T, ctx->st);
            };
            CK(run());
            CK(cudaEventRecord(a, ctx->st));
            for (int r = 0; r < reps; ++r) CK(run());
            CK(cudaEventRecord(b, ctx->st));
            CK(cudaEventSynchronize(b));
            float t = 0;
            CK(cudaEventElapsedTime(&t, a, b));
            const double mean = t / reps;
            if (ms) ms[3 * kind + plan] = mean;
            if (plan == 0 || mean < best) {
                best = mean;
                pick = plan;
            }
        }
        set_tau_tile(kind, d.nw0, pick);
    }
    g->have_chi0 = g->have_V = g->have_S = g->have_mom = g->have_U = false;
    return TPSC_OK;
}

// the tiling of one tau transform for one Nw0 (kind 0 chi0, 1 V, 2 Sigma;
// tile 0 one column pair per CTA, 1 four columns per CTA, 2 one pair per CTA
// with radix-8 FFT passes, Nw0 <= 2048)
int tpsc_set_tau_tile(int kind, int nw0, int tile) {
    if (kind < 0 || kind > 2 || tile < 0 || tile > 2 || !supported_grid(8, nw0) || (tile == 2 && nw0 > 2048))
        return fail(nullptr, TPSC_ERR_ARG, "need kind 0..2, tile 0..2 (2: Nw0 <= 2048) and a supported Nw0");
    set_tau_tile(kind, nw0, tile);
    return TPSC_OK;
}

int tpsc_set_slice_plan(int kind, int nk0, int plan) {
    const int nbk = nk0 / 2 + 1;
    if (kind < 0 || kind > 3 || plan < 0 || plan > 2 || !supported_grid(nk0, 16) ||
        !slice_plan_supported(kind, plan, nbk))
        return fail(nullptr, TPSC_ERR_ARG,
                    "need kind 0..3, plan 0, 1 (nk0 64, 128, 256) or 2 (kinds 2, 3 at nk0 256) and a supported nk0");
    set_slice_plan(kind, nbk, plan);
    return TPSC_OK;
}

// Times every supported plan of the four FP32 slice transforms on the
// current grid (after a mixed-form solve) and keeps the fastest per kind.
int tpsc_tune_slice_plans(tpsc_ctx *ctx, int reps, double ms[12]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g || !g->have_S || !g->g_mixed || !g->Grt32)
        return fail(ctx, TPSC_ERR_STATE, "tune after a mixed-form solve on the current grid");
    if (reps < 1 || reps > 100) return fail(ctx, TPSC_ERR_ARG, "need 1 <= reps <= 100");
    cudaSetDevice(ctx->device);
    const GridDev &d = g->d;
    cudaEvent_t a = ctx->ev[0], b = ctx->ev[1];
    for (int kind = 0; kind < 4; ++kind) {
        double best = 0.0;
        int pick = -1;
        for (int plan = 0; plan < 3; ++plan) {
            if (ms) ms[3 * kind + plan] = 0.0;
            if (!slice_plan_supported(kind, plan, d.nbk)) continue;
            set_slice_plan(kind, d.nbk, plan);
            auto run = [&]() -> cudaError_t {
                if (kind == kSliceG) return launch_gslice32(d, g->Grt32, g->mu0, ctx->T, ctx->st);
                if (kind == kSliceChi0) return launch_chi0_slice32(d, g->Grt32, g->chirt, g->chiq, ctx->st);
                if (kind == kSliceVertex)
                    return launch_vertex_q32(d, g->chiq, g->V, ctx->U, ctx->dres, ctx->T, ctx->st);
                return launch_sigma_slice32(d, g->Grt32, g->V, g->sigt, ctx->st);
            };
            CK(run());
            CK(cudaEventRecord(a, ctx->st));
            for (int r = 0; r < reps; ++r) CK(run());
            CK(cudaEventRecord(b, ctx->st));
            CK(cudaEventSynchronize(b));
            float t = 0;
            CK(cudaEventElapsedTime(&t, a, b));
            const double mean = t / reps;
            if (ms) ms[3 * kind + plan] = mean;
            if (pick < 0 || mean < best) {
                best = mean;
                pick = plan;
            }
        }
        set_slice_plan(kind, d.nbk, pick);
    }
    unsigned word = 0;
    if (tensor_plan_errors(&word, false) == 0 && word)
        return fail(ctx, TPSC_ERR_CUDA, "a tensor-plan kernel gave up waiting on the tensor cores");
    // the transforms overwrote the grid's stages: the next solve recomputes them
    g->have_chi0 = g->have_V = g->have_S = g->have_mom = g->have_U = false;
    return TPSC_OK;
}

int tpsc_tensor_plan_errors(unsigned *word, int clear) {
    if (!word) return fail(nullptr, TPSC_ERR_ARG, "null output");
    if (tensor_plan_errors(word, clear != 0)) return fail(nullptr, TPSC_ERR_CUDA, "reading the error word failed");
    return TPSC_OK;
}

int tpsc_get_slice_plan(int kind, int nk0) {
    if (kind < 0 || kind > 3 || !supported_grid(nk0, 16))
        return -fail(nullptr, TPSC_ERR_ARG, "need kind 0..3 and a supported nk0");
    return slice_plan(kind, nk0 / 2 + 1);
}

// green0::find_mu_inf_syst (src/green0.cpp:265-287): mu0 of the infinite
// lattice at the model's density and temperature (tpsc_lattice.cu)
int tpsc_mu0_infinite(tpsc_ctx *ctx, double *mu, int *L_used) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!mu) return fail(ctx, TPSC_ERR_ARG, "null output");
    cudaSetDevice(ctx->device);
    rc = lattice_mu0(ctx->n, ctx->T, ctx->tp, ctx->tpp, ctx->t3, ctx->st, mu, L_used);
    return rc ? fail(ctx, rc, g_static_err) : TPSC_OK;
}

// chi0::chiqw (src/chi0.cpp:211-276): chi0(q, i w_n) of the infinite lattice
// at npts points qw[p] = (qx, qy, w_n) for the chemical potential mu; L > 0:
// the L x L lattice's sum (chi0::chiqw_discret, src/chi0.cpp:1587-1612)
int tpsc_chi0_infinite(tpsc_ctx *ctx, double mu, int npts, const double *qw, int L, double *out, int *L_used) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (npts < 1 || npts > 65535 || !qw || !out || L < 0 || L > 65536)
        return fail(ctx, TPSC_ERR_ARG, "need 1 <= npts <= 65535, 0 <= L <= 65536 and arrays");
    cudaSetDevice(ctx->device);
    rc = lattice_chi0(mu, ctx->T, ctx->tp, ctx->tpp, ctx->t3, npts, qw, L, ctx->st, out, L_used);
    return rc ? fail(ctx, rc, g_static_err) : TPSC_OK;
}

// Warm start from saved results (green::load_Self_bin / load_Self,
// src/green.cpp:1517-1541, 1637-1670): the reference's Self_kw_array layout
// [Nw0/2][N8] complex into the device's blocked S; each tail array (and
// Sigma_inf) replaced only when given, as the reference's loaders leave them.
int tpsc_set_self(tpsc_ctx *ctx, const double *self_kw, const double *s2, const double *s3, const double *s4,
                  const double *sigma_inf) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!self_kw) return fail(ctx, TPSC_ERR_ARG, "null self_kw");
    cudaSetDevice(ctx->device);
    Grid *g = ctx->cur;
    const GridDev &d = g->d;
    const size_t bytes = (size_t)(d.nw0 / 2) * d.n8 * sizeof(double2);
    if ((rc = ensure_stage(ctx, bytes))) return rc;
    CK(cudaMemcpyAsync(ctx->stage, self_kw, bytes, cudaMemcpyHostToDevice, ctx->st));
    CK(launch_block_c((const double2 *)ctx->stage, g->S, d.nw0 / 2, d.nw0 / 2, d.n8, ctx->st));
    const size_t vb = (size_t)d.n8 * sizeof(double);
    if (s2) CK(cudaMemcpyAsync(g->s2, s2, vb, cudaMemcpyHostToDevice, ctx->st));
    if (s3) CK(cudaMemcpyAsync(g->s3, s3, vb, cudaMemcpyHostToDevice, ctx->st));
    if (s4) CK(cudaMemcpyAsync(g->s4, s4, vb, cudaMemcpyHostToDevice, ctx->st));
    if (sigma_inf) {
        CK(cudaMemcpyAsync(g->sinf, sigma_inf, sizeof(double), cudaMemcpyHostToDevice, ctx->st));
        ctx->scal[TPSC_S_SIGMA_INF] = *sigma_inf;
    }
    CK(cudaStreamSynchronize(ctx->st));
    g->have_S = true;
    ctx->scal[TPSC_S_EVALS_MU] = 0;  // mu belongs to the Sigma before this one
    return TPSC_OK;
}

// chi0::loadChi0 (src/chi0.cpp:99-154): chi0(q, iqn) [Nw0/2 + 1][N8] of the
// current grid replaces the device's; chi0max and qmax are found again; the
// tail coefficients and chi0(r, tau) stay those of the last chi0 stage, as the
// reference's loader leaves them.
int tpsc_set_chi0(tpsc_ctx *ctx, const double *chiqw) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!chiqw) return fail(ctx, TPSC_ERR_ARG, "null chiqw");
    cudaSetDevice(ctx->device);
    Grid *g = ctx->cur;
    const GridDev &d = g->d;
    const size_t bytes = (size_t)d.nb * d.n8 * sizeof(double);
    if ((rc = ensure_stage(ctx, bytes))) return rc;
    CK(cudaMemcpyAsync(ctx->stage, chiqw, bytes, cudaMemcpyHostToDevice, ctx->st));
    CK(launch_block((const double *)ctx->stage, g->chiq, d.nb, d.nb, d.n8, ctx->st));
    CK(launch_chi0max(d, g->chiq, ctx->red, ctx->st));
    double r[3];
    if ((rc = read_result(ctx, 3, r))) return rc;
    g->have_chi0 = true;
    g->have_V = g->have_S = g->have_mom = g->have_U = false;
    return set_chi0max(ctx, r);
}

namespace {
// The asynchronous copy-out of S and the three tail vectors (FP64), or, with
// f32, of the full Sigma(k, i w_n) formed in FP64 and rounded to FP32: a
// device snapshot, then copies on the copy stream.
int get_self_async(tpsc_ctx *ctx, void *self_kw, bool f32, double *s2, double *s3, double *s4) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g->have_S) return fail(ctx, TPSC_ERR_STATE, "the self-energy has not been computed");
    if (!self_kw) return fail(ctx, TPSC_ERR_ARG, "null self_kw");
    cudaSetDevice(ctx->device);
    const GridDev &d = g->d;
    if (!ctx->cst) {
        CK(cudaStreamCreateWithFlags(&ctx->cst, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) {
            CK(cudaEventCreateWithFlags(&ctx->snap_ev[k], cudaEventDisableTiming));
            CK(cudaEventCreateWithFlags(&ctx->copy_ev[k], cudaEventDisableTiming));
        }
    }
    const int k = ctx->snap_next;
    const size_t sbytes = (size_t)(d.nw0 / 2) * d.n8 * (f32 ? sizeof(float2) : sizeof(double2));
    const size_t vbytes = (size_t)d.n8 * sizeof(double);
    const size_t need = ((sbytes + 15) & ~(size_t)15) + 3 * vbytes;
    // snapshot buffer k is free once its previous copy has finished
    CK(cudaStreamWaitEvent(ctx->st, ctx->copy_ev[k], 0));
    if (ctx->snap_bytes[k] < need) {
        CK(cudaStreamSynchronize(ctx->st));
        if (ctx->snap[k]) cudaFree(ctx->snap[k]);
        ctx->snap[k] = nullptr;
        ctx->snap_bytes[k] = 0;
        CK(cudaMalloc(&ctx->snap[k], need));
        ctx->snap_bytes[k] = need;
    }
    char *base = static_cast<char *>(ctx->snap[k]);
    double *vs = reinterpret_cast<double *>(base + ((sbytes + 15) & ~(size_t)15));
    if (f32)
        CK(launch_sigma_full32(d, g->S, g->s2, g->s3, g->sinf, ctx->T, reinterpret_cast<float2 *>(base), ctx->st));
    else
        CK(launch_unblock_c(g->S, reinterpret_cast<double2 *>(base), d.nw0 / 2, d.nw0 / 2, d.n8, ctx->st));
    // the three vectors by the SMs too: a device-to-device copy may take a
    // copy engine, where it could wait behind the previous step's copy-out
    GatherPieces gp;
    const double *vsrc[3] = {g->s2, g->s3, g->s4};
    for (int i = 0; i < 3; ++i) {
        gp.src[i] = reinterpret_cast<const unsigned *>(vsrc[i]);
        gp.words[i] = 2LL * d.n8;
        gp.dst[i] = 2LL * i * d.n8;
    }
    gp.n = 3;
    CK(launch_gather(gp, reinterpret_cast<unsigned *>(vs), 32, ctx->st));
    CK(cudaEventRecord(ctx->snap_ev[k], ctx->st));
    CK(cudaStreamWaitEvent(ctx->cst, ctx->snap_ev[k], 0));
    CK(cudaMemcpyAsync(self_kw, base, sbytes, cudaMemcpyDeviceToHost, ctx->cst));
    if (s2) CK(cudaMemcpyAsync(s2, vs, vbytes, cudaMemcpyDeviceToHost, ctx->cst));
    if (s3) CK(cudaMemcpyAsync(s3, vs + d.n8, vbytes, cudaMemcpyDeviceToHost, ctx->cst));
    if (s4) CK(cudaMemcpyAsync(s4, vs + 2 * d.n8, vbytes, cudaMemcpyDeviceToHost, ctx->cst));
    CK(cudaEventRecord(ctx->copy_ev[k], ctx->cst));
    ctx->snap_next = k ^ 1;
    ctx->copies_pending = true;
    return TPSC_OK;
}
}  // namespace

int tpsc_get_self_async(tpsc_ctx *ctx, double *self_kw, double *s2, double *s3, double *s4) {
    return get_self_async(ctx, self_kw, false, s2, s3, s4);
}

int tpsc_get_sigma32_async(tpsc_ctx *ctx, float *sigma_kw) {
    return get_self_async(ctx, sigma_kw, true, nullptr, nullptr, nullptr);
}

int tpsc_wait_copies(tpsc_ctx *ctx, int join_stream) {
    if (!ctx) return fail(nullptr, TPSC_ERR_ARG, "null context");
    if (!ctx->copies_pending) return TPSC_OK;
    cudaSetDevice(ctx->device);
    if (join_stream) {
        // the last copy recorded copy_ev[snap_next ^ 1]; the stream waits for it
        CK(cudaStreamWaitEvent(ctx->st, ctx->copy_ev[ctx->snap_next ^ 1], 0));
        return TPSC_OK;
    }
    CK(cudaStreamSynchronize(ctx->cst));
    ctx->copies_pending = false;
    return TPSC_OK;
}

int tpsc_pade_sigma(tpsc_ctx *ctx, const int *n_idx, int Nn, const double *z, int Nz, int mode, double *out_sigma,
                    double *out_A) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g->have_S || ctx->scal[TPSC_S_EVALS_MU] == 0)
        return fail(ctx, TPSC_ERR_STATE, "the self-energy and mu must be computed first");
    if (!n_idx || !z || !out_A || Nn < 2 || Nn > 32 || Nn > g->d.nw0 / 2 || Nz < 1 || (mode != 0 && mode != 1))
        return fail(ctx, TPSC_ERR_ARG, "need 2 <= Nn <= min(32, Nw0/2), Nz >= 1, mode 0 (Pade) or 1 (polynomial)");
    const size_t n8 = g->d.n8;
    const size_t bytes = Nn * sizeof(int) + 16 + Nz * sizeof(double2) + n8 * Nz * (sizeof(double2) + sizeof(double));
    if ((rc = ensure_stage(ctx, bytes))) return rc;
    char *base = (char *)ctx->stage;
    double2 *dz = (double2 *)base;
    double2 *dsig = dz + Nz;
    double *dA = (double *)(dsig + n8 * Nz);
    int *didx = (int *)(dA + n8 * Nz);
    CK(cudaMemcpyAsync(didx, n_idx, Nn * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dz, z, Nz * sizeof(double2), cudaMemcpyHostToDevice, ctx->st));
    CK(launch_pade_sigma(g->d, g->S, g->s2, g->s3, g->sinf, didx, Nn, dz, Nz, mode, ctx->scal[TPSC_S_MU], ctx->T,
                         dsig, dA, ctx->st));
    if (out_sigma) CK(cudaMemcpyAsync(out_sigma, dsig, n8 * Nz * sizeof(double2), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(out_A, dA, n8 * Nz * sizeof(double), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return TPSC_OK;
}

int tpsc_gwn_local(tpsc_ctx *ctx, double *out) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g->have_S || ctx->scal[TPSC_S_EVALS_MU] == 0)
        return fail(ctx, TPSC_ERR_STATE, "the self-energy and mu must be computed first");
    const size_t bytes = (size_t)(g->d.nw0 / 2) * sizeof(double2);
    if ((rc = ensure_stage(ctx, bytes))) return rc;
    CK(launch_gwn_local(g->d, g->S, g->s2, g->s3, g->sinf, ctx->scal[TPSC_S_MU], ctx->T, (double2 *)ctx->stage,
                        ctx->st));
    CK(cudaMemcpyAsync(out, ctx->stage, bytes, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return TPSC_OK;
}

int tpsc_chijj(tpsc_ctx *ctx, int n_theta) {
    int rc = need_model(ctx);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    Grid *g = ctx->cur;
    if (!g->have_S || ctx->scal[TPSC_S_EVALS_MU] == 0)
        return fail(ctx, TPSC_ERR_STATE, "the self-energy and mu must be computed first");
    if (n_theta < 1 || n_theta > 64) return fail(ctx, TPSC_ERR_ARG, "need 1 <= n_theta <= 64");
    if (g->d.nk0 < 8) return fail(ctx, TPSC_ERR_ARG, "need nk0 >= 8");
    g->cond_bins = 0;
    return run_cond(ctx, n_theta);
}

int tpsc_barrier_probe(tpsc_ctx *ctx, int withhold, int *err_flag, int *timed_out, int *blocks, double *ms) {
    if (!ctx) return fail(nullptr, TPSC_ERR_ARG, "null context");
    cudaSetDevice(ctx->device);
    unsigned *words = nullptr;
    CK(cudaMallocAsync(reinterpret_cast<void **>(&words), 4 * sizeof(unsigned), ctx->st));
    int nblk = 0;
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    cudaError_t e = launch_barrier_probe(words, withhold, &nblk, ctx->st);
    if (e == cudaSuccess) e = cudaEventRecord(ctx->ev[1], ctx->st);
    unsigned h[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, words, sizeof(h), cudaMemcpyDeviceToHost, ctx->st);
    cudaFreeAsync(words, ctx->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "barrier probe");
    float t = 0.0f;
    CK(cudaEventElapsedTime(&t, ctx->ev[0], ctx->ev[1]));
    if (err_flag) *err_flag = (int)h[2];
    if (timed_out) *timed_out = (int)h[3];
    if (blocks) *blocks = nblk;
    if (ms) *ms = t;
    return TPSC_OK;
}

int tpsc_chijj3(tpsc_ctx *ctx, int mmin, int n_theta) {
    int rc = need_model(ctx);
    if (rc) return rc;
    cudaSetDevice(ctx->device);
    Grid *g = ctx->cur;
    if (!g->have_S || ctx->scal[TPSC_S_EVALS_MU] == 0)
        return fail(ctx, TPSC_ERR_STATE, "the self-energy and mu must be computed first");
    if (n_theta < 1 || n_theta > 64) return fail(ctx, TPSC_ERR_ARG, "need 1 <= n_theta <= 64");
    if (mmin < 0 || mmin > 24) return fail(ctx, TPSC_ERR_ARG, "need 0 <= mmin <= 24");
    if (g->d.nk0 < 8) return fail(ctx, TPSC_ERR_ARG, "need nk0 >= 8");
    g->al_bins = 0;
    return run_al(ctx, mmin, n_theta);
}

int tpsc_get_chijj3(tpsc_ctx *ctx, int cap, int *n_freq, int *ind_freq, double *chijj3, double *chijj3_k) {
    int rc = need_model(ctx);
    if (rc) return rc;
    const Grid *g = ctx->cur;
    if (g->al_bins == 0) return fail(ctx, TPSC_ERR_STATE, "tpsc_chijj3 has not been run on the current grid");
    const int N = (int)g->al_ind.size(), nb = g->al_bins;
    if (n_freq) *n_freq = N;
    if ((ind_freq || chijj3 || chijj3_k) && cap < N) return fail(ctx, TPSC_ERR_ARG, "cap is below the grid size");
    for (int j = 0; j < N; ++j) {
        if (ind_freq) ind_freq[j] = g->al_ind[j];
        if (chijj3) chijj3[j] = g->al_host[(size_t)j * (1 + nb)];
        for (int p = 0; p < nb; ++p)
            if (chijj3_k) chijj3_k[p + j * nb] = g->al_host[(size_t)j * (1 + nb) + 1 + p];
    }
    return TPSC_OK;
}

int tpsc_get_chijj(tpsc_ctx *ctx, double *chijj1, double *chijj2, double *kx0, double *chijj1_k, double *chijj2_k) {
    int rc = need_model(ctx);
    if (rc) return rc;
    const Grid *g = ctx->cur;
    if (g->cond_bins == 0) return fail(ctx, TPSC_ERR_STATE, "tpsc_chijj has not been run on the current grid");
    const int NB = g->d.nw0 / 2 + 1, nb = g->cond_bins;
    const double *tot = g->cond_host.data() + (size_t)nb * 2 * NB;
    if (chijj1) std::memcpy(chijj1, tot, NB * sizeof(double));
    if (chijj2) std::memcpy(chijj2, tot + NB, NB * sizeof(double));
    if (kx0) *kx0 = tot[2 * NB];
    for (int j = 0; j < NB; ++j)
        for (int p = 0; p < nb; ++p) {
            if (chijj1_k) chijj1_k[p + j * nb] = g->cond_host[(size_t)p * 2 * NB + j];
            if (chijj2_k) chijj2_k[p + j * nb] = g->cond_host[(size_t)p * 2 * NB + NB + j];
        }
    return TPSC_OK;
}

int tpsc_sigma_iqn(tpsc_ctx *ctx, int nq, double *sigma, double *sigma_bubble) {
    int rc = need_model(ctx);
    if (rc) return rc;
    const Grid *g = ctx->cur;
    if (g->cond_bins == 0) return fail(ctx, TPSC_ERR_STATE, "tpsc_chijj has not been run on the current grid");
    const int NB = g->d.nw0 / 2 + 1;
    if (nq < 1 || nq > NB - 1) return fail(ctx, TPSC_ERR_ARG, "need 1 <= nq <= Nw0/2");
    const double *tot = g->cond_host.data() + (size_t)g->cond_bins * 2 * NB;
    const double kx0 = tot[2 * NB];
    for (int n = 1; n <= nq; ++n) {
        const double qn = 2.0 * PI * n * ctx->T;
        if (sigma) sigma[n - 1] = (-kx0 - (tot[n] + tot[NB + n])) / qn;
        if (sigma_bubble) sigma_bubble[n - 1] = (-kx0 - tot[n]) / qn;
    }
    return TPSC_OK;
}

// d sigma(iq_n) / d{U, mu, t'} and d D / d{U, mu, t'} by central differences
// of full device solves (FP64 Newton form), each followed by tpsc_chijj with
// one angle bin and tpsc_sigma_iqn; mu is the shift of mu0 at fixed n
// (tpsc_set_mu_shift), t' moves at fixed n.  The model, mu shift and form are
// put back and the base point solved again, so the context ends as a plain
// solve + tpsc_chijj(1) of its model would leave it.
int tpsc_sigma_iqn_fd(tpsc_ctx *ctx, int nq, const double h[3], double *dsigma, double dD[3]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!h || !dsigma) return fail(ctx, TPSC_ERR_ARG, "null step or output");
    for (int p = 0; p < 3; ++p)
        if (!(h[p] > 0.0) || !std::isfinite(h[p])) return fail(ctx, TPSC_ERR_ARG, "steps must be positive");
    if (nq < 1 || nq > ctx->Nw0 / 2) return fail(ctx, TPSC_ERR_ARG, "need 1 <= nq <= Nw0/2");
    if (ctx->nk0 < 8) return fail(ctx, TPSC_ERR_ARG, "need nk0 >= 8");
    const int nk0 = ctx->nk0, Nw0 = ctx->Nw0, form = ctx->form;
    const double n = ctx->n, T = ctx->T, tp = ctx->tp, tpp = ctx->tpp, t3 = ctx->t3, U = ctx->U;
    const double dmu0 = ctx->mu_shift;
    std::vector<double> sp(nq), sm(nq);
    auto point = [&](double Uv, double dmu, double tpv, double *sig, double *D) -> int {
        int r = tpsc_set_model(ctx, nk0, Nw0, n, T, tpv, tpp, t3, Uv);
        if (!r) r = tpsc_set_mu_shift(ctx, dmu);
        if (!r) r = tpsc_solve(ctx);
        if (!r) r = tpsc_chijj(ctx, 1);
        if (!r && sig) r = tpsc_sigma_iqn(ctx, nq, sig, nullptr);
        if (!r && D) *D = ctx->scal[TPSC_S_DBLOCC];
        return r;
    };
    rc = tpsc_set_form(ctx, form & ~TPSC_FORM_MIXED);
    for (int p = 0; p < 3 && !rc; ++p) {
        double Dp = 0.0, Dm = 0.0;
        const double e[3] = {p == 0 ? h[0] : 0.0, p == 1 ? h[1] : 0.0, p == 2 ? h[2] : 0.0};
        rc = point(U + e[0], dmu0 + e[1], tp + e[2], sp.data(), &Dp);
        if (!rc) rc = point(U - e[0], dmu0 - e[1], tp - e[2], sm.data(), &Dm);
        if (rc) break;
        for (int k = 0; k < nq; ++k) dsigma[(size_t)p * nq + k] = (sp[k] - sm[k]) / (2.0 * h[p]);
        if (dD) dD[p] = (Dp - Dm) / (2.0 * h[p]);
    }
    // the base point, whatever happened above; the first error is the one reported
    const std::string err = rc ? ctx->err : std::string();
    tpsc_set_form(ctx, form);
    const int rc2 = point(U, dmu0, tp, nullptr, nullptr);
    if (rc) {
        ctx->err = err;
        return rc;
    }
    return rc2;
}

// buffers of the reverse pass, on first use per grid (the cond tables first)
int ensure_adj(tpsc_ctx *ctx, Grid *g) {
    if (g->adj_alloc) return TPSC_OK;
    const GridDev &d = g->d;
    const CondDev &c = g->cond;
    AdjDev &a = g->adj;
    int nblk = 0;
    CK(cond_bwd_blocks(d, &nblk));
    a.nblk = std::max(1, std::min(nblk, c.K4));
    const size_t NO = d.nw0 / 2, NJ = d.nw0 + 1, nb = d.nb, K4 = c.K4, K4p = c.K4p, n8 = d.n8, n8p = d.n8p;
    a.row_ct = 0;
    a.row_cl = a.row_ct + a.nblk;
    a.row_cb = a.row_cl + 2 * d.nbk;
    a.row_cs = a.row_cb + 2;
    a.row_sg = a.row_cs + (int)nb;
    a.row_ss = a.row_sg + (int)n8;
    a.row_sb = a.row_ss + (int)nb;
    a.row_vt = a.row_sb + 1;
    a.row_vq = a.row_vt + (int)n8;
    a.rows = a.row_vq + (int)nb;
    cudaError_t e = cudaSuccess;
#define A(x)                \
    if (e == cudaSuccess) { \
        e = (x);            \
    }
    A(dalloc(g, &a.cw, NO + 1));
    A(dalloc(g, &a.ws, (size_t)a.nblk * 2 * NO));
    A(dalloc(g, &a.hVb, K4p * NJ));
    A(dalloc(g, &a.dbb, 2 * K4p));
    A(dalloc(g, &a.sigc, K4 * NO));
    A(dalloc(g, &a.sigl, (size_t)2 * d.nbk * NO));
    A(dalloc(g, &a.tmpB, 2 * K4p));
    A(dalloc(g, &a.vbk, 2 * K4p));
    A(dalloc(g, &a.preb, 2 * K4p));
    A(dalloc(g, &a.dchb, 2 * K4p));
    A(dalloc(g, &a.tmpU, nb * K4p));
    A(dalloc(g, &a.vcond, nb * K4p));
    A(dalloc(g, &a.htab, 8 * K4));
    A(dalloc(g, &a.Sb, n8 * NO));
    A(dalloc(g, &a.s2b, n8));
    A(dalloc(g, &a.s3b, n8));
    A(dalloc(g, &a.stb, NJ * n8p));
    A(dalloc(g, &a.dSb, 2 * n8p));
    A(dalloc(g, &a.Vb, nb * n8p));
    A(dalloc(g, &a.part, (size_t)a.rows * kAdjW));
#undef A
    if (e != cudaSuccess) return cuda_fail(ctx, e, "reverse-pass allocation");
    g->adj_alloc = true;
    return TPSC_OK;
}

// sums of the partial-row slots over rows [r0, r1) of the reverse pass, in row order
int adj_rows(tpsc_ctx *ctx, const AdjDev &a, int r0, int r1, std::vector<double> &rows) {
    rows.assign((size_t)(r1 - r0) * kAdjW, 0.0);
    CK(cudaMemcpyAsync(rows.data(), a.part + (size_t)r0 * kAdjW, rows.size() * sizeof(double),
                       cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return TPSC_OK;
}
double adj_slot(const std::vector<double> &rows, int slot) {
    double s = 0.0, c = 0.0;  // compensated, in row order
    for (size_t i = slot; i < rows.size(); i += kAdjW) {
        const double y = rows[i] - c, t = s + y;
        c = (t - s) - y;
        s = t;
    }
    return s;
}

int tpsc_sigma_iqn_bwd(tpsc_ctx *ctx, int nq, const double *cot, double grad[3], double dD[3]) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!cot || !grad) return fail(ctx, TPSC_ERR_ARG, "null cotangent or gradient");
    Grid *g = ctx->cur;
    if (!g->have_S || ctx->scal[TPSC_S_EVALS_MU] == 0)
        return fail(ctx, TPSC_ERR_STATE, "the self-energy and mu must be computed first");
    if (nq < 1 || nq > ctx->Nw0 / 2) return fail(ctx, TPSC_ERR_ARG, "need 1 <= nq <= Nw0/2");
    if (ctx->nk0 < 8) return fail(ctx, TPSC_ERR_ARG, "need nk0 >= 8");
    for (int n = 0; n < nq; ++n)
        if (!std::isfinite(cot[n])) return fail(ctx, TPSC_ERR_ARG, "non-finite cotangent");
    cudaSetDevice(ctx->device);
    // forward tangents of the chi0 stage and the roots' sensitivities (also
    // leaves the FP64 G(r, tau) in g->Grt)
    double J[9];
    if ((rc = tpsc_sumrule_tangents(ctx, J))) return rc;
    if ((rc = ensure_cond(ctx, g, std::max(1, g->cond_bins)))) return rc;
    if ((rc = ensure_adj(ctx, g))) return rc;
    const GridDev &d = g->d;
    const CondDev &c = g->cond;
    AdjDev &a = g->adj;
    const double T = ctx->T, U = ctx->U, Usp = ctx->Usp, Uch = ctx->Uch, mu = ctx->scal[TPSC_S_MU], mu0 = g->mu0;
    const double fact4 = U * (3.0 * Usp + Uch) / 4.0, fact8 = U * (3.0 * Usp + Uch) / 8.0;
    const double dmu0_2 = g->t_dmu0_tp;
    const int NO = d.nw0 / 2;
    // d L / d chi_jj(iq_n) and d L / d kx0 for L = sum_n cot_n sigma(iq_n)
    std::vector<double> cw(NO + 1, 0.0);
    double kx0b = 0.0;
    for (int n = 1; n <= nq; ++n) {
        cw[n] = -cot[n - 1] / (2.0 * PI * n * T);
        kx0b += cw[n];
    }
    CK(cudaMemcpyAsync(a.cw, cw.data(), cw.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->st));
    // the h slices at the solved point, then chi_jj backward
    CK(launch_cond_slices_h(d, c, g->V, g->dchirt0, mu0, T, fact4, ctx->st));
    CondBwdArgs ca;
    ca.hV = c.hV;
    ca.dbound = c.dbound;
    ca.S = g->S;
    ca.s2 = g->s2;
    ca.s3 = g->s3;
    ca.sinf = g->sinf;
    ca.ek = d.ek;
    ca.dek = c.dek;
    ca.d2ek = c.d2ek;
    ca.spl_full = d.spl_full;
    ca.spl_half = d.spl_half;
    ca.tw = d.tw_w;
    ca.ht = d.ht_w;
    ca.cw = a.cw;
    ca.kx0b = kx0b;
    ca.ws = a.ws;
    ca.hVb = a.hVb;
    ca.dbb = a.dbb;
    ca.sigc = a.sigc;
    ca.part = a.part + (size_t)a.row_ct * kAdjW;
    ca.K4 = c.K4;
    ca.K4p = c.K4p;
    ca.nbk = d.nbk;
    ca.mu = mu;
    ca.T = T;
    ca.nf = 1.0 / ((double)d.nk0 * d.nk0);
    CK(launch_cond_tau_bwd(d, ca, a.nblk, ctx->st));
    CK(launch_cond_lines_bwd(d, c, a, g->S, g->s2, g->s3, g->sinf, mu, T, kx0b, ctx->st));
    // mu is the root of traceDiffG: its cotangent moves to Sigma, eps and mu0
    // through lam = -(d L / d mu) / (d traceDiffG / d mu)
    std::vector<double> rows;
    if ((rc = adj_rows(ctx, a, a.row_ct, a.row_cb, rows))) return rc;
    const double mub = adj_slot(rows, kAdjMu);
    const double sinfb_c = adj_slot(rows, kAdjSinf);
    CK(launch_trace_diff_G(d, g->S, g->s2, g->s3, g->s4, g->sinf, mu0, mu, T, ctx->red, ctx->st));
    double fr[2];
    if ((rc = read_result(ctx, 2, fr))) return rc;
    if (!(fr[1] != 0.0) || !std::isfinite(fr[1])) return fail(ctx, TPSC_ERR_NONFINITE, "d traceDiffG / d mu is zero");
    const double lam = -mub / fr[1];
    CK(launch_cond_slices_bwd(d, c, a, g->V, g->dchirt0, mu0, T, fact4, dmu0_2, ctx->st));
    CK(launch_sigbar(d, c, a, g->S, g->s2, g->s3, g->s4, g->sinf, mu0, mu, lam, T, dmu0_2, ctx->st));
    if ((rc = adj_rows(ctx, a, a.row_sg, a.row_sg + d.n8, rows))) return rc;
    const double sinfb = sinfb_c + adj_slot(rows, kAdjSinf);
    CK(launch_sigma_tau_bwd(d, a, sinfb, T, ctx->st));
    CK(launch_sigma_slices_bwd(d, c, a, g->Grt, g->V, g->dchirt0, g->dG0p, mu0, fact8, dmu0_2, ctx->st));
    CK(launch_vertex_bwd(d, a, g->chirt, g->chiq, g->Grt, U, Usp, Uch, T, ctx->st));
    if ((rc = adj_rows(ctx, a, 0, a.rows, rows))) return rc;
    // assembly: the mu0-shift and t' directions from the contractions; U, and
    // the roots' sensitivities d{Usp, Uch}/d theta (J) for every direction
    const double f4b = adj_slot(rows, kAdjFact4), f8b = adj_slot(rows, kAdjFact8);
    const double Uspb = adj_slot(rows, kAdjUsp) + f4b * 3.0 * U / 4.0 + f8b * 3.0 * U / 8.0;
    const double Uchb = adj_slot(rows, kAdjUch) + f4b * U / 4.0 + f8b * U / 8.0;
    const double Ub = adj_slot(rows, kAdjU) + f4b * (3.0 * Usp + Uch) / 4.0 + f8b * (3.0 * Usp + Uch) / 8.0;
    const double th[3] = {Ub, adj_slot(rows, kAdjTh1), adj_slot(rows, kAdjTh2)};
    for (int p = 0; p < 3; ++p) {
        grad[p] = th[p] + Uspb * J[3 * p] + Uchb * J[3 * p + 1];
        if (dD) dD[p] = J[3 * p + 2];
        if (!std::isfinite(grad[p])) return fail(ctx, TPSC_ERR_NONFINITE, "non-finite gradient");
    }
    return TPSC_OK;
}

int pade_batch(tpsc_ctx *ctx, int nf, int Nn, const double *x, const double *y, int Nz, const double *z,
               double *out) {
    const size_t bx = (size_t)nf * Nn * sizeof(double2), bz = (size_t)Nz * sizeof(double2),
                 bo = (size_t)nf * Nz * sizeof(double2);
    int rc = ensure_stage(ctx, 2 * bx + bz + bo);
    if (rc) return rc;
    char *base = (char *)ctx->stage;
    double2 *dx = (double2 *)base, *dy = (double2 *)(base + bx), *dz = (double2 *)(base + 2 * bx),
            *dout = (double2 *)(base + 2 * bx + bz);
    CK(cudaMemcpyAsync(dx, x, bx, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dy, y, bx, cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(dz, z, bz, cudaMemcpyHostToDevice, ctx->st));
    CK(launch_pade_batch(dx, dy, nf, Nn, dz, Nz, dout, ctx->st));
    CK(cudaMemcpyAsync(out, dout, bo, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return TPSC_OK;
}

int tpsc_pade_batch(tpsc_ctx *ctx, int nf, int Nn, const double *x, const double *y, int Nz, const double *z,
                    double *out) {
    if (!ctx) return fail(nullptr, TPSC_ERR_ARG, "null context");
    if (!x || !y || !z || !out || nf < 1 || Nn < 2 || Nn > kPadeBatchMax || Nz < 1)
        return fail(ctx, TPSC_ERR_ARG, "need nf >= 1, 2 <= Nn <= 4096, Nz >= 1 and non-NULL arrays");
    cudaSetDevice(ctx->device);
    return pade_batch(ctx, nf, Nn, x, y, Nz, z, out);
}

int tpsc_sigma_pade(tpsc_ctx *ctx, int Nn, const double *w, int Nw, double eta, double *out) {
    int rc = need_model(ctx);
    if (rc) return rc;
    if (!w || !out || Nw < 1 || Nn < 2) return fail(ctx, TPSC_ERR_ARG, "need Nn >= 2, Nw >= 1");
    std::vector<double> s(Nn), sb(Nn);
    if ((rc = tpsc_sigma_iqn(ctx, Nn, s.data(), sb.data()))) return rc;
    std::vector<double2> x(2 * Nn), y(2 * Nn), z(Nw);
    for (int j = 0; j < Nn; ++j) {
        const double qn = 2.0 * PI * (j + 1) * ctx->T;
        x[j] = x[Nn + j] = make_double2(0.0, qn);
        y[j] = make_double2(s[j], 0.0);
        y[Nn + j] = make_double2(sb[j], 0.0);
    }
    for (int i = 0; i < Nw; ++i) z[i] = make_double2(w[i], eta);
    cudaSetDevice(ctx->device);
    return pade_batch(ctx, 2, Nn, (const double *)x.data(), (const double *)y.data(), Nw, (const double *)z.data(),
                      out);
}

int tpsc_stage_times(tpsc_ctx *ctx, double *ms, int n) {
    if (!ctx || !ms) return fail(ctx, TPSC_ERR_ARG, "bad arguments");
    for (int i = 0; i < n && i < 8; ++i) ms[i] = ctx->stage_ms[i];
    return TPSC_OK;
}

int tpsc_launch_count(tpsc_ctx *ctx, long long *count) {
    if (!count) return fail(ctx, TPSC_ERR_ARG, "bad arguments");
    *count = launches_total();
    return TPSC_OK;
}

int tpsc_set_form(tpsc_ctx *ctx, int form) {
    if (!ctx) return fail(nullptr, TPSC_ERR_ARG, "null context");
    if (form < 0 || form > (TPSC_FORM_NEWTON | TPSC_FORM_MIXED)) return fail(ctx, TPSC_ERR_ARG, "unknown form");
    // mu0 comes from the root search of the form (host find_zero or the
    // device Newton kernel; they agree to an ulp or so): when that changes,
    // the next grid switch (every solve and chi0 stage) derives it again, so
    // a result does not depend on whether the form was set before the model
    if ((ctx->form ^ form) & TPSC_FORM_NEWTON)
        for (auto &kv : ctx->grids) kv.second->model_id = -1;
    ctx->form = form;
    return TPSC_OK;
}

int tpsc_get_stream(tpsc_ctx *ctx, void **stream) {
    if (!ctx || !stream) return fail(ctx, TPSC_ERR_ARG, "bad arguments");
    *stream = (void *)ctx->st;
    return TPSC_OK;
}

int tpsc_run_kernel(tpsc_ctx *ctx, int which) {
    int rc = need_model(ctx);
    if (rc) return rc;
    Grid *g = ctx->cur;
    if (!g->have_S) return fail(ctx, TPSC_ERR_STATE, "run tpsc_solve first");
    const GridDev &d = g->d;
    switch (which) {
        case 0:
            if (g->g_mixed)
                CK(launch_gslice32(d, g->Grt32, g->mu0, ctx->T, ctx->st));
            else
                CK(launch_gslice(d, g->Grt, g->mu0, ctx->T, ctx->st));
            break;
        case 1:
            if (g->g_mixed)
                CK(launch_chi0_slice32(d, g->Grt32, g->chirt, g->chiq, ctx->st));
            else
                CK(launch_chi0_slice(d, g->Grt, g->chirt, g->chiq, ctx->st));
            break;
        case 2: CK(launch_chi0_tau(d, g->chiq, g->dchiqt0, g->cinf, g->cinf2, ctx->T, ctx->st)); break;
        case 3:
            if (g->g_mixed)
                CK(launch_vertex_q32(d, g->chiq, g->V, ctx->U, ctx->dres, ctx->T, ctx->st));
            else
                CK(launch_vertex_q(d, g->chiq, g->V, ctx->U, ctx->dres, ctx->T, ctx->st));
            break;
        case 4: CK(launch_vertex_tau(d, g->V, g->chirt, ctx->U, ctx->dres, ctx->st)); break;
        case 5:
            if (g->g_mixed)
                CK(launch_sigma_slice32(d, g->Grt32, g->V, g->sigt, ctx->st));
            else
                CK(launch_sigma_slice(d, (const double *)g->Grt, g->V, g->sigt, ctx->st));
            break;
        case 6:
            CK(launch_sigma_tau(d, g->sigt, g->dS, g->S, g->s2, g->s3, g->s4, g->sinf, ctx->T, ctx->st));
            break;
        case 7:
            CK(launch_sumrule(d, g->chiq, g->cinf, g->cinf2, ctx->Usp, -1.0, ctx->T, ctx->red, ctx->st));
            break;
        case 8:
            CK(launch_trace_diff_G(d, g->S, g->s2, g->s3, g->s4, g->sinf, g->mu0, ctx->scal[TPSC_S_MU], ctx->T,
                                   ctx->red, ctx->st));
            break;
        case 9:
            // chi0 slices followed by the in-place chi0 tau transform
            if (g->g_mixed)
                CK(launch_chi0_slice32(d, g->Grt32, g->chirt, g->chiq, ctx->st));
            else
                CK(launch_chi0_slice(d, g->Grt, g->chirt, g->chiq, ctx->st));
            CK(launch_chi0_tau(d, g->chiq, g->dchiqt0, g->cinf, g->cinf2, ctx->T, ctx->st));
            break;
        case 10: {
            // one Newton-form sum-rule evaluation at Usp: low frequencies, series above
            int rc2 = ensure_moments_host(ctx, g);
            if (rc2) return rc2;
            int jdir, tail;
            series_cut(g, ctx->Usp, &jdir, &tail);
            CK(launch_sumrule(d, g->chiq, g->cinf, g->cinf2, ctx->Usp, -1.0, ctx->T, ctx->red, ctx->st, jdir, tail));
            break;
        }
        case 11: {
            // one Newton-form Tr(G - G0) evaluation at mu: frequencies below the series
            int jc;
            double wc;
            mu_series_cut(ctx, &jc, &wc);
            CK(launch_trace_diff_G(d, g->S, g->s2, g->s3, g->s4, g->sinf, g->mu0, ctx->scal[TPSC_S_MU], ctx->T,
                                   ctx->red, ctx->st, jc));
            break;
        }
        case 12:
            // the Newton-form sum-rule moments: per-frequency moments, tail, suffix sums
            g->have_mom = false;
            if ((rc = ensure_moments(ctx, g))) return rc;
            break;
        case 13:
            // the device Usp/Uch root search of the Newton form
            if ((rc = ensure_moments(ctx, g))) return rc;
            CK(launch_sumrule_roots(d, g->chiq, g->cinf, g->cinf2, g->d_mom_suf, g->d_cmax_suf, g->d_tailm, ctx->T,
                                    ctx->n, ctx->nsr, ctx->U, 2.0 / ctx->scal[TPSC_S_CHI0MAX] - 2 * EPS, ctx->roots,
                                    ctx->st));
            ctx->roots.reset_sr = true;
            break;
        case 14:
        case 15: {
            // 14: the Sigma moment pass (Tr Sigma G0 and the find_mu series);
            // 15: that pass followed by the device mu search
            int jc;
            double wc;
            mu_series_cut(ctx, &jc, &wc);
            CK(launch_sigma_moments(d, g->S, g->s2, g->s3, g->s4, g->sinf, g->mu0, ctx->T, jc, ctx->redm, ctx->st));
            if (which == 15) {
                CK(launch_mu_roots(d, g->S, g->s2, g->s3, g->s4, g->sinf, ctx->redm.result, g->mu0, ctx->T, jc, wc,
                                   ctx->roots, ctx->st));
                ctx->roots.reset_mu = true;
            }
            break;
        }
        default: return fail(ctx, TPSC_ERR_ARG, "unknown stage");
    }
    return TPSC_OK;
}

int tpsc_kernel_bytes(tpsc_ctx *ctx, int which, double *bytes) {
    int rc = need_model(ctx);
    if (rc) return rc;
    const GridDev &d = ctx->cur->d;
    const double s = sizeof(double), n8 = d.n8, nb = d.nb, nw = d.nw0;
    const double tau = (nw + 1) * n8 * s;   // one (Nw0+1) x N8 real array
    // G(r, tau) as the last solve stored it (FP32 in the mixed form)
    const double gtau = ctx->cur->g_mixed ? tau / 2 : tau;
    const double half = nb * n8 * s;        // one (Nw0/2+1) x N8 real array
    const double cplx = (nw / 2) * n8 * 2 * s;
    double b;
    switch (which) {
        case 0: b = gtau; break;                      // write G(r, tau)
        case 1: b = gtau + 2 * half; break;           // read G, write chi0(r,tau), chi0(q,tau)
        case 2: b = 2 * half; break;                  // read + write chi0(q, .)
        case 3: b = 2 * half; break;                  // read chi0(q, iqn), write V(r, iqn)
        case 4: b = 3 * half; break;                  // read V, chi0(r, tau); write V
        case 5: b = gtau + half + tau; break;         // read G, V; write Sigma(k, tau)
        case 6: b = tau + cplx; break;                // read Sigma(k, tau); write S
        case 7: b = half; break;                      // read chi0(q, iqn)
        case 8: b = cplx; break;                      // read S
        case 9: b = gtau + 2 * half + 2 * half; break; // stages 1 and 2
        case 10: {                                     // read chi0(q, iqn), j < jdir
            Grid *g = ctx->cur;
            int rc2 = ensure_moments_host(ctx, g);
            if (rc2) return rc2;
            int jdir, tail;
            series_cut(g, ctx->Usp, &jdir, &tail);
            b = (double)jdir * d.n8 * s + (tail ? 2 * d.n8 * s : 0.0);
            break;
        }
        case 11: {                                     // read S, j < jc
            int jc;
            double wc;
            mu_series_cut(ctx, &jc, &wc);
            b = (double)jc * d.n8 * 2 * s;
            break;
        }
        case 12: b = half + 2 * d.n8 * s; break;       // read chi0(q, iqn), chi0_inf, chi0_inf2
        case 13: {                                     // every evaluation reads chi0(q, iqn), j < jdir
            Grid *g = ctx->cur;
            int rc2 = ensure_moments_host(ctx, g);
            if (rc2) return rc2;
            int js, jch, tail;
            series_cut(g, ctx->Usp, &js, &tail);
            series_cut(g, ctx->Uch, &jch, &tail);
            b = (ctx->scal[TPSC_S_EVALS_SP] * js + ctx->scal[TPSC_S_EVALS_CH] * jch) * d.n8 * s;
            break;
        }
        case 14: b = cplx; break;                      // read S
        case 15: {                                     // the pass, then per evaluation S, j < jc, and one full pass
            int jc;
            double wc;
            mu_series_cut(ctx, &jc, &wc);
            b = 2 * cplx + ctx->scal[TPSC_S_EVALS_MU] * jc * d.n8 * 2 * s;
            break;
        }
        default: return fail(ctx, TPSC_ERR_ARG, "unknown stage");
    }
    *bytes = b;
    return TPSC_OK;
}

}  // extern "C"

// Cap on the cooperative root-search grids of one context, for callers that
// run several contexts' solves at once on one GPU (tpsc_batch.cpp).
void tpsc_ctx_set_coop_cap(tpsc_ctx *ctx, int blocks) {
    if (ctx) ctx->roots.max_blocks = blocks;
}

int tpsc_set_graph_mode(tpsc_ctx *ctx, int mode) {
    if (!ctx) return fail(nullptr, TPSC_ERR_ARG, "null context");
    if (mode < 0 || mode > 2) return fail(ctx, TPSC_ERR_ARG, "graph mode must be 0, 1 or 2");
    ctx->graph_mode = mode;
    return TPSC_OK;
}

int tpsc_graph_stats(tpsc_ctx *ctx, long long out[4]) {
    if (!ctx || !out) return fail(ctx, TPSC_ERR_ARG, "bad arguments");
    out[0] = ctx->graph_captures;
    out[1] = ctx->graph_replays;
    out[2] = ctx->graph_kernels;
    out[3] = ctx->graph_off ? 1 : 0;
    return TPSC_OK;
}
