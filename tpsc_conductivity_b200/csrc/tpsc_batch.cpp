// tpsc_batch.cpp -- the batched sweep: many independent TPSC solves, with
// uneven lattices and Matsubara cutoffs, on one GPU.
//
// A batch owns S solver contexts, each with its own CUDA streams, device
// scratch and grid cache (one allocation per lattice/cutoff shape, kept across
// calls), and one host thread per context.  The points of a call run largest
// first (nk0^2 Nw0) and each goes to the next free context, so that the small
// solves of a sweep -- launch- and round-trip-bound on their own -- overlap
// on the GPU with one another and with the large ones.  The cooperative root
// searches of the S contexts are capped at 2 SMs/S blocks each so that all of
// them fit on the GPU at once.  The number of contexts is set at creation or
// chosen by tpsc_batch_tune, which times a sample of points at 1, 2, 4, ...
// contexts.  Each point's results are those of tpsc_solve on that point.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <mutex>
#include <random>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tpsc_b200.h"

void tpsc_ctx_set_coop_cap(tpsc_ctx *ctx, int blocks);

struct tpsc_batch {
    int device = 0;
    int nstreams = 1;
    int sms = 0;
    int graph_mode = 1;  // tpsc_set_graph_mode of every context
    std::vector<tpsc_ctx *> ctxs;
    std::string err;
};

namespace {

constexpr int kParamCols = 8;  // nk0, Nw0, n, T, tp, tpp, t3, U
constexpr int kMaxStreams = 32;
constexpr int kCorrCols = 19;  // the columns of a corrLgth line

// contexts 0..n-1 exist, with their root grids capped for n concurrent solvers
int ensure_contexts(tpsc_batch *b, int n) {
    while ((int)b->ctxs.size() < n) {
        int st = TPSC_OK;
        tpsc_ctx *c = tpsc_create(b->device, &st);
        if (!c) {
            b->err = std::string("context creation failed: ") + tpsc_last_error(nullptr);
            return st ? st : TPSC_ERR_CUDA;
        }
        b->ctxs.push_back(c);
    }
    const int cap = n > 1 ? std::max(8, 2 * b->sms / n) : 0;
    for (int i = 0; i < n; ++i) {
        tpsc_ctx_set_coop_cap(b->ctxs[i], cap);
        tpsc_set_graph_mode(b->ctxs[i], b->graph_mode);
    }
    return TPSC_OK;
}

// Runs task(ctx, i) for every i < npts on contexts 0..n-1, one host thread
// per context, in the given order (each point on the next free context);
// per-point status in status[].  The wall time of the whole call (host clock
// from a device-idle start to a device-idle end) in *ms.  *first_fail (if
// given) receives the status of the first failing point in index order, and
// b->err its message.  Returns a context-level failure only.
template <class Task>
int run_tasks(tpsc_batch *b, int n, int npts, const std::vector<int> &order, Task task, int *status, double *ms,
              int *first_fail) {
    int rc = ensure_contexts(b, n);
    if (rc) return rc;
    std::atomic<int> next{0};
    std::mutex err_mu;
    std::string first_msg;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    const auto t0 = std::chrono::steady_clock::now();
    auto worker = [&](int w) {
        cudaSetDevice(b->device);
        tpsc_ctx *c = b->ctxs[w];
        for (;;) {
            const int k = next.fetch_add(1);
            if (k >= npts) break;
            const int i = order[k];
            const int r = task(c, i);
            if (r) {
                std::lock_guard<std::mutex> lk(err_mu);
                if (first_msg.empty()) first_msg = tpsc_last_error(c);
            }
            status[i] = r;
        }
    };
    if (n == 1) {
        worker(0);
    } else {
        std::vector<std::thread> th;
        th.reserve(n);
        for (int w = 0; w < n; ++w) th.emplace_back(worker, w);
        for (auto &t : th) t.join();
    }
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    const auto t1 = std::chrono::steady_clock::now();
    if (ms) *ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (first_fail) *first_fail = TPSC_OK;
    for (int i = 0; i < npts; ++i)
        if (status[i]) {
            b->err = "point " + std::to_string(i) + " failed with status " + std::to_string(status[i]) +
                     " (first failure seen: " + first_msg + ")";
            if (first_fail) *first_fail = status[i];
            break;
        }
    return TPSC_OK;
}

// the solves of one call on n contexts, largest first (nk0^2 Nw0)
int run_points(tpsc_batch *b, int n, int form, int npts, const double *params, double *results, int *status,
               double *ms, int *first_fail) {
    std::vector<int> order(npts);
    for (int i = 0; i < npts; ++i) order[i] = i;
    auto cost = [&](int i) {
        const double *p = params + (size_t)i * kParamCols;
        return p[0] * p[0] * p[1];
    };
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
    auto task = [&](tpsc_ctx *c, int i) -> int {
        tpsc_set_form(c, form);
        const double *p = params + (size_t)i * kParamCols;
        int r = TPSC_ERR_ARG;
        if (p[0] == std::floor(p[0]) && p[1] == std::floor(p[1]))
            r = tpsc_set_model(c, (int)p[0], (int)p[1], p[2], p[3], p[4], p[5], p[6], p[7]);
        if (!r) r = tpsc_solve(c);
        double *out = results + (size_t)i * TPSC_S_COUNT;
        if (!r) r = tpsc_get_scalars(c, out, TPSC_S_COUNT);
        if (r == TPSC_ERR_NONFINITE) {
            tpsc_get_scalars(c, out, TPSC_S_COUNT);  // keep them: they show which one
        } else if (r) {
            for (int q = 0; q < TPSC_S_COUNT; ++q) out[q] = NAN;
        }
        return r;
    };
    return run_tasks(b, n, npts, order, task, status, ms, first_fail);
}

bool valid_args(tpsc_batch *b, int npts, const double *params, const double *results, const int *status) {
    if (!b) return false;
    if (npts < 0 || (npts > 0 && (!params || !results || !status))) {
        b->err = "bad arguments";
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

tpsc_batch *tpsc_batch_create(int device, int nstreams, int *status) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0 || device < 0 || device >= ndev) {
        if (status) *status = ndev == 0 ? TPSC_ERR_CUDA : TPSC_ERR_ARG;
        return nullptr;
    }
    if (nstreams < 1 || nstreams > kMaxStreams) {
        if (status) *status = TPSC_ERR_ARG;
        return nullptr;
    }
    tpsc_batch *b = new tpsc_batch;
    b->device = device;
    b->nstreams = nstreams;
    cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, device);
    const int rc = ensure_contexts(b, nstreams);
    if (rc) {
        if (status) *status = rc;
        tpsc_batch_destroy(b);
        return nullptr;
    }
    if (status) *status = TPSC_OK;
    return b;
}

void tpsc_batch_destroy(tpsc_batch *b) {
    if (!b) return;
    for (tpsc_ctx *c : b->ctxs) tpsc_destroy(c);
    delete b;
}

const char *tpsc_batch_last_error(const tpsc_batch *b) { return b ? b->err.c_str() : "null batch"; }

int tpsc_batch_set_graph_mode(tpsc_batch *b, int mode) {
    if (!b) return TPSC_ERR_ARG;
    if (mode < 0 || mode > 3) {
        b->err = "graph mode must be 0, 1, 2 or 3";
        return TPSC_ERR_ARG;
    }
    b->graph_mode = mode;
    for (tpsc_ctx *c : b->ctxs) tpsc_set_graph_mode(c, mode == 3 ? 2 : mode);
    return TPSC_OK;
}

int tpsc_batch_streams(const tpsc_batch *b, int *nstreams) {
    if (!b || !nstreams) return TPSC_ERR_ARG;
    *nstreams = b->nstreams;
    return TPSC_OK;
}

int tpsc_batch_solve(tpsc_batch *b, int form, int npts, const double *params, double *results, int *status,
                     double *ms) {
    if (!valid_args(b, npts, params, results, status)) return TPSC_ERR_ARG;
    if (b->graph_mode == 3 && form == (TPSC_FORM_NEWTON | TPSC_FORM_MIXED)) {
        // every shape group in one launch per stage (tpsc_solve_points)
        cudaSetDevice(b->device);
        int rc = tpsc_solve_points(b->ctxs[0], npts, params, results, status, ms);
        if (rc) {
            b->err = tpsc_last_error(b->ctxs[0]);
            return rc;
        }
        for (int i = 0; i < npts; ++i)
            if (status[i]) {
                b->err = "point " + std::to_string(i) + " failed with status " + std::to_string(status[i]) + " (" +
                         tpsc_last_error(b->ctxs[0]) + ")";
                return status[i];
            }
        return TPSC_OK;
    }
    int first = TPSC_OK;
    const int rc = run_points(b, b->nstreams, form, npts, params, results, status, ms, &first);
    return rc ? rc : first;
}

int tpsc_batch_tune(tpsc_batch *b, int form, int npts, const double *params, int max_streams, double *ms) {
    if (!b || npts <= 0 || !params || max_streams < 1 || max_streams > kMaxStreams) {
        if (b) b->err = "bad arguments";
        return TPSC_ERR_ARG;
    }
    std::vector<double> res((size_t)npts * TPSC_S_COUNT);
    std::vector<int> st(npts);
    // one untimed pass allocates every shape's grid on every context used
    // (failing points are timed like the others: their status is the same at
    // every count)
    int rc = run_points(b, max_streams, form, npts, params, res.data(), st.data(), nullptr, nullptr);
    if (rc) return rc;
    // the tau transforms' tiling of every shape, timed on its first good point
    std::set<std::pair<int, int>> tuned;
    tpsc_ctx *c0 = b->ctxs[0];
    for (int i = 0; i < npts; ++i) {
        const double *p = params + (size_t)i * kParamCols;
        const std::pair<int, int> shape((int)p[0], (int)p[1]);
        if (st[i] || tuned.count(shape)) continue;
        tuned.insert(shape);
        tpsc_set_form(c0, form);
        if (tpsc_set_model(c0, shape.first, shape.second, p[2], p[3], p[4], p[5], p[6], p[7]) == TPSC_OK &&
            tpsc_solve(c0) == TPSC_OK)
            tpsc_tune_tau_plans(c0, 3, nullptr);
    }
    double best = 0.0;
    int best_n = 1, k = 0;
    for (int n = 1; n <= max_streams; n *= 2, ++k) {
        double t = 0.0;
        rc = run_points(b, n, form, npts, params, res.data(), st.data(), &t, nullptr);
        if (rc) return rc;
        if (ms) ms[k] = t;
        if (n == 1 || t < best) {
            best = t;
            best_n = n;
        }
    }
    b->nstreams = best_n;
    return ensure_contexts(b, best_n);
}

int tpsc_batch_corr_length(tpsc_batch *b, int form, int nk0, int Nw0, double tp, double tpp, double t3, double U,
                           const double *dens, int nD, const double *Temp, int nT, double nsr, double mu_fs,
                           double *rows, int *status, double *ms) {
    if (!b) return TPSC_ERR_ARG;
    if (!dens || !Temp || nD < 1 || nT < 1 || !rows || !status) {
        b->err = "bad arguments";
        return TPSC_ERR_ARG;
    }
    // the grid of chi::calc_corr_length (src/chi.cpp:940-959), density-major
    const double n0 = dens[0], dn = nD > 1 ? (dens[1] - n0) / (nD - 1) : 0.0;
    const double T0 = Temp[0], dT = nT > 1 ? (Temp[1] - T0) / (nT - 1) : 0.0;
    const int npts = nD * nT;
    std::vector<int> order(npts);
    for (int i = 0; i < npts; ++i) order[i] = i;
    auto task = [&](tpsc_ctx *c, int i) -> int {
        const int l = i / nT, j = i % nT;
        const double n = n0 + l * dn, T = T0 + j * dT;
        double *row = rows + (size_t)i * kCorrCols;
        for (int q = 0; q < kCorrCols; ++q) row[q] = NAN;
        int r = tpsc_set_form(c, form);
        if (!r) r = tpsc_set_model(c, nk0, Nw0, n, T, tp, tpp, t3, U);
        if (!r && nsr > 0.0) r = tpsc_set_nsr(c, nsr);
        if (!r) r = tpsc_find_Usp_Uch(c);
        double sc[TPSC_S_COUNT], xi[7];
        if (!r) r = tpsc_get_scalars(c, sc, TPSC_S_COUNT);
        if (!r) r = tpsc_sp_corr_length_fs(c, std::isnan(mu_fs) ? sc[TPSC_S_MU0] : mu_fs, xi);
        if (r) return r;
        // the columns of the reference's corrLgth line (src/chi.cpp:967-975)
        const double v[kCorrCols] = {n, T, sc[TPSC_S_MU0], xi[0], sc[TPSC_S_USP], sc[TPSC_S_DIFRELSP],
                                     sc[TPSC_S_UCH], sc[TPSC_S_DIFRELCH], sc[TPSC_S_DBLOCC], xi[2], xi[1], xi[4],
                                     xi[3], xi[6], xi[5], (double)(nk0 / 2 + 1), sc[TPSC_S_QMAX0], sc[TPSC_S_QMAX1],
                                     sc[TPSC_S_CHI0MAX]};
        std::copy(v, v + kCorrCols, row);
        return TPSC_OK;
    };
    int first = TPSC_OK;
    const int rc = run_tasks(b, b->nstreams, npts, order, task, status, ms, &first);
    return rc ? rc : first;
}

int tpsc_sweep_points(int npts, unsigned long long seed, double *params) {
    if (npts < 0 || (npts > 0 && !params)) return TPSC_ERR_ARG;
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> lat(0, 3);
    std::uniform_real_distribution<double> uU(1.0, 6.0), un(0.7, 1.0), ulT(std::log(0.03), std::log(0.5)),
        utp(-0.3, 0.0);
    for (int i = 0; i < npts; ++i) {
        double *p = params + (size_t)i * kParamCols;
        const int L = 32 << lat(rng);
        const double U = uU(rng), n = un(rng), T = std::exp(ulT(rng)), tp = utp(rng);
        int pos = 1;
        const double need = std::ceil(40.0 / (3.141592653589793 * T));
        while (pos < need) pos *= 2;
        p[0] = L;
        p[1] = 2.0 * pos;
        p[2] = n;
        p[3] = T;
        p[4] = tp;
        p[5] = 0.0;
        p[6] = 0.0;
        p[7] = U;
    }
    return TPSC_OK;
}

}  // extern "C"
