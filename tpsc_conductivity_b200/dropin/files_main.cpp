// files_main.cpp -- the saved-run formats through the drop-in classes.
//
//   files_main_b200 save|load|corr|rew|edc|chi0inf U tp tpp t3 n T nk0 Nw0
//
// save: the model is solved as src/tpsc_main.cpp solves it
// (calc_Self_FFT_spline, traceSelfG, find_mu), then written with the
// reference's writers chi0::save_chi, green::save_Self(0), green::save_Self_bin
// and green::save_Green({2, 1}); a second object of the same model then loads
// the self_bin file back (green::load_Self_bin) and finds mu again.
// load: only that second part, on a self_bin file already in the directory
// (for instance one the reference wrote).
// corr: chi::calc_corr_length({n, n + 0.05}, 2, {T, 1.5 T}, 2), the (n, T)
// scan that writes the corrLgth file.
// rew: the solve, then green::calc_Self_Re_w_BZ(n = 0..15, 16, w = -4..4
// (9 points), 9, eta = {0.05, 0.01}, 2): the real-frequency Sigma and A(k, w)
// files of every k of the reduced zone.
// edc: the solve, then green::EDC over the reduced zone and over the k list
// {(-3, 1), (10, 2)} (non-uniform grid m = 1, NP_max = 8, w = -2..2, eta =
// {0.05, 0.1}; prefixes edc and edcl) and green::EDC({3}, {1}, 1, "edc2").
// chi0inf: chi0::chiqw_discret({2, 1}, 1), then chi0::calc_chi0_qlims(n,
// {0, 0, pi, pi}, {3, 3}) for n = 0, 1 (the infinite lattice); prints
// "chi_discret", "mu0_finite" and, after the scans, "mu0_inf".
// Prints "mu <value>" per find_mu, 17 significant digits.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "cond_opt.h"

// reaches the protected loader and binary writer, as a program deriving from
// green would
class files_green : public green {
public:
    files_green(int nk0, int Nw0, double n, double T, double eta, double *p) : green(nk0, Nw0, n, T, eta, p) {}
    void warm_start() { load_Self_bin(); }
    void save_bin() { save_Self_bin(); }
    double mu0_now() const { return mu0; }
};

int main(int argc, char **argv) {
    if (argc != 10 ||
        (strcmp(argv[1], "save") && strcmp(argv[1], "load") && strcmp(argv[1], "corr") && strcmp(argv[1], "rew") &&
         strcmp(argv[1], "edc") && strcmp(argv[1], "chi0inf"))) {
        fprintf(stderr, "usage: %s save|load|corr|rew|edc|chi0inf U tp tpp t3 n T nk0 Nw0\n", argv[0]);
        return 1;
    }
    const bool save = !strcmp(argv[1], "save");
    double params[] = {atof(argv[3]), atof(argv[4]), atof(argv[5]), atof(argv[2])};
    const double n = atof(argv[6]), T = atof(argv[7]);
    const int nk0 = atoi(argv[8]), Nw0 = atoi(argv[9]);
    if (!strcmp(argv[1], "chi0inf")) {
        files_green g(nk0, Nw0, n, T, 0.1, params);
        int q[2] = {2, 1};
        printf("chi_discret %.17g\nmu0_finite %.17g\n", g.chiqw_discret(q, 1), g.mu0_now());
        const double pi = acos(-1.0);
        double qlims[4] = {0.0, 0.0, pi, pi};
        int Nq[2] = {3, 3};
        g.calc_chi0_qlims(0, qlims, Nq);
        g.calc_chi0_qlims(1, qlims, Nq);
        printf("mu0_inf %.17g\n", g.mu0_now());
        return 0;
    }
    if (!strcmp(argv[1], "edc")) {
        files_green g(nk0, Nw0, n, T, 0.1, params);
        g.calc_Self_FFT_spline();
        g.traceSelfG();
        g.find_mu();
        double w[5] = {-2.0, -1.0, 0.0, 1.0, 2.0}, eta[2] = {0.05, 0.1};
        char f1[] = "edc", f2[] = "edcl", f3[] = "edc2";
        g.EDC(NULL, NULL, 0, w, 5, 1, 8, eta, 2, f1);
        int kx[2] = {-3, 10}, ky[2] = {1, 2};
        g.EDC(kx, ky, 2, w, 5, 1, 8, eta, 2, f2);
        int kx2[1] = {3}, ky2[1] = {1};
        g.EDC(kx2, ky2, 1, f3);
        return 0;
    }
    if (!strcmp(argv[1], "rew")) {
        files_green g(nk0, Nw0, n, T, 0.1, params);
        g.calc_Self_FFT_spline();
        g.traceSelfG();
        g.find_mu();
        int nn[16];
        for (int j = 0; j < 16; j++) nn[j] = j;
        double w[9], eta[2] = {0.05, 0.01};
        for (int j = 0; j < 9; j++) w[j] = -4.0 + j;
        g.calc_Self_Re_w_BZ(nn, 16, w, 9, eta, 2);
        return 0;
    }
    if (!strcmp(argv[1], "corr")) {
        files_green c(nk0, Nw0, n, T, 0.1, params);
        double dens[2] = {n, n + 0.05}, temp[2] = {T, 1.5 * T};
        c.calc_corr_length(dens, 2, temp, 2);
        return 0;
    }
    if (save) {
        files_green g(nk0, Nw0, n, T, 0.1, params);
        g.set_keep_chiqw(true);
        g.calc_Self_FFT_spline();
        g.traceSelfG();
        g.find_mu();
        printf("mu %.17g\n", g.get_mu());
        g.save_chi();
        g.save_Self(0);
        g.save_bin();
        int k[2] = {2, 1};
        g.save_Green(k);
    }
    // warm start: the tails come from this object's own Sigma stage, S from the file
    files_green h(nk0, Nw0, n, T, 0.1, params);
    h.calc_Self_FFT_spline();
    h.warm_start();
    h.find_mu();
    printf("mu %.17g\n", h.get_mu());
    return 0;
}
