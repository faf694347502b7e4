/*
 * probe.cpp -- driver for the CPU oracle binary oracle/_ref/tpsc_ref_probe.
 *
 * TEST INFRASTRUCTURE.  It is compiled together with the UNMODIFIED reference
 * sources (src/*.cpp of dbergeron1/TPSC_conductivity, read in place) and the
 * FFTW shim in this folder.  It derives from the reference's cond_opt class
 * only to reach the protected result arrays, runs the reference's own public
 * methods in the order src/tpsc_main.cpp:61-75 uses, times them with
 * omp_get_wtime, and dumps the results as raw little-endian doubles.
 *
 * usage: tpsc_ref_probe OUTDIR MODE U tp tpp t3 n T nk0 Nw0
 *   MODE chi0   chi0::calc_chiqw_FFT_spline(nk0, Nw0)            (chi0.cpp:279)
 *        solve  green::calc_Self_FFT_spline(); traceSelfG(); find_mu()
 *               (green.cpp:1673, 3001, 3185) -- the full TPSC solve -- then
 *               chi::sp_corr_length() (chi.cpp:450) on the full-grid chi0
 *        cond   solve + cond_opt::calc_chijj_vertex_corr_all_optim(false,3,N,NULL,0)
 *               (cond_opt.cpp:2537), N = $TPSC_PROBE_NTHETA (default 1) angle bins
 *        cond3  the same with chi3 = true and mmin = $TPSC_PROBE_MMIN (default 3):
 *               also the Aslamazov-Larkin correction chijj3 on the non-uniform
 *               iqn grid (cond_opt.cpp:4292-6529)
 *        post   solve + find_FS_inter, MDC(10 points, w=0, 4 etas), Gwn_local
 *               (src/tpsc_main.cpp:77-114)
 *        bench  timings only: the half-grid pre-pass alone, then the solve
 *        corr   chi::calc_corr_length({n, n + 0.05}, 2, {T, 1.5 T}, 2)
 *               (src/chi.cpp:931-981): the (n, T) scan of Usp, Uch and the
 *               correlation lengths; the reference writes its corrLgth file
 *        rew    solve, then green::calc_Self_Re_w_BZ(n = 0..15, 16, w = -4..4
 *               (9 points), 9, eta = {0.05, 0.01}, 2) (src/green.cpp:386-542):
 *               Pade and J-fraction Sigma(k, w + i eta) and A(k, w) files for
 *               every k of the reduced zone
 *        edc    solve, then green::EDC over the reduced zone and over a k list
 *               (non-uniform grid m = 1, NP_max = 8, w = -2..2 (5 points),
 *               eta = {0.05, 0.1}) and green::EDC({3}, {1}, 1, "edc2")
 *               (src/green.cpp:589-812), on one OpenMP thread: the first
 *               overload shares its Pade buffers (members) between threads
 *        chi0inf  chi0::calc_chi0_qlims(n, {0, 0, pi, pi}, {3, 3}) for n = 0, 1
 *               (the infinite lattice by adaptive quadrature, src/chi0.cpp:157-276)
 *               and chi0::chiqw_discret({2, 1}, 1) on the constructor's lattice
 *        fftbench  timings of the FFTW shim alone, single thread, on the
 *               transforms the reference runs: 2D REDFT00 of nk0/2+1 points
 *               square, 2D RODFT00 x REDFT00 of (nk0/2-1) x (nk0/2+1), 1D
 *               complex DFT of Nw0 points (seconds per transform in meta.txt)
 *        files  solve, then the reference's own writers of the saved-run
 *               formats: chi0::save_chi, green::save_Self(0),
 *               green::save_Self_bin, green::save_Green({2, 1})
 *               (src/chi0.cpp:61, src/green.cpp:1496-1633)
 * The reference writes its own text files into the current directory; the
 * probe chdir()s into OUTDIR/work first so they land there.
 */
#include "cond_opt.h"

#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

// transforms the FFTW shim has executed, per kind (fftw_shim.cpp)
extern "C" void oracle_fftw_counts(long out[4]);

class tpsc_probe : public cond_opt {
public:
    tpsc_probe(int nk0, int Nw0, double n, double T, double eta, double *p)
        : cond_opt(nk0, Nw0, n, T, eta, p) {}

    int nk8() const { return (nbq * (nbq + 1)) / 2; }

    void dump_chi0(FILE *meta, const std::string &dir) {
        const long n8 = nk8();
        const long nw = nwmax + 1;
        fprintf(meta, "nbq %d\nnwmax %d\nmu0 %.17g\nchi0max %.17g\nqmax0 %d\nqmax1 %d\n", nbq,
                nwmax, mu0, chi0max, qmax[0], qmax[1]);
        write(dir + "/chiqw.bin", chiqw_array, n8 * nw);
        write(dir + "/chi0_inf.bin", chi0_inf, n8);
        write(dir + "/chi0_inf2.bin", chi0_inf2, n8);
        write(dir + "/dtau_chirt0.bin", dtau_chirt0, n8);
        write(dir + "/dtau_Grt0p.bin", dtau_Grt0p, n8);
        if (chirt) write(dir + "/chirt.bin", chirt, n8 * nw);
        write(dir + "/ek.bin", ek, (long)nbk * nbk);
    }

    void dump_solve(FILE *meta, const std::string &dir) {
        const long n8 = nk8();
        fprintf(meta, "Usp %.17g\nUch %.17g\ndblOcc %.17g\nSigma_inf %.17g\nmu %.17g\nnbw %d\n",
                Usp, Uch, dblOcc, Sigma_inf, mu, nbw);
        write(dir + "/vertex_rt.bin", vertex_rt_array, n8 * (nwmax + 1));
        write(dir + "/self.bin", reinterpret_cast<double *>(Self_kw_array), 2 * n8 * (nbw / 2));
        write(dir + "/sigma_inf2.bin", Sigma_inf2, n8);
        write(dir + "/sigma_inf3.bin", Sigma_inf3, n8);
        write(dir + "/sigma_inf4.bin", Sigma_inf4, n8);
    }

    // chi::sp_corr_length (src/chi.cpp:450-718) on the full-grid chi0 and Usp,
    // with the Fermi surface green0::find_FS(10001) computed at construction
    void dump_corr(FILE *meta) {
        sp_corr_length();
        fprintf(meta, "vF %.17g\nxi_y %.17g\nxi_x %.17g\nxiAs_y %.17g\nxiAs_x %.17g\nxi0_y %.17g\nxi0_x %.17g\n",
                vF, spCorrLgth_y, spCorrLgth_x, spCorrLgthAs_y, spCorrLgthAs_x, xi0_y, xi0_x);
    }

    // the infinite-lattice chi0 files, the infinite mu0 they leave in mu0,
    // and the finite-lattice sum at q = (2, 1), n = 1
    void chi0_infinite(FILE *meta) {
        int q[2] = {2, 1};
        fprintf(meta, "chi_discret %.17g\nmu0_finite %.17g\n", chiqw_discret(q, 1), mu0);
        const double pi = acos(-1.0);
        double qlims[4] = {0.0, 0.0, pi, pi};
        int Nq[2] = {3, 3};
        calc_chi0_qlims(0, qlims, Nq);
        calc_chi0_qlims(1, qlims, Nq);
        fprintf(meta, "mu0_inf %.17g\n", mu0);
    }

    // the saved-run formats, written by the reference's own methods
    void save_files() {
        save_chi();
        save_Self(0);
        save_Self_bin();
        int k[2] = {2, 1};
        save_Green(k);
    }

    void dump_cond(FILE *meta, const std::string &dir) {
        fprintf(meta, "kx0 %.17g\n", kx0);
        write(dir + "/chijj1.bin", chijj1_qn, nbw / 2 + 1);
        write(dir + "/chijj2.bin", chijj2_qn, nbw / 2 + 1);
    }

    // chijj3_qn holds the AL correction at the first N entries, N the size of
    // the non-uniform grid of src/cond_opt.cpp:5123-5126
    void dump_cond3(FILE *meta, const std::string &dir, int mmin) {
        const int N0 = nbw / 2 + 1;
        const int N = mmin * ((N0 - 1) / (1 << (mmin + 1))) + (N0 - 1) / (1 << mmin) + 1;
        fprintf(meta, "mmin %d\nn_al %d\n", mmin, N);
        write(dir + "/chijj3.bin", chijj3_qn, N);
    }

private:
    static void write(const std::string &path, const double *p, long n) {
        if (!p) return;
        FILE *f = fopen(path.c_str(), "wb");
        if (!f) {
            perror(path.c_str());
            exit(2);
        }
        fwrite(p, sizeof(double), n, f);
        fclose(f);
    }
};

int main(int argc, char **argv) {
    if (argc != 11) {
        fprintf(stderr, "usage: %s OUTDIR MODE U tp tpp t3 n T nk0 Nw0\n", argv[0]);
        return 1;
    }
    std::string dir = argv[1];
    std::string mode = argv[2];
    double U = atof(argv[3]), tp = atof(argv[4]), tpp = atof(argv[5]), t3 = atof(argv[6]);
    double n = atof(argv[7]), T = atof(argv[8]);
    int nk0 = atoi(argv[9]), Nw0 = atoi(argv[10]);
    double params[] = {tp, tpp, t3, U};

    mkdir(dir.c_str(), 0755);
    std::string work = dir + "/work";
    mkdir(work.c_str(), 0755);
    char cwd[4096];
    if (!getcwd(cwd, sizeof cwd)) return 2;
    std::string absdir = dir[0] == '/' ? dir : std::string(cwd) + "/" + dir;
    if (chdir(work.c_str())) return 2;

    // capture the reference's stdout (it prints the sum-rule traces there)
    std::stringstream captured;
    std::streambuf *orig = std::cout.rdbuf(captured.rdbuf());
    std::cout << std::setprecision(17);

    double t0 = omp_get_wtime();
    tpsc_probe *g = new tpsc_probe(nk0, Nw0, n, T, 0.1, params);
    double t_ctor = omp_get_wtime() - t0;

    FILE *meta = fopen((absdir + "/meta.txt").c_str(), "w");
    fprintf(meta, "mode %s\nU %.17g\ntp %.17g\ntpp %.17g\nt3 %.17g\nn %.17g\nT %.17g\nnk0 %d\nNw0 %d\n",
            mode.c_str(), U, tp, tpp, t3, n, T, nk0, Nw0);
    fprintf(meta, "omp_threads %d\nt_ctor %.6f\n", omp_get_max_threads(), t_ctor);

    if (mode == "chi0") {
        g->set_keep_chirt(true);
        t0 = omp_get_wtime();
        g->calc_chiqw_FFT_spline(nk0, Nw0);
        fprintf(meta, "t_chi0 %.6f\n", omp_get_wtime() - t0);
        g->dump_chi0(meta, absdir);
    } else if (mode == "chi0inf") {
        t0 = omp_get_wtime();
        g->chi0_infinite(meta);
        fprintf(meta, "t_chi0inf %.6f\n", omp_get_wtime() - t0);
    } else if (mode == "fftbench") {
        const int nb = nk0 / 2 + 1;
        std::vector<double> a((size_t)nb * nb, 0.5), b((size_t)(nb - 2) * nb, 0.5);
        std::vector<fftw_complex> c(Nw0);
        for (int j = 0; j < Nw0; j++) c[j][0] = c[j][1] = 1.0 / (j + 1);
        for (size_t j = 0; j < a.size(); j++) a[j] = 1.0 / (j + 1);
        for (size_t j = 0; j < b.size(); j++) b[j] = 1.0 / (j + 2);
        fftw_plan p1 = fftw_plan_r2r_2d(nb, nb, a.data(), a.data(), FFTW_REDFT00, FFTW_REDFT00, FFTW_MEASURE);
        fftw_plan p2 = fftw_plan_r2r_2d(nb - 2, nb, b.data(), b.data(), FFTW_RODFT00, FFTW_REDFT00, FFTW_MEASURE);
        fftw_plan p3 = fftw_plan_dft_1d(Nw0, c.data(), c.data(), FFTW_FORWARD, FFTW_MEASURE);
        auto time_it = [&](fftw_plan p, const char *key) {
            int reps = 1;
            double dt = 0.0;
            for (;;) {
                t0 = omp_get_wtime();
                for (int r = 0; r < reps; r++) fftw_execute(p);
                dt = omp_get_wtime() - t0;
                if (dt > 0.5) break;
                reps *= 2;
            }
            fprintf(meta, "%s %.9g\n", key, dt / reps);
        };
        time_it(p1, "t_dct2d");
        time_it(p2, "t_dstdct2d");
        time_it(p3, "t_dft1d");
        fftw_destroy_plan(p1);
        fftw_destroy_plan(p2);
        fftw_destroy_plan(p3);
    } else if (mode == "corr") {
        double dens[2] = {n, n + 0.05}, temp[2] = {T, 1.5 * T};
        t0 = omp_get_wtime();
        g->calc_corr_length(dens, 2, temp, 2);
        fprintf(meta, "t_corr %.6f\n", omp_get_wtime() - t0);
    } else if (mode == "bench") {
        // timing only: the solve exactly as src/tpsc_main.cpp:71-75 runs it, then
        // the half-grid Usp/Uch pass that calc_Self_FFT_spline runs first
        // (src/chi.cpp:285-297) timed on its own so it can be subtracted (it
        // re-grids the object, so it must come after the solve)
        double Usc[2] = {0, 0};
        g->set_keep_chiqw(false);
        t0 = omp_get_wtime();
        g->calc_Self_FFT_spline();
        double t_self = omp_get_wtime() - t0;
        t0 = omp_get_wtime();
        g->traceSelfG();
        double t_tr = omp_get_wtime() - t0;
        t0 = omp_get_wtime();
        g->find_mu();
        double t_mu = omp_get_wtime() - t0;
        fprintf(meta, "t_self %.6f\nt_traceSelfG %.6f\nt_find_mu %.6f\n", t_self, t_tr, t_mu);
        fprintf(meta, "mu %.17g\n", g->get_mu());
        long cnt[4];
        oracle_fftw_counts(cnt);
        fprintf(meta, "n_r2r_2d %ld\nn_r2r_1d %ld\nn_dft_1d %ld\nn_dft_2d %ld\n", cnt[0], cnt[1], cnt[2], cnt[3]);
        t0 = omp_get_wtime();
        g->find_Usp_Uch(nk0 / 2, Nw0 / 2, Usc);
        fprintf(meta, "t_half %.6f\n", omp_get_wtime() - t0);
    } else if (mode == "solve" || mode == "post" || mode == "cond" || mode == "cond3" || mode == "files" ||
               mode == "rew" || mode == "edc") {
        g->set_keep_chiqw(true);
        t0 = omp_get_wtime();
        g->calc_Self_FFT_spline();
        double t_self = omp_get_wtime() - t0;
        std::cout << std::setprecision(17);
        t0 = omp_get_wtime();
        g->traceSelfG();
        double t_tr = omp_get_wtime() - t0;
        std::cout << std::setprecision(17);
        t0 = omp_get_wtime();
        g->find_mu();
        double t_mu = omp_get_wtime() - t0;
        fprintf(meta, "t_self %.6f\nt_traceSelfG %.6f\nt_find_mu %.6f\n", t_self, t_tr, t_mu);
        g->dump_chi0(meta, absdir);
        g->dump_solve(meta, absdir);
        g->dump_corr(meta);
        if (mode == "files") g->save_files();
        if (mode == "edc") {
            omp_set_num_threads(1);
            double w[5] = {-2.0, -1.0, 0.0, 1.0, 2.0}, eta[2] = {0.05, 0.1};
            char f1[] = "edc", f2[] = "edcl", f3[] = "edc2";
            g->EDC(NULL, NULL, 0, w, 5, 1, 8, eta, 2, f1);
            int kx[2] = {-3, 10}, ky[2] = {1, 2};
            g->EDC(kx, ky, 2, w, 5, 1, 8, eta, 2, f2);
            int kx2[1] = {3}, ky2[1] = {1};
            g->EDC(kx2, ky2, 1, f3);
        }
        if (mode == "rew") {
            int nn[16];
            for (int j = 0; j < 16; j++) nn[j] = j;
            double w[9], eta[2] = {0.05, 0.01};
            for (int j = 0; j < 9; j++) w[j] = -4.0 + j;
            g->calc_Self_Re_w_BZ(nn, 16, w, 9, eta, 2);
        }
        if (mode == "post" || mode == "cond" || mode == "cond3") {
            // the post-processing tpsc_main.cpp runs after find_mu (lines 77-114)
            g->find_FS_inter();
            int NP = 10;
            double eta_p[] = {0.01, 0.001, 0.0001, 0.00001};
            int *n_qn = new int[Nw0 / 2];
            for (int j = 0; j < Nw0 / 2; j++) n_qn[j] = j;
            g->MDC(n_qn, NP, 0.0, eta_p, 4, true);
            delete[] n_qn;
            g->Gwn_local();
        }
        if (mode == "cond") {
            std::cout << std::setprecision(17);
            t0 = omp_get_wtime();
            const char *nt = getenv("TPSC_PROBE_NTHETA");
            const int ntheta = nt ? atoi(nt) : 1;
            fprintf(meta, "ntheta %d\n", ntheta);
            g->calc_chijj_vertex_corr_all_optim(false, 3, ntheta, NULL, 0);
            fprintf(meta, "t_cond %.6f\n", omp_get_wtime() - t0);
            g->dump_cond(meta, absdir);
        }
        if (mode == "cond3") {
            std::cout << std::setprecision(17);
            t0 = omp_get_wtime();
            const char *nt = getenv("TPSC_PROBE_NTHETA");
            const int ntheta = nt ? atoi(nt) : 1;
            const char *mm = getenv("TPSC_PROBE_MMIN");
            const int mmin = mm ? atoi(mm) : 3;
            fprintf(meta, "ntheta %d\n", ntheta);
            g->calc_chijj_vertex_corr_all_optim(true, mmin, ntheta, NULL, 0);
            fprintf(meta, "t_cond %.6f\n", omp_get_wtime() - t0);
            g->dump_cond(meta, absdir);
            g->dump_cond3(meta, absdir, mmin);
        }
    } else {
        fprintf(stderr, "unknown mode %s\n", mode.c_str());
        return 1;
    }
    fclose(meta);
    delete g;

    std::cout.rdbuf(orig);
    FILE *log = fopen((absdir + "/stdout.txt").c_str(), "w");
    std::string s = captured.str();
    fwrite(s.data(), 1, s.size(), log);
    fclose(log);
    return 0;
}
