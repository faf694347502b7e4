// tpsc_dropin.h -- C++ drop-in for the reference's TPSC class chain.
//
// The reference (dbergeron1/TPSC_conductivity) exposes its computation as the
// classes generique -> hamiltonien -> green0 -> chi0 -> chi -> green ->
// cond_opt.  These classes keep those names, that inheritance order and the
// public member functions a driver calls (src/tpsc_main.cpp and the
// commented-out blocks there), with the same argument meaning, so the
// reference's tpsc_main.cpp compiles unchanged against this directory.  Every
// computation goes through the C ABI of include/tpsc_b200.h on a CUDA device;
// the result files keep the reference's names and column layouts.
//
// Error behaviour follows the reference: failures print a message and the
// member function returns (the reference prints French messages and returns).
#ifndef TPSC_B200_DROPIN_H
#define TPSC_B200_DROPIN_H

#include <sys/stat.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <string>
#include <vector>

#include "../../include/tpsc_b200.h"

using namespace std;

typedef complex<double> dcomplex;

// numerical routines base class (root search, spline, Pade live in the engine)
class generique {
public:
    generique() {}
};

// lattice and model parameters (src/hamiltonien.h:24-57)
class hamiltonien : public generique {
public:
    hamiltonien(int nk0 = 8, double n = 1.0, double T = 1.0, double params[] = NULL);
    void set_U(double Up) { U = Up; }
    void set_tem(double T) { tem = T; }
    void set_density(double n) { density = n; }
    void get_params() const;

protected:
    double density, U, tp, tpp, t3, tem;
    int nbk;
};

// non-interacting Green's function; owns the device context (src/green0.h)
class green0 : public hamiltonien {
public:
    green0(int nk0 = 8, int Nw0 = 32, double n = 0.0, double T = 1.0, double params[] = NULL);
    virtual ~green0();
    void get_params() const;
    double get_mu() const { return mu0; }
    // hamiltonien::set_tem / set_density, then mu0 again (src/green0.h:35-38)
    void set_tem(double T);
    void set_density(double n);

protected:
    void find_mu_inf_syst();
    bool check(int status, const char *what) const;
    void set_model();
    virtual void model_changed() {}  // after set_model: the derived classes' own model state
    tpsc_ctx *ctx_;
    double mu0;
    double mu0_fs_;  // mu0 of the constructor: the Fermi surface's (src/green0.cpp:35)
    int nbw, nwmax;
    double scal_[TPSC_S_COUNT];
    void refresh();
};

// Lindhard function (src/chi0.h)
class chi0 : public green0 {
public:
    chi0(int nk0 = 8, int Nw0 = 32, double n = 1.0, double T = 1.0, double params[] = NULL);
    void set_keep_chirt(bool v) { keep_chirt = v; }
    void set_keep_chiqw(bool v) { keep_chiqw = v; }
    void set_save_chi0_q(bool v) { save_chi0_q = v; }
    void set_save_chi0_to_file(bool v) { save_chi0_to_file = v; }
    void calc_chiqw_FFT_spline(int nq0, int nw0);
    void traceChi0();
    void save_chi();
    double chiqw(double qx, double par[]);
    double chiqw_discret(int *q, int n);
    void calc_chi0_qlims(int n, double qlims[], int Nq[]);

protected:
    void loadChi0();
    bool keep_chirt, keep_chiqw, save_chi0_q, save_chi0_to_file;
    double chi0max;
    int qmax[2];
    int nbq;
};

// spin and charge response, Usp and Uch (src/chi.h)
class chi : public chi0 {
public:
    chi(int nk0 = 8, int Nw0 = 32, double n = 0.0, double T = 1.0, double *params = NULL);
    void get_params() const;
    void find_Usp_Uch();
    void find_Usp_Uch(int nq0, int nw0, double Usc[]);
    void sp_corr_length();
    void calc_corr_length(double dens[], int nD, double Temp[], int nT);

protected:
    void calc_chirt();
    void model_changed() override;  // keeps the constructor's nsr, as the reference does
    double Uch, Usp, dblOcc, nsr;
    double errUs, errUc;  // never assigned by the reference's find_Usp_Uch (src/chi.cpp:361-362 are commented out)
    double spCorrLgth_x, spCorrLgth_y, spCorrLgthAs_x, spCorrLgthAs_y, xi0_x, xi0_y, vF;
    char paramsFileName[200];
};

// interacting Green's function (src/green.h)
class green : public chi {
public:
    green(int nk0 = 8, int Nw0 = 32, double n = 1.0, double T = 1.0, double eta = 0.1, double *params = NULL);
    void get_params() const;
    double get_mu() { return mu; }
    void calc_Self_FFT_spline();
    void traceSelfG();
    void traceSelfG2();
    void find_mu();
    void find_FS_inter();
    void MDC(int *n, int Nn, double w, double *eta, int Neta, bool use_Pade = false);
    void Gwn_local();
    void save_self_ikn(int *k_save, int nk_save, int Nwn);
    void save_Green(int *k);
    void save_Self(int Nfreq);
    void calc_Self_Re_w(int *k, int *n, int Nn, double *w, int Nw, double *eta, int Neta);
    void calc_Self_Re_w_BZ(int *n, int Nn, double *w, int Nw, double *eta, int Neta);
    // spectral weight and energy distribution curves (src/green.cpp:554-812, 1073-1260)
    void calc_spectral_weight(int *k, double *w, int nw0, int N, double *spectr_w);
    void calc_spectral_weight(double *x, double *w, int nw0, double *spectr_w) {
        int k[2];
        double eps = 0.5 / nbk;
        double f = (x[0] + eps) * nbk;
        k[0] = (int)f;
        f = (x[1] + eps) * nbk;
        k[1] = (int)f;
        calc_spectral_weight(k, w, nw0, nbw / 2, spectr_w);
    }
    void calc_spectral_weight(int *k, double *w, int nw0, int N, double *eta_p, int N_eta, double *spectr_w);
    void EDC(int *kx, int *ky, int Nk, char *fname);
    void create_non_uniform_ind_freq(int m);
    void EDC(int *kx, int *ky, int Nk, double *w, int nw0, int m_freq, int NP_max, double *eta_p, int N_eta,
             char *fname);

protected:
    void self_re_w(const int *ks, int nk, int *n, int Nn, double *w, int Nw, double *eta, int Neta);
    // A(k, w + i eta) at the nk octant points ks (folded pairs) from the N-point
    // continued fraction through z0[0..N) with Sigma read at the stored
    // frequencies 0..N-1: out[(p nw0 + j) neta + l]; one batched device Pade
    bool spectra(const int *ks, int nk, const double *z0, int N, const double *w, int nw0, const double *eta, int neta,
                 double *out);
    std::vector<int> ind_freq;   // create_non_uniform_ind_freq
    std::vector<double> pade_z0; // i (2 ind_freq[j] + 1) pi T, interleaved
    int N_freq = 0, m_freq = 0;
    void load_Self();
    void save_Self_bin();
    void load_Self_bin();
    double eta, mu, Sigma_inf;
    bool mu_calcule, have_self;
};

// optical conductivity (src/cond_opt.h)
class cond_opt : public green {
public:
    cond_opt(int nk0 = 8, int Nw0 = 256, double n = 1.0, double T = 1.0, double eta = 0.1, double *params = NULL);
    virtual ~cond_opt();
    // the bubble and the Maki-Thompson correction; with chi3 also the
    // Aslamazov-Larkin correction on the non-uniform iqn grid of mmin
    void calc_chijj_vertex_corr_all_optim(bool chi3, int mmin, int N_theta_k, int *k_chijj, int nk_chijj);

protected:
    // the chi3 branch (device AL correction and its files)
    void calc_chijj3(int mmin, int N_theta_k);
    double *chijj1_qn, *chijj2_qn;  // [Nw0/2 + 1]
    double *chijj3_qn;              // [Nw0/2 + 1]: the AL correction at the first N entries (grid order)
    double kx0;
};

#endif
