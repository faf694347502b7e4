// cond_main.cpp -- driver for the conductivity block of the reference's
// src/tpsc_main.cpp (lines 220-249, shipped there commented out): read the
// model from ../../input.dat as the reference's driver does
// (U tp tpp t3 n T nk0 Nw0 chijj3 mmin, src/tpsc_main.cpp:33), plus an
// optional N_theta_k, and run cond_opt::calc_chijj_vertex_corr_all_optim.
// Written against the class interface only, so the same file builds against
// the reference's cond_opt.h or this directory's.
#include "cond_opt.h"

int main() {
    double U, tp, tpp, t3, n, T;
    int nk0, Nw0, mmin, N_theta_k = 1;
    bool chijj3;
    fstream inputFile;
    inputFile.open("../../input.dat", ios::in);
    if (!inputFile) {
        cout << "echec d'ouverture de input.dat" << '\n';
        return 0;
    }
    inputFile >> U >> tp >> tpp >> t3 >> n >> T >> nk0 >> Nw0 >> chijj3 >> mmin;
    if (!(inputFile >> N_theta_k)) N_theta_k = 1;
    inputFile.close();
    double paramsHub[] = {tp, tpp, t3, U};
    const double eta = 0.1;
    cond_opt *sigma1 = new cond_opt(nk0, Nw0, n, T, eta, paramsHub);
    sigma1->calc_chijj_vertex_corr_all_optim(chijj3, mmin, N_theta_k, NULL, 0);
    delete sigma1;
    return 0;
}
