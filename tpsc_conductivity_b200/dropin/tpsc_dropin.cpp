// tpsc_dropin.cpp -- the drop-in classes of tpsc_dropin.h over the C ABI.
//
// Result files keep the reference's names (sprintf formats) and column
// layouts so that tools reading the reference's output read these too:
// TPSC_infos_* / TPSCparams_* (src/chi.cpp:375-415), the traces
// (src/green.cpp:3091-3102, 2982-2995), mu0_mu_D_* (src/green.cpp:3272-3279),
// FS_inter_* (src/green.cpp:2227-2330), Akw/Self_Pade_k_* and *_poly_k_*
// (src/green.cpp:838-1060), Gwn_loc_* (src/green.cpp:225-263) and the chi0
// dumps (src/chi0.cpp:720-742).
#include "tpsc_dropin.h"

#include <complex>
#include <vector>

namespace {

int device_from_env() {
    const char *d = getenv("TPSC_DEVICE");
    return d ? atoi(d) : 0;
}

}  // namespace

// ---------------------------------------------------------------------------
hamiltonien::hamiltonien(int nk0, double n, double T, double params[]) {
    nbk = nk0 / 2 + 1;
    density = n;
    tem = T;
    if (params) {
        tp = params[0];
        tpp = params[1];
        t3 = params[2];
        U = params[3];
    } else {
        tp = tpp = t3 = 0;
        U = 1;
    }
}

void hamiltonien::get_params() const {
    cout << setiosflags(ios::left) << "U: " << setw(10) << U << "tp: " << setw(10) << tp << "tpp: " << setw(10)
         << tpp << "t3: " << setw(10) << t3 << "density: " << setw(10) << density << "T: " << tem << endl;
}

// ---------------------------------------------------------------------------
green0::green0(int nk0, int Nw0, double n, double T, double params[]) : hamiltonien(nk0, n, T, params) {
    nbw = Nw0;
    nwmax = (nbw - 2) / 2;
    mu0 = 0.0;
    for (double &s : scal_) s = 0.0;
    int st = 0;
    ctx_ = tpsc_create(device_from_env(), &st);
    if (!ctx_) {
        cout << "tpsc: no CUDA context (" << tpsc_last_error(NULL) << ")" << endl;
        return;
    }
    if (check(tpsc_set_model(ctx_, nk0, Nw0, n, T, tp, tpp, t3, U), "tpsc_set_model")) {
        refresh();
        mu0 = scal_[TPSC_S_MU0];
        cout << "mu0 du systeme fini: " << mu0 << endl;
    }
    mu0_fs_ = mu0;
}

// the model of the current members on the current grid; mu0 again
void green0::set_model() {
    if (!ctx_ || !check(tpsc_set_model(ctx_, 2 * (nbk - 1), nbw, density, tem, tp, tpp, t3, U), "tpsc_set_model"))
        return;
    refresh();
    mu0 = scal_[TPSC_S_MU0];
    model_changed();
}

void green0::set_tem(double T) {
    tem = T;
    set_model();
}

void green0::set_density(double n) {
    density = n;
    set_model();
}

green0::~green0() {
    if (ctx_) tpsc_destroy(ctx_);
}

bool green0::check(int status, const char *what) const {
    if (status == TPSC_OK) return true;
    cout << what << ": " << tpsc_last_error(ctx_) << " (status " << status << ")" << endl;
    return false;
}

void green0::refresh() {
    if (ctx_) tpsc_get_scalars(ctx_, scal_, TPSC_S_COUNT);
}

void green0::get_params() const {
    hamiltonien::get_params();
    cout << "mu0: " << mu0 << '\n';
}

// ---------------------------------------------------------------------------
chi0::chi0(int nk0, int Nw0, double n, double T, double params[]) : green0(nk0, Nw0, n, T, params) {
    nbq = nk0 / 2 + 1;
    nwmax = Nw0 / 2;
    keep_chirt = keep_chiqw = save_chi0_q = save_chi0_to_file = true;
    chi0max = 0.0;
    qmax[0] = qmax[1] = 0;
}

void chi0::calc_chiqw_FFT_spline(int nq0, int nw0) {
    cout << "calcul de chi0 par calc_chiqw_FFT_spline()\n";
    if (!ctx_ || !check(tpsc_chi0(ctx_, nq0, nw0), "calc_chiqw_FFT_spline")) return;
    nbq = nbk = nq0 / 2 + 1;
    nbw = nw0;
    nwmax = nw0 / 2;
    refresh();
    mu0 = scal_[TPSC_S_MU0];
    chi0max = scal_[TPSC_S_CHI0MAX];
    qmax[0] = (int)scal_[TPSC_S_QMAX0];
    qmax[1] = (int)scal_[TPSC_S_QMAX1];
    cout << "qxmax, qymax: " << qmax[0] << ",  " << qmax[1] << '\n';
    if (save_chi0_q) {
        const int nw = nwmax + 1, n8 = nbq * (nbq + 1) / 2;
        std::vector<double> c((size_t)nw * n8);
        if (check(tpsc_get_chi0(ctx_, c.data(), NULL, NULL, NULL), "tpsc_get_chi0")) {
            char name[300];
            fstream file;
            int l = qmax[0], m = qmax[1];
            sprintf(name, "./chi0_qmax_wn_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%d_%d_%d_%d.dat", tp, tpp, t3, density, tem,
                    nq0, nw0, l, m);
            file.open(name, ios::out);
            file << setiosflags(ios::left) << setprecision(16);
            for (int j = 0; j < nw; j++) file << setw(10) << j << c[m + (l * (l + 1)) / 2 + (size_t)j * n8] << '\n';
            file.close();
            sprintf(name, "./chi0_wn0_q_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%d_%d.dat", tp, tpp, t3, density, tem, nq0,
                    nw0);
            file.open(name, ios::out);
            file << setiosflags(ios::left) << setprecision(16);
            for (l = 0; l < nbq; l++)
                for (m = 0; m <= l; m++) file << setw(10) << l << setw(10) << m << c[m + (l * (l + 1)) / 2] << '\n';
            file.close();
        }
    }
    traceChi0();
}

void chi0::traceChi0() {
    double tr[2];
    if (!ctx_ || !check(tpsc_trace_chi0(ctx_, tr), "traceChi0")) return;
    const double ex = density - density * density / 2.0;
    cout << setprecision(14);
    cout << "trace(chi0(q,iwn)):   " << tr[0] << "\tn-n^2/2:   " << ex << "\tdifference relative:  "
         << (ex - tr[0]) / ex << '\n';
    cout << "trace(chi0(q,iwn))(+correction asymptotique):   " << tr[1] << "\tn-n^2/2:   " << ex
         << "\tdifference relative:  " << (ex - tr[1]) / ex << '\n';
}

// green0::find_mu_inf_syst (src/green0.cpp:265-287): mu0 of the infinite
// lattice becomes the object's mu0, as in the reference (chiqw reads it); the
// engine's finite-lattice mu0 for the TPSC stages is not changed
void green0::find_mu_inf_syst() {
    double mu;
    if (!ctx_ || tpsc_mu0_infinite(ctx_, &mu, NULL) != TPSC_OK) {
        cout << "mu0 non trouve\n";
        return;
    }
    mu0 = mu;
    cout << "mu0 du systeme infini: " << mu0 << endl;
}

// chi0::chiqw (src/chi0.cpp:211-276): chi0(q, i w_n) of the infinite lattice,
// q = (qx, par[0]), w_n = par[1], at the object's mu0
double chi0::chiqw(double qx, double par[]) {
    double qw[3] = {qx, par[0], par[1]}, out = 0.0;
    if (ctx_) check(tpsc_chi0_infinite(ctx_, mu0, 1, qw, 0, &out, NULL), "chiqw");
    return out;
}

// chi0::chiqw_discret (src/chi0.cpp:1587-1612): the same sum on this object's
// nq0 x nq0 lattice at q = 2 pi q[] / nq0, w_n = 2 n pi T
double chi0::chiqw_discret(int *q, int n) {
    const int nq0 = 2 * (nbq - 1);
    const double pi = acos(-1.0);
    double qw[3] = {q[0] * 2 * pi / nq0, q[1] * 2 * pi / nq0, 2 * n * pi * tem}, out = 0.0;
    if (ctx_) check(tpsc_chi0_infinite(ctx_, mu0, 1, qw, nq0, &out, NULL), "chiqw_discret");
    return out;
}

// chi0::calc_chi0_qlims (src/chi0.cpp:157-209): the infinite lattice's chi0 at
// w_n = 2 n pi T on the q grid from (qlims[0], qlims[1]) to (qlims[2],
// qlims[3]), Nq points per direction, qy <= qx; all points in one call
void chi0::calc_chi0_qlims(int n, double qlims[], int Nq[]) {
    find_mu_inf_syst();
    const double pi = acos(-1.0), eps = numeric_limits<double>::epsilon();
    const double wn = 2 * n * pi * tem;
    const int Nqx = Nq[0], Nqy = Nq[1];
    const double dqx = Nqx > 1 ? (qlims[2] - qlims[0]) / (Nqx - 1) : 0.0;
    const double dqy = Nqy > 1 ? (qlims[3] - qlims[1]) / (Nqy - 1) : 0.0;
    char name[200];
    sprintf(name, "./chi0_q_%5.3f_%5.3f_%5.3f_%7.5f_%7.5f_%7.5f_%7.5f_%7.5f_%7.5f_%d_%d_%d.dat", tp, tpp, t3, density, tem,
            qlims[0] / pi, qlims[1] / pi, qlims[2] / pi, qlims[3] / pi, Nqx, Nqy, n);
    cout << "calcul de chi0(q,wn=" << wn << ")" << '\n';
    std::vector<double> qw;
    double qx = qlims[0];
    for (int jx = 1; qx <= qlims[2] + eps; jx++) {
        double qy = qlims[1];
        for (int jy = 1; qy <= qlims[3] + eps && qy <= qx + eps; jy++) {
            qw.insert(qw.end(), {qx, qy, wn});
            qy = qlims[1] + jy * dqy;
            if (dqy == 0.0) break;  // the reference would repeat this point forever
        }
        qx = qlims[0] + jx * dqx;
        if (dqx == 0.0) break;
    }
    const int np = (int)qw.size() / 3;
    std::vector<double> chi(np);
    if (!np || !ctx_ || !check(tpsc_chi0_infinite(ctx_, mu0, np, qw.data(), 0, chi.data(), NULL), "calc_chi0_qlims"))
        return;
    fstream file;
    file.open(name, ios::out);
    file << setiosflags(ios::left) << setprecision(16);
    for (int p = 0; p < np; p++) file << setw(25) << qw[3 * p] << setw(25) << qw[3 * p + 1] << chi[p] << '\n';
    file.close();
}

// chi0::save_chi (src/chi0.cpp:61-95): the chi0 binary of the current grid
void chi0::save_chi() {
    if (!ctx_) return;
    const size_t n8 = (size_t)nbq * (nbq + 1) / 2;
    std::vector<double> chi(n8 * (size_t)(nwmax + 1));
    if (!check(tpsc_get_chi0(ctx_, chi.data(), NULL, NULL, NULL), "save_chi")) return;
    char name[200];
    tpsc_file_name(TPSC_FILE_CHI0_BIN, name, sizeof name, U, tp, tpp, t3, density, tem, 2 * (nbq - 1), 2 * nwmax,
                   0, 0);
    if (tpsc_write_chi0_bin(name, nbq, nwmax, chi.data()) != TPSC_OK) std::cout << "Error in chi0::save_chi" << std::endl;
}

// chi0::loadChi0 (src/chi0.cpp:99-154): the chi0 binary of this grid's name
// back into the device, chi0max and qmax found again
void chi0::loadChi0() {
    char name[200];
    tpsc_file_name(TPSC_FILE_CHI0_BIN, name, sizeof name, U, tp, tpp, t3, density, tem, 2 * (nbq - 1), 2 * nwmax,
                   0, 0);
    int fq = 0, fw = 0;
    if (tpsc_read_chi0_bin(name, &fq, &fw, NULL, 0) != TPSC_OK) {
        cout << "chi0::loadChi0():  fichier  " << name << "   inexistant \n";
        return;
    }
    if (fq != nbq || fw != nwmax) {
        cout << "chi0::loadChi0(): " << name << " holds nbq " << fq << ", nwmax " << fw << ", not this grid's\n";
        return;
    }
    std::vector<double> chi((size_t)fq * (fq + 1) / 2 * (size_t)(fw + 1));
    if (!check(tpsc_read_chi0_bin(name, &fq, &fw, chi.data(), (long long)chi.size()), "loadChi0")) return;
    if (!ctx_ || !check(tpsc_set_chi0(ctx_, chi.data()), "loadChi0")) return;
    refresh();
    chi0max = scal_[TPSC_S_CHI0MAX];
    qmax[0] = (int)scal_[TPSC_S_QMAX0];
    qmax[1] = (int)scal_[TPSC_S_QMAX1];
    cout << "chi0 charge,  nbq: " << nbq << "  nwmax: " << nwmax << '\n';
    cout << "qmax: " << qmax[0] << "  " << qmax[1] << "  chi0max: " << chi0max << '\n';
}

// ---------------------------------------------------------------------------
chi::chi(int nk0, int Nw0, double n, double T, double *params) : chi0(nk0, Nw0, n, T, params) {
    nsr = n > 1.0 ? 2.0 - n : n;
    Usp = Uch = dblOcc = 0.0;
    errUs = errUc = 0.0;
    paramsFileName[0] = 0;
}

void chi::get_params() const { green0::get_params(); }

void chi::find_Usp_Uch(int nq0, int nw0, double Usc[]) {
    double u[2];
    if (!ctx_ || !check(tpsc_find_Usp_Uch_grid(ctx_, nq0, nw0, u), "find_Usp_Uch")) return;
    nbq = nbk = nq0 / 2 + 1;
    nbw = nw0;
    nwmax = nw0 / 2;
    refresh();
    mu0 = scal_[TPSC_S_MU0];
    chi0max = scal_[TPSC_S_CHI0MAX];
    qmax[0] = (int)scal_[TPSC_S_QMAX0];
    qmax[1] = (int)scal_[TPSC_S_QMAX1];
    Usc[0] = Usp = u[0];
    Usc[1] = u[1];
    cout << "Usp: " << Usc[0] << '\n' << "Uch: " << Usc[1] << '\n';
}

void chi::find_Usp_Uch() {
    cout << "calcul de Usp et Uch\n";
    if (!ctx_ || !check(tpsc_find_Usp_Uch(ctx_), "find_Usp_Uch")) return;
    refresh();
    nbq = nbk;
    nwmax = nbw / 2;
    mu0 = scal_[TPSC_S_MU0];
    chi0max = scal_[TPSC_S_CHI0MAX];
    qmax[0] = (int)scal_[TPSC_S_QMAX0];
    qmax[1] = (int)scal_[TPSC_S_QMAX1];
    Usp = scal_[TPSC_S_USP];
    Uch = scal_[TPSC_S_UCH];
    dblOcc = scal_[TPSC_S_DBLOCC];
    const double difRelsp = scal_[TPSC_S_DIFRELSP], difRelch = scal_[TPSC_S_DIFRELCH];
    cout << "iteration q: 1  difRelsp: " << difRelsp << "  difRelch: " << difRelch << '\n';
    if (save_chi0_to_file) {
        // the full-grid chi0 dumps calc_chiqw_FFT_spline writes on the second grid
        const bool keep = save_chi0_q;
        save_chi0_q = true;
        const int nq0 = 2 * (nbq - 1), nw0 = 2 * nwmax;
        const int nw = nwmax + 1, n8 = nbq * (nbq + 1) / 2;
        std::vector<double> c((size_t)nw * n8);
        if (check(tpsc_get_chi0(ctx_, c.data(), NULL, NULL, NULL), "tpsc_get_chi0")) {
            char name[300];
            fstream file;
            int l = qmax[0], m = qmax[1];
            sprintf(name, "./chi0_qmax_wn_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%d_%d_%d_%d.dat", tp, tpp, t3, density, tem,
                    nq0, nw0, l, m);
            file.open(name, ios::out);
            file << setiosflags(ios::left) << setprecision(16);
            for (int j = 0; j < nw; j++) file << setw(10) << j << c[m + (l * (l + 1)) / 2 + (size_t)j * n8] << '\n';
            file.close();
            sprintf(name, "./chi0_wn0_q_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%d_%d.dat", tp, tpp, t3, density, tem, nq0,
                    nw0);
            file.open(name, ios::out);
            file << setiosflags(ios::left) << setprecision(16);
            for (l = 0; l < nbq; l++)
                for (m = 0; m <= l; m++) file << setw(10) << l << setw(10) << m << c[m + (l * (l + 1)) / 2] << '\n';
            file.close();
        }
        save_chi0_q = keep;
    }
    const double chispmax = chi0max / (1.0 - Usp * chi0max / 2.0);
    char name[300];
    sprintf(name, "./TPSC_infos_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%d_%d.dat", U, tp, tpp, t3, density, tem,
            2 * (nbq - 1), 2 * nwmax);
    fstream infos;
    infos << setprecision(16);
    infos.open(name, ios::out);
    infos << "Usp:  " << Usp << "   difRelsp:  " << difRelsp << '\n';
    infos << "Uch:  " << Uch << "   difRelch:  " << difRelch << '\n';
    infos << "chi0max: " << chi0max << "   chispmax: " << chispmax << "   rapport: " << chispmax / chi0max << '\n';
    infos << "double occupation (ansatz): " << dblOcc << '\n';
    infos << "qxmax, qymax:   " << qmax[0] << ",  " << qmax[1] << '\n';
    infos.close();
    cout << "chi0max: " << chi0max << "  chispmax: " << chispmax << "  rapport: " << chispmax / chi0max << '\n';
    cout << "double occupation: " << dblOcc << '\n';
    sprintf(paramsFileName, "./TPSCparams_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%d_%d.dat", U, tp, tpp, t3, density,
            tem, 2 * (nbq - 1), 2 * nwmax);
    fstream params;
    params.open(paramsFileName, ios::out);
    if (!params) {
        cout << "echec de creation du fichier de parametres\n";
        return;
    }
    params << setprecision(16);
    params << "Usp  " << Usp << "   difRelsp:  " << difRelsp << '\n';
    params << "Uch  " << Uch << "   difRelch:  " << difRelch << '\n';
    params << "nbq  " << nbq << '\n';
    params << "nbw  " << nwmax + 1 << '\n';
    params << "dblOcc_ansatz  " << dblOcc << '\n';
    params << "qxmax  " << qmax[0] << '\n';
    params << "qymax  " << qmax[1] << '\n';
    params << "chispmax_over_chi0max  " << chispmax / chi0max << '\n';
    params << "mu0  " << mu0 << '\n';
    params.close();
}

// chi::sp_corr_length (src/chi.cpp:450-718): the lengths from the engine, the
// reference's lines on stdout and appended to TPSC_infos_*
void chi::sp_corr_length() {
    if (!ctx_) return;
    double r[7];
    // the Fermi surface of the constructor's mu0, as the reference keeps it
    if (!check(tpsc_sp_corr_length_fs(ctx_, mu0_fs_, r), "sp_corr_length")) return;
    vF = r[0];
    spCorrLgth_y = r[1];
    spCorrLgth_x = r[2];
    spCorrLgthAs_y = r[3];
    spCorrLgthAs_x = r[4];
    xi0_y = r[5];
    xi0_x = r[6];
    if (qmax[0] != (nbq - 1) || qmax[1] != (nbq - 1))
        cout << "chisp incommensurable (formule asymptotique non valable)\n";
    char name[300];
    sprintf(name, "./TPSC_infos_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%d_%d.dat", U, tp, tpp, t3, density, tem,
            2 * (nbq - 1), 2 * nwmax);
    fstream infos;
    infos.open(name, ios::out | ios::app);
    infos << setprecision(16);
    struct Line {
        const char *what;
        double xi;
        bool th;
    };
    const Line lines[] = {
        {"longueur de correlation de spin (1/(larg.mi-haut.)) (axe y):  ", spCorrLgth_y, true},
        {"longueur de correlation de spin (1/(larg.mi-haut.)) (axe x):  ", spCorrLgth_x, true},
        {"longueur de correlation de spin (formule asymptotique) (axe y):  ", spCorrLgthAs_y, false},
        {"longueur de correlation de spin (formule asymptotique) (axe x):  ", spCorrLgthAs_x, false},
    };
    cout << "vitesse de Fermi aux points chauds:  " << vF << endl;
    infos << "vitesse de Fermi aux points chauds:  " << vF << endl;
    for (const Line &L : lines) {
        const char *ratio = L.th ? "xi_sp/xi_th:  " : "xi_sp_As/xi_th:  ";
        const char *prod = L.th ? "xi_sp*T:  " : "xi_sp_As*T:  ";
        cout << L.what << L.xi << '\n' << ratio << L.xi * acos(-1.0) * tem / vF << '\n' << prod << L.xi * tem << '\n';
        infos << L.what << L.xi << '\n' << ratio << L.xi * acos(-1.0) * tem / vF << '\n' << prod << L.xi * tem << '\n';
    }
    const double chisp_max = chi0max / (1.0 - Usp * chi0max / 2.0);
    cout << "(max(chi_sp)/max(chi_0))^0.5:  " << sqrt(chisp_max / chi0max) << endl;
    infos.close();
}

// the reference's chi computes nsr once, in its constructor (src/chi.cpp:18-19)
void chi::model_changed() { check(tpsc_set_nsr(ctx_, nsr), "set_density"); }

// chi::calc_corr_length (src/chi.cpp:931-981): Usp, Uch and the spin
// correlation lengths on the (n, T) grid dens[0]..dens[1] (nD points) x
// Temp[0]..Temp[1] (nT points), one line per point in the corrLgth file
void chi::calc_corr_length(double dens[], int nD, double Temp[], int nT) {
    const double T0 = Temp[0], Tf = Temp[1], dT = (Tf - T0) / (nT - 1);
    const double n0 = dens[0], nf = dens[1], dn = (nf - n0) / (nD - 1);
    char name[100];
    sprintf(name, "./corrLgth_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%7.5f_%6.4f_%6.4f.dat", U, tp, tpp, t3, n0, nf, T0, Tf);
    fstream file;
    file.open(name, ios::out);
    file << setiosflags(ios::left) << setprecision(15);
    for (int l = 0; l < nD; l++) {
        set_density(n0 + l * dn);
        for (int j = 0; j < nT; j++) {
            set_tem(T0 + j * dT);
            find_Usp_Uch();
            sp_corr_length();
            file << setw(25) << density << setw(25) << tem << setw(25) << mu0;
            file << setw(25) << vF << setw(25) << Usp << setw(25) << errUs;
            file << setw(25) << Uch << setw(25) << errUc << setw(25) << dblOcc;
            file << setw(25) << spCorrLgth_x << setw(25) << spCorrLgth_y;
            file << setw(25) << spCorrLgthAs_x << setw(25) << spCorrLgthAs_y;
            file << setw(25) << xi0_x << setw(25) << xi0_y << setw(25) << nbq;
            file << setw(25) << qmax[0] << setw(25) << qmax[1];
            file << chi0max << '\n';
        }
    }
    file.close();
}

void chi::calc_chirt() {
    cout << "calcul de vertex_rt_array\n";
    if (!ctx_) return;
    check(tpsc_vertex(ctx_), "calc_chirt");
}

// ---------------------------------------------------------------------------
green::green(int nk0, int Nw0, double n, double T, double eta0, double *params) : chi(nk0, Nw0, n, T, params) {
    eta = eta0;
    mu = 0;
    Sigma_inf = 0;
    mu_calcule = have_self = false;
}

void green::get_params() const {
    chi::get_params();
    cout << "mu: " << mu << '\n';
}

void green::calc_Self_FFT_spline() {
    find_Usp_Uch();
    calc_chirt();
    cout << "calcul de la self-energie par calc_Self_FFT_spline()\n";
    if (!ctx_ || !check(tpsc_self_energy(ctx_), "calc_Self_FFT_spline")) return;
    refresh();
    Sigma_inf = scal_[TPSC_S_SIGMA_INF];
    have_self = true;
    cout << "self-energie calculee\n";
}

void green::traceSelfG() {
    double tr[2];
    if (!ctx_ || !check(tpsc_trace_self_G(ctx_, tr), "traceSelfG")) return;
    const double ud = U * dblOcc - U * density * density / 4.0;
    cout << "U*dblOcc-U*n^2/4:  " << ud << '\n';
    cout << "trace Self*G: " << tr[0] << '\n';
    cout << "trace Self*G (avec correction asymptotique): " << tr[1] << '\n';
    char name[300];
    sprintf(name, "./TPSC_infos_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, density, tem,
            2 * (nbk - 1), nbw);
    fstream f;
    f.open(name, ios::out | ios::app);
    f << setprecision(16);
    f << "U*dblOcc-U*n^2/4:   " << ud << '\n';
    f << "trace Self*G:  " << tr[0] << '\n';
    f.close();
}

void green::traceSelfG2() {
    refresh();
    const double sum = scal_[TPSC_S_TR_SG2];
    cout << "trace Self*G2: " << sum << "  U*dblOcc-U*n^2/4:  " << U * dblOcc - U * density * density / 4.0 << '\n';
    cout << "double occupation (Self*G2): " << (sum + U * density * density / 4.0) / U << '\n';
    char name[300];
    sprintf(name, "./TPSC_infos_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, density, tem,
            2 * (nbk - 1), nbw);
    fstream f;
    f.open(name, ios::out | ios::app);
    f << setprecision(16);
    f << "trace Self*G2:  " << sum << '\n';
    f << "double occupation (Self*G2): " << (sum + U * density * density / 4.0) / U << '\n';
    f << "mu0:  " << mu0 << '\n';
    f << "mu:  " << mu << '\n';
    f.close();
}

void green::find_mu() {
    if (!ctx_) return;
    if (check(tpsc_find_mu(ctx_), "find_mu")) {
        refresh();
        mu = scal_[TPSC_S_MU];
        mu_calcule = true;
        cout << "mu:  " << mu << '\n';
    } else {
        cout << "Attention! mu non calcule!\n";
    }
    char pname[300], mname[300];
    sprintf(pname, "./TPSCparams_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, density, tem,
            2 * (nbk - 1), nbw);
    sprintf(mname, "./mu0_mu_D_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, density, tem,
            2 * (nbk - 1), nbw);
    fstream pf;
    pf.open(pname, ios::out | ios::app);
    if (pf) {
        pf << setprecision(14);
        pf << "mu  " << mu << '\n';
        pf.close();
    } else {
        cout << "echec d'ouverture du fichier de parametres\n";
    }
    fstream mf;
    mf.open(mname, ios::out);
    if (mf) {
        mf << setprecision(15) << setiosflags(ios::left);
        mf << setw(25) << mu0 << setw(25) << mu << dblOcc << '\n';
        mf.close();
    }
    if (mu_calcule) traceSelfG2();
}

void green::find_FS_inter() {
    cout << "calcul des coordonnees de la surface de Fermi avec interaction\n";
    if (!have_self) {
        cout << "find_FS_inter(): self-energy non calculee\n";
        return;
    }
    if (!mu_calcule) {
        cout << "find_FS_inter(): mu n'a pas ete calcule\n";
        return;
    }
    const int n8 = nbk * (nbk + 1) / 2;
    const double z[2] = {0.0, 0.000001};
    int idx[4] = {0, 1, 2, 3};
    std::vector<double> Apoly(n8), Apade(n8);
    if (!check(tpsc_pade_sigma(ctx_, idx, 3, z, 1, 1, NULL, Apoly.data()), "find_FS_inter")) return;
    if (!check(tpsc_pade_sigma(ctx_, idx, 4, z, 1, 0, NULL, Apade.data()), "find_FS_inter")) return;
    const char *forms[4] = {"./FS_inter_AkF_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat",
                            "./FS_inter_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat",
                            "./FS_inter_AkF_Pade_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat",
                            "./FS_inter_Pade_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat"};
    fstream f[4];
    for (int i = 0; i < 4; ++i) {
        char name[300];
        sprintf(name, forms[i], U, tp, tpp, t3, density, tem, 2 * (nbk - 1), nbw);
        f[i].open(name, ios::out);
        f[i] << setiosflags(ios::left) << setprecision(8);
    }
    for (int l = 0; l < nbk; l++) {
        double best[2] = {0, 0};
        int bm[2] = {0, 0};
        for (int m = 0; m < nbk - l; m++) {
            const int x = l + m, y = m;
            const double a[2] = {Apoly[y + (x * (x + 1)) / 2], Apade[y + (x * (x + 1)) / 2]};
            for (int k = 0; k < 2; ++k)
                if (a[k] > best[k]) {
                    best[k] = a[k];
                    bm[k] = m;
                }
        }
        f[0] << setw(10) << l + bm[0] << setw(10) << bm[0] << best[0] << endl;
        f[1] << setw(10) << l + bm[0] << setw(10) << bm[0] << endl;
        f[2] << setw(10) << l + bm[1] << setw(10) << bm[1] << best[1] << endl;
        f[3] << setw(10) << l + bm[1] << setw(10) << bm[1] << endl;
    }
    for (auto &x : f) x.close();
}

void green::MDC(int *n, int Nn, double w, double *eta_p, int Neta, bool use_Pade) {
    if (!have_self) {
        cout << "MDC(): la self-energie n'a pas ete calculee\n";
        return;
    }
    if (Nn < 2) Nn = 2;
    const int npts = use_Pade ? Nn : (Nn >= 4 ? 4 : 3);
    const int n8 = nbk * (nbk + 1) / 2;
    std::vector<double> z(2 * Neta), sig((size_t)2 * n8 * Neta), A((size_t)n8 * Neta);
    for (int j = 0; j < Neta; ++j) {
        z[2 * j] = w;
        z[2 * j + 1] = eta_p[j];
    }
    if (!check(tpsc_pade_sigma(ctx_, n, npts, z.data(), Neta, use_Pade ? 0 : 1, sig.data(), A.data()), "MDC"))
        return;
    char name[300];
    fstream af, sf;
    sprintf(name,
            use_Pade ? "Akw_Pade_k_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%5.3e_%1d_%1d.dat"
                     : "Akw_poly_k_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%5.3e_%1d_%1d.dat",
            U, tp, tpp, t3, density, tem, w, 2 * (nbk - 1), nbw);
    af.open(name, ios::out);
    af << setprecision(12) << setiosflags(ios::left);
    sprintf(name,
            use_Pade ? "Self_Pade_k_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%5.3e_%1d_%1d.dat"
                     : "Self_poly_k_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%5.3e_%1d_%1d.dat",
            U, tp, tpp, t3, density, tem, w, 2 * (nbk - 1), nbw);
    sf.open(name, ios::out);
    sf << setprecision(12) << setiosflags(ios::left);
    for (int l = 0; l < nbk; l++)
        for (int m = 0; m <= l; m++) {
            const size_t o = m + (l * (l + 1)) / 2;
            sf << setw(10) << l << setw(20) << m << setw(20) << sig[2 * (o * Neta)] << setw(25)
               << sig[2 * (o * Neta) + 1];
            af << setw(10) << l << setw(20) << m << setw(20) << A[o * Neta];
            for (int j = 1; j < Neta; j++) {
                sf << setw(20) << sig[2 * (o * Neta + j)] << setw(25) << sig[2 * (o * Neta + j) + 1];
                af << setw(20) << A[o * Neta + j];
            }
            sf << endl;
            af << endl;
        }
    sf.close();
    af.close();
}

void green::Gwn_local() {
    if (!mu_calcule || !have_self) {
        cout << "G_local(): mu non calcule ou Self_kw_array inexistant\n";
        return;
    }
    std::vector<double> g(nbw);
    if (!check(tpsc_gwn_local(ctx_, g.data()), "Gwn_local")) return;
    char name[300];
    sprintf(name, "./Gwn_loc_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%d_%d.dat", U, tp, tpp, t3, density, tem,
            2 * (nbk - 1), nbw);
    fstream file;
    file.open(name, ios::out);
    file << setprecision(10) << setiosflags(ios::left);
    for (int j = 0; j < nbw / 2; j++) file << setw(10) << j << setw(25) << g[2 * j] << g[2 * j + 1] << endl;
    file.close();
}

// Sigma(k, i k_n) at the listed k points, n <= Nwn (green::save_self_ikn,
// src/green.cpp:127-180)
void green::save_self_ikn(int *k_save, int nk_save, int Nwn) {
    if (!have_self) {
        set_keep_chiqw(false);
        calc_Self_FFT_spline();
        traceSelfG();
        green::find_mu();
    }
    if (!have_self) return;
    const size_t n8 = (size_t)nbk * (nbk + 1) / 2;
    std::vector<double> S((size_t)2 * n8 * (nbw / 2)), c2(n8), c3(n8);
    if (!check(tpsc_get_self(ctx_, S.data(), c2.data(), c3.data(), NULL), "save_self_ikn")) return;
    char name[200];
    sprintf(name, "./self_k_ikn_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, density, tem,
            2 * (nbk - 1), nbw);
    fstream file;
    file.open(name, ios::out);
    file << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
    const double pi = acos(-1.0);
    for (int j = 0; j <= Nwn && j < nbw / 2; j++) {
        const double kn = (2.0 * j + 1) * pi * tem;
        for (int p = 0; p < nk_save; p++) {
            long x = k_save[2 * p], y = k_save[2 * p + 1];
            if (y > x) std::swap(x, y);
            if (x >= 0 && x < nbk && y >= 0) {
                const size_t o = y + (x * (x + 1)) / 2;
                const double re = -c2[o] / (kn * kn) + S[2 * (o + j * n8)] / (kn * kn * kn * kn);
                const double im = -Sigma_inf / kn + c3[o] / (kn * kn * kn) + S[2 * (o + j * n8) + 1] / (kn * kn * kn * kn);
                file << setw(10) << j << setw(10) << x << setw(10) << y << setw(25) << re << im << endl;
            }
        }
    }
    file.close();
}

// green::calc_Self_Re_w (src/green.cpp:407-542) at one k, and
// calc_Self_Re_w_BZ (src/green.cpp:386-404) at every k of the reduced zone
void green::calc_Self_Re_w(int *k, int *n, int Nn, double *w, int Nw, double *eta, int Neta) {
    self_re_w(k, 1, n, Nn, w, Nw, eta, Neta);
}

void green::calc_Self_Re_w_BZ(int *n, int Nn, double *w, int Nw, double *eta, int Neta) {
    std::vector<int> ks;
    const int nk2 = (nbk - 1) / 2 + 1;
    for (int l = 0; l < nk2; l++)
        for (int m = 0; l + m <= nbk - m - 1; m++) {
            ks.push_back(nbk - m - 1);
            ks.push_back(l + m);
        }
    self_re_w(ks.data(), (int)ks.size() / 2, n, Nn, w, Nw, eta, Neta);
}

// For the nk points k = (ks[2p], ks[2p+1]): the Pade continuation of
// Sigma(k, z) = Sigma_inf/z + C2/z^2 + C3/z^3 + S/z^4 from the Nn points
// z_j = i (2 n[j] + 1) pi T (S read at the stored frequency j, as the
// reference does) to z = w + i eta, and A(k, w) = -Im 1/(pi (z - eps + mu -
// Sigma)); then the same from the J-fraction Sigma = a1/(z + b1 + F(z)),
// a1 = Sigma_inf, b1 = -C2/Sigma_inf, F continued from max(4, Nn/8) points
// (src/green.cpp:487-540).  All k in two batched Pade launches; the
// reference's four files per k.
void green::self_re_w(const int *ks, int nk, int *n, int Nn, double *w, int Nw, double *eta, int Neta) {
    if (!have_self) {
        cout << "calc_Self_Re_w(): la self-energie n'a pas ete calculee\n";
        return;
    }
    const int Nn2 = std::max(4, Nn / 8);
    if (Nn < Nn2 || Nn > nbw / 2 || Neta < 1 || Nw < 1) {
        cout << "calc_Self_Re_w(): need " << Nn2 << " <= Nn <= " << nbw / 2 << ", Nw >= 1 and Neta >= 1\n";
        return;
    }
    const size_t n8 = (size_t)nbk * (nbk + 1) / 2;
    std::vector<double> S((size_t)2 * n8 * (nbw / 2)), c2(n8), c3(n8), ek((size_t)nbk * nbk);
    if (!check(tpsc_get_self(ctx_, S.data(), c2.data(), c3.data(), NULL), "calc_Self_Re_w")) return;
    if (!check(tpsc_get_ek(ctx_, ek.data()), "calc_Self_Re_w")) return;
    typedef std::complex<double> cx;
    const double pi = acos(-1.0);
    const int nk0 = 2 * (nbk - 1);
    auto fold = [&](int x) {
        while (x < 0) x += nk0;
        return x > nbk - 1 ? nk0 - x : x;
    };
    std::vector<cx> z0(Nn), x1((size_t)nk * Nn), y1((size_t)nk * Nn), x2((size_t)nk * Nn2), y2((size_t)nk * Nn2);
    std::vector<cx> zs((size_t)Nw * Neta);
    for (int j = 0; j < Nn; j++) z0[j] = cx(0.0, (2 * n[j] + 1) * pi * tem);
    for (int j = 0; j < Nw; j++)
        for (int l = 0; l < Neta; l++) zs[(size_t)j * Neta + l] = cx(w[j], eta[l]);
    std::vector<double> a1(nk), b1(nk), ekmu(nk);
    for (int p = 0; p < nk; p++) {
        long x = ks[2 * p], y = ks[2 * p + 1];
        if (y > x) std::swap(x, y);
        const size_t o = y + (x * (x + 1)) / 2;
        auto fk = [&](int j) { return cx(S[2 * (o + j * n8)], S[2 * (o + j * n8) + 1]); };
        for (int j = 0; j < Nn; j++) {
            const cx z = z0[j];
            x1[(size_t)p * Nn + j] = z;
            y1[(size_t)p * Nn + j] = Sigma_inf / z + c2[o] / (z * z) + c3[o] / (z * z * z) + fk(j) / (z * z * z * z);
        }
        const double c1 = Sigma_inf, cc3 = c3[o];
        a1[p] = c1;
        b1[p] = -c2[o] / c1;
        const double b = b1[p];
        for (int j = 0; j < Nn2; j++) {
            const cx z = z0[j], f = fk(j);
            x2[(size_t)p * Nn2 + j] = z;
            y2[(size_t)p * Nn2 + j] =
                (b * f + (f + b * cc3) * z + (cc3 - c1 * b * b) * z * z) / (-f - cc3 * z + c1 * b * z * z - c1 * z * z * z);
        }
        ekmu[p] = ek[fold(ks[2 * p + 1]) + (size_t)fold(ks[2 * p]) * nbk] - mu;
    }
    const int Nz = Nw * Neta;
    std::vector<cx> s1((size_t)nk * Nz), s2((size_t)nk * Nz);
    if (!check(tpsc_pade_batch(ctx_, nk, Nn, (double *)x1.data(), (double *)y1.data(), Nz, (double *)zs.data(),
                               (double *)s1.data()),
               "calc_Self_Re_w"))
        return;
    if (!check(tpsc_pade_batch(ctx_, nk, Nn2, (double *)x2.data(), (double *)y2.data(), Nz, (double *)zs.data(),
                               (double *)s2.data()),
               "calc_Self_Re_w"))
        return;
    char name[200];
    for (int p = 0; p < nk; p++) {
        for (int variant = 0; variant < 2; variant++) {
            const char *fs = variant ? "Self_Re_w_Jfrac_U%4.2f_tp%5.3f_tpp%5.3f_tt%5.3f_dens%7.5f_tem%6.4f_Nk%1d_Nwn%1d_%1d_%1d.dat"
                                     : "Self_Re_w_U%4.2f_tp%5.3f_tpp%5.3f_tt%5.3f_dens%7.5f_tem%6.4f_Nk%1d_Nwn%1d_%1d_%1d.dat";
            const char *fa = variant
                                 ? "spectr_wgt_Jfrac_U%4.2f_tp%5.3f_tpp%5.3f_tt%5.3f_dens%7.5f_tem%6.4f_Nk%1d_Nwn%1d_%1d_%1d.dat"
                                 : "spectr_wgt_U%4.2f_tp%5.3f_tpp%5.3f_tt%5.3f_dens%7.5f_tem%6.4f_Nk%1d_Nwn%1d_%1d_%1d.dat";
            fstream fileSelf, fileAkw;
            sprintf(name, fs, U, tp, tpp, t3, density, tem, nk0, nbw, ks[2 * p], ks[2 * p + 1]);
            fileSelf.open(name, ios::out);
            fileSelf << setiosflags(ios::left) << setprecision(10);
            sprintf(name, fa, U, tp, tpp, t3, density, tem, nk0, nbw, ks[2 * p], ks[2 * p + 1]);
            fileAkw.open(name, ios::out);
            fileAkw << setiosflags(ios::left) << setprecision(10);
            for (int j = 0; j < Nw; j++) {
                for (int l = 0; l < Neta; l++) {
                    const size_t q = (size_t)p * Nz + (size_t)j * Neta + l;
                    const cx z = zs[(size_t)j * Neta + l];
                    const cx self_w = variant ? a1[p] / (z + b1[p] + s2[q]) : s1[q];
                    const double Akw = -imag((1.0 / pi) / (z - ekmu[p] - self_w));
                    if (l == 0) {
                        fileSelf << setw(25) << w[j] << setw(20) << real(self_w) << setw(25) << imag(self_w);
                        fileAkw << setw(25) << w[j] << setw(20) << Akw;
                    } else {
                        fileSelf << setw(20) << real(self_w) << setw(25) << imag(self_w);
                        fileAkw << setw(20) << Akw;
                    }
                }
                fileSelf << endl;
                fileAkw << endl;
            }
            fileSelf.close();
            fileAkw.close();
        }
    }
}

bool green::spectra(const int *ks, int nk, const double *z0, int N, const double *w, int nw0, const double *eta,
                    int neta, double *out) {
    typedef std::complex<double> cx;
    const size_t n8 = (size_t)nbk * (nbk + 1) / 2;
    std::vector<double> S((size_t)2 * n8 * (nbw / 2)), c2(n8), c3(n8), ek((size_t)nbk * nbk);
    if (!check(tpsc_get_self(ctx_, S.data(), c2.data(), c3.data(), NULL), "calc_spectral_weight")) return false;
    if (!check(tpsc_get_ek(ctx_, ek.data()), "calc_spectral_weight")) return false;
    std::vector<cx> X((size_t)nk * N), Y((size_t)nk * N), Z((size_t)nw0 * neta), F((size_t)nk * nw0 * neta);
    for (int j = 0; j < nw0; j++)
        for (int l = 0; l < neta; l++) Z[(size_t)j * neta + l] = cx(w[j], eta[l]);
    for (int p = 0; p < nk; p++) {
        int x = ks[2 * p], y = ks[2 * p + 1];
        if (y > x) std::swap(x, y);
        const size_t o = y + ((size_t)x * (x + 1)) / 2;
        for (int n = 0; n < N; n++) {
            const cx z(z0[2 * n], z0[2 * n + 1]);
            X[(size_t)p * N + n] = z;
            Y[(size_t)p * N + n] = Sigma_inf / z + c2[o] / (z * z) + c3[o] / (z * z * z) +
                                   cx(S[2 * (o + n * n8)], S[2 * (o + n * n8) + 1]) / (z * z * z * z);
        }
    }
    if (!check(tpsc_pade_batch(ctx_, nk, N, (double *)X.data(), (double *)Y.data(), nw0 * neta, (double *)Z.data(),
                               (double *)F.data()),
               "calc_spectral_weight"))
        return false;
    const double pi = acos(-1.0);
    for (int p = 0; p < nk; p++) {
        // hamiltonien::ek_val on the folded point (src/hamiltonien.cpp:107-116)
        const double ekmu = ek[ks[2 * p + 1] + (size_t)ks[2 * p] * nbk] - mu;
        for (int j = 0; j < nw0; j++)
            for (int l = 0; l < neta; l++) {
                const size_t q = ((size_t)p * nw0 + j) * neta + l;
                out[q] = -imag(1.0 / (cx(w[j] - ekmu, eta[l]) - F[q])) / pi;
            }
    }
    return true;
}

// green::calc_spectral_weight (src/green.cpp:1152-1260): A(k, w + i eta) from
// the N-point Pade through i (2n + 1) pi T, n < N; k folded by |.|
void green::calc_spectral_weight(int *k, double *w, int nw0, int N, double *spectr_w) {
    if (w[0] > w[nw0 - 1]) {
        cout << "calc_spectral_weight: wi>wf!\n";
        return;
    }
    if (N > nbw / 2) {
        cout << "calc_spectral_weight: Value N larger than nw=" << nbw / 2 << '\n';
        return;
    }
    if (N <= 0) {
        cout << "calc_spectral_weight: Value N too small: " << N << '\n';
        return;
    }
    if (k[0] < 0) k[0] *= -1;
    if (k[1] < 0) k[1] *= -1;
    if (k[0] >= nbk || k[1] >= nbk) {
        cout << "calc_spectral_weight: invalid wave vector k=(" << k[0] << "," << k[1] << ")" << '\n';
        return;
    }
    if (!have_self) {
        cout << "calc_spectral_weight: Self-energy not computed" << '\n';
        return;
    }
    const double pi = acos(-1.0);
    std::vector<double> z0(2 * (size_t)N);
    for (int n = 0; n < N; n++) {
        z0[2 * n] = 0.0;
        z0[2 * n + 1] = (2 * n + 1) * pi * tem;
    }
    spectra(k, 1, z0.data(), N, w, nw0, &eta, 1, spectr_w);
}

// green::calc_spectral_weight with several eta (src/green.cpp:1073-1150): the
// Pade through the non-uniform points of create_non_uniform_ind_freq; k
// folded into the zone
void green::calc_spectral_weight(int *k, double *w, int nw0, int N, double *eta_p, int N_eta, double *spectr_w) {
    if (w[0] > w[nw0 - 1]) {
        cout << "calc_spectral_weight: wi>wf!\n";
        return;
    }
    if (N > nbw / 2) {
        cout << "calc_spectral_weight: Value N larger than nw=" << nbw / 2 << '\n';
        return;
    }
    if (N <= 0) {
        cout << "calc_spectral_weight: Value N too small: " << N << '\n';
        return;
    }
    const int Nk = 2 * (nbk - 1);
    while (k[0] < 0) k[0] += Nk;
    while (k[1] < 0) k[1] += Nk;
    if (k[0] > nbk - 1) k[0] = Nk - k[0];
    if (k[1] > nbk - 1) k[1] = Nk - k[1];
    if (!have_self) {
        cout << "calc_spectral_weight: Self-energy not computed" << '\n';
        return;
    }
    if ((int)pade_z0.size() < 2 * N) {
        cout << "calc_spectral_weight: create_non_uniform_ind_freq has not been called\n";
        return;
    }
    spectra(k, 1, pade_z0.data(), N, w, nw0, eta_p, N_eta, spectr_w);
}

// green::create_non_uniform_ind_freq (src/green.cpp:554-582): the first N1 =
// nbw / 2^(m+1) indices, then m runs of N1/2 indices spaced 2^(l+1)
void green::create_non_uniform_ind_freq(int m_freq_p) {
    m_freq = m_freq_p;
    const int N1 = nbw / ((int)pow(2, m_freq + 1)), N2 = N1 / 2;
    N_freq = N1 + m_freq * N2;
    cout << "non uniform frequency grid parameters:\n";
    cout << "N1: " << N1 << endl;
    cout << "N_freq: " << N_freq << endl;
    ind_freq.assign(N_freq, 0);
    for (int j = 0; j < N1; j++) ind_freq[j] = j;
    for (int j = N1; j < N_freq; j++) {
        const int lj = (j - N1) / N2, p2lj = (int)pow(2, lj);
        ind_freq[j] = p2lj * N1 + p2lj * 2 * ((j - N1) % N2);
    }
    const double pi = acos(-1.0);
    pade_z0.assign(2 * (size_t)N_freq, 0.0);
    for (int j = 0; j < N_freq; j++) pade_z0[2 * j + 1] = (2 * ind_freq[j] + 1) * pi * tem;
}

// green::EDC (src/green.cpp:589-711): A(k, w + i eta_p) from the Pade through
// up to NP_max points of the non-uniform grid, for the listed k or (kx or ky
// NULL) every other point of the reduced zone; one file per k.  All k in one
// batched device Pade.
void green::EDC(int *kx, int *ky, int Nk, double *w, int nw0, int m_freq_p, int NP_max, double *eta_p, int N_eta,
                char *fname) {
    if (!have_self) {
        cout << "EDC(): la self-energie n'a pas ete calculee\n";
        return;
    }
    create_non_uniform_ind_freq(m_freq_p);
    const double pi = acos(-1.0);
    const int NP = N_freq > NP_max ? NP_max : N_freq;
    cout << setprecision(5);
    cout << "frequence maximale incluse dans le prolongement analytique: " << (2 * ind_freq[NP - 1] + 1) * pi * tem
         << endl;
    std::string form = fname ? fname : "spectral_weight";
    form += "_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d_%1d_%1d_%3.1e_%3.1e.dat";
    std::vector<int> ks;
    if (!kx || !ky) {
        cout << "calcul du poids spectral dans la zone reduite\n";
        for (int l = 0; l < nbk; l += 2)
            for (int m = 0; m <= l; m += 2) {
                ks.push_back(l);
                ks.push_back(m);
            }
    } else {
        cout << "calcul du poids spectral pour les vecteurs d'onde entre k=(" << (pi * kx[0]) / (nbk - 1) << ","
             << (pi * ky[0]) / (nbk - 1) << ") et (" << (pi * kx[Nk - 1]) / (nbk - 1) << ","
             << (pi * ky[Nk - 1]) / (nbk - 1) << ")\n";
        const int NK = 2 * (nbk - 1);
        for (int p = 0; p < Nk; p++) {
            int k[2] = {kx[p], ky[p]};
            for (int c = 0; c < 2; c++) {
                while (k[c] < 0) k[c] += NK;
                if (k[c] > nbk - 1) k[c] = NK - k[c];
            }
            ks.push_back(k[0]);
            ks.push_back(k[1]);
        }
    }
    const int nk = (int)ks.size() / 2;
    std::vector<double> A((size_t)nk * nw0 * N_eta);
    if (NP <= 0 || NP > nbw / 2 || w[0] > w[nw0 - 1] ||
        !spectra(ks.data(), nk, pade_z0.data(), NP, w, nw0, eta_p, N_eta, A.data()))
        return;
    char name[400];
    for (int p = 0; p < nk; p++) {
        sprintf(name, form.c_str(), U, tp, tpp, t3, density, tem, 2 * (nbk - 1), nbw, ks[2 * p], ks[2 * p + 1], w[0],
                w[nw0 - 1]);
        fstream f;
        f.open(name, ios::out);
        f << setprecision(10) << setiosflags(ios::left);
        for (int j = 0; j < nw0; j++) {
            f << setw(20) << w[j];
            for (int n = 0; n < N_eta; n++) f << setw(20) << A[((size_t)p * nw0 + j) * N_eta + n];
            f << endl;
        }
        f.close();
    }
}

// green::EDC (src/green.cpp:714-812): A(k, w + i eta) on w = -10..10 (step
// 0.01) from the nbw/2-point Pade, the object's eta; fname is the prefix
void green::EDC(int *kx, int *ky, int Nk, char *fname) {
    if (!have_self) {
        cout << "EDC(): la self-energie n'a pas ete calculee\n";
        return;
    }
    const double Dw = 10.0, dw = 0.01;
    const int nw0 = (int)(2 * Dw / dw) + 1;
    std::vector<double> w(nw0);
    w[0] = -Dw;
    for (int j = 1; j < nw0; j++) w[j] = w[0] + j * dw;
    const int N = nbw / 2;
    std::vector<int> ks;
    if (!kx || !ky) {
        cout << "calcul du poids spectral dans la zone reduite\n";
        for (int l = 0; l < nbk; l += 2)
            for (int m = 0; m <= l; m += 2) {
                ks.push_back(l);
                ks.push_back(m);
            }
    } else {
        cout << "calcul du poids spectral pour les vecteurs d'onde donnes\n";
        for (int p = 0; p < Nk; p++) {
            const int a = kx[p] < 0 ? -kx[p] : kx[p], b = ky[p] < 0 ? -ky[p] : ky[p];
            if (a >= nbk || b >= nbk) {
                // the reference would write a file of uninitialised values here
                cout << "calc_spectral_weight: invalid wave vector k=(" << a << "," << b << ")" << '\n';
                continue;
            }
            ks.push_back(a);
            ks.push_back(b);
        }
    }
    const int nk = (int)ks.size() / 2;
    if (!nk) return;
    const double pi = acos(-1.0);
    std::vector<double> z0(2 * (size_t)N), A((size_t)nk * nw0);
    for (int n = 0; n < N; n++) z0[2 * n + 1] = (2 * n + 1) * pi * tem;
    if (!spectra(ks.data(), nk, z0.data(), N, w.data(), nw0, &eta, 1, A.data())) return;
    std::string form = fname;
    form += "_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%3.1e_%1d_%1d_%1d_%1d.dat";
    char name[400];
    for (int p = 0; p < nk; p++) {
        sprintf(name, form.c_str(), U, tp, tpp, t3, density, tem, eta, 2 * (nbk - 1), nbw, ks[2 * p], ks[2 * p + 1]);
        fstream f;
        f.open(name, ios::out);
        f << setprecision(15) << setiosflags(ios::left);
        for (int j = 0; j < nw0; j++) f << setw(30) << w[j] << A[(size_t)p * nw0 + j] << '\n';
        f.close();
    }
}

// green::save_Self (src/green.cpp:1544-1574): ascii, Nfreq frequencies
void green::save_Self(int Nfreq) {
    if (!have_self) {
        cout << "save_Self(): Self_kw_array n'existe pas\n";
        return;
    }
    const size_t n8 = (size_t)nbk * (nbk + 1) / 2;
    std::vector<double> S((size_t)2 * n8 * (nbw / 2));
    if (!check(tpsc_get_self(ctx_, S.data(), NULL, NULL, NULL), "save_Self")) return;
    char name[200];
    tpsc_file_name(TPSC_FILE_SELF_ASCII, name, sizeof name, U, tp, tpp, t3, density, tem, 2 * (nbk - 1), nbw, 0, 0);
    check(tpsc_write_self_ascii(name, nbk, nbw, Nfreq, S.data()), "save_Self");
}

// green::save_Self_bin (src/green.cpp:1496-1515): S, then the frame the
// reference's Sigma stage leaves after it, (Sigma(k, beta/2), 0)
void green::save_Self_bin() {
    if (!have_self) {
        cout << "Self_kw_array n'existe pas\n";
        return;
    }
    const size_t n8 = (size_t)nbk * (nbk + 1) / 2;
    std::vector<double> S((size_t)2 * n8 * (nbw / 2)), mid(n8), last(2 * n8, 0.0);
    if (!check(tpsc_get_self(ctx_, S.data(), NULL, NULL, NULL), "save_Self_bin")) return;
    if (!check(tpsc_get_sigma_tau(ctx_, nbw / 2, mid.data()), "save_Self_bin")) return;
    for (size_t o = 0; o < n8; ++o) last[2 * o] = mid[o];
    char name[200];
    tpsc_file_name(TPSC_FILE_SELF_BIN, name, sizeof name, U, tp, tpp, t3, density, tem, 2 * (nbk - 1), nbw, 0, 0);
    check(tpsc_write_self_bin(name, nbk, nbw, S.data(), last.data()), "save_Self_bin");
}

// green::load_Self_bin (src/green.cpp:1517-1541): S from this model's
// self_bin file; the tails stay as they are
void green::load_Self_bin() {
    const size_t n8 = (size_t)nbk * (nbk + 1) / 2;
    std::vector<double> S((size_t)2 * n8 * (nbw / 2 + 1));
    char name[200];
    tpsc_file_name(TPSC_FILE_SELF_BIN, name, sizeof name, U, tp, tpp, t3, density, tem, 2 * (nbk - 1), nbw, 0, 0);
    if (tpsc_read_self_bin(name, nbk, nbw, S.data()) != TPSC_OK) {
        cout << "fichier  " << name << "  inexistant\n";
        return;
    }
    if (ctx_ && check(tpsc_set_self(ctx_, S.data(), NULL, NULL, NULL, NULL), "load_Self_bin")) have_self = true;
}

// green::load_Self (src/green.cpp:1637-1670): S from this model's self_tpsc
// ascii file; the tails stay as they are
void green::load_Self() {
    const size_t n8 = (size_t)nbk * (nbk + 1) / 2;
    std::vector<double> S((size_t)2 * n8 * (nbw / 2));
    char name[200];
    tpsc_file_name(TPSC_FILE_SELF_ASCII, name, sizeof name, U, tp, tpp, t3, density, tem, 2 * (nbk - 1), nbw, 0, 0);
    if (tpsc_read_self_ascii(name, nbk, nbw, S.data()) != TPSC_OK) {
        cout << "load_Self():  fichier  " << name << "  inexistant\n";
        return;
    }
    if (ctx_ && check(tpsc_set_self(ctx_, S.data(), NULL, NULL, NULL, NULL), "load_Self")) have_self = true;
}

// green::save_Green (src/green.cpp:1577-1633): G(k, i w_n) at one k, the
// lattice point folded into the octant, eps_k - mu with the current mu
void green::save_Green(int *k) {
    if (!have_self) {
        cout << "save_Green(): Self_kw_array n'existe pas\n";
        return;
    }
    const int nk0 = 2 * (nbk - 1);
    long l = k[0] < 0 ? -k[0] : k[0], m = k[1] < 0 ? -k[1] : k[1];
    if (l > nk0 || m > nk0) {
        cout << "save_Green(): k[0] et k[1] doivent etre entre 0 et nk0\n";
        return;
    }
    if (l > nbk - 1) l = nk0 - l;
    if (m > nbk - 1) m = nk0 - m;
    if (m > l) std::swap(l, m);
    // hamiltonien::ek_val (src/hamiltonien.cpp:107-116) on the unfolded k
    auto fold = [&](int x) {
        while (x < 0) x += nk0;
        return x > nbk - 1 ? nk0 - x : x;
    };
    std::vector<double> ek((size_t)nbk * nbk);
    const size_t n8 = (size_t)nbk * (nbk + 1) / 2;
    std::vector<double> S((size_t)2 * n8 * (nbw / 2)), c2(n8), c3(n8);
    if (!check(tpsc_get_ek(ctx_, ek.data()), "save_Green")) return;
    if (!check(tpsc_get_self(ctx_, S.data(), c2.data(), c3.data(), NULL), "save_Green")) return;
    const double ek_mu = ek[fold(k[1]) + (size_t)fold(k[0]) * nbk] - mu;
    const size_t o = m + (l * (l + 1)) / 2;
    char name[200];
    tpsc_file_name(TPSC_FILE_GREEN, name, sizeof name, U, tp, tpp, t3, density, tem, nk0, nbw, (int)l, (int)m);
    check(tpsc_write_green_ascii(name, nbw, tem, ek_mu, Sigma_inf, c2[o], c3[o], S.data() + 2 * o, (long long)n8),
          "save_Green");
}

// ---------------------------------------------------------------------------
cond_opt::cond_opt(int nk0, int Nw0, double n, double T, double eta0, double *params)
    : green(nk0, Nw0, n, T, eta0, params), chijj1_qn(NULL), chijj2_qn(NULL), chijj3_qn(NULL), kx0(0.0) {}

cond_opt::~cond_opt() {
    delete[] chijj1_qn;
    delete[] chijj2_qn;
    delete[] chijj3_qn;
}

// cond_opt::calc_chijj_vertex_corr_all_optim (src/cond_opt.cpp:2537-6529):
// Sigma and mu first when missing, Sigma at the listed k points, the Fermi
// surface files, then chi_jj on the device and the reference's result files
// (chijj*_k_qn_*, chijj*_k_tot_qn_*, kx0_*, kx0_bin_*, chijj1_qn_*,
// chijj_with_vc1_qn_*, chijj2_qn_*) with its column layouts and stdout lines.
// With chi3, the Aslamazov-Larkin correction on the non-uniform grid of mmin
// and its files (chijj3_qn_*, chijj_with_all_vc_qn_*, and with angle bins
// chijj3_k_qn_*, chijj3_k_tot_qn_*; src/cond_opt.cpp:6448-6521).
void cond_opt::calc_chijj_vertex_corr_all_optim(bool chi3, int mmin, int N_theta_k, int *k_chijj, int nk_chijj) {
    cout << "calcul de chijj par calc_chijj_vertex_corr_all_optim()\n";
    const int nw = nbw / 2, nk0 = 2 * (nbk - 1);
    if (!have_self) {
        calc_Self_FFT_spline();
        traceSelfG();
        green::find_mu();
    }
    if (!mu_calcule) {
        cout << "calc_chijj_vertex_corr_all_optim(): mu non calcule\n";
        return;
    }
    if (k_chijj && nk_chijj) save_self_ikn(k_chijj, nk_chijj, nw / 16);
    find_FS_inter();
    if (N_theta_k < 1) N_theta_k = 1;
    if (!check(tpsc_chijj(ctx_, N_theta_k), "calc_chijj_vertex_corr_all_optim")) return;
    delete[] chijj1_qn;
    delete[] chijj2_qn;
    chijj1_qn = new double[nw + 1];
    chijj2_qn = new double[nw + 1];
    std::vector<double> k1((size_t)(nw + 1) * N_theta_k), k2((size_t)(nw + 1) * N_theta_k);
    if (!check(tpsc_get_chijj(ctx_, chijj1_qn, chijj2_qn, &kx0, k1.data(), k2.data()), "tpsc_get_chijj")) return;

    char name[200];
    fstream file, file2, file3, file4;
    const double dn = density;
    sprintf(name, "./chijj1_k_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, dn, tem, nk0, nbw);
    file.open(name, ios::out);
    file << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
    sprintf(name, "./chijj1_k_tot_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, dn, tem, nk0,
            nbw);
    file2.open(name, ios::out);
    file2 << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
    sprintf(name, "./chijj2_k_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, dn, tem, nk0, nbw);
    file3.open(name, ios::out);
    file3 << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
    sprintf(name, "./chijj2_k_tot_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, dn, tem, nk0,
            nbw);
    file4.open(name, ios::out);
    file4 << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
    for (int j = 0; j <= nw; j++) {
        double t1 = 0, t2 = 0;
        for (int p = 0; p < N_theta_k; p++) {
            t1 += k1[p + (size_t)j * N_theta_k];
            t2 += k2[p + (size_t)j * N_theta_k];
        }
        file2 << setw(10) << j << setw(30) << t1 << setw(30) << chijj1_qn[j] << t1 / chijj1_qn[j] << '\n';
        file4 << setw(10) << j << setw(30) << t2 << setw(30) << chijj2_qn[j] << t2 / chijj2_qn[j] << '\n';
        for (int p = 0; p < N_theta_k; p++) {
            file << setw(10) << j << setw(10) << p + 1 << k1[p + (size_t)j * N_theta_k] << '\n';
            file3 << setw(10) << j << setw(10) << p + 1 << k2[p + (size_t)j * N_theta_k] << '\n';
        }
    }
    file.close();
    file2.close();
    file3.close();
    file4.close();

    sprintf(name, "kx0_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, dn, tem, nk0, nbw);
    file.open(name, ios::out);
    file << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific) << kx0 << '\n';
    file.close();
    sprintf(name, "kx0_bin_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, dn, tem, nk0, nbw);
    file.open(name, ios::out | ios::binary);
    file.write((char *)&kx0, sizeof(kx0));
    file.close();

    for (int j = 0; j <= nw; j++)
        if (chijj1_qn[j] < 0.0) {
            cout << "attention! valeur non-physique de chi_jj\n";
            cout << setw(30) << chijj1_qn[j] << '\n';
            break;
        }
    sprintf(name, "./chijj1_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, dn, tem, nk0, nbw);
    file.open(name, ios::out);
    file << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
    sprintf(name, "./chijj_with_vc1_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, dn, tem,
            nk0, nbw);
    file2.open(name, ios::out);
    file2 << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
    sprintf(name, "./chijj2_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, dn, tem, nk0, nbw);
    file4.open(name, ios::out);
    file4 << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
    for (int j = 0; j <= nw; j++) {
        file << setw(10) << j << chijj1_qn[j] << '\n';
        file4 << setw(10) << j << chijj2_qn[j] << '\n';
        file2 << setw(10) << j << chijj1_qn[j] + chijj2_qn[j] << '\n';
    }
    file.close();
    file2.close();
    file4.close();
    cout << "-k0:  " << -kx0 << '\n';
    cout << "chijj1(iqn=0):  " << chijj1_qn[0] << '\n';
    cout << "chijj2(iqn=0):  " << chijj2_qn[0] << '\n';
    cout << "chijj1(iqn=0)+chijj2(iqn=0):  " << chijj1_qn[0] + chijj2_qn[0] << '\n';
    cout << "difference relative avec -k0:  " << (chijj1_qn[0] + chijj2_qn[0] + kx0) / kx0 << '\n';
    if (chi3) calc_chijj3(mmin, N_theta_k);
}

// The chi3 branch of calc_chijj_vertex_corr_all_optim (src/cond_opt.cpp:4292-6529)
// after chijj1, chijj2: the AL correction on the device, then the reference's
// files with their formats.
void cond_opt::calc_chijj3(int mmin, int N_theta_k) {
    cout << "calcul de la seconde correction de vertex\n";
    const int nw = nbw / 2, nk0 = 2 * (nbk - 1);
    if (!check(tpsc_chijj3(ctx_, mmin, N_theta_k), "calc_chijj_vertex_corr_all_optim")) return;
    int N = 0;
    if (!check(tpsc_get_chijj3(ctx_, 0, &N, NULL, NULL, NULL), "tpsc_get_chijj3")) return;
    std::vector<int> ind(N);
    std::vector<double> c3(N), k3((size_t)N * N_theta_k);
    if (!check(tpsc_get_chijj3(ctx_, N, &N, ind.data(), c3.data(), k3.data()), "tpsc_get_chijj3")) return;
    cout << "2^M:  " << (1 << mmin) << "  (N0-1)/((int)pow(2.0,M)):  " << (nw >> mmin) << "   N:  " << N << '\n';
    delete[] chijj3_qn;
    chijj3_qn = new double[nw + 1];
    for (int j = 0; j <= nw; j++) chijj3_qn[j] = j < N ? c3[j] : 0.0;

    char name[200];
    fstream file, file2;
    const double dn = density;
    sprintf(name, "./chijj3_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d_%1d.dat", U, tp, tpp, t3, dn, tem, nk0, nbw,
            mmin);
    file.open(name, ios::out);
    file << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
    for (int j = 0; j < N; j++) file << setw(10) << (long)ind[j] << chijj3_qn[j] << '\n';
    file.close();

    sprintf(name, "./chijj_with_all_vc_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d_%1d.dat", U, tp, tpp, t3, dn, tem,
            nk0, nbw, mmin);
    file.open(name, ios::out);
    file << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
    for (int j = 0; j < N; j++) {
        const double v = j == 0 ? chijj1_qn[0] + chijj2_qn[0]
                                : chijj1_qn[ind[j]] + chijj2_qn[ind[j]] + chijj3_qn[j];
        file << setw(10) << (long)ind[j] << v << '\n';
    }
    file.close();

    if (N_theta_k > 1) {
        sprintf(name, "./chijj3_k_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d_%1d.dat", U, tp, tpp, t3, dn, tem, nk0,
                nbw, mmin);
        file.open(name, ios::out);
        file << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
        sprintf(name, "./chijj3_k_tot_qn_%5.3f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d_%1d.dat", U, tp, tpp, t3, dn, tem,
                nk0, nbw, mmin);
        file2.open(name, ios::out);
        file2 << setprecision(16) << setiosflags(ios::left) << setiosflags(ios::scientific);
        for (int j = 1; j < N; j++) {
            double tot = 0;
            for (int p = 0; p < N_theta_k; p++) tot += k3[p + (size_t)j * N_theta_k];
            file2 << setw(10) << (long)ind[j] << setw(30) << tot << setw(30) << chijj3_qn[j] << tot / chijj3_qn[j]
                  << '\n';
            for (int p = 0; p < N_theta_k; p++)
                file << setw(10) << (long)ind[j] << setw(10) << (p + 1) << k3[p + (size_t)j * N_theta_k] << '\n';
        }
        file.close();
        file2.close();
    }
}
