// tpsc_files.cpp -- the reference's on-disk formats for chi0 and Sigma, on
// the host (no device work): the files a saved run leaves and a warm start
// reads, in the reference's names and layouts so that either program reads
// the other's files.
//
//  * chi0 binary (chi0::save_chi / loadChi0, src/chi0.cpp:61-154): int nbq,
//    int nwmax, then nwmax + 1 frames of N8 doubles, chi0(q, iqn) at octant
//    index m + l(l+1)/2 of frame n;
//  * self_bin (green::save_Self_bin / load_Self_bin, src/green.cpp:1496-1541):
//    nbw/2 + 1 frames of N8 complex doubles, the S coefficient of
//    Sigma = Sigma_inf/z + C2/z^2 + C3/z^3 + S/z^4 for n < nbw/2; the last
//    frame is what calc_Self_FFT_spline leaves there from packing Sigma(k, tau)
//    (src/green.cpp:1872-1885): (Sigma(k, beta/2), 0);
//  * self_tpsc ascii (green::save_Self / load_Self, src/green.cpp:1544-1574,
//    1637-1670): one line "n l m Re Im" per frequency and octant point;
//  * Green ascii (green::save_Green, src/green.cpp:1577-1633): one line
//    "n Re G Im G" per frequency at one k.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <string>
#include <vector>

#include "../../include/tpsc_b200.h"
#include "tpsc_host.h"

namespace {

using tpsc::static_fail;
using cplx = std::complex<double>;

long long n8_of(int nbk) { return (long long)nbk * (nbk + 1) / 2; }

bool grid_ok(int nbk, int nbw) { return nbk >= 2 && nbw >= 2 && nbw % 2 == 0; }

int open_fail(const char *what, const char *path) {
    return static_fail(TPSC_ERR_ARG, std::string(what) + ": cannot open " + (path ? path : "(null)"));
}

}  // namespace

extern "C" {

int tpsc_file_name(int kind, char *out, int cap, double U, double tp, double tpp, double t3, double n, double T,
                   int nk0, int nbw, int l, int m) {
    if (!out || cap <= 0) return static_fail(TPSC_ERR_ARG, "tpsc_file_name: no buffer");
    int w = -1;
    switch (kind) {
        case TPSC_FILE_CHI0_BIN:
            w = snprintf(out, cap, "./chi0_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%d_%d.dat", tp, tpp, t3, n, T, nk0, nbw);
            break;
        case TPSC_FILE_SELF_BIN:
            w = snprintf(out, cap, "./self_bin_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, n, T,
                         nk0, nbw);
            break;
        case TPSC_FILE_SELF_ASCII:
            w = snprintf(out, cap, "./self_tpsc_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d.dat", U, tp, tpp, t3, n,
                         T, nk0, nbw);
            break;
        case TPSC_FILE_GREEN:
            w = snprintf(out, cap, "./Green_%4.2f_%5.3f_%5.3f_%5.3f_%7.5f_%6.4f_%1d_%1d_%1d_%1d.dat", U, tp, tpp, t3,
                         n, T, nk0, nbw, l, m);
            break;
        default: return static_fail(TPSC_ERR_ARG, "tpsc_file_name: unknown kind");
    }
    if (w < 0 || w >= cap) return static_fail(TPSC_ERR_ARG, "tpsc_file_name: buffer too small");
    return TPSC_OK;
}

int tpsc_write_chi0_bin(const char *path, int nbq, int nwmax, const double *chiqw) {
    if (!path || !chiqw || nbq < 2 || nwmax < 1) return static_fail(TPSC_ERR_ARG, "tpsc_write_chi0_bin: bad arguments");
    std::ofstream f(path, std::ios::out | std::ios::binary);
    if (!f) return open_fail("tpsc_write_chi0_bin", path);
    f.write(reinterpret_cast<const char *>(&nbq), sizeof nbq);
    f.write(reinterpret_cast<const char *>(&nwmax), sizeof nwmax);
    f.write(reinterpret_cast<const char *>(chiqw), (std::streamsize)((nwmax + 1) * n8_of(nbq) * sizeof(double)));
    return f ? TPSC_OK : static_fail(TPSC_ERR_ARG, std::string("tpsc_write_chi0_bin: write failed: ") + path);
}

int tpsc_read_chi0_bin(const char *path, int *nbq, int *nwmax, double *chiqw, long long cap) {
    if (!path || !nbq || !nwmax) return static_fail(TPSC_ERR_ARG, "tpsc_read_chi0_bin: bad arguments");
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f) return open_fail("tpsc_read_chi0_bin", path);
    int b = 0, w = 0;
    f.read(reinterpret_cast<char *>(&b), sizeof b);
    f.read(reinterpret_cast<char *>(&w), sizeof w);
    if (!f || b < 2 || w < 1) return static_fail(TPSC_ERR_ARG, std::string("tpsc_read_chi0_bin: bad header: ") + path);
    *nbq = b;
    *nwmax = w;
    if (!chiqw) return TPSC_OK;
    const long long need = (long long)(w + 1) * n8_of(b);
    if (cap < need) return static_fail(TPSC_ERR_ARG, "tpsc_read_chi0_bin: buffer smaller than the file's frames");
    f.read(reinterpret_cast<char *>(chiqw), (std::streamsize)(need * sizeof(double)));
    return f ? TPSC_OK : static_fail(TPSC_ERR_ARG, std::string("tpsc_read_chi0_bin: short file: ") + path);
}

int tpsc_write_self_bin(const char *path, int nbk, int nbw, const double *self_kw, const double *last) {
    if (!path || !self_kw || !grid_ok(nbk, nbw)) return static_fail(TPSC_ERR_ARG, "tpsc_write_self_bin: bad arguments");
    std::ofstream f(path, std::ios::out | std::ios::binary);
    if (!f) return open_fail("tpsc_write_self_bin", path);
    const long long frame = n8_of(nbk);
    f.write(reinterpret_cast<const char *>(self_kw), (std::streamsize)((nbw / 2) * frame * sizeof(cplx)));
    std::vector<cplx> tail((size_t)frame);
    if (last) std::copy(reinterpret_cast<const cplx *>(last), reinterpret_cast<const cplx *>(last) + frame, tail.begin());
    f.write(reinterpret_cast<const char *>(tail.data()), (std::streamsize)(frame * sizeof(cplx)));
    return f ? TPSC_OK : static_fail(TPSC_ERR_ARG, std::string("tpsc_write_self_bin: write failed: ") + path);
}

int tpsc_read_self_bin(const char *path, int nbk, int nbw, double *self_kw) {
    if (!path || !self_kw || !grid_ok(nbk, nbw)) return static_fail(TPSC_ERR_ARG, "tpsc_read_self_bin: bad arguments");
    std::ifstream f(path, std::ios::in | std::ios::binary);
    if (!f) return open_fail("tpsc_read_self_bin", path);
    f.read(reinterpret_cast<char *>(self_kw), (std::streamsize)((nbw / 2 + 1) * n8_of(nbk) * sizeof(cplx)));
    return f ? TPSC_OK : static_fail(TPSC_ERR_ARG, std::string("tpsc_read_self_bin: short file: ") + path);
}

int tpsc_write_self_ascii(const char *path, int nbk, int nbw, int nfreq, const double *self_kw) {
    if (!path || !self_kw || !grid_ok(nbk, nbw) || nfreq < 0)
        return static_fail(TPSC_ERR_ARG, "tpsc_write_self_ascii: bad arguments");
    if (nfreq > nbw / 2 || nfreq == 0) nfreq = nbw / 2;
    std::ofstream f(path, std::ios::out);
    if (!f) return open_fail("tpsc_write_self_ascii", path);
    const long long frame = n8_of(nbk);
    const cplx *S = reinterpret_cast<const cplx *>(self_kw);
    f << std::left << std::scientific << std::setprecision(16);
    for (long j = 0; j < nfreq; ++j)
        for (long l = 0; l < nbk; ++l)
            for (long m = 0; m <= l; ++m) {
                const cplx v = S[m + l * (l + 1) / 2 + j * frame];
                f << std::setw(10) << j << std::setw(10) << l << std::setw(10) << m << std::setw(25) << v.real()
                  << v.imag() << '\n';
            }
    return f ? TPSC_OK : static_fail(TPSC_ERR_ARG, std::string("tpsc_write_self_ascii: write failed: ") + path);
}

int tpsc_read_self_ascii(const char *path, int nbk, int nbw, double *self_kw) {
    if (!path || !self_kw || !grid_ok(nbk, nbw)) return static_fail(TPSC_ERR_ARG, "tpsc_read_self_ascii: bad arguments");
    std::ifstream f(path, std::ios::in);
    if (!f) return open_fail("tpsc_read_self_ascii", path);
    const long long frame = n8_of(nbk);
    cplx *S = reinterpret_cast<cplx *>(self_kw);
    // the frames in file order; each line names its own (n, l, m)
    for (long long i = 0; i < (nbw / 2) * frame; ++i) {
        long j, l, m;
        double re, im;
        if (!(f >> j >> l >> m >> re >> im))
            return static_fail(TPSC_ERR_ARG, std::string("tpsc_read_self_ascii: short file: ") + path);
        if (j < 0 || j >= nbw / 2 || l < 0 || l >= nbk || m < 0 || m > l)
            return static_fail(TPSC_ERR_ARG, std::string("tpsc_read_self_ascii: index out of range: ") + path);
        S[m + l * (l + 1) / 2 + j * frame] = cplx(re, im);
    }
    return TPSC_OK;
}

int tpsc_write_green_ascii(const char *path, int nbw, double T, double ek_mu, double sigma_inf, double s2, double s3,
                           const double *self_col, long long stride) {
    if (!path || !self_col || nbw < 2 || !(T > 0) || stride < 1)
        return static_fail(TPSC_ERR_ARG, "tpsc_write_green_ascii: bad arguments");
    std::ofstream f(path, std::ios::out);
    if (!f) return open_fail("tpsc_write_green_ascii", path);
    const double pi = std::acos(-1.0);
    const cplx *S = reinterpret_cast<const cplx *>(self_col);
    f << std::left << std::setprecision(16);
    for (long j = 0; j < nbw / 2; ++j) {
        const cplx z(0, (2 * j + 1) * pi * T);
        const cplx sig = sigma_inf / z + s2 / (z * z) + s3 / (z * z * z) + S[j * stride] / (z * z * z * z);
        const cplx G = 1.0 / (z - ek_mu - sig);
        f << std::setw(10) << j << std::setw(25) << G.real() << G.imag() << '\n';
    }
    return f ? TPSC_OK : static_fail(TPSC_ERR_ARG, std::string("tpsc_write_green_ascii: write failed: ") + path);
}

}  // extern "C"
