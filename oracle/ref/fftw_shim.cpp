/*
 * fftw_shim.cpp -- the FFTW3 subset declared in fftw3.h, written from the
 * transform definitions in the FFTW 3 manual (section "What FFTW Really
 * Computes").  TEST INFRASTRUCTURE: linked only into the CPU oracle binary
 * built from the unmodified reference sources; never into the product.
 *
 * Method (standard, published): a length-2^p complex FFT (iterative radix-2
 * decimation in time, twiddles from long-double sin/cos) drives
 *   - DFT of any power-of-two length (sign +-1, unnormalised);
 *   - DCT-I of length n as the DFT of the length-2(n-1) even extension;
 *   - DST-I of length n as the DFT of the length-2(n+1) odd extension.
 * Two real lines are packed into one complex transform (real even input has a
 * real spectrum, real odd input an imaginary one), so a DCT-I line costs about
 * one complex FFT of length n-1, the same as FFTW's r2hc-based REDFT00.
 * Non power-of-two lengths fall back to a direct O(N^2) sum.
 * Plans are immutable after creation, so concurrent fftw_execute_* calls from
 * OpenMP threads (as the reference makes) are safe.
 */
#include "fftw3.h"

#include <cmath>
#include <complex>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <vector>

typedef std::complex<double> cplx;

namespace {

struct CFFT {
    int n = 0;
    bool pow2 = false;
    std::vector<cplx> tw;    // exp(-2 pi i k / n), k < n/2 (pow2) or k < n (direct)
    std::vector<int> rev;    // bit reversal permutation

    explicit CFFT(int n_) : n(n_) {
        pow2 = n > 0 && (n & (n - 1)) == 0;
        if (pow2) {
            tw.resize(n / 2 > 0 ? n / 2 : 1);
            for (int k = 0; k < n / 2; ++k) {
                long double a = -2.0L * 3.141592653589793238462643383279502884L * k / n;
                tw[k] = cplx((double)cosl(a), (double)sinl(a));
            }
            rev.resize(n);
            int bits = 0;
            while ((1 << bits) < n) ++bits;
            for (int i = 0; i < n; ++i) {
                int r = 0;
                for (int b = 0; b < bits; ++b)
                    if (i & (1 << b)) r |= 1 << (bits - 1 - b);
                rev[i] = r;
            }
        } else {
            tw.resize(n);
            for (int k = 0; k < n; ++k) {
                long double a = -2.0L * 3.141592653589793238462643383279502884L * k / n;
                tw[k] = cplx((double)cosl(a), (double)sinl(a));
            }
        }
    }

    // in-place transform of x[0..n), exponent sign `sign` (-1 forward, +1 backward)
    void run(cplx *x, int sign) const {
        if (n <= 1) return;
        if (!pow2) {
            std::vector<cplx> y(n);
            for (int k = 0; k < n; ++k) {
                cplx s = 0;
                for (int j = 0; j < n; ++j) {
                    cplx w = tw[(long)j * k % n];
                    if (sign > 0) w = std::conj(w);
                    s += x[j] * w;
                }
                y[k] = s;
            }
            for (int k = 0; k < n; ++k) x[k] = y[k];
            return;
        }
        for (int i = 0; i < n; ++i)
            if (i < rev[i]) std::swap(x[i], x[rev[i]]);
        for (int len = 2; len <= n; len <<= 1) {
            int half = len >> 1, step = n / len;
            for (int i = 0; i < n; i += len) {
                for (int k = 0; k < half; ++k) {
                    cplx w = tw[k * step];
                    if (sign > 0) w = std::conj(w);
                    cplx u = x[i + k];
                    cplx v = x[i + k + half] * w;
                    x[i + k] = u + v;
                    x[i + k + half] = u - v;
                }
            }
        }
    }
};

enum PlanType { P_R2R_1D, P_R2R_2D, P_DFT_1D, P_DFT_2D };

struct R2RLine {
    fftw_r2r_kind kind;
    int len;
    CFFT *fft;   // length of the symmetric extension
};

}  // namespace

struct oracle_fftw_plan_s {
    PlanType type;
    int n0 = 0, n1 = 0;
    int sign = -1;
    double *rin = nullptr, *rout = nullptr;
    fftw_complex *cin = nullptr, *cout = nullptr;
    R2RLine line0{}, line1{};
    CFFT *f0 = nullptr, *f1 = nullptr;
    ~oracle_fftw_plan_s() {
        delete line0.fft;
        delete line1.fft;
        delete f0;
        delete f1;
    }
};

static R2RLine make_line(fftw_r2r_kind kind, int len) {
    R2RLine l;
    l.kind = kind;
    l.len = len;
    if (kind == FFTW_REDFT00)
        l.fft = new CFFT(2 * (len - 1));
    else if (kind == FFTW_RODFT00)
        l.fft = new CFFT(2 * (len + 1));
    else
        std::abort();   // kinds the reference never uses
    return l;
}

// Transform `count` real lines of length line.len; line p starts at data+p*dist,
// consecutive elements are `stride` apart.  Lines are processed two at a time.
static void r2r_lines(const R2RLine &line, double *in, double *out, int count, long stride,
                      long dist) {
    const int len = line.len;
    const int L = line.fft->n;
    std::vector<cplx> z(L);
    for (int p = 0; p < count; p += 2) {
        const bool two = (p + 1 < count);
        const double *a = in + p * dist;
        const double *b = two ? in + (p + 1) * dist : nullptr;
        if (line.kind == FFTW_REDFT00) {
            // even extension e_j = x_j (j<len), x_{L-j} (j>=len)
            for (int j = 0; j < L; ++j) {
                int s = j < len ? j : L - j;
                z[j] = cplx(a[s * stride], two ? b[s * stride] : 0.0);
            }
            line.fft->run(z.data(), -1);
            double *oa = out + p * dist;
            double *ob = two ? out + (p + 1) * dist : nullptr;
            for (int k = 0; k < len; ++k) {
                oa[k * stride] = z[k].real();
                if (two) ob[k * stride] = z[k].imag();
            }
        } else {
            // odd extension o = [0, x_0..x_{n-1}, 0, -x_{n-1}..-x_0]; DFT_k = -2i S_k
            for (int j = 0; j < L; ++j) z[j] = 0;
            for (int j = 0; j < len; ++j) {
                cplx v(a[j * stride], two ? b[j * stride] : 0.0);
                z[j + 1] = v;
                z[L - 1 - j] = -v;
            }
            line.fft->run(z.data(), -1);
            double *oa = out + p * dist;
            double *ob = two ? out + (p + 1) * dist : nullptr;
            for (int k = 0; k < len; ++k) {
                // Z = -2i S_a + 2 S_b  ->  Y_a = 2 S_a = -Im Z, Y_b = 2 S_b = Re Z
                oa[k * stride] = -z[k + 1].imag();
                if (two) ob[k * stride] = z[k + 1].real();
            }
        }
    }
}

extern "C" {

fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind, unsigned) {
    fftw_plan p = new oracle_fftw_plan_s;
    p->type = P_R2R_1D;
    p->n0 = n;
    p->rin = in;
    p->rout = out;
    p->line0 = make_line(kind, n);
    return p;
}

fftw_plan fftw_plan_r2r_2d(int n0, int n1, double *in, double *out, fftw_r2r_kind kind0,
                           fftw_r2r_kind kind1, unsigned) {
    fftw_plan p = new oracle_fftw_plan_s;
    p->type = P_R2R_2D;
    p->n0 = n0;
    p->n1 = n1;
    p->rin = in;
    p->rout = out;
    p->line0 = make_line(kind0, n0);
    p->line1 = make_line(kind1, n1);
    return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned) {
    fftw_plan p = new oracle_fftw_plan_s;
    p->type = P_DFT_1D;
    p->n0 = n;
    p->sign = sign;
    p->cin = in;
    p->cout = out;
    p->f0 = new CFFT(n);
    return p;
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned) {
    fftw_plan p = new oracle_fftw_plan_s;
    p->type = P_DFT_2D;
    p->n0 = n0;
    p->n1 = n1;
    p->sign = sign;
    p->cin = in;
    p->cout = out;
    p->f0 = new CFFT(n0);
    p->f1 = new CFFT(n1);
    return p;
}

// transforms executed, per kind (2D r2r, 1D r2r, 1D dft, 2D dft), for the
// probe's account of where the reference's CPU time goes
static std::atomic<long> g_exec_count[4];
extern "C" void oracle_fftw_counts(long out[4]) {
    for (int i = 0; i < 4; ++i) out[i] = g_exec_count[i].load();
}

void fftw_execute_r2r(const fftw_plan p, double *in, double *out) {
    g_exec_count[p->type == P_R2R_2D ? 0 : 1].fetch_add(1, std::memory_order_relaxed);
    if (p->type == P_R2R_1D) {
        r2r_lines(p->line0, in, out, 1, 1, 0);
    } else if (p->type == P_R2R_2D) {
        // dimension 1 (contiguous) first, then dimension 0 (stride n1), in place on out
        r2r_lines(p->line1, in, out, p->n0, 1, p->n1);
        r2r_lines(p->line0, out, out, p->n1, p->n1, 1);
    } else {
        std::abort();
    }
}

void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) {
    g_exec_count[p->type == P_DFT_1D ? 2 : 3].fetch_add(1, std::memory_order_relaxed);
    if (p->type == P_DFT_1D) {
        const int n = p->n0;
        std::vector<cplx> z(n);
        for (int j = 0; j < n; ++j) z[j] = cplx(in[j][0], in[j][1]);
        p->f0->run(z.data(), p->sign);
        for (int j = 0; j < n; ++j) {
            out[j][0] = z[j].real();
            out[j][1] = z[j].imag();
        }
    } else if (p->type == P_DFT_2D) {
        const int n0 = p->n0, n1 = p->n1;
        std::vector<cplx> z((size_t)n0 * n1), line(n0);
        for (size_t j = 0; j < z.size(); ++j) z[j] = cplx(in[j][0], in[j][1]);
        for (int r = 0; r < n0; ++r) p->f1->run(&z[(size_t)r * n1], p->sign);
        for (int c = 0; c < n1; ++c) {
            for (int r = 0; r < n0; ++r) line[r] = z[(size_t)r * n1 + c];
            p->f0->run(line.data(), p->sign);
            for (int r = 0; r < n0; ++r) z[(size_t)r * n1 + c] = line[r];
        }
        for (size_t j = 0; j < z.size(); ++j) {
            out[j][0] = z[j].real();
            out[j][1] = z[j].imag();
        }
    } else {
        std::abort();
    }
}

void fftw_execute(const fftw_plan p) {
    if (p->type == P_R2R_1D || p->type == P_R2R_2D)
        fftw_execute_r2r(p, p->rin, p->rout);
    else
        fftw_execute_dft(p, p->cin, p->cout);
}

void fftw_destroy_plan(fftw_plan p) { delete p; }

}  // extern "C"
