/*
 * fftw3.h -- minimal FFTW3-API shim used ONLY to compile the unmodified
 * reference sources into the CPU oracle binary (oracle/_ref/).
 *
 * TEST INFRASTRUCTURE: nothing in the product links this file.
 *
 * FFTW 3.x itself (unpinned in the reference, src/CMakeLists.txt:11) is not
 * installed in this image.  This header declares exactly the subset of the
 * public FFTW 3 interface the reference calls (grep of src/*.cpp):
 *   fftw_plan_r2r_2d / fftw_plan_r2r_1d   kinds REDFT00 (DCT-I), RODFT00 (DST-I)
 *   fftw_plan_dft_1d / fftw_plan_dft_2d   sign FFTW_FORWARD (-1) / FFTW_BACKWARD (+1)
 *   fftw_execute / fftw_execute_r2r / fftw_execute_dft / fftw_destroy_plan
 * The enum and macro values are FFTW's published API values so that source
 * code written against FFTW compiles unchanged.  The transforms follow the
 * definitions in the FFTW manual (unnormalised, row-major multi-d):
 *   REDFT00, n:  Y_k = X_0 + (-1)^k X_{n-1} + 2 sum_{j=1}^{n-2} X_j cos(pi j k/(n-1))
 *   RODFT00, n:  Y_k = 2 sum_{j=0}^{n-1} X_j sin(pi (j+1)(k+1)/(n+1))
 *   DFT, sign s: Y_k = sum_j X_j exp(s * 2 pi i j k / n)
 * The implementation (fftw_shim.cpp) is an O(N log N) radix-2 FFT for power
 * of two lengths (the only ones the reference uses) with an O(N^2) fallback.
 */
#ifndef TPSC_ORACLE_FFTW3_SHIM_H
#define TPSC_ORACLE_FFTW3_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];

typedef enum {
    FFTW_R2HC = 0, FFTW_HC2R = 1, FFTW_DHT = 2,
    FFTW_REDFT00 = 3, FFTW_REDFT01 = 4, FFTW_REDFT10 = 5, FFTW_REDFT11 = 6,
    FFTW_RODFT00 = 7, FFTW_RODFT01 = 8, FFTW_RODFT10 = 9, FFTW_RODFT11 = 10
} fftw_r2r_kind;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

typedef struct oracle_fftw_plan_s *fftw_plan;

fftw_plan fftw_plan_r2r_1d(int n, double *in, double *out, fftw_r2r_kind kind, unsigned flags);
fftw_plan fftw_plan_r2r_2d(int n0, int n1, double *in, double *out,
                           fftw_r2r_kind kind0, fftw_r2r_kind kind1, unsigned flags);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_execute_r2r(const fftw_plan p, double *in, double *out);
void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
