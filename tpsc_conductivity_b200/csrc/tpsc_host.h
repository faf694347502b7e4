// tpsc_host.h -- host-side helpers shared by the library's C++ files.
#pragma once
#include <cuda_runtime.h>

#include <string>

namespace tpsc {
// sets the message tpsc_last_error(NULL) returns; returns code
int static_fail(int code, const std::string &msg);

// the infinite lattice (tpsc_lattice.cu): mu0 at density n, and chi0 at
// np points qw[p] = (qx, qy, w_n); L_out the lattice size the sums converged at
int lattice_mu0(double n, double T, double tp, double tpp, double t3, cudaStream_t st, double *mu_out, int *L_out);
// (L_fixed > 0: that lattice only, no convergence loop)
int lattice_chi0(double mu, double T, double tp, double tpp, double t3, int np, const double *qw, int L_fixed,
                 cudaStream_t st, double *out, int *L_out);
}  // namespace tpsc
