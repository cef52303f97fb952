// Device eigensolvers (solvers.cu) and the density kernel (rho.cu).
#pragma once

#include "common.cuh"
#include "engine.h"

namespace pspw {

void random_col_host(double2 *A, int nelem, long seed);
int gen_prec_dev(pspw_cell *c, double *d_prec, int nbasis, double tau);
// X: device FP64 block nbasis x nstates (ld nbasis), overwritten with the
// solver's random start and then the eigenvectors.
int davidson_dev(pspw_cell *c, int hprec, double *evals_host, double2 *X, int nbasis, int nstates,
                 const double *d_prec, int nempty, int max_iter, double *res_host, int *iters);
int lobpcg_dev(pspw_cell *c, int hprec, double *lambda_host, double2 *X, int nbasis, int nstates,
               const double *d_prec, int nempty, int max_iter, double *res_host, int *iters);
// LOBPCG with an orthonormal [X W P] basis and a standard Rayleigh-Ritz
// eigenproblem (an opt-in alternative to lobpcg_dev; same start, same test).
int lobpcg_ortho_dev(pspw_cell *c, int hprec, double *lambda_host, double2 *X, int nbasis,
                     int nstates, const double *d_prec, int nempty, int max_iter, double *res_host,
                     int *iters, bool from_x = false);
// v0: device, normalised in place; T_host k x k (ldT); f_out device or null.
// hprec: precision of the H*v products (PSPW_PREC_F64 reproduces lanczos.cpp;
// PSPW_PREC_F32 for bounds that only shape a filter); the recurrence, the
// reorthogonalisation and T stay FP64.
int lanczos_dev(pspw_cell *c, double2 *v0, int ngw, int k, double *T_host, int ldT, double2 *f_out,
                int hprec = PSPW_PREC_F64);

// EvalRhoPsi / EvalENL on device blocks (capi_solvers.cu); see pspw_gpu.h.
int eval_rho_psi_dev(pspw_cell *c, const double2 *dX, int ld, int ngw, int nx, const double *focc,
                     double wkpt, double omega, double *d_rho, double *ekin);
int eval_enl_dev(pspw_cell *c, const double2 *dX, int ld, int ngw, int nx, const double *focc,
                 double wkpt, double *enl, double *fnl);

}  // namespace pspw
