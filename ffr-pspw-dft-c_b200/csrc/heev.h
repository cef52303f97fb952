// Small dense Hermitian eigensolver and tridiagonal eigenvalues on the
// device (heev.cu).
#pragma once

#include <cstddef>

#include "common.cuh"
#include "engine.h"

namespace pspw {

// largest order of dev_heev_small and dev_chol_inv_upper (their one-block
// kernels keep the packed lower triangle, n (n+1)/2 complex values, in
// shared memory)
constexpr int kHeevMax = 150;
// largest order of dev_tri_eigvals
constexpr int kTriEigMax = 4096;

// bytes of device workspace dev_heev_small needs for order n
size_t heev_small_workspace(int n);

// A (n x n, lda; upper triangle read, as zheevd 'V','U') <- orthonormal
// eigenvectors, w[n] (device) <- eigenvalues ascending.  n <= kHeevMax;
// `work` holds heev_small_workspace(n) bytes.  Enqueued on the cell stream.
int dev_heev_small(pspw_cell *c, double2 *A, int lda, double *w, int n, void *work);

// Cholesky factor and its inverse for CholeskyQR: G (n x n, ldg, upper
// triangle read) = U^H U; Uinv (n x n, ldu) <- U^-1 (upper, zeros below);
// stat[0] (device) <- 0, or k + 1 if the k-th pivot is not positive;
// stat[1] <- max |U_kk| / min |U_kk|.  n <= kHeevMax: the factor in one
// block, the inverse on ceil(n / 4) blocks (one warp per column); Uinv is
// left untouched when the factorisation fails.
int dev_chol_inv_upper(pspw_cell *c, const double2 *G, int ldg, int n, double2 *Uinv, int ldu,
                       double *stat);

// Eigenvalues (ascending) of the real symmetric tridiagonal matrix with
// diagonal d[n] and off-diagonal e[n-1] (device arrays), by bisection.
int dev_tri_eigvals(pspw_cell *c, const double *d, const double *e, int n, double *w);

}  // namespace pspw
