// Device dense linear algebra for the eigensolvers (dense.cu): the small
// Hermitian eigenproblems, QR and Cholesky of the reference's eig_zheevd.cpp,
// eig_zhegv.cpp, ortho_qr.cpp and lobpcg_cpu.cpp, plus column-wise helpers.
// All FP64 complex, column-major, on the cell stream.
#pragma once

#include <cublas_v2.h>

#include "common.cuh"
#include "engine.h"

namespace pspw {

// the cell's cuBLAS handle, bound to the cell's current stream
int cublas_handle(pspw_cell *c, cublasHandle_t *h);
// A (n x n, lda) <- eigenvectors, w[n] (device) <- ascending eigenvalues;
// upper triangle of A is read (zheevd 'V','U').  *info_out = LAPACK info.
// n <= 160: the engine's kernels (heev.cu, info always 0); else cuSOLVER.
int dev_zheevd(pspw_cell *c, double2 *A, int lda, double *w, int n, int *info_out);
// Householder QR of X (m x n, ld) replaced by its explicit Q (zgeqrf+zungqr).
int dev_ortho_qr(pspw_cell *c, double2 *X, int ld, int m, int n, int *info_out);
// Upper Cholesky of the n x n Hermitian A (zpotrf 'U'); A overwritten.
int dev_potrf_upper(pspw_cell *c, double2 *A, int lda, int n, int *info_out);
// B (m x n, ldb) <- B * U^-1 with U upper (ztrsm 'R','U','N','N').
int dev_trsm_right_upper(pspw_cell *c, const double2 *U, int ldu, double2 *B, int ldb, int m,
                         int n);
// Generalised problem of eig_zhegv.cpp:5-161: B's eigenvectors scaled by
// 1/sqrt(eval) where eval > SMALL; A' = S^H (A S); eig(A'); evec = S U.
// A and B are overwritten as in the reference; eval (device, n) may be null.
int dev_zhegv(pspw_cell *c, double2 *A, int lda, double2 *B, int ldb, double *eval,
              double2 *evec, int lde, int n, int *nindep_out);
// v(0:n,0:n) <- (v + v^H)/2 (lobpcg_cpu.cpp:15-27)
int dev_symmetrize(pspw_cell *c, double2 *v, int ldv, int n);
// out[j] = Re(sum_i conj(x(i,j)) y(i,j)) for j < n (column dot products)
int dev_coldot(pspw_cell *c, const double2 *x, int ldx, const double2 *y, int ldy, int m, int n,
               double *out);
// R(:,j) = lam[j] X(:,j) - HX(:,j)
int dev_residual(pspw_cell *c, const double *lam, const double2 *X, int ldx, const double2 *HX,
                 int ldh, double2 *R, int ldr, int m, int n);
// R(i,j) = prec[i] * (s[j] * R(i,j))   (s may be null: s = 1)
int dev_scale_prec(pspw_cell *c, const double *s, const double *prec, double2 *R, int ldr, int m,
                   int n);
// identity / diagonal fill of an n x n block
int dev_diag(pspw_cell *c, double2 *A, int lda, int n, const double *d);

}  // namespace pspw
