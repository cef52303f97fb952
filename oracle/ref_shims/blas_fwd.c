/*
 * TEST INFRASTRUCTURE (oracle build only) -- never linked into the product.
 *
 * BLAS/LAPACK entry points with the names and argument lists the reference
 * declares (common_pspw.h:268-344), forwarded to the LP64 OpenBLAS that
 * scipy bundles (symbols prefixed `scipy_`).  Two adaptations:
 *   - zdotc_/zdotu_: the reference declares the MKL form that returns the
 *     result through a leading pointer (common_pspw.h:273-274); OpenBLAS
 *     returns the complex value, so the adapter stores it.
 *   - LAPACK routines get their hidden Fortran CHARACTER lengths (1 each).
 */
#include <stddef.h>

typedef double _Complex zc;

extern double scipy_ddot_(int *, double *, int *, double *, int *);
extern double scipy_dnrm2_(int *, double *, int *);
extern zc scipy_zdotc_(int *, zc *, int *, zc *, int *);
extern zc scipy_zdotu_(int *, zc *, int *, zc *, int *);
extern void scipy_zscal_(int *, zc *, zc *, int *);
extern void scipy_zdscal_(int *, double *, zc *, int *);
extern void scipy_dcopy_(int *, double *, int *, double *, int *);
extern void scipy_zcopy_(int *, zc *, int *, zc *, int *);
extern void scipy_zaxpy_(int *, zc *, zc *, int *, zc *, int *);
extern void scipy_zgemv_(char *, int *, int *, zc *, zc *, int *, zc *, int *, zc *, zc *, int *,
                         size_t);
extern void scipy_dgemv_(char *, int *, int *, double *, double *, int *, double *, int *,
                         double *, double *, int *, size_t);
extern void scipy_zgemm_(char *, char *, int *, int *, int *, zc *, zc *, int *, zc *, int *, zc *,
                         zc *, int *, size_t, size_t);
extern void scipy_ztrsm_(char *, char *, char *, char *, int *, int *, zc *, zc *, int *, zc *,
                         int *, size_t, size_t, size_t, size_t);
extern void scipy_zheevd_(char *, char *, int *, zc *, int *, double *, zc *, int *, double *,
                          int *, int *, int *, int *, size_t, size_t);
extern void scipy_zgeqrf_(int *, int *, zc *, int *, zc *, zc *, int *, int *);
extern void scipy_zungqr_(int *, int *, int *, zc *, int *, zc *, zc *, int *, int *);
extern void scipy_zpotrf_(char *, int *, zc *, int *, int *, size_t);
extern void scipy_dgetrf_(int *, int *, double *, int *, int *, int *);
extern void scipy_dgetri_(int *, double *, int *, int *, double *, int *, int *);
extern void scipy_dsysv_(char *, int *, int *, double *, int *, int *, double *, int *, double *,
                         int *, int *, size_t);
extern void scipy_dgeev_(char *, char *, int *, double *, int *, double *, double *, double *,
                         int *, double *, int *, double *, int *, int *, size_t, size_t);
extern void scipy_dsyev_(char *, char *, int *, double *, int *, double *, double *, int *, int *,
                         size_t, size_t);

double ddot_(int *n, double *x, int *incx, double *y, int *incy) {
  return scipy_ddot_(n, x, incx, y, incy);
}
double dnrm2_(int *n, double *x, int *incx) { return scipy_dnrm2_(n, x, incx); }
void zdotc_(zc *pres, int *n, zc *x, int *incx, zc *y, int *incy) {
  *pres = scipy_zdotc_(n, x, incx, y, incy);
}
void zdotu_(zc *pres, int *n, zc *x, int *incx, zc *y, int *incy) {
  *pres = scipy_zdotu_(n, x, incx, y, incy);
}
void zscal_(int *n, zc *a, zc *x, int *incx) { scipy_zscal_(n, a, x, incx); }
void zdscal_(int *n, double *a, zc *x, int *incx) { scipy_zdscal_(n, a, x, incx); }
void dcopy_(int *n, double *x, int *incx, double *y, int *incy) {
  scipy_dcopy_(n, x, incx, y, incy);
}
void zcopy_(int *n, zc *x, int *incx, zc *y, int *incy) { scipy_zcopy_(n, x, incx, y, incy); }
void zaxpy_(int *n, zc *a, zc *x, int *incx, zc *y, int *incy) {
  scipy_zaxpy_(n, a, x, incx, y, incy);
}
void zgemv_(char *t, int *m, int *n, zc *al, zc *a, int *lda, zc *x, int *incx, zc *be, zc *y,
            int *incy) {
  scipy_zgemv_(t, m, n, al, a, lda, x, incx, be, y, incy, 1);
}
void dgemv_(char *t, int *m, int *n, double *al, double *a, int *lda, double *x, int *incx,
            double *be, double *y, int *incy) {
  scipy_dgemv_(t, m, n, al, a, lda, x, incx, be, y, incy, 1);
}
void zgemm_(char *ta, char *tb, int *m, int *n, int *k, zc *al, zc *a, int *lda, zc *b, int *ldb,
            zc *be, zc *c, int *ldc) {
  scipy_zgemm_(ta, tb, m, n, k, al, a, lda, b, ldb, be, c, ldc, 1, 1);
}
void ztrsm_(char *side, char *uplo, char *ta, char *diag, int *m, int *n, zc *al, zc *a, int *lda,
            zc *b, int *ldb) {
  scipy_ztrsm_(side, uplo, ta, diag, m, n, al, a, lda, b, ldb, 1, 1, 1, 1);
}
void zheevd_(char *jobz, char *uplo, int *n, zc *a, int *lda, double *w, zc *work, int *lwork,
             double *rwork, int *lrwork, int *iwork, int *liwork, int *info) {
  scipy_zheevd_(jobz, uplo, n, a, lda, w, work, lwork, rwork, lrwork, iwork, liwork, info, 1, 1);
}
void zgeqrf_(int *m, int *n, zc *a, int *lda, zc *tau, zc *work, int *lwork, int *info) {
  scipy_zgeqrf_(m, n, a, lda, tau, work, lwork, info);
}
void zungqr_(int *m, int *n, int *k, zc *a, int *lda, zc *tau, zc *work, int *lwork, int *info) {
  scipy_zungqr_(m, n, k, a, lda, tau, work, lwork, info);
}
void zpotrf_(char *uplo, int *n, zc *a, int *lda, int *info) {
  scipy_zpotrf_(uplo, n, a, lda, info, 1);
}
void dgetrf_(int *m, int *n, double *a, int *lda, int *ipiv, int *info) {
  scipy_dgetrf_(m, n, a, lda, ipiv, info);
}
void dgetri_(int *n, double *a, int *lda, int *ipiv, double *work, int *lwork, int *info) {
  scipy_dgetri_(n, a, lda, ipiv, work, lwork, info);
}
void dsysv_(char *uplo, int *n, int *nrhs, double *a, int *lda, int *ipiv, double *b, int *ldb,
            double *work, int *lwork, int *info) {
  scipy_dsysv_(uplo, n, nrhs, a, lda, ipiv, b, ldb, work, lwork, info, 1);
}
void dgeev_(char *jobvl, char *jobvr, int *n, double *a, int *lda, double *wr, double *wi,
            double *vl, int *ldvl, double *vr, int *ldvr, double *work, int *lwork, int *info) {
  scipy_dgeev_(jobvl, jobvr, n, a, lda, wr, wi, vl, ldvl, vr, ldvr, work, lwork, info, 1, 1);
}
void dsyev_(char *jobz, char *uplo, int *n, double *a, int *lda, double *w, double *work,
            int *lwork, int *info) {
  scipy_dsyev_(jobz, uplo, n, a, lda, w, work, lwork, info, 1, 1);
}
