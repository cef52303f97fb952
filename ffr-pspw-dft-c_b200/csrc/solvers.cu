// Device-resident eigensolvers and their C ABI: block Davidson
// (davidson_cpu.cpp:9-266), LOBPCG (lobpcg_cpu.cpp:31-395), Lanczos
// (lanczos.cpp:8-101), plus ortho_qr, eig_zheevd, eig_zhegv(_eval), GenPrec
// and random_col.
//
// Every block (X, HX, residuals, Q, HQ) stays on the device in FP64; the
// reduced matrices are formed by the engine's GEMMs and diagonalised by
// cuSOLVER on the device.  The host only sees the per-iteration residual
// norms it needs for the reference's convergence tests.  H*psi inside the
// solvers runs in FP64, or in FP32 (`hprec`) with the block converted on the
// way in and out -- the mixed form where orthonormalisation and the subspace
// eigensolve stay FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "dense.h"
#include "engine.h"
#include "gemm.h"
#include "solvers.h"

namespace pspw {

namespace {

const double2 kOne = {1.0, 0.0}, kZero = {0.0, 0.0}, kMOne = {-1.0, 0.0};

__global__ void k_z2c(const double2 *__restrict__ a, float2 *__restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = make_float2((float)a[i].x, (float)a[i].y);
}
__global__ void k_c2z(const float2 *__restrict__ a, double2 *__restrict__ b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = make_double2((double)a[i].x, (double)a[i].y);
}

// GenPrec.cpp:5-24, with the reference's operation order (no contraction)
__global__ void k_gen_prec(const double *__restrict__ xkg, double tpiba2, int n, double tau,
                           double *prec) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    if (tau <= 0.0) {
      const double x = __dmul_rn(xkg[i], tpiba2);
      const double y =
          __dadd_rn(27.0, __dmul_rn(x, __dadd_rn(18.0, __dmul_rn(x, __dadd_rn(12.0, __dmul_rn(8.0, x))))));
      const double x4 = __dmul_rn(__dmul_rn(__dmul_rn(x, x), x), x);
      prec[i] = __ddiv_rn(y, __dadd_rn(y, __dmul_rn(16.0, x4)));
    } else {
      prec[i] = __ddiv_rn(tau, __dmul_rn(__dmul_rn(0.5, __dadd_rn(xkg[i], 1.0)), tpiba2));
    }
  }
}

// Lanczos helpers: T(j, j-1) = sqrt(nf); V_j = f / sqrt(nf)
__global__ void k_lanczos_next(const double2 *__restrict__ f, double2 *__restrict__ vj, int n,
                               const double *__restrict__ nf, double *T, int ldT, int j) {
  const double s = sqrt(nf[0]);
  if (j > 0 && blockIdx.x == 0 && threadIdx.x == 0) T[(size_t)(j - 1) * ldT + j] = s;
  const double beta = 1.0 / s;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    vj[i] = make_double2(beta * f[i].x, beta * f[i].y);
}
// y += x
__global__ void k_axpy1(const double2 *__restrict__ x, double2 *y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    y[i] = make_double2(y[i].x + x[i].x, y[i].y + x[i].y);
}
// f = x - V h over the nj columns of V (lanczos.cpp:60-70): one thread per
// row, the columns summed in order
__global__ void k_lz_sub(int n, int nj, const double2 *__restrict__ V, int ldv,
                         const double2 *__restrict__ h, const double2 *__restrict__ x,
                         double2 *__restrict__ f) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double2 t = make_double2(0.0, 0.0);
    for (int q = 0; q < nj; q++) cfma(t, V[(size_t)q * ldv + i], h[q]);
    f[i] = make_double2(x[i].x - t.x, x[i].y - t.y);
  }
}
// The end of Lanczos step j (lanczos.cpp:72-91): f -= V s, and (block 0)
// h += s with column j of T = Re h, taken before the correction for the
// first column (:36-38) and after it for the others (:89-91)
__global__ void k_lz_update(int n, int nj, const double2 *__restrict__ V, int ldv, double2 *h,
                            const double2 *__restrict__ s, double2 *f, double *T, int ldT,
                            int j) {
  if (blockIdx.x == 0)
    for (int i = threadIdx.x; i < nj; i += blockDim.x) {
      double2 hv = h[i];
      if (j == 0) T[(size_t)j * ldT + i] = hv.x;
      hv = make_double2(hv.x + s[i].x, hv.y + s[i].y);
      h[i] = hv;
      if (j > 0) T[(size_t)j * ldT + i] = hv.x;
    }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double2 t = make_double2(0.0, 0.0);
    for (int q = 0; q < nj; q++) cfma(t, V[(size_t)q * ldv + i], s[q]);
    f[i] = make_double2(f[i].x - t.x, f[i].y - t.y);
  }
}

inline int gridn(size_t n) { return (int)std::min<size_t>(4 * 148, (n + 255) / 256 + 1); }

int block(pspw_cell *c, int slot, size_t elems, double2 **p) {
  return ws_reserve(c, kWsSolverBase + slot, sizeof(double2) * std::max<size_t>(1, elems),
                    (void **)p);
}
int dblock(pspw_cell *c, int slot, size_t elems, double **p) {
  return ws_reserve(c, kWsSolverBase + slot, sizeof(double) * std::max<size_t>(1, elems),
                    (void **)p);
}

// HX = H X for a device FP64 block (m x n, ld m), FP64 or FP32 arithmetic.
int apply_h(pspw_cell *c, int hprec, const double2 *X, double2 *HX, int m, int n) {
  if (hprec == PSPW_PREC_F64)
    return hpsi_apply<double>(c, X, m, HX, m, m, n, 1.0, 0.0, 0.0, nullptr, m);
  float2 *xf = nullptr, *hf = nullptr;
  int rc;
  if ((rc = ws_reserve(c, kWsConv, sizeof(float2) * (size_t)m * n, (void **)&xf)) ||
      (rc = ws_reserve(c, kWsSolverBase + 15, sizeof(float2) * (size_t)m * n, (void **)&hf)))
    return rc;
  k_z2c<<<gridn((size_t)m * n), 256, 0, c->stream>>>(X, xf, (size_t)m * n);
  if ((rc = hpsi_apply<float>(c, xf, m, hf, m, m, n, 1.0, 0.0, 0.0, nullptr, m))) return rc;
  k_c2z<<<gridn((size_t)m * n), 256, 0, c->stream>>>(hf, HX, (size_t)m * n);
  c->kernel_launches += 2;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int d2h(pspw_cell *c, void *dst, const void *src, size_t bytes) {
  PSPW_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, c->stream));
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  return device_status(c);
}
int h2d(pspw_cell *c, void *dst, const void *src, size_t bytes) {
  PSPW_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, c->stream));
  return PSPW_OK;
}
int d2d(pspw_cell *c, void *dst, const void *src, size_t bytes) {
  PSPW_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c->stream));
  return PSPW_OK;
}

void random_start(std::vector<double2> &X, int nbasis, int nstates) {
  X.resize((size_t)nbasis * nstates);
  for (int ist = 0; ist < nstates; ist++) random_col_host(&X[(size_t)ist * nbasis], nbasis, 100 + ist);
}

int default_maxiter(int nstates, int max_iter) {
  if (max_iter > 0) return max_iter;
  return std::max(30, nstates / 2);
}

}  // namespace

// util_random_cpu.cpp:5-23: state a <- ((a*214013 + 2531011) >> 16) & 32767;
// each value is ((a mod 100) + 1) / a with the updated state, real then
// imaginary part.
void random_col_host(double2 *A, int nelem, long seed) {
  long a = seed;
  for (int i = 0; i < nelem; i++) {
    a = (((a * 214013L + 2531011L) >> 16) & 32767);
    const double re = (double)((a % 100) + 1) / (double)a;
    a = (((a * 214013L + 2531011L) >> 16) & 32767);
    const double im = (double)((a % 100) + 1) / (double)a;
    A[i] = make_double2(re, im);
  }
}

int gen_prec_dev(pspw_cell *c, double *d_prec, int nbasis, double tau) {
  if (nbasis > c->basis.ngw) return fail(PSPW_ERR_SHAPE, "GenPrec: nbasis exceeds the cell");
  k_gen_prec<<<gridn(nbasis), 256, 0, c->stream>>>(c->basis.d_xkg64, c->tpiba2, nbasis, tau, d_prec);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

// ------------------------------------------------------------ Davidson
int davidson_dev(pspw_cell *c, int hprec, double *evals_host, double2 *X, int nbasis, int nstates,
                 const double *d_prec, int nempty, int max_iter, double *res_host, int *iters) {
  const int nb = nstates, n2 = 2 * nstates;
  const size_t blk = (size_t)nbasis * nb;
  double2 *HX, *R, *HR, *Xt, *h, *o, *ev;
  double *evals, *evals_red, *rnorm_d, *dots;
  int rc;
  if ((rc = block(c, 0, blk, &HX)) || (rc = block(c, 1, blk, &R)) || (rc = block(c, 2, blk, &HR)) ||
      (rc = block(c, 3, blk, &Xt)) || (rc = block(c, 4, (size_t)n2 * n2, &h)) ||
      (rc = block(c, 5, (size_t)n2 * n2, &o)) || (rc = block(c, 6, (size_t)n2 * n2, &ev)) ||
      (rc = dblock(c, 7, nb, &evals)) || (rc = dblock(c, 8, n2, &evals_red)) ||
      (rc = dblock(c, 9, nb, &rnorm_d)) || (rc = dblock(c, 10, nb, &dots)))
    return rc;
  // random start (davidson_cpu.cpp:47-51) and orthonormalisation (:53)
  std::vector<double2> X0;
  random_start(X0, nbasis, nb);
  if ((rc = h2d(c, X, X0.data(), sizeof(double2) * blk))) return rc;
  int info = 0;
  if ((rc = dev_ortho_qr(c, X, nbasis, nbasis, nb, &info))) return rc;
  if (info) return fail(PSPW_ERR_LAPACK, "zgeqrf/zungqr: info = " + std::to_string(info));
  if ((rc = apply_h(c, hprec, X, HX, nbasis, nb))) return rc;                   // :56
  if ((rc = dev_coldot(c, X, nbasis, HX, nbasis, nbasis, nb, evals))) return rc;  // :59-62
  if ((rc = dev_residual(c, evals, X, nbasis, HX, nbasis, R, nbasis, nbasis, nb))) return rc;
  std::vector<double> res(nb), rn(nb);
  auto residual_norms = [&]() -> int {
    int r = dev_coldot(c, R, nbasis, R, nbasis, nbasis, nb, dots);
    if (r) return r;
    if ((r = d2h(c, res.data(), dots, sizeof(double) * nb))) return r;
    for (auto &v : res) v = std::sqrt(v);
    return PSPW_OK;
  };
  if ((rc = residual_norms())) return rc;
  const int max_dir = default_maxiter(nb, max_iter);
  const double machine_zero = 2.220446049250313e-16, TOL = 1.0e-6;
  int istep = 0;
  for (istep = 1; istep <= max_dir; istep++) {
    for (int i = 0; i < nb; i++) rn[i] = res[i] > machine_zero ? 1.0 / res[i] : 1.0;  // :89-93
    if ((rc = h2d(c, rnorm_d, rn.data(), sizeof(double) * nb))) return rc;
    if ((rc = dev_scale_prec(c, rnorm_d, d_prec, R, nbasis, nbasis, nb))) return rc;  // :96-105
    if ((rc = apply_h(c, hprec, R, HR, nbasis, nb))) return rc;                       // :118
    // reduced Hamiltonian (:120-147) and overlap (:160-178)
    if (istep == 1)
      rc = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, X, nbasis, HX, nbasis, kZero, h, n2);
    else
      rc = dev_diag(c, h, n2, nb, evals);
    if (rc) return rc;
    if ((rc = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, X, nbasis, HR, nbasis, kZero,
                            h + (size_t)nb * n2, n2)) ||
        (rc = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, HR, nbasis, X, nbasis, kZero, h + nb, n2)) ||
        (rc = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, R, nbasis, HR, nbasis, kZero,
                            h + (size_t)nb * n2 + nb, n2)) ||
        (rc = dev_diag(c, o, n2, nb, nullptr)) ||
        (rc = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, X, nbasis, R, nbasis, kZero,
                            o + (size_t)nb * n2, n2)) ||
        (rc = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, R, nbasis, X, nbasis, kZero, o + nb, n2)) ||
        (rc = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, R, nbasis, R, nbasis, kZero,
                            o + (size_t)nb * n2 + nb, n2)))
      return rc;
    if ((rc = dev_zhegv(c, h, n2, o, n2, evals_red, ev, n2, n2, nullptr))) return rc;  // :181
    if ((rc = d2d(c, evals, evals_red, sizeof(double) * nb))) return rc;             // :184
    // X = X c1 + R c2, HX = HX c1 + HR c2 (:189-207)
    if ((rc = zgemm<double>(c, 'N', nbasis, nb, nb, kOne, X, nbasis, ev, n2, kZero, Xt, nbasis)) ||
        (rc = d2d(c, X, Xt, sizeof(double2) * blk)) ||
        (rc = zgemm<double>(c, 'N', nbasis, nb, nb, kOne, HX, nbasis, ev, n2, kZero, Xt, nbasis)) ||
        (rc = d2d(c, HX, Xt, sizeof(double2) * blk)) ||
        (rc = zgemm<double>(c, 'N', nbasis, nb, nb, kOne, R, nbasis, ev + nb, n2, kOne, X, nbasis)) ||
        (rc = zgemm<double>(c, 'N', nbasis, nb, nb, kOne, HR, nbasis, ev + nb, n2, kOne, HX, nbasis)))
      return rc;
    if ((rc = dev_residual(c, evals, X, nbasis, HX, nbasis, R, nbasis, nbasis, nb))) return rc;
    if ((rc = residual_norms())) return rc;
    int nconv = 0;
    double rnorm = 0.0;
    for (int i = 0; i < nb; i++) {
      nconv += res[i] < TOL;
      rnorm += res[i];
    }
    if (nconv >= nb - nempty) break;   // :224-227
    if (rnorm / nb < TOL / 10.0) break;  // :229-238
  }
  if (iters) *iters = std::min(istep, max_dir);
  if (res_host) std::copy(res.begin(), res.end(), res_host);
  return d2h(c, evals_host, evals, sizeof(double) * nb);
}

// ------------------------------------------------------------ LOBPCG
int lobpcg_dev(pspw_cell *c, int hprec, double *lambda_host, double2 *X, int nbasis, int nstates,
               const double *d_prec, int nempty, int max_iter, double *res_host, int *iters) {
  const int nb = nstates, n2 = 2 * nb, n3 = 3 * nb;
  const size_t blk = (size_t)nbasis * nb;
  double2 *Q, *HQ, *t1, *T, *G, *U, *tX;
  double *lam, *dots;
  int rc;
  if ((rc = block(c, 0, (size_t)nbasis * n3, &Q)) || (rc = block(c, 1, (size_t)nbasis * n3, &HQ)) ||
      (rc = block(c, 2, (size_t)nb * nb, &t1)) || (rc = block(c, 3, (size_t)n3 * n3, &T)) ||
      (rc = block(c, 4, (size_t)n3 * n3, &G)) || (rc = block(c, 5, (size_t)n3 * n3, &U)) ||
      (rc = block(c, 6, blk, &tX)) || (rc = dblock(c, 7, nb, &lam)) || (rc = dblock(c, 8, nb, &dots)))
    return rc;
  double2 *Xq = Q, *W = Q + blk, *P = Q + 2 * blk;
  double2 *HXq = HQ, *HW = HQ + blk, *HP = HQ + 2 * blk;
  std::vector<double2> X0;
  random_start(X0, nbasis, nb);  // :82-86
  if ((rc = h2d(c, Xq, X0.data(), sizeof(double2) * blk))) return rc;
  int info = 0;
  if ((rc = dev_ortho_qr(c, Xq, nbasis, nbasis, nb, &info))) return rc;  // :90
  if (info) return fail(PSPW_ERR_LAPACK, "zgeqrf/zungqr: info = " + std::to_string(info));
  if ((rc = apply_h(c, hprec, Xq, HXq, nbasis, nb))) return rc;  // :95
  std::vector<double> res(nb);
  const int maxiter = default_maxiter(nb, max_iter);
  const double TOL = 1.0e-6;
  // residuals W = HX - X (X^H HX), lambda = eig(X^H HX); true = converged
  auto check = [&](bool *done) -> int {
    int r;
    if ((r = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, Xq, nbasis, HXq, nbasis, kZero, t1, nb)) ||
        (r = d2d(c, W, HXq, sizeof(double2) * blk)) ||
        (r = zgemm<double>(c, 'N', nbasis, nb, nb, kMOne, Xq, nbasis, t1, nb, kOne, W, nbasis)))
      return r;
    int inf = 0;
    if ((r = dev_zheevd(c, t1, nb, lam, nb, &inf))) return r;
    if (inf) return fail(PSPW_ERR_LAPACK, "zheevd: info = " + std::to_string(inf));
    if ((r = dev_coldot(c, W, nbasis, W, nbasis, nbasis, nb, dots))) return r;
    if ((r = d2h(c, res.data(), dots, sizeof(double) * nb))) return r;
    int nconv = 0;
    double rn = 0.0;
    for (auto &v : res) {
      v = std::sqrt(v);
      nconv += v < TOL;
      rn += v;
    }
    *done = (nconv >= nb - nempty) || (rn / nb < TOL);
    return PSPW_OK;
  };
  // Cholesky orthonormalisation of a block and its H image (:153-180)
  auto chol = [&](double2 *Y, double2 *HY) -> int {
    int r;
    if ((r = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, Y, nbasis, Y, nbasis, kZero, t1, nb)) ||
        (r = dev_symmetrize(c, t1, nb, nb)))
      return r;
    int inf = 0;
    if ((r = dev_potrf_upper(c, t1, nb, nb, &inf))) return r;
    if (inf) return fail(PSPW_ERR_LAPACK, "ERROR calculating Cholesky decomposition");
    if ((r = dev_trsm_right_upper(c, t1, nb, Y, nbasis, nbasis, nb)) ||
        (r = dev_trsm_right_upper(c, t1, nb, HY, nbasis, nbasis, nb)))
      return r;
    return PSPW_OK;
  };
  int iter = 1;
  bool done = false;
  for (;;) {
    if ((rc = check(&done))) return rc;
    if (done) break;
    if ((rc = dev_scale_prec(c, nullptr, d_prec, W, nbasis, nbasis, nb))) return rc;  // :142-146
    if ((rc = apply_h(c, hprec, W, HW, nbasis, nb))) return rc;                        // :149
    if ((rc = chol(W, HW))) return rc;
    const int nq = (iter == 1) ? n2 : n3;  // first iteration without P (:183-196)
    if ((rc = zgemm<double>(c, 'C', nq, nq, nbasis, kOne, Q, nbasis, HQ, nbasis, kZero, T, n3)) ||
        (rc = dev_symmetrize(c, T, n3, nq)) ||
        (rc = zgemm<double>(c, 'C', nq, nq, nbasis, kOne, Q, nbasis, Q, nbasis, kZero, G, n3)) ||
        (rc = dev_symmetrize(c, G, n3, nq)) ||
        (rc = dev_zhegv(c, T, n3, G, n3, nullptr, U, n3, nq, nullptr)))
      return rc;
    // X = Q U(:, 0:nb), HX = HQ U(:, 0:nb)
    if ((rc = zgemm<double>(c, 'N', nbasis, nb, nq, kOne, Q, nbasis, U, n3, kZero, tX, nbasis)) ||
        (rc = d2d(c, Xq, tX, sizeof(double2) * blk)) ||
        (rc = zgemm<double>(c, 'N', nbasis, nb, nq, kOne, HQ, nbasis, U, n3, kZero, tX, nbasis)) ||
        (rc = d2d(c, HXq, tX, sizeof(double2) * blk)))
      return rc;
    if (iter == 1) {
      if ((rc = d2d(c, P, W, sizeof(double2) * blk)) || (rc = d2d(c, HP, HW, sizeof(double2) * blk)))
        return rc;
    } else {
      // P = W U(nb:2nb, :) + P U(2nb:3nb, :), same for HP (:328-345), then
      // Cholesky-orthonormalise P and HP (:348-370)
      if ((rc = zgemm<double>(c, 'N', nbasis, nb, nb, kOne, P, nbasis, U + 2 * nb, n3, kZero, tX,
                              nbasis)) ||
          (rc = zgemm<double>(c, 'N', nbasis, nb, nb, kOne, W, nbasis, U + nb, n3, kZero, P, nbasis)))
        return rc;
      k_axpy1<<<gridn(blk), 256, 0, c->stream>>>(tX, P, blk);
      if ((rc = zgemm<double>(c, 'N', nbasis, nb, nb, kOne, HP, nbasis, U + 2 * nb, n3, kZero, tX,
                              nbasis)) ||
          (rc = zgemm<double>(c, 'N', nbasis, nb, nb, kOne, HW, nbasis, U + nb, n3, kZero, HP, nbasis)))
        return rc;
      k_axpy1<<<gridn(blk), 256, 0, c->stream>>>(tX, HP, blk);
      c->kernel_launches += 2;
      if ((rc = chol(P, HP))) return rc;
    }
    iter++;
    if (iter > maxiter) break;
  }
  if (iters) *iters = iter;
  if (res_host) std::copy(res.begin(), res.end(), res_host);
  if ((rc = d2d(c, X, Xq, sizeof(double2) * blk))) return rc;
  return d2h(c, lambda_host, lam, sizeof(double) * nb);
}

// ------------------------------------------------------------ Lanczos
// LOBPCG with an orthonormal search basis (an opt-in alternative to the
// reference's lobpcg_cpu; no counterpart in the reference).  The reference
// orthonormalises W and P each on its own, so near convergence the overlap
// of [X W P] becomes nearly singular and eig_zhegv (which scales overlap
// directions by 1/sqrt(eigenvalue) down to 1.2e-15) amplifies rounding.
// Here W and P are made orthogonal to X (and W to P) by two block
// projections and then orthonormalised (Cholesky QR, Householder QR when
// the Cholesky factorisation fails), so [X W P] is orthonormal and the
// Rayleigh-Ritz step is a standard Hermitian eigenproblem; P is the
// component of the new Ritz vectors along [W P] (Hetmaniuk and Lehoucq,
// "Basis selection in LOBPCG", J. Comput. Phys. 218 (2006) 324-332;
// Knyazev, SIAM J. Sci. Comput. 23 (2001) 517-541).  Same random start,
// preconditioner and convergence test as the reference (lobpcg_cpu.cpp:82-86,
// 142-146, 239-262).
int lobpcg_ortho_dev(pspw_cell *c, int hprec, double *lambda_host, double2 *X, int nbasis,
                     int nstates, const double *d_prec, int nempty, int max_iter, double *res_host,
                     int *iters, bool from_x) {
  const int nb = nstates, n3 = 3 * nb;
  const size_t blk = (size_t)nbasis * nb;
  double2 *Q, *HQ, *t1, *T, *tX, *tH, *tY;
  double *lam, *lam3, *dots;
  int rc;
  if ((rc = block(c, 0, (size_t)nbasis * n3, &Q)) || (rc = block(c, 1, (size_t)nbasis * n3, &HQ)) ||
      (rc = block(c, 2, (size_t)nb * nb, &t1)) || (rc = block(c, 3, (size_t)n3 * n3, &T)) ||
      (rc = block(c, 6, blk, &tX)) || (rc = block(c, 9, blk, &tH)) || (rc = block(c, 11, blk, &tY)) ||
      (rc = dblock(c, 7, nb, &lam)) || (rc = dblock(c, 8, nb, &dots)) ||
      (rc = dblock(c, 10, n3, &lam3)))
    return rc;
  double2 *Xq = Q, *W = Q + blk, *P = Q + 2 * blk;
  double2 *HXq = HQ, *HW = HQ + blk, *HP = HQ + 2 * blk;
  if (from_x) {  // the caller's start block
    if ((rc = d2d(c, Xq, X, sizeof(double2) * blk))) return rc;
  } else {
    std::vector<double2> X0;
    random_start(X0, nbasis, nb);
    if ((rc = h2d(c, Xq, X0.data(), sizeof(double2) * blk))) return rc;
  }
  int info = 0;
  if ((rc = dev_ortho_qr(c, Xq, nbasis, nbasis, nb, &info))) return rc;
  if (info) return fail(PSPW_ERR_LAPACK, "zgeqrf/zungqr: info = " + std::to_string(info));
  if ((rc = apply_h(c, hprec, Xq, HXq, nbasis, nb))) return rc;
  // Y -= B (B^H Y) and HY -= HB (B^H Y)
  auto project_out = [&](double2 *Y, double2 *HY, const double2 *Bm, const double2 *HB) -> int {
    int r;
    if ((r = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, Bm, nbasis, Y, nbasis, kZero, t1, nb)) ||
        (r = zgemm<double>(c, 'N', nbasis, nb, nb, kMOne, Bm, nbasis, t1, nb, kOne, Y, nbasis)))
      return r;
    if (HY && (r = zgemm<double>(c, 'N', nbasis, nb, nb, kMOne, HB, nbasis, t1, nb, kOne, HY,
                                 nbasis)))
      return r;
    return PSPW_OK;
  };
  // orthonormalise Y (and its H image HY, when given) by Cholesky QR;
  // *ok = false when the Gram matrix is not positive definite
  auto cholqr = [&](double2 *Y, double2 *HY, bool *ok) -> int {
    int r;
    if ((r = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, Y, nbasis, Y, nbasis, kZero, t1, nb)) ||
        (r = dev_symmetrize(c, t1, nb, nb)))
      return r;
    int inf = 0;
    if ((r = dev_potrf_upper(c, t1, nb, nb, &inf))) return r;
    *ok = inf == 0;
    if (!*ok) return PSPW_OK;
    if ((r = dev_trsm_right_upper(c, t1, nb, Y, nbasis, nbasis, nb))) return r;
    if (HY && (r = dev_trsm_right_upper(c, t1, nb, HY, nbasis, nbasis, nb))) return r;
    return PSPW_OK;
  };
  std::vector<double> res(nb);
  const int maxiter = default_maxiter(nb, max_iter);
  const double TOL = 1.0e-6;
  bool have_p = false;
  int iter = 1;
  for (;;) {
    // Rayleigh-Ritz on the current basis: X orthonormal, T = X^H HX
    // (first pass), then residuals W = HX - X diag(lambda)
    if (iter == 1) {
      if ((rc = zgemm<double>(c, 'C', nb, nb, nbasis, kOne, Xq, nbasis, HXq, nbasis, kZero, t1,
                              nb)) ||
          (rc = dev_symmetrize(c, t1, nb, nb)) || (rc = dev_zheevd(c, t1, nb, lam, nb, &info)))
        return rc;
      if (info) return fail(PSPW_ERR_LAPACK, "zheevd: info = " + std::to_string(info));
      if ((rc = zgemm<double>(c, 'N', nbasis, nb, nb, kOne, Xq, nbasis, t1, nb, kZero, tX,
                              nbasis)) ||
          (rc = d2d(c, Xq, tX, sizeof(double2) * blk)) ||
          (rc = zgemm<double>(c, 'N', nbasis, nb, nb, kOne, HXq, nbasis, t1, nb, kZero, tX,
                              nbasis)) ||
          (rc = d2d(c, HXq, tX, sizeof(double2) * blk)))
        return rc;
    }
    if ((rc = dev_residual(c, lam, Xq, nbasis, HXq, nbasis, W, nbasis, nbasis, nb)) ||
        (rc = dev_coldot(c, W, nbasis, W, nbasis, nbasis, nb, dots)) ||
        (rc = d2h(c, res.data(), dots, sizeof(double) * nb)))
      return rc;
    int nconv = 0;
    double rn = 0.0;
    for (auto &v : res) {
      v = std::sqrt(v);
      nconv += v < TOL;
      rn += v;
    }
    if ((nconv >= nb - nempty) || (rn / nb < TOL)) break;
    if (iter > maxiter) break;
    // W = prec (X lambda - HX), orthogonal to X and P, orthonormal
    if ((rc = dev_scale_prec(c, nullptr, d_prec, W, nbasis, nbasis, nb))) return rc;
    for (int pass = 0; pass < 2; pass++) {
      if ((rc = project_out(W, nullptr, Xq, nullptr))) return rc;
      if (have_p && (rc = project_out(W, nullptr, P, nullptr))) return rc;
    }
    bool ok = false;
    if ((rc = cholqr(W, nullptr, &ok))) return rc;
    if (!ok) {
      if ((rc = dev_ortho_qr(c, W, nbasis, nbasis, nb, &info))) return rc;
      if (info) return fail(PSPW_ERR_LAPACK, "zgeqrf/zungqr: info = " + std::to_string(info));
    }
    if ((rc = apply_h(c, hprec, W, HW, nbasis, nb))) return rc;
    // standard Rayleigh-Ritz on the orthonormal [X W P]
    const int nq = have_p ? n3 : 2 * nb;
    if ((rc = zgemm<double>(c, 'C', nq, nq, nbasis, kOne, Q, nbasis, HQ, nbasis, kZero, T, n3)) ||
        (rc = dev_symmetrize(c, T, n3, nq)) || (rc = dev_zheevd(c, T, n3, lam3, nq, &info)))
      return rc;
    if (info) return fail(PSPW_ERR_LAPACK, "zheevd: info = " + std::to_string(info));
    if ((rc = d2d(c, lam, lam3, sizeof(double) * nb))) return rc;
    // P = [W P] U(nb:, 0:nb), HP likewise (before X is overwritten)
    if ((rc = zgemm<double>(c, 'N', nbasis, nb, nq - nb, kOne, W, nbasis, T + nb, n3, kZero, tX,
                            nbasis)) ||
        (rc = zgemm<double>(c, 'N', nbasis, nb, nq - nb, kOne, HW, nbasis, T + nb, n3, kZero, tH,
                            nbasis)))
      return rc;
    // X = Q U(:, 0:nb), HX = HQ U(:, 0:nb)
    if ((rc = zgemm<double>(c, 'N', nbasis, nb, nq, kOne, Q, nbasis, T, n3, kZero, tY, nbasis)) ||
        (rc = d2d(c, Xq, tY, sizeof(double2) * blk)) ||
        (rc = zgemm<double>(c, 'N', nbasis, nb, nq, kOne, HQ, nbasis, T, n3, kZero, tY, nbasis)) ||
        (rc = d2d(c, HXq, tY, sizeof(double2) * blk)) ||
        (rc = d2d(c, P, tX, sizeof(double2) * blk)) || (rc = d2d(c, HP, tH, sizeof(double2) * blk)))
      return rc;
    // P orthogonal to the new X, orthonormal; dropped when that fails
    for (int pass = 0; pass < 2; pass++)
      if ((rc = project_out(P, HP, Xq, HXq))) return rc;
    if ((rc = cholqr(P, HP, &ok))) return rc;
    have_p = ok;
    iter++;
  }
  if (iters) *iters = iter;
  if (res_host) std::copy(res.begin(), res.end(), res_host);
  if ((rc = d2d(c, X, Xq, sizeof(double2) * blk))) return rc;
  return d2h(c, lambda_host, lam, sizeof(double) * nb);
}

int lanczos_dev(pspw_cell *c, double2 *v0, int ngw, int k, double *T_host, int ldT, double2 *f_out,
                int hprec) {
  double2 *V, *Hv, *f, *h, *s, *ns;
  double *T, *nf;
  int rc;
  if ((rc = block(c, 0, (size_t)ngw * k, &V)) || (rc = block(c, 1, ngw, &Hv)) ||
      (rc = block(c, 2, ngw, &f)) || (rc = block(c, 3, k, &h)) || (rc = block(c, 4, k, &s)) ||
      (rc = block(c, 5, k, &ns)) || (rc = dblock(c, 6, (size_t)k * k, &T)) ||
      (rc = dblock(c, 7, 4, &nf)))
    return rc;
  PSPW_CUDA(cudaMemsetAsync(T, 0, sizeof(double) * (size_t)k * k, c->stream));
  // v0 /= ||v0|| (lanczos.cpp:24-26); V(:,1) = v0
  if ((rc = dev_coldot(c, v0, ngw, v0, ngw, ngw, 1, nf))) return rc;
  k_lanczos_next<<<gridn(ngw), 256, 0, c->stream>>>(v0, v0, ngw, nf, T, k, 0);
  if ((rc = d2d(c, V, v0, sizeof(double2) * ngw))) return rc;
  for (int j = 0; j < k; j++) {
    double2 *vj = V + (size_t)j * ngw;
    if (j > 0) {
      // T(j, j-1) = ||f||, V(:,j) = f/||f|| (:53-58)
      if ((rc = dev_coldot(c, f, ngw, f, ngw, ngw, 1, nf))) return rc;
      k_lanczos_next<<<gridn(ngw), 256, 0, c->stream>>>(f, vj, ngw, nf, T, k, j);
      c->kernel_launches++;
    }
    if ((rc = apply_h(c, hprec, vj, Hv, ngw, 1))) return rc;
    // h = V^H Hv; f = Hv - V h; s = V^H f; h += s; f -= V s (:60-87), four
    // launches
    const int nj = j + 1;
    if ((rc = zgemm<double>(c, 'C', nj, 1, ngw, kOne, V, ngw, Hv, ngw, kZero, h, nj))) return rc;
    k_lz_sub<<<gridn(ngw), 256, 0, c->stream>>>(ngw, nj, V, ngw, h, Hv, f);
    if ((rc = zgemm<double>(c, 'C', nj, 1, ngw, kOne, V, ngw, f, ngw, kZero, s, nj))) return rc;
    k_lz_update<<<gridn(ngw), 256, 0, c->stream>>>(ngw, nj, V, ngw, h, s, f, T, k, j);
    c->kernel_launches += 2;
  }
  PSPW_CUDA(cudaGetLastError());
  if (f_out && (rc = d2d(c, f_out, f, sizeof(double2) * ngw))) return rc;
  std::vector<double> Th((size_t)k * k);
  if ((rc = d2h(c, Th.data(), T, sizeof(double) * Th.size()))) return rc;
  for (int j = 0; j < k; j++)
    for (int i = 0; i < k; i++) T_host[(size_t)j * ldT + i] = Th[(size_t)j * k + i];
  return PSPW_OK;
}

}  // namespace pspw
