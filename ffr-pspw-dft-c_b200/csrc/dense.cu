// Device dense linear algebra for the eigensolvers.  Hermitian eigensolves
// of order <= 160 (the Rayleigh-Ritz matrices of the SCF loop and of small
// blocks) run on the engine's own kernels (heev.cu); larger ones, QR and
// Cholesky are cuSOLVER calls (the reference calls LAPACK
// zheevd/zgeqrf/zungqr/zpotrf at eig_zheevd.cpp:24, ortho_qr.cpp:19-26,
// lobpcg_cpu.cpp:163); the triangular solve is cuBLAS ztrsm; the GEMMs and
// the small column-wise kernels are this engine's own.
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <algorithm>
#include <vector>

#include "common.cuh"
#include "dense.h"
#include "engine.h"
#include "gemm.h"
#include "heev.h"

namespace pspw {

namespace {

int solver_handle(pspw_cell *c, cusolverDnHandle_t *h) {
  if (!c->cusolver) {
    cusolverDnHandle_t s;
    if (cusolverDnCreate(&s) != CUSOLVER_STATUS_SUCCESS)
      return fail(PSPW_ERR_CUDA, "cusolverDnCreate failed");
    // the same bits on every run: the SCF loop's stopping iteration depends
    // on differences far below the results' own accuracy
    if (cusolverDnSetDeterministicMode(s, CUSOLVER_DETERMINISTIC_RESULTS) !=
        CUSOLVER_STATUS_SUCCESS) {
      cusolverDnDestroy(s);
      return fail(PSPW_ERR_CUDA, "cusolverDnSetDeterministicMode failed");
    }
    c->cusolver = s;
  }
  *h = static_cast<cusolverDnHandle_t>(c->cusolver);
  if (cusolverDnSetStream(*h, c->stream) != CUSOLVER_STATUS_SUCCESS)
    return fail(PSPW_ERR_CUDA, "cusolverDnSetStream failed");
  return PSPW_OK;
}

int blas_handle(pspw_cell *c, cublasHandle_t *h) {
  if (!c->cublas) {
    cublasHandle_t s;
    if (cublasCreate(&s) != CUBLAS_STATUS_SUCCESS) return fail(PSPW_ERR_CUDA, "cublasCreate failed");
    if (cublasSetAtomicsMode(s, CUBLAS_ATOMICS_NOT_ALLOWED) != CUBLAS_STATUS_SUCCESS) {
      cublasDestroy(s);
      return fail(PSPW_ERR_CUDA, "cublasSetAtomicsMode failed");
    }
    c->cublas = s;
  }
  *h = static_cast<cublasHandle_t>(c->cublas);
  if (cublasSetStream(*h, c->stream) != CUBLAS_STATUS_SUCCESS)
    return fail(PSPW_ERR_CUDA, "cublasSetStream failed");
  return PSPW_OK;
}

int read_info(pspw_cell *c, const int *d_info, int *info_out) {
  int info = 0;
  PSPW_CUDA(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  if (info_out) *info_out = info;
  return PSPW_OK;
}

// a failed cuSOLVER call reports its status and the thread's pending CUDA
// error (a library call fails with EXECUTION_FAILED when one is pending)
#define SOLVER_CHECK(call, what)                                                        \
  do {                                                                                  \
    cusolverStatus_t _s = (call);                                                       \
    if (_s != CUSOLVER_STATUS_SUCCESS)                                                  \
      return fail(PSPW_ERR_CUDA, std::string(what) + ": cusolver status " +             \
                                     std::to_string((int)_s) + ", pending CUDA error: " + \
                                     cudaGetErrorString(cudaPeekAtLastError()));        \
  } while (0)

__global__ void k_symmetrize(double2 *v, int ldv, int n) {
  const size_t tot = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    if (i > j) continue;  // (i, j) with i <= j handles the pair
    const double2 a = v[(size_t)j * ldv + i], b = v[(size_t)i * ldv + j];
    const double2 t = make_double2(0.5 * (a.x + b.x), 0.5 * (a.y - b.y));
    v[(size_t)j * ldv + i] = t;
    v[(size_t)i * ldv + j] = make_double2(t.x, -t.y);
  }
}

// column dots: one block per column, fixed-order tree reduction
// one block per column; four independent partial sums per thread keep four
// loads in flight, then a fixed-order warp and block reduction
__global__ void k_coldot(const double2 *__restrict__ x, int ldx, const double2 *__restrict__ y,
                         int ldy, int m, double *out) {
  __shared__ double red[32];
  const int j = blockIdx.x, nt = blockDim.x;
  const double2 *xc = x + (size_t)j * ldx, *yc = y + (size_t)j * ldy;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  int i = threadIdx.x;
  for (; i + 3 * nt < m; i += 4 * nt) {
    const double2 a0 = xc[i], b0 = yc[i], a1 = xc[i + nt], b1 = yc[i + nt];
    const double2 a2 = xc[i + 2 * nt], b2 = yc[i + 2 * nt], a3 = xc[i + 3 * nt],
                  b3 = yc[i + 3 * nt];
    s0 += a0.x * b0.x + a0.y * b0.y;
    s1 += a1.x * b1.x + a1.y * b1.y;
    s2 += a2.x * b2.x + a2.y * b2.y;
    s3 += a3.x * b3.x + a3.y * b3.y;
  }
  for (; i < m; i += nt) {
    const double2 a = xc[i], b = yc[i];
    s0 += a.x * b.x + a.y * b.y;
  }
  double s = (s0 + s1) + (s2 + s3);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = nt >> 5;
  if (lane == 0) red[warp] = s;
  __syncthreads();
  if (warp == 0) {
    s = lane < nw ? red[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) out[j] = s;
  }
}

__global__ void k_residual(const double *__restrict__ lam, const double2 *__restrict__ X, int ldx,
                           const double2 *__restrict__ HX, int ldh, double2 *R, int ldr, int m,
                           int n) {
  const size_t tot = (size_t)m * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot;
       e += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / m), i = (int)(e - (size_t)j * m);
    const double l = lam[j];
    const double2 x = X[(size_t)j * ldx + i], h = HX[(size_t)j * ldh + i];
    R[(size_t)j * ldr + i] = make_double2(l * x.x - h.x, l * x.y - h.y);
  }
}

__global__ void k_scale_prec(const double *__restrict__ s, const double *__restrict__ prec,
                             double2 *R, int ldr, int m, int n) {
  const size_t tot = (size_t)m * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot;
       e += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / m), i = (int)(e - (size_t)j * m);
    double2 r = R[(size_t)j * ldr + i];
    if (s) r = make_double2(s[j] * r.x, s[j] * r.y);
    const double p = prec[i];
    R[(size_t)j * ldr + i] = make_double2(p * r.x, p * r.y);
  }
}

__global__ void k_diag(double2 *A, int lda, int n, const double *d) {
  const size_t tot = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    A[(size_t)j * lda + i] = make_double2(i == j ? (d ? d[i] : 1.0) : 0.0, 0.0);
  }
}

// column i of B scaled by 1/sqrt(ev[i]) where ev[i] > small (eig_zhegv.cpp:39-47)
__global__ void k_scale_cols_rsqrt(double2 *B, int ldb, int n, const double *ev, double small) {
  const size_t tot = (size_t)n * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot;
       e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % n), j = (int)(e / n);
    if (ev[j] > small) {
      const double s = 1.0 / sqrt(ev[j]);
      double2 *p = B + (size_t)j * ldb + i;
      *p = make_double2(s * p->x, s * p->y);
    }
  }
}

inline int grid_for(size_t n) { return (int)std::min<size_t>(4 * 148, (n + 255) / 256 + 1); }

}  // namespace

int dev_zheevd(pspw_cell *c, double2 *A, int lda, double *w, int n, int *info_out) {
  if (n >= 1 && n <= kHeevMax) {
    // the engine's own one-block reduction + bisection + inverse iteration
    void *work = nullptr;
    int rc = ws_reserve(c, kWsHeev, heev_small_workspace(n), &work);
    if (rc) return rc;
    if (info_out) *info_out = 0;
    return dev_heev_small(c, A, lda, w, n, work);
  }
  cusolverDnHandle_t h;
  int rc = solver_handle(c, &h);
  if (rc) return rc;
  int lwork = 0;
  SOLVER_CHECK(cusolverDnZheevd_bufferSize(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n,
                                           A, lda, w, &lwork),
               "zheevd buffer size");
  double2 *work = nullptr;
  int *d_info = nullptr;
  if ((rc = ws_reserve(c, kWsSolver, sizeof(double2) * (size_t)std::max(1, lwork), (void **)&work)) ||
      (rc = ws_reserve(c, kWsInfo, 64, (void **)&d_info)))
    return rc;
  SOLVER_CHECK(cusolverDnZheevd(h, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_UPPER, n, A, lda, w,
                                work, lwork, d_info),
               "zheevd");
  c->kernel_launches++;
  return read_info(c, d_info, info_out);
}

int dev_ortho_qr(pspw_cell *c, double2 *X, int ld, int m, int n, int *info_out) {
  cusolverDnHandle_t h;
  int rc = solver_handle(c, &h);
  if (rc) return rc;
  int l1 = 0, l2 = 0;
  double2 *tau = nullptr, *work = nullptr;
  int *d_info = nullptr;
  if ((rc = ws_reserve(c, kWsTau, sizeof(double2) * (size_t)n, (void **)&tau))) return rc;
  SOLVER_CHECK(cusolverDnZgeqrf_bufferSize(h, m, n, X, ld, &l1), "zgeqrf buffer size");
  SOLVER_CHECK(cusolverDnZungqr_bufferSize(h, m, n, n, X, ld, tau, &l2), "zungqr buffer size");
  const int lwork = std::max(1, std::max(l1, l2));
  if ((rc = ws_reserve(c, kWsSolver, sizeof(double2) * (size_t)lwork, (void **)&work)) ||
      (rc = ws_reserve(c, kWsInfo, 64, (void **)&d_info)))
    return rc;
  SOLVER_CHECK(cusolverDnZgeqrf(h, m, n, X, ld, tau, work, lwork, d_info), "zgeqrf");
  int info = 0;
  if ((rc = read_info(c, d_info, &info))) return rc;
  if (info != 0) {
    if (info_out) *info_out = info;
    return PSPW_OK;
  }
  SOLVER_CHECK(cusolverDnZungqr(h, m, n, n, X, ld, tau, work, lwork, d_info), "zungqr");
  c->kernel_launches += 2;
  return read_info(c, d_info, info_out);
}

int dev_potrf_upper(pspw_cell *c, double2 *A, int lda, int n, int *info_out) {
  cusolverDnHandle_t h;
  int rc = solver_handle(c, &h);
  if (rc) return rc;
  int lwork = 0;
  SOLVER_CHECK(cusolverDnZpotrf_bufferSize(h, CUBLAS_FILL_MODE_UPPER, n, A, lda, &lwork),
               "zpotrf buffer size");
  double2 *work = nullptr;
  int *d_info = nullptr;
  if ((rc = ws_reserve(c, kWsSolver, sizeof(double2) * (size_t)std::max(1, lwork), (void **)&work)) ||
      (rc = ws_reserve(c, kWsInfo, 64, (void **)&d_info)))
    return rc;
  SOLVER_CHECK(cusolverDnZpotrf(h, CUBLAS_FILL_MODE_UPPER, n, A, lda, work, lwork, d_info), "zpotrf");
  c->kernel_launches++;
  return read_info(c, d_info, info_out);
}

int dev_trsm_right_upper(pspw_cell *c, const double2 *U, int ldu, double2 *B, int ldb, int m,
                         int n) {
  cublasHandle_t h;
  int rc = blas_handle(c, &h);
  if (rc) return rc;
  const double2 one = make_double2(1.0, 0.0);
  if (cublasZtrsm(h, CUBLAS_SIDE_RIGHT, CUBLAS_FILL_MODE_UPPER, CUBLAS_OP_N, CUBLAS_DIAG_NON_UNIT, m,
                  n, &one, U, ldu, B, ldb) != CUBLAS_STATUS_SUCCESS)
    return fail(PSPW_ERR_CUDA, "cublasZtrsm failed");
  c->kernel_launches++;
  return PSPW_OK;
}

int dev_symmetrize(pspw_cell *c, double2 *v, int ldv, int n) {
  k_symmetrize<<<grid_for((size_t)n * n), 256, 0, c->stream>>>(v, ldv, n);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int dev_coldot(pspw_cell *c, const double2 *x, int ldx, const double2 *y, int ldy, int m, int n,
               double *out) {
  if (n <= 0) return PSPW_OK;
  // few columns (Lanczos, single vectors): wide blocks, so one column's
  // loads spread over 32 warps
  k_coldot<<<n, n < 148 ? 1024 : 256, 0, c->stream>>>(x, ldx, y, ldy, m, out);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int dev_residual(pspw_cell *c, const double *lam, const double2 *X, int ldx, const double2 *HX,
                 int ldh, double2 *R, int ldr, int m, int n) {
  k_residual<<<grid_for((size_t)m * n), 256, 0, c->stream>>>(lam, X, ldx, HX, ldh, R, ldr, m, n);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int dev_scale_prec(pspw_cell *c, const double *s, const double *prec, double2 *R, int ldr, int m,
                   int n) {
  k_scale_prec<<<grid_for((size_t)m * n), 256, 0, c->stream>>>(s, prec, R, ldr, m, n);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int dev_diag(pspw_cell *c, double2 *A, int lda, int n, const double *d) {
  k_diag<<<grid_for((size_t)n * n), 256, 0, c->stream>>>(A, lda, n, d);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int dev_zhegv(pspw_cell *c, double2 *A, int lda, double2 *B, int ldb, double *eval,
              double2 *evec, int lde, int n, int *nindep_out) {
  const double SMALL = 12.220446049250313e-16;  // eig_zhegv.cpp:7
  double *ev = nullptr;
  int rc = ws_reserve(c, kWsEval, sizeof(double) * (size_t)n, (void **)&ev);
  if (rc) return rc;
  int info = 0;
  if ((rc = dev_zheevd(c, B, ldb, ev, n, &info))) return rc;
  if (info != 0) return fail(PSPW_ERR_LAPACK, "zheevd in eig_zhegv: info = " + std::to_string(info));
  if (nindep_out) {
    std::vector<double> h(n);
    PSPW_CUDA(cudaMemcpyAsync(h.data(), ev, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
    PSPW_CUDA(cudaStreamSynchronize(c->stream));
    int nn = 0;
    for (double v : h) nn += v > SMALL;
    *nindep_out = nn;
  }
  k_scale_cols_rsqrt<<<grid_for((size_t)n * n), 256, 0, c->stream>>>(B, ldb, n, ev, SMALL);
  c->kernel_launches++;
  const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
  if ((rc = zgemm<double>(c, 'N', n, n, n, one, A, lda, B, ldb, zero, evec, lde))) return rc;
  if ((rc = zgemm<double>(c, 'C', n, n, n, one, B, ldb, evec, lde, zero, A, lda))) return rc;
  double *w = eval ? eval : ev;
  if ((rc = dev_zheevd(c, A, lda, w, n, &info))) return rc;
  if (info != 0) return fail(PSPW_ERR_LAPACK, "zheevd in eig_zhegv: info = " + std::to_string(info));
  return zgemm<double>(c, 'N', n, n, n, one, B, ldb, A, lda, zero, evec, lde);
}

int cublas_handle(pspw_cell *c, cublasHandle_t *h) { return blas_handle(c, h); }

}  // namespace pspw
