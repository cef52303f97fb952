// C ABI of the eigensolvers, dense steps, preconditioner, random start and
// density (host-buffer entry points mirroring the reference signatures).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "common.cuh"
#include "dense.h"
#include "engine.h"
#include "fftpath.h"
#include "gemm.h"
#include "solvers.h"

namespace pspw {
namespace {

int enter(pspw_cell *c) {
  if (!c) return fail(PSPW_ERR_ARG, "null cell");
  PSPW_CUDA(cudaSetDevice(c->device));
  return PSPW_OK;
}

// upload an m x n column-major host matrix (ld) into a compact device buffer
int up_mat(pspw_cell *c, int slot, const double *h, int ld, int m, int n, double2 **d) {
  int rc = ws_reserve(c, slot, sizeof(double2) * (size_t)std::max(1, m) * std::max(1, n), (void **)d);
  if (rc) return rc;
  PSPW_CUDA(cudaMemcpy2DAsync(*d, sizeof(double2) * m, h, sizeof(double2) * ld, sizeof(double2) * m,
                              n, cudaMemcpyHostToDevice, c->stream));
  return PSPW_OK;
}

int down_mat(pspw_cell *c, double *h, int ld, const double2 *d, int m, int n) {
  PSPW_CUDA(cudaMemcpy2DAsync(h, sizeof(double2) * ld, d, sizeof(double2) * m, sizeof(double2) * m,
                              n, cudaMemcpyDeviceToHost, c->stream));
  return PSPW_OK;
}

int sync(pspw_cell *c) {
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  return device_status(c);
}

// ss[j] = sum_{i<m} |c|^2, sk[j] = sum_{i<m} xkg[i] |c|^2 (EvalRhoPsi.cpp:117-126)
__global__ void k_charge_sums(const double2 *__restrict__ X, int ld, int m,
                              const double *__restrict__ xkg, double *ss, double *sk) {
  __shared__ double r1[256], r2[256];
  const int j = blockIdx.x;
  const double2 *col = X + (size_t)j * ld;
  double a = 0.0, b = 0.0;
  for (int i = threadIdx.x; i < m; i += blockDim.x) {
    const double2 v = col[i];
    const double q = v.x * v.x + v.y * v.y;
    a += q;
    b += xkg[i] * q;
  }
  r1[threadIdx.x] = a;
  r2[threadIdx.x] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      r1[threadIdx.x] += r1[threadIdx.x + w];
      r2[threadIdx.x] += r2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    ss[j] = r1[0];
    sk[j] = r2[0];
  }
}

constexpr int kSlotA = kWsSolverBase + 11;
constexpr int kSlotB = kWsSolverBase + 12;
constexpr int kSlotC = kWsSolverBase + 13;
constexpr int kSlotD = kWsSolverBase + 14;
constexpr int kSlotE = kWsEnl;

}  // namespace

// EvalRhoPsi.cpp:83-157 on a device block (ld >= ngw): the charge check and
// EKIN from column sums, and d_rho += sum_i wkpt focc_i |psi_i(r)|^2 / omega
// with the scatter stopping at ig < ngw - 1 (EvalRhoPsi.cpp:117).
// *ekin += the kinetic energy (x TPIBA2).  The band weights do not depend on
// the sums, so the sums and the density pass are enqueued together and the
// host reads the sums once, after both (on a wrong charge d_rho has been
// accumulated when the error returns).
int eval_rho_psi_dev(pspw_cell *c, const double2 *dX, int ld, int ngw, int nx, const double *focc,
                     double wkpt, double omega, double *d_rho, double *ekin) {
  const Basis &B = c->basis;
  const int m = ngw - 1;  // the scatter stops at ig < NGW_ik (EvalRhoPsi.cpp:117)
  double *dsum, *dw;
  int rc;
  if ((rc = ws_reserve(c, kSlotB, sizeof(double) * 2 * (size_t)nx, (void **)&dsum)) ||
      (rc = ws_reserve(c, kSlotD, sizeof(double) * (size_t)nx, (void **)&dw)))
    return rc;
  std::vector<double> wband(nx);
  for (int i = 0; i < nx; i++) wband[i] = (wkpt * focc[i]) / omega;
  PSPW_CUDA(cudaMemcpyAsync(dw, wband.data(), sizeof(double) * nx, cudaMemcpyHostToDevice, c->stream));
  k_charge_sums<<<nx, 256, 0, c->stream>>>(dX, ld, m, B.d_xkg64, dsum, dsum + nx);
  c->kernel_launches++;
  if (B.fast) {
    const FastGeo g{B.ncol,    B.nxa,       B.d_col_start, B.d_sg_ig,
                    B.d_sg_z,  B.d_sg_col,  B.d_xa_list,   B.d_col_x,
                    B.d_col_y, B.d_xa_of_x, false,         B.d_sg_off};
    if ((rc = rho_fast<double>(c, g, dX, ld, m, nx, dw, d_rho))) return rc;
  } else if ((rc = rho_generic(c, dX, ld, m, nx, dw, d_rho))) {
    return rc;
  }
  // (a copy into pageable memory returns when it is done: the one wait)
  std::vector<double> sums(2 * (size_t)nx);
  PSPW_CUDA(cudaMemcpyAsync(sums.data(), dsum, sizeof(double) * 2 * nx, cudaMemcpyDeviceToHost,
                            c->stream));
  if ((rc = sync(c))) return rc;
  double xkin = 0.0;
  for (int i = 0; i < nx; i++) {
    const double ss = sums[i];
    if (std::fabs(ss - 1.0) > 6.e-3) {  // EvalRhoPsi.cpp:129-133
      char msg[160];
      std::snprintf(msg, sizeof msg,
                    "Wrong charge density in G-space: %18.10f for k-point 1 and states %d", ss,
                    i + 1);
      return fail(PSPW_ERR_CHARGE, msg);
    }
    const double wdotf = wkpt * focc[i];
    xkin = xkin + sums[nx + i] * (wdotf * 0.5);
  }
  if (ekin) *ekin = *ekin + xkin * c->tpiba2;  // EvalRhoPsi.cpp:154
  return PSPW_OK;
}

// enl_p[p] = sum_ist focc[ist] |P(p, ist)|^2: one warp per projector, lanes
// over the states in a fixed order, then a fixed shuffle tree
__global__ void k_enl_per_projector(const double2 *__restrict__ P, const double *__restrict__ focc,
                                    int nx, int nproj, double *enl_p) {
  const int p = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (p >= nproj) return;  // uniform per warp
  double acc = 0.0;
  for (int ist = lane; ist < nx; ist += 32) {
    const double2 sf = P[(size_t)ist * nproj + p];
    const double a = hypot(sf.x, sf.y);
    acc += focc[ist] * (a * a);
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, d);
  if (lane == 0) enl_p[p] = acc;
}

// EvalENL.cpp:5-49 for one k-point on a device block X (ngw x nx, ld).
int eval_enl_dev(pspw_cell *c, const double2 *dX, int ld, int ngw, int nx, const double *focc,
                 double wkpt, double *enl, double *fnl) {
  const int nproj = c->proj.nproj;
  *enl = 0.0;
  if (nx == 0 || nproj == 0) return PSPW_OK;
  double2 *dP;
  int rc;
  if ((rc = ws_reserve(c, kSlotE, sizeof(double2) * (size_t)nx * nproj, (void **)&dP))) return rc;
  if ((rc = project_fp64(c, dX, ld, ngw, nx, dP))) return rc;
  if (!fnl) {
    // only the energy: the per-projector sums over states on the device (a
    // fixed lane-strided order, not the reference's sequential one: equal to
    // rounding), the sum over projectors in the reference's order on the host
    double *dfo, *dep;
    if ((rc = ws_reserve(c, kSlotD, sizeof(double) * ((size_t)nx + nproj), (void **)&dfo)))
      return rc;
    dep = dfo + nx;
    PSPW_CUDA(cudaMemcpyAsync(dfo, focc, sizeof(double) * nx, cudaMemcpyHostToDevice, c->stream));
    k_enl_per_projector<<<(nproj * 32 + 255) / 256, 256, 0, c->stream>>>(dP, dfo, nx, nproj, dep);
    c->kernel_launches++;
    std::vector<double> ep(nproj), w(nproj);
    PSPW_CUDA(cudaMemcpyAsync(ep.data(), dep, sizeof(double) * nproj, cudaMemcpyDeviceToHost,
                              c->stream));
    PSPW_CUDA(cudaMemcpyAsync(w.data(), c->proj.d_pw64, sizeof(double) * nproj,
                              cudaMemcpyDeviceToHost, c->stream));
    if ((rc = sync(c))) return rc;
    double e = 0.0;
    for (int p = 0; p < nproj; p++) e = e + wkpt * ep[p] * w[p];
    *enl = e;
    return PSPW_OK;
  }
  std::vector<double2> P((size_t)nx * nproj);
  std::vector<double> w(nproj);
  PSPW_CUDA(cudaMemcpyAsync(P.data(), dP, sizeof(double2) * P.size(), cudaMemcpyDeviceToHost,
                            c->stream));
  PSPW_CUDA(cudaMemcpyAsync(w.data(), c->proj.d_pw64, sizeof(double) * nproj,
                            cudaMemcpyDeviceToHost, c->stream));
  if ((rc = sync(c))) return rc;
  // projectors are species-major, then atom, then lm: the reference's loop
  // order (EvalENL.cpp:21-45) for one k-point
  double e = 0.0;
  for (int p = 0; p < nproj; p++) {
    double enl_m = 0.0;
    for (int ist = 0; ist < nx; ist++) {
      const double2 sf = P[(size_t)ist * nproj + p];
      const double a = std::hypot(sf.x, sf.y);
      enl_m = enl_m + focc[ist] * (a * a);
    }
    e = e + wkpt * enl_m * w[p];
  }
  *enl = e;
  if (fnl)
    for (int p = 0; p < nproj; p++)
      for (int ist = 0; ist < nx; ist++) {
        const double2 sf = P[(size_t)ist * nproj + p];
        fnl[2 * ((size_t)p * nx + ist)] = sf.x;
        fnl[2 * ((size_t)p * nx + ist) + 1] = sf.y;
      }
  return PSPW_OK;
}

}  // namespace pspw

using namespace pspw;

extern "C" {

int pspw_random_col(double *A, int nelem, long seed) {
  if (!A || nelem < 0) return fail(PSPW_ERR_ARG, "random_col: bad argument");
  random_col_host(reinterpret_cast<double2 *>(A), nelem, seed);
  return PSPW_OK;
}

int pspw_gen_prec(pspw_cell *c, double *prec, int nbasis, double tau) {
  int rc = enter(c);
  if (rc) return rc;
  double *d = nullptr;
  if ((rc = ws_reserve(c, kSlotA, sizeof(double) * (size_t)std::max(1, nbasis), (void **)&d)) ||
      (rc = gen_prec_dev(c, d, nbasis, tau)))
    return rc;
  PSPW_CUDA(cudaMemcpyAsync(prec, d, sizeof(double) * nbasis, cudaMemcpyDeviceToHost, c->stream));
  return sync(c);
}

int pspw_ortho_qr(pspw_cell *c, double *X, int nbasis, int nstates) {
  int rc = enter(c);
  if (rc) return rc;
  if (!X || nbasis < nstates || nstates < 0) return fail(PSPW_ERR_ARG, "ortho_qr: bad shape");
  double2 *d;
  if ((rc = up_mat(c, kSlotA, X, nbasis, nbasis, nstates, &d))) return rc;
  int info = 0;
  if ((rc = dev_ortho_qr(c, d, nbasis, nbasis, nstates, &info))) return rc;
  if (info) return fail(PSPW_ERR_LAPACK, "zgeqrf/zungqr: info = " + std::to_string(info));
  if ((rc = down_mat(c, X, nbasis, d, nbasis, nstates))) return rc;
  return sync(c);
}

int pspw_eig_zheevd(pspw_cell *c, double *A, int lda, double *lambda, int n) {
  int rc = enter(c);
  if (rc) return rc;
  double2 *d;
  double *w;
  if ((rc = up_mat(c, kSlotA, A, lda, n, n, &d)) ||
      (rc = ws_reserve(c, kSlotB, sizeof(double) * (size_t)std::max(1, n), (void **)&w)))
    return rc;
  int info = 0;
  if ((rc = dev_zheevd(c, d, n, w, n, &info))) return rc;
  if (info) return fail(PSPW_ERR_LAPACK, "zheevd: info = " + std::to_string(info));
  if ((rc = down_mat(c, A, lda, d, n, n))) return rc;
  PSPW_CUDA(cudaMemcpyAsync(lambda, w, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  return sync(c);
}

int pspw_eig_zhegv_eval(pspw_cell *c, double *A, int lda, double *B, int ldb, double *eval,
                        double *evec, int lde, int n) {
  int rc = enter(c);
  if (rc) return rc;
  double2 *dA, *dB, *dE;
  double *w;
  if ((rc = up_mat(c, kSlotA, A, lda, n, n, &dA)) || (rc = up_mat(c, kSlotB, B, ldb, n, n, &dB)) ||
      (rc = ws_reserve(c, kSlotC, sizeof(double2) * (size_t)n * n, (void **)&dE)) ||
      (rc = ws_reserve(c, kSlotD, sizeof(double) * (size_t)n, (void **)&w)))
    return rc;
  int nn = 0;
  if ((rc = dev_zhegv(c, dA, n, dB, n, w, dE, n, n, &nn))) return rc;
  if (nn < n)
    std::printf("Warning: Number of linearly independent vectors = %d\n         while size of the "
                "problem: %d\n", nn, n);
  if ((rc = down_mat(c, A, lda, dA, n, n)) || (rc = down_mat(c, B, ldb, dB, n, n)) ||
      (rc = down_mat(c, evec, lde, dE, n, n)))
    return rc;
  if (eval) PSPW_CUDA(cudaMemcpyAsync(eval, w, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  return sync(c);
}

int pspw_eig_zhegv(pspw_cell *c, double *A, int lda, double *B, int ldb, double *evec, int lde,
                   int n) {
  return pspw_eig_zhegv_eval(c, A, lda, B, ldb, nullptr, evec, lde, n);
}

static int solver_entry(int kind, pspw_cell *c, double *evals, double *X, int nbasis,
                        int nstates, const double *prec, int nempty, int max_iter, int hprec,
                        double *resnrm, int *iters) {
  int rc = enter(c);
  if (rc) return rc;
  if (!evals || !X || !prec || nstates <= 0 || nbasis < nstates)
    return fail(PSPW_ERR_ARG, "eigensolver: bad argument");
  if (nbasis > c->basis.ngw) return fail(PSPW_ERR_SHAPE, "eigensolver: nbasis exceeds the cell");
  if (hprec != PSPW_PREC_F64 && hprec != PSPW_PREC_F32) return fail(PSPW_ERR_ARG, "bad precision");
  double2 *dX;
  double *dp;
  if ((rc = ws_reserve(c, kSlotA, sizeof(double2) * (size_t)nbasis * nstates, (void **)&dX)) ||
      (rc = ws_reserve(c, kSlotB, sizeof(double) * (size_t)nbasis, (void **)&dp)))
    return rc;
  PSPW_CUDA(cudaMemcpyAsync(dp, prec, sizeof(double) * nbasis, cudaMemcpyHostToDevice, c->stream));
  if (kind == 3)
    PSPW_CUDA(cudaMemcpyAsync(dX, X, sizeof(double2) * (size_t)nbasis * nstates,
                              cudaMemcpyHostToDevice, c->stream));
  if (kind == 1)
    rc = lobpcg_dev(c, hprec, evals, dX, nbasis, nstates, dp, nempty, max_iter, resnrm, iters);
  else if (kind == 2 || kind == 3)
    rc = lobpcg_ortho_dev(c, hprec, evals, dX, nbasis, nstates, dp, nempty, max_iter, resnrm,
                          iters, kind == 3);
  else
    rc = davidson_dev(c, hprec, evals, dX, nbasis, nstates, dp, nempty, max_iter, resnrm, iters);
  if (rc) return rc;
  PSPW_CUDA(cudaMemcpyAsync(X, dX, sizeof(double2) * (size_t)nbasis * nstates,
                            cudaMemcpyDeviceToHost, c->stream));
  return sync(c);
}

int pspw_davidson(pspw_cell *c, double *evals, double *X, int nbasis, int nstates,
                  const double *prec, int nempty, int max_iter, int hprec, double *resnrm,
                  int *iters) {
  return solver_entry(0, c, evals, X, nbasis, nstates, prec, nempty, max_iter, hprec, resnrm,
                      iters);
}

int pspw_lobpcg(pspw_cell *c, double *lambda, double *X, int nbasis, int nstates,
                const double *prec, int nempty, int max_iter, int hprec, double *resnrm,
                int *iters) {
  return solver_entry(1, c, lambda, X, nbasis, nstates, prec, nempty, max_iter, hprec, resnrm,
                      iters);
}

int pspw_lobpcg_ortho(pspw_cell *c, double *lambda, double *X, int nbasis, int nstates,
                      const double *prec, int nempty, int max_iter, int hprec, double *resnrm,
                      int *iters) {
  return solver_entry(2, c, lambda, X, nbasis, nstates, prec, nempty, max_iter, hprec, resnrm,
                      iters);
}

int pspw_lobpcg_ortho_from(pspw_cell *c, double *lambda, double *X, int nbasis, int nstates,
                           const double *prec, int nempty, int max_iter, int hprec,
                           double *resnrm, int *iters) {
  return solver_entry(3, c, lambda, X, nbasis, nstates, prec, nempty, max_iter, hprec, resnrm,
                      iters);
}

int pspw_lanczos(pspw_cell *c, double *v0, int ngw, int k, double *T, int ldT, double *f) {
  int rc = enter(c);
  if (rc) return rc;
  if (!v0 || !T || k < 1 || ldT < k || ngw < 1) return fail(PSPW_ERR_ARG, "lanczos: bad argument");
  double2 *dv, *df;
  if ((rc = ws_reserve(c, kSlotA, sizeof(double2) * (size_t)ngw, (void **)&dv)) ||
      (rc = ws_reserve(c, kSlotB, sizeof(double2) * (size_t)ngw, (void **)&df)))
    return rc;
  PSPW_CUDA(cudaMemcpyAsync(dv, v0, sizeof(double2) * ngw, cudaMemcpyHostToDevice, c->stream));
  if ((rc = lanczos_dev(c, dv, ngw, k, T, ldT, df))) return rc;
  PSPW_CUDA(cudaMemcpyAsync(v0, dv, sizeof(double2) * ngw, cudaMemcpyDeviceToHost, c->stream));
  if (f) PSPW_CUDA(cudaMemcpyAsync(f, df, sizeof(double2) * ngw, cudaMemcpyDeviceToHost, c->stream));
  return sync(c);
}

int pspw_eval_rho_psi(pspw_cell *c, double *rhoe, const double *eigvec, int ld, int ngw, int nx,
                      const double *focc, double wkpt, double omega, double *ekin) {
  int rc = enter(c);
  if (rc) return rc;
  if (!rhoe || !eigvec || !focc || nx < 0 || ld < ngw || ngw < 1)
    return fail(PSPW_ERR_ARG, "EvalRhoPsi: bad argument");
  if (nx == 0) return PSPW_OK;
  const Basis &B = c->basis;
  if (ngw > B.ngw) return fail(PSPW_ERR_SHAPE, "EvalRhoPsi: NGW exceeds the cell");
  double2 *dX;
  double *drho;
  if ((rc = ws_reserve(c, kSlotA, sizeof(double2) * (size_t)ld * nx, (void **)&dX)) ||
      (rc = ws_reserve(c, kSlotC, sizeof(double) * (size_t)B.nnr, (void **)&drho)))
    return rc;
  PSPW_CUDA(cudaMemcpyAsync(dX, eigvec, sizeof(double2) * ((size_t)ld * (nx - 1) + ngw),
                            cudaMemcpyHostToDevice, c->stream));
  PSPW_CUDA(cudaMemcpyAsync(drho, rhoe, sizeof(double) * B.nnr, cudaMemcpyHostToDevice, c->stream));
  if ((rc = eval_rho_psi_dev(c, dX, ld, ngw, nx, focc, wkpt, omega, drho, ekin))) return rc;
  PSPW_CUDA(cudaMemcpyAsync(rhoe, drho, sizeof(double) * B.nnr, cudaMemcpyDeviceToHost, c->stream));
  return sync(c);
}

int pspw_eval_enl(pspw_cell *c, const double *c0, int ld, int ngw, int nx, const double *focc,
                  double wkpt, double *enl, double *fnl) {
  int rc = enter(c);
  if (rc) return rc;
  if (!c0 || !focc || !enl || nx < 0 || ld < ngw || ngw < 1)
    return fail(PSPW_ERR_ARG, "EvalENL: bad argument");
  if (ngw > c->basis.ngw) return fail(PSPW_ERR_SHAPE, "EvalENL: NGW exceeds the cell");
  *enl = 0.0;
  if (nx == 0 || c->proj.nproj == 0) return PSPW_OK;
  double2 *dX;
  if ((rc = up_mat(c, kSlotA, c0, ld, ngw, nx, &dX))) return rc;
  return eval_enl_dev(c, dX, ngw, ngw, nx, focc, wkpt, enl, fnl);
}

int pspw_eval_rho_psi_dev(pspw_cell *c, double *d_rhoe, const double *d_eigvec, int ld, int ngw,
                          int nx, const double *focc, double wkpt, double omega, double *ekin) {
  int rc = enter(c);
  if (rc) return rc;
  if (!d_rhoe || !d_eigvec || !focc || nx < 0 || ld < ngw || ngw < 1)
    return fail(PSPW_ERR_ARG, "EvalRhoPsi: bad argument");
  if (ngw > c->basis.ngw) return fail(PSPW_ERR_SHAPE, "EvalRhoPsi: NGW exceeds the cell");
  if (nx == 0) return PSPW_OK;
  if ((rc = eval_rho_psi_dev(c, reinterpret_cast<const double2 *>(d_eigvec), ld, ngw, nx, focc,
                             wkpt, omega, d_rhoe, ekin)))
    return rc;
  return sync(c);
}

int pspw_eval_enl_dev(pspw_cell *c, const double *d_c0, int ld, int ngw, int nx,
                      const double *focc, double wkpt, double *enl, double *fnl) {
  int rc = enter(c);
  if (rc) return rc;
  if (!d_c0 || !focc || !enl || nx < 0 || ld < ngw || ngw < 1)
    return fail(PSPW_ERR_ARG, "EvalENL: bad argument");
  if (ngw > c->basis.ngw) return fail(PSPW_ERR_SHAPE, "EvalENL: NGW exceeds the cell");
  *enl = 0.0;
  if (nx == 0 || c->proj.nproj == 0) return PSPW_OK;
  return eval_enl_dev(c, reinterpret_cast<const double2 *>(d_c0), ld, ngw, nx, focc, wkpt, enl,
                      fnl);
}

}  // extern "C"

extern "C" int pspw_zgemm_dev(pspw_cell *c, char opa, int m, int n, int k, const double *alpha,
                              const double *d_A, int lda, const double *d_B, int ldb,
                              const double *beta, double *d_C, int ldc) {
  int rc = enter(c);
  if (rc) return rc;
  if (!alpha || !beta || m < 0 || n < 0 || k < 0)
    return fail(PSPW_ERR_ARG, "zgemm_dev: bad arguments");
  if (m == 0 || n == 0) return PSPW_OK;
  const bool conj = opa == 'C' || opa == 'c';
  if ((k > 0 && (!d_A || !d_B)) || !d_C || lda < std::max(1, conj ? k : m) ||
      ldb < std::max(1, k) || ldc < m)
    return fail(PSPW_ERR_ARG, "zgemm_dev: null matrix or leading dimension too small");
  return zgemm<double>(c, opa, m, n, k, make_double2(alpha[0], alpha[1]),
                       reinterpret_cast<const double2 *>(d_A), lda,
                       reinterpret_cast<const double2 *>(d_B), ldb,
                       make_double2(beta[0], beta[1]), reinterpret_cast<double2 *>(d_C), ldc);
}

extern "C" int pspw_eig_zheevd_dev(pspw_cell *c, double *d_A, int lda, double *d_w, int n) {
  int rc = enter(c);
  if (rc) return rc;
  if (n < 0 || lda < std::max(1, n) || (n > 0 && (!d_A || !d_w)))
    return fail(PSPW_ERR_ARG, "eig_zheevd_dev: bad arguments");
  if (n == 0) return PSPW_OK;
  int info = 0;
  if ((rc = dev_zheevd(c, reinterpret_cast<double2 *>(d_A), lda, d_w, n, &info))) return rc;
  if (info) return fail(PSPW_ERR_LAPACK, "zheevd: info = " + std::to_string(info));
  return PSPW_OK;
}
