// The Chebyshev-filtered SCF loop of ChebySCFLoop.cpp:36-378 with every
// array on the device: V_eff, the densities and the mixing history stay in
// HBM between iterations, and the host only steers (bounds, convergence).
// Step for step:
//   EvalEnergy(start density) -> V_eff; Lanczos (k = max(2 NX, 10) steps)
//   and the eigenvalues of its T for the filter bounds lb, ub;
//   first iteration by Davidson (IDIAG >= 0) or the caller's random block;
//   then per iteration: Chebyshev filter of the NX+2 block, QR, Rayleigh-Ritz
//   (H X, X^H H X, symmetrize, eigendecomposition, rotation), EvalRhoPsi,
//   EvalENL, mixing, EvalEnergy, |dETOT| test, new bounds from the Ritz
//   values and a 10-step Lanczos (ChebySCFLoop.cpp:351-366).
// The filter may run in FP32 (the mixed-precision mode), and with it the
// H*v products of the Lanczos bounds, which only set the filter's window;
// everything else is FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "dense.h"
#include "engine.h"
#include "gemm.h"
#include "heev.h"
#include "scf.h"
#include "solvers.h"

namespace pspw {
namespace {

__global__ void k_z2c(const double2 *__restrict__ a, float2 *b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = make_float2((float)a[i].x, (float)a[i].y);
}
__global__ void k_c2z(const float2 *__restrict__ a, double2 *b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    b[i] = make_double2(a[i].x, a[i].y);
}
__global__ void k_real_to_z(const double *__restrict__ a, double2 *b, int k, int lda) {
  // the upper triangle of the k x k real matrix a (lda) as a complex matrix
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= k * k) return;
  const int r = i % k, col = i / k;
  b[i] = make_double2(r <= col ? a[r + (size_t)lda * col] : 0.0, 0.0);
}

// column j of X (m rows, ld) scaled by 1/sqrt(d[j]) where d[j] > 0
__global__ void k_unit_cols(double2 *X, int ld, int m, int n, const double *__restrict__ d) {
  const size_t tot = (size_t)m * n;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < tot;
       e += (size_t)gridDim.x * blockDim.x) {
    const int j = (int)(e / m), i = (int)(e - (size_t)j * m);
    const double dj = d[j];
    if (dj > 0.0) {
      const double s = 1.0 / sqrt(dj);
      double2 *p = X + (size_t)j * ld + i;
      *p = make_double2(s * p->x, s * p->y);
    }
  }
}

// ChebySCFLoop.cpp:7-34: |A v1|^2 with v1 = 1/sqrt(N) (ones), A the leading
// N x N block of the lda-strided matrix
double induced_norm_mat(const double *A, int lda, int N) {
  const double d = 1.0 / std::sqrt((double)N);
  std::vector<double> v(N, 0.0);
  for (int j = 0; j < N; j++)
    for (int i = 0; i < N; i++) v[i] += A[i + (size_t)lda * j] * d;
  double res = 0.0;
  for (int i = 0; i < N; i++) res += v[i] * v[i];
  return res;
}

// An orthonormal basis of span(X) (X: ngw x n, ld ngw) in place, for the
// Rayleigh-Ritz step that follows the filter (ChebySCFLoop.cpp:288-307):
// the reference's Householder QR (ortho_qr.cpp) and any other orthonormal
// basis of the same span give the same Ritz pairs, since Rayleigh-Ritz
// depends on the span only (Q and Q D, D a diagonal of unit-modulus
// phases, differ in the phases of the Ritz vectors alone).  CholeskyQR2:
// twice G = X^H X = U^H U, X <- X U^-1, with the Gram matrices and the
// products by U^-1 on the FP64 tensor-core GEMM and the factorisation and
// inversion of U in one block (heev.cu).  Stable while cond(X) stays well
// below 1/sqrt(eps); the ratio of the largest to the smallest diagonal of
// the first U bounds cond(X) from below, and above 1e6 (or when the
// factorisation fails) the block goes to the Householder QR instead.  The
// columns are first scaled to unit norm (the span is unchanged): the filter
// multiplies the eigen-components of its block by factors that span orders
// of magnitude, so the filtered columns are nearly orthogonal but of very
// different lengths, an ill-conditioning that the scaling removes.
// Both passes are enqueued before the host reads the two pivot statuses
// (one synchronisation): the first pass writes W only, so X is intact for
// the Householder fallback, and a failed first factorisation leaves U as it
// was, which only makes the second pass's numbers meaningless.
// G, U: n x n scratch (ld n); dn: n doubles; stat: 4 doubles; W: ngw x n.
int span_orthonormalize(pspw_cell *c, double2 *X, int ngw, int n, double2 *G, double2 *U,
                        double *dn, double *stat, double2 *W, int *info) {
  const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
  int rc;
  if ((rc = dev_coldot(c, X, ngw, X, ngw, ngw, n, dn))) return rc;
  k_unit_cols<<<4 * 148, 256, 0, c->stream>>>(X, ngw, ngw, n, dn);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  if (n > kHeevMax) {  // beyond the one-block factorisation: Householder
    return dev_ortho_qr(c, X, ngw, ngw, n, info);
  }
  for (int pass = 0; pass < 2; pass++) {
    double2 *src = pass == 0 ? X : W;
    // the factorisation reads the upper triangle of G only
    if ((rc = zgemm_tri(c, 'C', kZgemmUpperC, n, n, ngw, one, src, ngw, src, ngw, zero, G, n)))
      return rc;
    if ((rc = dev_chol_inv_upper(c, G, n, n, U, n, stat + 2 * pass))) return rc;
    // U^-1 is upper triangular (zeros stored below the diagonal)
    if (pass == 0 &&
        (rc = zgemm_tri(c, 'N', kZgemmUpperB, ngw, n, n, one, X, ngw, U, n, zero, W, ngw)))
      return rc;
  }
  double h[4];
  PSPW_CUDA(cudaMemcpyAsync(h, stat, sizeof h, cudaMemcpyDeviceToHost, c->stream));
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  const bool fallback = h[0] != 0.0 || !(h[1] <= 1.0e6) || h[2] != 0.0;
  if (fallback) return dev_ortho_qr(c, X, ngw, ngw, n, info);
  if ((rc = zgemm_tri(c, 'N', kZgemmUpperB, ngw, n, n, one, W, ngw, U, n, zero, X, ngw)))
    return rc;
  *info = 0;
  return PSPW_OK;
}

}  // namespace

// C entry of the span orthonormalisation (scratch from the cell's workspaces)
int ortho_span_dev(pspw_cell *c, double2 *X, int ngw, int n, int *info) {
  double2 *G, *U, *W;
  double *dn, *stat;
  int rc;
  if ((rc = ws_reserve(c, kWsSpan, sizeof(double2) * (size_t)n * n, (void **)&G)) ||
      (rc = ws_reserve(c, kWsSpan + 1, sizeof(double2) * (size_t)n * n, (void **)&U)) ||
      (rc = ws_reserve(c, kWsSpan + 2, sizeof(double2) * (size_t)ngw * n, (void **)&W)) ||
      (rc = ws_reserve(c, kWsSpan + 3, sizeof(double) * ((size_t)n + 4), (void **)&dn)))
    return rc;
  stat = dn + n;
  return span_orthonormalize(c, X, ngw, n, G, U, dn, stat, W, info);
}

namespace {

struct DevBuf {
  std::vector<void *> p;
  ~DevBuf() {
    for (void *q : p) cudaFree(q);
  }
  template <typename T>
  bool get(T **out, size_t n) {
    void *q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(1, n) * sizeof(T)) != cudaSuccess) return false;
    p.push_back(q);
    *out = static_cast<T *>(q);
    return true;
  }
};

// Fermi-Dirac occupations of the nx states (ascending Ritz values, Ha) at
// the electronic temperature ekt (eV): f_i = 2 / (1 + exp((e_i - ef) / ekt))
// with the eigenvalues in eV (AU = 2 x 13.6058), cut to 2 and 0 beyond
// |x| = 30, and the Fermi level ef found by bisection until sum_i f_i w
// equals nel within 1e-7 (FermiEnergy.cpp:69-107).  The reference starts
// its bisection from the interval [-40000, 40000] eV; any bracket of the
// spectrum gives the same level.
void fermi_occupations(const double *eig, int nx, double nel, double w, double ekt, double *f) {
  const double au = 2.0 * 13.6058;
  auto fill = [&](double ef) {
    double sum = 0.0;
    for (int i = 0; i < nx; i++) {
      const double x = (eig[i] * au - ef) / ekt;
      f[i] = x <= -30.0 ? 2.0 : (x < 30.0 ? 2.0 / (1.0 + std::exp(x)) : 0.0);
      sum += f[i] * w;
    }
    return sum;
  };
  double lo = eig[0] * au - 40.0 * ekt, hi = eig[nx - 1] * au + 40.0 * ekt;
  for (int it = 0; it < 200; it++) {
    const double ef = 0.5 * (lo + hi), sum = fill(ef);
    if (std::fabs(sum - nel) < 1e-7) return;
    if (sum > nel) hi = ef; else lo = ef;
  }
  fill(0.5 * (lo + hi));
}

}  // namespace
}  // namespace pspw

using namespace pspw;

extern "C" int pspw_cheby_scf(pspw_scf *s, const pspw_scf_params *p, const double *focc,
                              const double *rho_start, const double *v0, double *X_io,
                              double *eig, double *rho_out, double *hist, int *iterations,
                              int *converged, double *e6) {
  if (!s || !p || !focc || !rho_start || !v0 || !X_io || !eig || !iterations || !converged || !e6)
    return fail(PSPW_ERR_ARG, "cheby_scf: null argument");
  pspw_cell *c = s->cell;
  PSPW_CUDA(cudaSetDevice(c->device));
  const Basis &B = c->basis;
  const int nx = p->nx, nx2 = nx + 2, ngw = B.ngw, nnr = B.nnr;
  const int k = std::max(2 * nx, 10);
  if (nx < 1 || p->degree < 1 || p->max_scf_iter < 1 || nx2 > ngw || k > ngw)
    return fail(PSPW_ERR_ARG, "cheby_scf: bad sizes");
  if (p->filter_prec != PSPW_PREC_F64 && p->filter_prec != PSPW_PREC_F32)
    return fail(PSPW_ERR_ARG, "cheby_scf: unknown filter precision");
  if (p->tmetal && !(p->ekt > 0.0)) return fail(PSPW_ERR_ARG, "cheby_scf: TMETAL needs EKT > 0");
  if (p->tmetal && 2.0 * nx < s->nel) return fail(PSPW_ERR_ARG, "cheby_scf: too few states");
  // occupations: the caller's, or Fermi-Dirac ones after every Rayleigh-Ritz step
  std::vector<double> occ(focc, focc + nx);
  // precision of the filter and of the Lanczos bounds' H*v
  const int fprec = p->filter_prec;
  const int kind = (p->imix == PSPW_MIX_KERKER || p->imix == PSPW_MIX_ANDERSON ||
                    p->imix == PSPW_MIX_PULAY || p->imix == PSPW_MIX_BROYDEN)
                       ? p->imix
                       : PSPW_MIX_SIMPLE;
  const double beta =
      (kind == PSPW_MIX_PULAY || kind == PSPW_MIX_BROYDEN) ? p->pulay_beta : p->mix_beta;
  int rc;
  // ---- device arrays
  DevBuf mem;
  double2 *X, *HX, *T, *dU, *dv0, *df, *dRT;
  float2 *Xf = nullptr;
  double *veff, *rho, *wT, *dprec, *dcn, *dstat;
  if (!mem.get(&X, (size_t)ngw * nx2) || !mem.get(&dcn, nx2) || !mem.get(&HX, (size_t)ngw * nx2) ||
      !mem.get(&T, (size_t)nx2 * nx2) || !mem.get(&dU, (size_t)nx2 * nx2) ||
      !mem.get(&dstat, 4) || !mem.get(&dv0, ngw) || !mem.get(&df, ngw) ||
      !mem.get(&dRT, (size_t)k * k) || !mem.get(&veff, nnr) || !mem.get(&rho, nnr) ||
      !mem.get(&wT, std::max(k, nx2)) || !mem.get(&dprec, ngw) ||
      (fprec == PSPW_PREC_F32 && !mem.get(&Xf, (size_t)ngw * nx2)))
    return fail(PSPW_ERR_OOM, "cheby_scf: device memory");
  cudaStream_t st = c->stream;
  // rhoe2 = rho_old = the starting density (ChebySCFLoop.cpp:164-175)
  PSPW_CUDA(cudaMemcpyAsync(veff, rho_start, sizeof(double) * nnr, cudaMemcpyHostToDevice, st));
  PSPW_CUDA(cudaMemcpyAsync(dv0, v0, sizeof(double2) * ngw, cudaMemcpyHostToDevice, st));
  // simple and Kerker mixing start from rho_old = the start density; the
  // Anderson, Pulay and Broyden histories start at zero
  // (ChebySCFLoop.cpp:123-148), so the first Pulay step mixes the new density
  // with zero
  const bool mix_from_start = kind == PSPW_MIX_SIMPLE || kind == PSPW_MIX_KERKER;
  if ((rc = pspw_mix_init(s, kind, p->mixdim, beta, p->kerker_q0,
                          mix_from_start ? rho_start : nullptr)))
    return rc;
  double en[6];
  // EvalEnergy(rhoe2) with the EKIN, ENL of before the loop (zero)
  if ((rc = eval_energy_dev(s, veff, 0.0, 0.0, en))) return rc;
  double etot_old = en[0];
  if ((rc = pspw_cell_set_veff_device(c, veff, nnr))) return rc;
  // ---- Lanczos bounds (ChebySCFLoop.cpp:180-198)
  std::vector<double> rT((size_t)k * k, 0.0), evT(std::max(k, nx2));
  // the bounds only shape the filter, so in the mixed mode their H*v
  // products run in the filter's precision
  if ((rc = lanczos_dev(c, dv0, ngw, k, rT.data(), k, df, fprec))) return rc;
  {
    double *dr;
    if (!mem.get(&dr, (size_t)k * k)) return fail(PSPW_ERR_OOM, "cheby_scf: device memory");
    PSPW_CUDA(cudaMemcpyAsync(dr, rT.data(), sizeof(double) * k * k, cudaMemcpyHostToDevice, st));
    k_real_to_z<<<(k * k + 255) / 256, 256, 0, st>>>(dr, dRT, k, k);
    c->kernel_launches++;
    int info = 0;
    if ((rc = dev_zheevd(c, dRT, k, wT, k, &info))) return rc;  // dsyev('N','U') values
    PSPW_CUDA(cudaMemcpyAsync(evT.data(), wT, sizeof(double) * k, cudaMemcpyDeviceToHost, st));
    PSPW_CUDA(cudaStreamSynchronize(st));
    if (info) return fail(PSPW_ERR_LAPACK, "cheby_scf: eigenvalues of the Lanczos T");
  }
  double lb = evT[nx + 1], ub = evT[2 * nx - 1];
  std::vector<double> evals(nx2), res(nx2);
  int iter_start = 1, done_iters = 0;
  *converged = 0;
  const auto t_start = std::chrono::steady_clock::now();
  auto record = [&](int it, double etot, double detot, double drms) {
    if (hist && it >= 1 && it <= p->max_scf_iter) {
      double *h = hist + 4 * (size_t)(it - 1);
      h[0] = etot;
      h[1] = detot;
      h[2] = drms;
      // the iteration's results are on the host here (its last step
      // synchronised the stream), so the host clock marks its end
      h[3] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start)
                 .count();
    }
  };
  // density, EKIN, ENL of the first nx columns of X (ld ngw), then mixing
  // and EvalEnergy (ChebySCFLoop.cpp:232-262 and 321-348)
  auto density_step = [&](int it, double *etot, double *drms) -> int {
    int r;
    PSPW_CUDA(cudaMemsetAsync(rho, 0, sizeof(double) * nnr, st));
    double ekin = 0.0, enl = 0.0;
    cudaEvent_t e;
    timing_begin(c, kFamScfDensity, &e);
    if (p->tmetal) fermi_occupations(evals.data(), nx, s->nel, 1.0, p->ekt, occ.data());
    if ((r = eval_rho_psi_dev(c, X, ngw, ngw, nx, occ.data(), 1.0, s->omega, rho, &ekin))) return r;
    timing_end(c, kFamScfDensity, e);
    timing_begin(c, kFamScfEnl, &e);
    if ((r = eval_enl_dev(c, X, ngw, ngw, nx, occ.data(), 1.0, &enl, nullptr))) return r;
    timing_end(c, kFamScfEnl, e);
    timing_begin(c, kFamScfMixEnergy, &e);
    if ((r = mix_dev(s, it, rho, drms))) return r;
    PSPW_CUDA(cudaMemcpyAsync(veff, rho, sizeof(double) * nnr, cudaMemcpyDeviceToDevice, st));
    if ((r = eval_energy_dev(s, veff, ekin, enl, en))) return r;
    *etot = en[0];
    r = pspw_cell_set_veff_device(c, veff, nnr);
    timing_end(c, kFamScfMixEnergy, e);
    return r;
  };
  if (p->idiag < 0) {
    // the caller's random block, orthonormalised (ChebySCFLoop.cpp:201-209)
    PSPW_CUDA(cudaMemcpyAsync(X, X_io, sizeof(double2) * (size_t)ngw * nx2, cudaMemcpyHostToDevice,
                              st));
    int info = 0;
    if ((rc = dev_ortho_qr(c, X, ngw, ngw, nx2, &info))) return rc;
  } else {
    // first iteration by Davidson (ChebySCFLoop.cpp:210-262)
    if ((rc = gen_prec_dev(c, dprec, ngw, -10.0))) return rc;
    int its = 0;
    if ((rc = davidson_dev(c, PSPW_PREC_F64, evals.data(), X, ngw, nx2, dprec, p->nempty,
                           p->max_diag_iter, res.data(), &its)))
      return rc;
    double etot = 0.0, drms = 0.0;
    if ((rc = density_step(1, &etot, &drms))) return rc;
    const double detot = std::fabs(etot - etot_old);
    record(1, etot, detot, drms);
    etot_old = etot;
    iter_start = 2;
    done_iters = 1;
  }
  std::vector<double> rT10((size_t)k * k, 0.0);
  double *dfn;
  if (!mem.get(&dfn, 1)) return fail(PSPW_ERR_OOM, "cheby_scf: device memory");
  for (int it = iter_start; it <= p->max_scf_iter; it++) {
    cudaEvent_t ev;
    // filter the NX+2 block (ChebySCFLoop.cpp:285)
    timing_begin(c, kFamScfFilter, &ev);
    if (fprec == PSPW_PREC_F32) {
      const size_t n = (size_t)ngw * nx2;
      k_z2c<<<4 * 148, 256, 0, st>>>(X, Xf, n);
      if ((rc = pspw_chebyfilt_dev(c, PSPW_PREC_F32, Xf, ngw, ngw, nx2, p->degree, lb, ub)))
        return rc;
      k_c2z<<<4 * 148, 256, 0, st>>>(Xf, X, n);
      c->kernel_launches += 2;
    } else if ((rc = pspw_chebyfilt_dev(c, PSPW_PREC_F64, X, ngw, ngw, nx2, p->degree, lb, ub))) {
      return rc;
    }
    timing_end(c, kFamScfFilter, ev);
    int info = 0;
    timing_begin(c, kFamScfQr, &ev);
    if ((rc = span_orthonormalize(c, X, ngw, nx2, T, dU, dcn, dstat, HX, &info))) return rc;
    timing_end(c, kFamScfQr, ev);
    // Rayleigh-Ritz (ChebySCFLoop.cpp:293-307)
    timing_begin(c, kFamScfRayleigh, &ev);
    // H X in FP64: the Ritz pairs (and through them the density) carry no
    // FP32 rounding; with an FP32 H X the subspace matrix's error (~1e-6 Ha)
    // divided by the occupied-empty gap keeps |dETOT| of a 64-atom cell
    // above 1e-6
    if ((rc = hpsi_apply<double>(c, X, ngw, HX, ngw, ngw, nx2, 1.0, 0.0, 0.0, nullptr, ngw)))
      return rc;
    const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
    if ((rc = zgemm<double>(c, 'C', nx2, nx2, ngw, one, X, ngw, HX, ngw, zero, T, nx2))) return rc;
    timing_end(c, kFamScfRayleigh, ev);
    timing_begin(c, kFamScfEig, &ev);
    if ((rc = dev_symmetrize(c, T, nx2, nx2))) return rc;
    if ((rc = dev_zheevd(c, T, nx2, wT, nx2, &info))) return rc;
    timing_end(c, kFamScfEig, ev);
    timing_begin(c, kFamScfRayleigh, &ev);
    if ((rc = zgemm<double>(c, 'N', ngw, nx2, nx2, one, X, ngw, T, nx2, zero, HX, ngw))) return rc;
    timing_end(c, kFamScfRayleigh, ev);
    std::swap(X, HX);
    PSPW_CUDA(cudaMemcpyAsync(evals.data(), wT, sizeof(double) * nx2, cudaMemcpyDeviceToHost, st));
    PSPW_CUDA(cudaStreamSynchronize(st));
    if (info) return fail(PSPW_ERR_LAPACK, "cheby_scf: Rayleigh-Ritz eigensolver");
    double etot = 0.0, drms = 0.0;
    if ((rc = density_step(it, &etot, &drms))) return rc;
    const double detot = std::fabs(etot - etot_old);
    record(it, etot, detot, drms);
    etot_old = etot;
    done_iters = it;
    if (detot <= p->conv) {
      *converged = 1;
      break;
    }
    // new bounds (ChebySCFLoop.cpp:356-366)
    lb = evals[nx + 1];
    const int kl = k > 10 ? 10 : k;
    timing_begin(c, kFamScfLanczos, &ev);
    if ((rc = lanczos_dev(c, dv0, ngw, kl, rT10.data(), k, df, fprec))) return rc;
    double fn = 0.0;
    if ((rc = dev_coldot(c, df, ngw, df, ngw, ngw, 1, dfn))) return rc;
    PSPW_CUDA(cudaMemcpyAsync(&fn, dfn, sizeof(double), cudaMemcpyDeviceToHost, st));
    timing_end(c, kFamScfLanczos, ev);
    PSPW_CUDA(cudaStreamSynchronize(st));
    ub = induced_norm_mat(rT10.data(), k, kl) + std::sqrt(fn);
  }
  // results
  for (int i = 0; i < nx; i++) eig[i] = evals[i];
  PSPW_CUDA(cudaMemcpyAsync(X_io, X, sizeof(double2) * (size_t)ngw * nx2, cudaMemcpyDeviceToHost,
                            st));
  if (rho_out)
    PSPW_CUDA(cudaMemcpyAsync(rho_out, rho, sizeof(double) * nnr, cudaMemcpyDeviceToHost, st));
  PSPW_CUDA(cudaStreamSynchronize(st));
  for (int i = 0; i < 6; i++) e6[i] = en[i];
  *iterations = done_iters;
  return device_status(c);
}

extern "C" int pspw_ortho_span_dev(pspw_cell *c, double *d_X, int ngw, int n) {
  if (!c || !d_X || n < 1 || ngw < n) return fail(PSPW_ERR_ARG, "ortho_span_dev: bad arguments");
  PSPW_CUDA(cudaSetDevice(c->device));
  int info = 0;
  const int rc = ortho_span_dev(c, reinterpret_cast<double2 *>(d_X), ngw, n, &info);
  if (rc) return rc;
  if (info) return fail(PSPW_ERR_LAPACK, "ortho_span_dev: info = " + std::to_string(info));
  return PSPW_OK;
}
