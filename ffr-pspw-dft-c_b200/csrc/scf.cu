// SCF pieces around the eigensolver, on the device and in FP64:
//   EvalEnergy (EvalEnergy.cpp:5-163): Hartree + local pseudopotential through
//     a full-grid FFT, xc_PZ, V_eff = Re(V_H + V_loc) + V_xc, energy terms;
//   xc_PZ (xc_PZ.cpp:7-63), NormalizeRho (NormalizeRho.cpp:7-33),
//   KerkerPrec (KerkerRhoMix.cpp:53-81) and the density mixers
//   SimpleRhoMix, KerkerRhoMix, AndersonRhoMix, PulayRhoMix and BroydenRhoMix
//   (SimpleRhoMix.cpp, KerkerRhoMix.cpp:5-50, AndersonRhoMix.cpp:8-91,
//   PulayRhoMix.cpp:5-91).
// Every sum over the grid or the G list is a two-stage reduction with a
// fixed block count and a fixed tree, so results do not depend on
// scheduling.  The reference's quirks are kept and named where they occur.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "common.cuh"
#include "engine.h"
#include "fft.cuh"
#include "scf.h"

namespace pspw {
namespace {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 296;  // fixed: 2 per SM
constexpr int kMaxRedValues = 8;

FftArg arg_of(const FftDim &d) {
  FftArg a;
  a.n = d.n;
  a.nf = d.nf;
  for (int i = 0; i < kMaxStages; i++) a.rad[i] = d.rad[i];
  return a;
}

// ---------------------------------------------------------------- reductions
// Each block reduces its NV per-thread values with a fixed tree and writes
// part[q * gridDim.x + blockIdx.x].
template <int NV>
__device__ __forceinline__ void block_reduce_store(double (&v)[NV], double *part) {
  __shared__ double sh[NV][kRedThreads];
#pragma unroll
  for (int q = 0; q < NV; q++) sh[q][threadIdx.x] = v[q];
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int q = 0; q < NV; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) part[(size_t)q * gridDim.x + blockIdx.x] = sh[q][0];
}

// out[q] = sum over nb partials of value q (one block, fixed order)
template <int NV>
__global__ void __launch_bounds__(kRedThreads) k_reduce_final(const double *__restrict__ part,
                                                              int nb, double *out) {
  double v[NV];
#pragma unroll
  for (int q = 0; q < NV; q++) {
    double a = 0.0;
    for (int b = threadIdx.x; b < nb; b += kRedThreads) a += part[(size_t)q * nb + b];
    v[q] = a;
  }
  __shared__ double sh[NV][kRedThreads];
#pragma unroll
  for (int q = 0; q < NV; q++) sh[q][threadIdx.x] = v[q];
  __syncthreads();
  for (int w = kRedThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int q = 0; q < NV; q++) sh[q][threadIdx.x] += sh[q][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int q = 0; q < NV; q++) out[q] = sh[q][0];
}

// Reduce the partials of a launch of kRedBlocks blocks into s->h_part[0..NV).
template <int NV>
int finish_reduce(pspw_scf *s, double *out) {
  pspw_cell *c = s->cell;
  double *d_out = s->d_part + kMaxRedValues * kRedBlocks;
  k_reduce_final<NV><<<1, kRedThreads, 0, c->stream>>>(s->d_part, kRedBlocks, d_out);
  c->kernel_launches++;
  PSPW_CUDA(cudaMemcpyAsync(s->h_part, d_out, sizeof(double) * NV, cudaMemcpyDeviceToHost,
                            c->stream));
  PSPW_CUDA(cudaStreamSynchronize(c->stream));
  for (int q = 0; q < NV; q++) out[q] = s->h_part[q];
  return device_status(c);
}

// ---------------------------------------------------------------- grid FFT
// One pass of 1D transforms along AXIS over L consecutive lines.  Lines of
// the y and z passes are numbered with x fastest, so a warp reads
// consecutive addresses at every element position.
template <int AXIS>
__global__ void __launch_bounds__(256) k_grid_pass(double2 *grid, int n1, int n2, int n3,
                                                   FftArg f, const double2 *__restrict__ w,
                                                   int sign, int L, double scale) {
  extern __shared__ double2 gsm[];
  const int n = f.n, ls = n + 1;
  double2 *a = gsm, *b = gsm + L * ls;
  const int nlines = AXIS == 0 ? n2 * n3 : (AXIS == 1 ? n1 * n3 : n1 * n2);
  const int l0 = blockIdx.x * L;
  const int nl = min(L, nlines - l0);
  const size_t stride = AXIS == 0 ? 1 : (AXIS == 1 ? (size_t)n1 : (size_t)n1 * n2);
  auto base = [&](int l) -> size_t {
    if (AXIS == 0) return (size_t)l * n1;
    if (AXIS == 1) return (size_t)(l % n1) + (size_t)(l / n1) * n1 * n2;
    return (size_t)l;
  };
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    int l, i;
    if (AXIS == 0) {
      l = e / n;
      i = e - l * n;
    } else {
      l = e % nl;
      i = e / nl;
    }
    a[l * ls + i] = grid[base(l0 + l) + i * stride];
  }
  __syncthreads();
  const double2 *r = fft_lines(a, b, nl, ls, f, w, sign);
  for (int e = threadIdx.x; e < nl * n; e += blockDim.x) {
    int l, i;
    if (AXIS == 0) {
      l = e / n;
      i = e - l * n;
    } else {
      l = e % nl;
      i = e / nl;
    }
    double2 v = r[l * ls + i];
    if (scale != 1.0) v = make_double2(v.x * scale, v.y * scale);
    grid[base(l0 + l) + i * stride] = v;
  }
}

// ---------------------------------------------------------------- elementwise
__global__ void k_real_to_grid(const double *__restrict__ x, double2 *grid, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    grid[i] = make_double2(x[i], 0.0);
}
__global__ void k_grid_to_real(const double2 *__restrict__ grid, double *x, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    x[i] = grid[i].x;
}

// ---------------------------------------------------------------- EvalEnergy
__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cs(double s, double2 a) { return make_double2(s * a.x, s * a.y); }
__device__ __forceinline__ double2 cj(double2 a) { return make_double2(a.x, -a.y); }

// EvalEnergy.cpp:59-107 for every density G: read the transformed density at
// G, accumulate eh, eh2, eg2, eps, and write vtemp(G) = V_H + V_loc back to
// the same grid point.  Grid points outside the density sphere keep the
// transformed density, as in the reference (it scatters vtemp into c_fft
// without clearing it, EvalEnergy.cpp:115-118).
__global__ void __launch_bounds__(kRedThreads) k_energy_terms(
    const double2 *__restrict__ grid, const int *__restrict__ gidx,
    const double *__restrict__ g, const double2 *__restrict__ vp,
    const double2 *__restrict__ rp, int ng, double tpiba2, double2 *__restrict__ vg,
    double *part) {
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};  // eh, eh2, eg2, eps (re, im)
  const double fourpi = 4.0 * M_PI;
  for (int ig = blockIdx.x * blockDim.x + threadIdx.x; ig < ng; ig += gridDim.x * blockDim.x) {
    const int idx = gidx[ig];
    const double2 rhet = grid[idx];
    const double2 vpg = vp[ig];
    if (ig == 0) {
      const double2 e0 = cm(vpg, cj(rhet));  // eps = vp * conj(c_fft[0])
      v[6] += e0.x;
      v[7] += e0.y;
      vg[ig] = vpg;  // vtemp[0] = vp + vh0, vh0 = 0
      continue;
    }
    const double2 rpg = rp[ig];
    const double2 rhog = make_double2(rhet.x + rpg.x, rhet.y + rpg.y);
    const double2 rhets = cj(rhet), rhogs = cj(rhog), rps = cj(rpg);
    const double fpibg = fourpi / (tpiba2 * g[ig]);
    const double2 vcg = cs(fpibg, rhog);
    const double2 t1 = cm(cs(0.5, vcg), rhogs);
    const double2 t2 = cm(cs(0.5 * fpibg, rhet), rhets);
    const double2 t3 = cm(cs(0.5 * fpibg, rpg), rps);
    const double2 t4 = cm(rhets, vpg);
    v[0] += t1.x;
    v[1] += t1.y;
    v[2] += t2.x;
    v[3] += t2.y;
    v[4] += t3.x;
    v[5] += t3.y;
    v[6] += t4.x;
    v[7] += t4.y;
    vg[ig] = make_double2(vcg.x + vpg.x, vcg.y + vpg.y);
  }
  block_reduce_store<8>(v, part);
}

// c_fft(G) = vtemp(G) in G order (EvalEnergy.cpp:117-119): where density G
// alias onto one grid point the last one's value stays, so only it writes.
// A separate pass after k_energy_terms, which reads every rho(G) first.
__global__ void k_scatter_last(const double2 *__restrict__ vg, const int *__restrict__ gidx,
                               const unsigned char *__restrict__ last, int ng, double2 *grid) {
  for (int ig = blockIdx.x * blockDim.x + threadIdx.x; ig < ng; ig += gridDim.x * blockDim.x)
    if (last[ig]) grid[gidx[ig]] = vg[ig];
}

// ---------------------------------------------------------------- xc_PZ
// Perdew-Zunger LDA of one point (xc_PZ.cpp:24-59): returns v = ux + uc and
// e = ex + ec; zero for r <= 1e-13.  (Callers handle r < -0.1.)
__device__ __forceinline__ void pz_point(double r, double &v, double &e) {
  const double A = -0.1423, B = 1.0529, C = 0.3334;
  const double a = 0.0311, b = -0.0480, c = 0.0020, d = -0.0116;
  if (r <= 1.e-13) {
    v = 0.0;
    e = 0.0;
    return;
  }
  const double ax = -(3.0 / 4.0) * pow(3.0 / 2.0 / M_PI, 2.0 / 3.0);
  const double rs = pow(3.0 / (4.0 * M_PI * r), 1.0 / 3.0);
  const double rrs = sqrt(rs);
  const double ex = ax / rs;
  const double ux = 4.0 / 3.0 * ex;
  double ec, uc;
  if (rs >= 1.0) {
    const double bpr = 1.0 + B * rrs + C * rs;
    ec = A / bpr;
    uc = (1.0 + 7.0 / 6.0 * B * rrs + 4.0 / 3.0 * C * rs) * ec / bpr;
  } else {
    const double rsl = log(rs);
    ec = a * rsl + b + c * rs * rsl + d * rs;
    uc = (2.0 * d - c) / 3.0 * rs + b - a / 3.0 + a * rsl + 2.0 * c / 3.0 * rs * rsl;
  }
  v = ux + uc;
  e = ex + ec;
}

// vxc[i] and the sum of rho[i] (ex + ec).  A point with rho < -0.1 keeps the
// values of the nearest earlier point with rho >= -0.1 (the reference leaves
// its loop variables unchanged there, xc_PZ.cpp:27-30), or zeros if none.
__global__ void __launch_bounds__(kRedThreads) k_xc(const double *__restrict__ rho,
                                                    double *__restrict__ vxc, int n,
                                                    double *part) {
  double v[2] = {0.0, 0.0};  // Exc, count of stale points
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double r = rho[i];
    double vv = 0.0, ee = 0.0;
    if (r < -0.1) {
      v[1] += 1.0;
      for (int j = i - 1; j >= 0; j--) {
        const double rj = rho[j];
        if (rj >= -0.1) {
          pz_point(rj, vv, ee);
          break;
        }
      }
    } else {
      pz_point(r, vv, ee);
    }
    vxc[i] = vv;
    v[0] += r * ee;
  }
  block_reduce_store<2>(v, part);
}

// V_eff = Re(grid) + vxc, written over rho (EvalEnergy.cpp:130-134)
__global__ void k_veff(double *rho, const double2 *__restrict__ grid,
                       const double *__restrict__ vxc, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    rho[i] = grid[i].x + vxc[i];
}

// ---------------------------------------------------------------- NormalizeRho
__global__ void __launch_bounds__(kRedThreads) k_clamp_sum(double *rho, int n, double *part) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double r = rho[i];
    if (r < 0.0) {
      r = 0.0;
      rho[i] = 0.0;
    }
    v[0] += r;
  }
  block_reduce_store<1>(v, part);
}
__global__ void k_scale_ratio(double *rho, int n, double num, double den) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    rho[i] = rho[i] * num / den;
}

// ---------------------------------------------------------------- Kerker
// c(G) *= beta*gg/(gg + q0) for the wavefunction G's only (KerkerRhoMix.cpp:69-72)
__global__ void k_kerker(double2 *grid, const int *__restrict__ wg, const double *__restrict__ xkg,
                         int ngw, double beta, double q0) {
  for (int ig = blockIdx.x * blockDim.x + threadIdx.x; ig < ngw; ig += gridDim.x * blockDim.x) {
    const double gg = xkg[ig];
    const double f = beta * gg / (gg + q0);
    const double2 v = grid[wg[ig]];
    grid[wg[ig]] = make_double2(f * v.x, f * v.y);
  }
}

// ---------------------------------------------------------------- mixers
// sum of (a - b)^2 and a.b-type products over up to 3 vector pairs
__global__ void __launch_bounds__(kRedThreads) k_dots(const double *__restrict__ x0,
                                                      const double *__restrict__ y0,
                                                      const double *__restrict__ x1,
                                                      const double *__restrict__ y1,
                                                      const double *__restrict__ x2,
                                                      const double *__restrict__ y2, int n,
                                                      double *part) {
  double v[3] = {0.0, 0.0, 0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    v[0] += x0[i] * y0[i];
    if (x1) v[1] += x1[i] * y1[i];
    if (x2) v[2] += x2[i] * y2[i];
  }
  block_reduce_store<3>(v, part);
}

// Simple and Kerker mixing, the d sum of (rhoe - rho_old)^2 first
__global__ void __launch_bounds__(kRedThreads) k_diff_sq(const double *__restrict__ a,
                                                         const double *__restrict__ b, int n,
                                                         double *part) {
  double v[1] = {0.0};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double t = a[i] - b[i];
    v[0] += t * t;
  }
  block_reduce_store<1>(v, part);
}

// out = ca*a + cb*b (+ cc*c) elementwise; any of the outputs may alias inputs
// out = ca a + cb b + cc c; b and c may be null (their terms are dropped)
__global__ void k_lin3(double *out, double ca, const double *a, double cb, const double *b,
                       double cc, const double *c, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = ca * a[i];
    if (b) v += cb * b[i];
    if (c) v += cc * c[i];
    out[i] = v;
  }
}

int launch_blocks(int n) { return std::max(1, std::min(4 * 148, (n + 255) / 256)); }

// Small dense solve A x = b (A symmetric, given by its upper triangle, m x m
// column-major), LU with partial pivoting on the full matrix.  Used for the
// Pulay coefficients in place of the reference's dsysv (PulayRhoMix.cpp:69-79).
bool solve_small(int m, std::vector<double> a, std::vector<double> &b) {
  for (int j = 0; j < m; j++)
    for (int i = j + 1; i < m; i++) a[i + (size_t)m * j] = a[j + (size_t)m * i];
  for (int k = 0; k < m; k++) {
    int p = k;
    for (int i = k + 1; i < m; i++)
      if (std::fabs(a[i + (size_t)m * k]) > std::fabs(a[p + (size_t)m * k])) p = i;
    if (a[p + (size_t)m * k] == 0.0) return false;
    if (p != k) {
      for (int j = 0; j < m; j++) std::swap(a[k + (size_t)m * j], a[p + (size_t)m * j]);
      std::swap(b[k], b[p]);
    }
    for (int i = k + 1; i < m; i++) {
      const double l = a[i + (size_t)m * k] / a[k + (size_t)m * k];
      for (int j = k; j < m; j++) a[i + (size_t)m * j] -= l * a[k + (size_t)m * j];
      b[i] -= l * b[k];
    }
  }
  for (int i = m - 1; i >= 0; i--) {
    double t = b[i];
    for (int j = i + 1; j < m; j++) t -= a[i + (size_t)m * j] * b[j];
    b[i] = t / a[i + (size_t)m * i];
  }
  return true;
}

}  // namespace

// ---------------------------------------------------------------- grid FFT
int grid_fft(pspw_cell *c, double2 *grid, int sign) {
  const Basis &B = c->basis;
  const int n[3] = {B.n1, B.n2, B.n3};
  const int nlines[3] = {B.n2 * B.n3, B.n1 * B.n3, B.n1 * B.n2};
  for (int ax = 0; ax < 3; ax++) {
    const FftDim &d = B.dim[ax];
    const FftArg f = arg_of(d);
    const int L = std::max(1, 1536 / (n[ax] + 1));
    const size_t smem = sizeof(double2) * 2 * (size_t)L * (n[ax] + 1);
    const double scale = (sign < 0 && ax == 2) ? 1.0 / (double)B.nnr : 1.0;
    const int nb = (nlines[ax] + L - 1) / L;
    switch (ax) {
      case 0:
        k_grid_pass<0><<<nb, 256, smem, c->stream>>>(grid, B.n1, B.n2, B.n3, f, d.d_w64, sign, L,
                                                     scale);
        break;
      case 1:
        k_grid_pass<1><<<nb, 256, smem, c->stream>>>(grid, B.n1, B.n2, B.n3, f, d.d_w64, sign, L,
                                                     scale);
        break;
      default:
        k_grid_pass<2><<<nb, 256, smem, c->stream>>>(grid, B.n1, B.n2, B.n3, f, d.d_w64, sign, L,
                                                     scale);
    }
    c->kernel_launches++;
  }
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int xc_pz_dev(pspw_scf *s, const double *d_rho, double *d_vxc, double *exc) {
  pspw_cell *c = s->cell;
  const int n = c->basis.nnr;
  k_xc<<<kRedBlocks, kRedThreads, 0, c->stream>>>(d_rho, d_vxc, n, s->d_part);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  double r[2];
  int rc = finish_reduce<2>(s, r);
  if (rc) return rc;
  *exc = r[0];
  return PSPW_OK;
}

int eval_energy_dev(pspw_scf *s, double *d_rho, double ekin, double enl, double *e6) {
  pspw_cell *c = s->cell;
  const int n = c->basis.nnr;
  const int nbl = launch_blocks(n);
  k_real_to_grid<<<nbl, 256, 0, c->stream>>>(d_rho, s->d_grid, n);
  c->kernel_launches++;
  int rc = grid_fft(c, s->d_grid, -1);
  if (rc) return rc;
  k_energy_terms<<<kRedBlocks, kRedThreads, 0, c->stream>>>(s->d_grid, s->d_gidx, s->d_g, s->d_vp,
                                                            s->d_rp, s->ng, c->tpiba2, s->d_vg,
                                                            s->d_part);
  k_scatter_last<<<launch_blocks(s->ng), 256, 0, c->stream>>>(s->d_vg, s->d_gidx, s->d_glast,
                                                              s->ng, s->d_grid);
  c->kernel_launches += 2;
  PSPW_CUDA(cudaGetLastError());
  double t[8];
  if ((rc = finish_reduce<8>(s, t))) return rc;
  if ((rc = grid_fft(c, s->d_grid, +1))) return rc;
  double exc = 0.0;
  if ((rc = xc_pz_dev(s, d_rho, s->d_vxc, &exc))) return rc;
  k_veff<<<nbl, 256, 0, c->stream>>>(d_rho, s->d_grid, s->d_vxc, n);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  // EvalEnergy.cpp:142-147
  const double EXC = exc * s->omega / n;
  const double EHT = t[0] * s->omega + s->esr - s->eself;
  const double EPSEU = t[6] * s->omega;
  const double ETOT = ekin + EHT + EPSEU + enl + EXC;
  e6[0] = ETOT;
  e6[1] = ekin;
  e6[2] = EHT;
  e6[3] = EPSEU;
  e6[4] = enl;
  e6[5] = EXC;
  return PSPW_OK;
}

int normalize_rho_dev(pspw_scf *s, double *d_rho, double omega, double nel, int *warn) {
  pspw_cell *c = s->cell;
  const int n = c->basis.nnr;
  k_clamp_sum<<<kRedBlocks, kRedThreads, 0, c->stream>>>(d_rho, n, s->d_part);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  double sum;
  int rc = finish_reduce<1>(s, &sum);
  if (rc) return rc;
  const double truesum = n * nel / omega;
  if (sum < 1.0e-15) {
    char msg[128];
    std::snprintf(msg, sizeof msg, "NormalizeRho: sum(rho)=%f < %f", sum, 1.0e-15);
    return fail(PSPW_ERR_CHARGE, msg);
  }
  if (warn) *warn = std::fabs(truesum - sum) * omega / n > 1.0e-5 ? 1 : 0;
  k_scale_ratio<<<launch_blocks(n), 256, 0, c->stream>>>(d_rho, n, truesum, sum);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int kerker_prec_dev(pspw_scf *s, double *d_x, double beta, double q0) {
  pspw_cell *c = s->cell;
  const int n = c->basis.nnr, nbl = launch_blocks(n);
  k_real_to_grid<<<nbl, 256, 0, c->stream>>>(d_x, s->d_grid, n);
  int rc = grid_fft(c, s->d_grid, -1);
  if (rc) return rc;
  k_kerker<<<launch_blocks(c->basis.ngw), 256, 0, c->stream>>>(s->d_grid, c->basis.d_wgrid,
                                                               c->basis.d_xkg64, c->basis.ngw,
                                                               beta, q0);
  if ((rc = grid_fft(c, s->d_grid, +1))) return rc;
  k_grid_to_real<<<nbl, 256, 0, c->stream>>>(s->d_grid, d_x, n);
  c->kernel_launches += 3;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

int mix_dev(pspw_scf *s, int iter, double *d_rhoe, double *d_out) {
  pspw_cell *c = s->cell;
  const int n = c->basis.nnr, nbl = launch_blocks(n);
  const double beta = s->mix_beta;
  double *H = s->d_hist, *F = s->d_f, *Gm = s->d_gm;
  auto col = [&](double *base, int j1) { return base + (size_t)(j1 - 1) * n; };  // 1-based column
  auto sum1 = [&](const double *a, const double *b, double *out) -> int {
    k_diff_sq<<<kRedBlocks, kRedThreads, 0, c->stream>>>(a, b, n, s->d_part);
    c->kernel_launches++;
    return finish_reduce<1>(s, out);
  };
  auto dots = [&](const double *x0, const double *y0, const double *x1, const double *y1,
                  const double *x2, const double *y2, double *out3) -> int {
    k_dots<<<kRedBlocks, kRedThreads, 0, c->stream>>>(x0, y0, x1, y1, x2, y2, n, s->d_part);
    c->kernel_launches++;
    return finish_reduce<3>(s, out3);
  };
  auto lin = [&](double *out, double ca, const double *a, double cb, const double *b, double cc,
                 const double *cv) {
    k_lin3<<<nbl, 256, 0, c->stream>>>(out, ca, a, cb, b, cc, cv, n);
    c->kernel_launches++;
  };
  auto copy = [&](double *dst, const double *src) -> int {
    PSPW_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    return PSPW_OK;
  };
  int rc = PSPW_OK;
  double d = 0.0;
  switch (s->mix_kind) {
    case PSPW_MIX_SIMPLE: {  // SimpleRhoMix.cpp
      if ((rc = sum1(d_rhoe, H, &d))) return rc;
      lin(d_rhoe, beta, d_rhoe, 1.0 - beta, H, 0.0, nullptr);
      if ((rc = copy(H, d_rhoe))) return rc;
      d = std::sqrt(d / (double)n);
      break;
    }
    case PSPW_MIX_KERKER: {  // KerkerRhoMix.cpp:5-50: rhoe = rho_old + K(rhoe - rho_old)
      if ((rc = sum1(d_rhoe, H, &d))) return rc;
      lin(s->d_tmp, 1.0, d_rhoe, -1.0, H, 0.0, nullptr);
      if ((rc = kerker_prec_dev(s, s->d_tmp, beta, s->mix_q0))) return rc;
      lin(d_rhoe, 1.0, H, 1.0, s->d_tmp, 0.0, nullptr);
      if ((rc = copy(H, d_rhoe))) return rc;
      d = std::sqrt(d / (double)n);
      break;
    }
    case PSPW_MIX_ANDERSON: {  // AndersonRhoMix.cpp:8-91 (history of 3 columns)
      if (iter == 1) {
        if ((rc = copy(col(H, 1), d_rhoe))) return rc;
        PSPW_CUDA(cudaMemsetAsync(col(F, 1), 0, sizeof(double) * n, c->stream));
        d = 1.0;
        break;
      }
      const int j0 = (iter - 1) % 3 + 1, j1 = (iter - 2) % 3 + 1, j2 = (iter - 3) % 3 + 1;
      lin(col(F, j0), 1.0, d_rhoe, -1.0, col(H, j1), 0.0, nullptr);
      double t3[3];
      if ((rc = dots(col(F, j0), col(F, j0), nullptr, nullptr, nullptr, nullptr, t3))) return rc;
      d = t3[0];
      if (iter == 2) {
        lin(d_rhoe, beta, d_rhoe, 1.0 - beta, col(H, j1), 0.0, nullptr);
        if ((rc = copy(col(H, j0), d_rhoe))) return rc;
        break;  // the reference returns here without the final copy
      }
      lin(col(Gm, 1), 1.0, col(F, j1), -1.0, col(F, j0), 0.0, nullptr);
      if (iter == 3) {
        if ((rc = dots(col(Gm, 1), col(Gm, 1), col(F, j0), col(Gm, 1), nullptr, nullptr, t3)))
          return rc;
        const double d11 = t3[0], r1 = t3[1];
        const double t1 = -r1 / d11;
        // rhoe = (1-t1) rho_old(j1) + t1 rho_old(j2) + beta (f(j0) + t1 g1)
        lin(s->d_tmp, 1.0 - t1, col(H, j1), t1, col(H, j2), 0.0, nullptr);
        lin(d_rhoe, 1.0, s->d_tmp, beta, col(F, j0), beta * t1, col(Gm, 1));
      } else {
        lin(col(Gm, 2), 1.0, col(F, j2), -1.0, col(F, j0), 0.0, nullptr);
        double a3[3], b3[3];
        if ((rc = dots(col(Gm, 1), col(Gm, 1), col(F, j0), col(Gm, 1), col(Gm, 2), col(Gm, 2),
                       a3)))
          return rc;
        if ((rc = dots(col(Gm, 1), col(Gm, 2), col(F, j0), col(Gm, 2), nullptr, nullptr, b3)))
          return rc;
        const double d11 = a3[0], r1 = a3[1], d22 = a3[2], d12 = b3[0], r2 = b3[1];
        double t1 = d11 * d22;
        double t2 = t1 - d12 * d12;
        if (std::fabs(t2) > std::fabs(t1) * 1.0e-8) {
          const double u1 = (-r1 * d22 + r2 * d12) / t2;
          const double u2 = (r1 * d12 - r2 * d11) / t2;
          t1 = u1;
          t2 = u2;
        } else {
          t1 = 0.0;
          t2 = 0.0;
        }
        // the reference adds t2*g(:,1), not t2*g(:,2) (AndersonRhoMix.cpp:76)
        lin(s->d_tmp, 1.0 - t1 - t2, col(H, j1), t1, col(H, j2), t2, col(H, j0));
        lin(d_rhoe, 1.0, s->d_tmp, beta, col(F, j0), beta * (t1 + t2), col(Gm, 1));
      }
      if ((rc = copy(col(H, j0), d_rhoe))) return rc;
      break;
    }
    case PSPW_MIX_PULAY: {  // PulayRhoMix.cpp:5-91 (beta 0.25 in the reference)
      const int mixdim = s->mixdim;
      if (iter < mixdim) {
        // rhoe = beta rhoe + (1-beta) rho_old(iter); f(iter+1) = rhoe - rho_old(iter)
        lin(d_rhoe, beta, d_rhoe, 1.0 - beta, col(H, iter), 0.0, nullptr);
        lin(col(F, iter + 1), 1.0, d_rhoe, -1.0, col(H, iter), 0.0, nullptr);
        if ((rc = kerker_prec_dev(s, col(F, iter + 1), 1.0, s->mix_q0))) return rc;
        if ((rc = copy(col(H, iter + 1), d_rhoe))) return rc;
        double t3[3];
        if ((rc = dots(col(F, iter + 1), col(F, iter + 1), nullptr, nullptr, nullptr, nullptr, t3)))
          return rc;
        d = std::sqrt(t3[0] / (double)n);
        break;
      }
      const int jc = iter % mixdim + 1, jn = (iter + 1) % mixdim + 1;
      const int m = std::min(iter + 1, mixdim) + 1;
      lin(col(F, jc), 1.0, d_rhoe, -1.0, col(H, jc), 0.0, nullptr);
      if ((rc = kerker_prec_dev(s, col(F, jc), 1.0, s->mix_q0))) return rc;
      double t3[3];
      if ((rc = dots(col(F, jc), col(F, jc), nullptr, nullptr, nullptr, nullptr, t3))) return rc;
      d = std::sqrt(t3[0] / (double)n);
      std::vector<double> a((size_t)m * m, 0.0), alpha(m, 0.0);
      for (int i = 1; i <= m - 1; i++) {
        for (int j = i; j <= m - 1; j++) {
          if ((rc = dots(col(F, i), col(F, j), nullptr, nullptr, nullptr, nullptr, t3))) return rc;
          a[(i - 1) + (size_t)m * (j - 1)] = t3[0];
        }
        a[(i - 1) + (size_t)m * (m - 1)] = 1.0;
      }
      alpha[m - 1] = 1.0;
      if (!solve_small(m, a, alpha)) return fail(PSPW_ERR_LAPACK, "PulayRhoMix: singular system");
      PSPW_CUDA(cudaMemsetAsync(d_rhoe, 0, sizeof(double) * n, c->stream));
      for (int j = 1; j <= m - 1; j++)
        lin(d_rhoe, 1.0, d_rhoe, alpha[j - 1], col(H, j), alpha[j - 1], col(F, j));
      int warn = 0;
      if ((rc = normalize_rho_dev(s, d_rhoe, s->omega, s->nel, &warn))) return rc;
      if ((rc = copy(col(H, jn), d_rhoe))) return rc;
      break;
    }
    case PSPW_MIX_BROYDEN: {
      // BroydenRhoMix.cpp:10-104 with alpha = beta (0.25) and w0 = 0.01 as
      // the ChebySCF loop calls it (ChebySCFLoop.cpp:240,336).  H: rho_old
      // (2 columns), F: f (2 columns), Gm: df (mixdim columns) then u.
      const int mixdim = s->mixdim;
      const double w0 = 0.01;
      double *DF = Gm, *U = Gm + (size_t)mixdim * n;
      const int m = std::min(iter + 1, mixdim);
      const int jc = iter % m + 1, kp = (iter - 1) % 2 + 1, kc = iter % 2 + 1;
      lin(col(F, kc), 1.0, d_rhoe, -1.0, col(H, kp), 0.0, nullptr);
      double t3[3];
      if ((rc = dots(col(F, kc), col(F, kc), nullptr, nullptr, nullptr, nullptr, t3))) return rc;
      d = std::sqrt(t3[0] / (double)n);
      lin(col(DF, jc), 1.0, col(F, kc), -1.0, col(F, kp), 0.0, nullptr);
      if ((rc = dots(col(DF, jc), col(DF, jc), nullptr, nullptr, nullptr, nullptr, t3))) return rc;
      double t1 = std::sqrt(t3[0]);
      if (t1 > 1.e-8) t1 = 1.0 / t1;  // a norm below 1e-8 is used as it is (:45-46)
      lin(col(DF, jc), t1, col(DF, jc), 0.0, col(DF, jc), 0.0, nullptr);
      lin(s->d_tmp, 1.0, col(H, kp), -1.0, col(H, kc), 0.0, nullptr);
      lin(col(U, jc), beta, col(DF, jc), t1, s->d_tmp, 0.0, nullptr);
      std::vector<double> cvec(m), &A = s->mix_a;
      for (int k = 1; k <= m; k++) {
        if ((rc = dots(col(DF, k), col(F, kc), col(DF, jc), col(DF, k), nullptr, nullptr, t3)))
          return rc;
        cvec[k - 1] = t3[0];
        A[(k - 1) + (size_t)mixdim * (jc - 1)] = t3[1];
        A[(jc - 1) + (size_t)mixdim * (k - 1)] = t3[1];
      }
      // gamma = c^T beta^-1 with beta = a + w0^2 I (m x m), symmetric
      std::vector<double> bm((size_t)m * m);
      for (int j = 0; j < m; j++)
        for (int i = 0; i < m; i++)
          bm[i + (size_t)m * j] = A[i + (size_t)mixdim * j] + (i == j ? w0 * w0 : 0.0);
      std::vector<double> gamma = cvec;
      if (!solve_small(m, bm, gamma)) return fail(PSPW_ERR_LAPACK, "BroydenRhoMix: singular beta");
      lin(d_rhoe, 1.0, col(H, kp), beta, col(F, kc), 0.0, nullptr);
      for (int l = 1; l <= m; l++) lin(d_rhoe, 1.0, d_rhoe, -gamma[l - 1], col(U, l), 0.0, nullptr);
      if ((rc = copy(col(H, kc), d_rhoe))) return rc;
      break;
    }
    default:
      return fail(PSPW_ERR_ARG, "mix: mixer not initialised (pspw_mix_init)");
  }
  PSPW_CUDA(cudaGetLastError());
  if (d_out) *d_out = d;
  return PSPW_OK;
}

}  // namespace pspw

using namespace pspw;

extern "C" {

int pspw_scf_create(pspw_cell *c, int ng, const int *n1, const int *n2, const int *n3,
                    const double *g, int nsp, const double *sfac, const double *vps,
                    const double *rhops, double omega, double nel, double esr, double eself,
                    pspw_scf **out) {
  if (!c || !out || ng < 1 || nsp < 0 || !n1 || !n2 || !n3 || !g ||
      (nsp > 0 && (!sfac || !vps || !rhops)))
    return fail(PSPW_ERR_ARG, "scf_create: bad argument");
  *out = nullptr;
  PSPW_CUDA(cudaSetDevice(c->device));
  const Basis &B = c->basis;
  std::vector<int> gidx(ng);
  std::vector<double2> vp(ng), rp(ng);
  for (int ig = 0; ig < ng; ig++) {
    const int i1 = n1[ig] - 1, i2 = n2[ig] - 1, i3 = n3[ig] - 1;  // 1-based grid indices
    if (i1 < 0 || i1 >= B.n1 || i2 < 0 || i2 >= B.n2 || i3 < 0 || i3 >= B.n3)
      return fail(PSPW_ERR_SHAPE, "scf_create: G index outside the grid");
    gidx[ig] = i1 + B.n1 * (i2 + B.n2 * i3);
    // vp, rp = sum over species in order (EvalEnergy.cpp:63-70)
    double vr = 0.0, vi = 0.0, rr = 0.0, ri = 0.0;
    for (int is = 0; is < nsp; is++) {
      const size_t k = (size_t)is + (size_t)nsp * ig;  // SFAC(is, ig), NSP leading
      const double sr = sfac[2 * k], si = sfac[2 * k + 1];
      vr = vr + sr * vps[k];
      vi = vi + si * vps[k];
      rr = rr + sr * rhops[k];
      ri = ri + si * rhops[k];
    }
    vp[ig] = make_double2(vr, vi);
    rp[ig] = make_double2(rr, ri);
  }
  if (gidx[0] != 0) return fail(PSPW_ERR_SHAPE, "scf_create: the first G must be G = 0");
  // the last density G on each grid point (aliasing on small grids)
  std::vector<unsigned char> glast(ng, 0);
  {
    std::vector<int> last_of(B.nnr, -1);
    for (int ig = 0; ig < ng; ig++) last_of[gidx[ig]] = ig;
    for (int ig = 0; ig < ng; ig++) glast[ig] = last_of[gidx[ig]] == ig;
  }
  pspw_scf *s = new pspw_scf;
  s->cell = c;
  s->device = c->device;
  s->ng = ng;
  s->nsp = nsp;
  s->omega = omega;
  s->nel = nel;
  s->esr = esr;
  s->eself = eself;
  const size_t nnr = B.nnr;
  bool ok = cudaMalloc(&s->d_gidx, sizeof(int) * ng) == cudaSuccess &&
            cudaMalloc(&s->d_g, sizeof(double) * ng) == cudaSuccess &&
            cudaMalloc(&s->d_vp, sizeof(double2) * ng) == cudaSuccess &&
            cudaMalloc(&s->d_rp, sizeof(double2) * ng) == cudaSuccess &&
            cudaMalloc(&s->d_glast, ng) == cudaSuccess &&
            cudaMalloc(&s->d_vg, sizeof(double2) * ng) == cudaSuccess &&
            cudaMalloc(&s->d_grid, sizeof(double2) * nnr) == cudaSuccess &&
            cudaMalloc(&s->d_vxc, sizeof(double) * nnr) == cudaSuccess &&
            cudaMalloc(&s->d_tmp, sizeof(double) * nnr) == cudaSuccess &&
            cudaMalloc(&s->d_part, sizeof(double) * (kMaxRedValues * kRedBlocks + 16)) ==
                cudaSuccess &&
            cudaMallocHost(&s->h_part, sizeof(double) * 16) == cudaSuccess;
  if (ok)
    ok = cudaMemcpy(s->d_gidx, gidx.data(), sizeof(int) * ng, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(s->d_glast, glast.data(), ng, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(s->d_g, g, sizeof(double) * ng, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(s->d_vp, vp.data(), sizeof(double2) * ng, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(s->d_rp, rp.data(), sizeof(double2) * ng, cudaMemcpyHostToDevice) == cudaSuccess &&
         // the copies' DMA lands before any kernel on the (non-blocking)
         // cell streams reads the tables
         cudaStreamSynchronize(cudaStreamLegacy) == cudaSuccess;
  if (!ok) {
    pspw_scf_destroy(s);
    return fail(PSPW_ERR_OOM, "scf_create: device memory");
  }
  *out = s;
  return PSPW_OK;
}

int pspw_scf_destroy(pspw_scf *s) {
  if (!s) return PSPW_OK;
  // the cell may already be gone (a garbage collector finalises handles in
  // any order): only the device id is read, and the whole device is
  // synchronised instead of the cell's stream
  cudaSetDevice(s->device);
  cudaDeviceSynchronize();
  void *p[] = {s->d_gidx, s->d_glast, s->d_vg, s->d_g, s->d_vp, s->d_rp, s->d_grid, s->d_vxc,
               s->d_tmp,  s->d_part, s->d_hist, s->d_f, s->d_gm};
  for (void *q : p)
    if (q) cudaFree(q);
  if (s->h_part) cudaFreeHost(s->h_part);
  delete s;
  return PSPW_OK;
}

namespace {
int scf_enter(pspw_scf *s) {
  if (!s) return fail(PSPW_ERR_ARG, "null scf handle");
  PSPW_CUDA(cudaSetDevice(s->cell->device));
  return PSPW_OK;
}
int up(pspw_scf *s, double *d, const double *h) {
  PSPW_CUDA(cudaMemcpyAsync(d, h, sizeof(double) * s->cell->basis.nnr, cudaMemcpyHostToDevice,
                            s->cell->stream));
  return PSPW_OK;
}
int down(pspw_scf *s, double *h, const double *d) {
  PSPW_CUDA(cudaMemcpyAsync(h, d, sizeof(double) * s->cell->basis.nnr, cudaMemcpyDeviceToHost,
                            s->cell->stream));
  PSPW_CUDA(cudaStreamSynchronize(s->cell->stream));
  return device_status(s->cell);
}
// a device NNR vector of the cell's workspace for the host-buffer entry points
int host_vec(pspw_scf *s, int slot, double **d) {
  return ws_reserve(s->cell, slot, sizeof(double) * s->cell->basis.nnr, (void **)d);
}
constexpr int kSlotScfA = kWsScfA;
constexpr int kSlotScfB = kWsScfB;
}  // namespace

int pspw_eval_energy_dev(pspw_scf *s, double *d_rhoe, double ekin, double enl, double *e6) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (!d_rhoe || !e6) return fail(PSPW_ERR_ARG, "eval_energy: null argument");
  return eval_energy_dev(s, d_rhoe, ekin, enl, e6);
}

int pspw_eval_energy(pspw_scf *s, double *rhoe, double ekin, double enl, double *e6) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (!rhoe || !e6) return fail(PSPW_ERR_ARG, "eval_energy: null argument");
  double *d;
  if ((rc = host_vec(s, kSlotScfA, &d)) || (rc = up(s, d, rhoe)) ||
      (rc = eval_energy_dev(s, d, ekin, enl, e6)))
    return rc;
  return down(s, rhoe, d);
}

int pspw_xc_pz(pspw_scf *s, const double *rho, double *vxc, double *exc) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (!rho || !vxc || !exc) return fail(PSPW_ERR_ARG, "xc_pz: null argument");
  double *d, *dv;
  if ((rc = host_vec(s, kSlotScfA, &d)) || (rc = host_vec(s, kSlotScfB, &dv)) ||
      (rc = up(s, d, rho)) || (rc = xc_pz_dev(s, d, dv, exc)))
    return rc;
  return down(s, vxc, dv);
}

int pspw_normalize_rho(pspw_scf *s, double *rho, int *warn) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (!rho) return fail(PSPW_ERR_ARG, "normalize_rho: null argument");
  double *d;
  if ((rc = host_vec(s, kSlotScfA, &d)) || (rc = up(s, d, rho)) ||
      (rc = normalize_rho_dev(s, d, s->omega, s->nel, warn)))
    return rc;
  return down(s, rho, d);
}

int pspw_xc_pz_dev(pspw_scf *s, const double *d_rho, double *d_vxc, double *exc) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (!d_rho || !d_vxc || !exc) return fail(PSPW_ERR_ARG, "xc_pz: null argument");
  return xc_pz_dev(s, d_rho, d_vxc, exc);
}

int pspw_normalize_rho_dev(pspw_scf *s, double *d_rho, int *warn) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (!d_rho) return fail(PSPW_ERR_ARG, "normalize_rho: null argument");
  return normalize_rho_dev(s, d_rho, s->omega, s->nel, warn);
}

int pspw_kerker_prec_dev(pspw_scf *s, double *d_x, double beta, double q0) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (!d_x) return fail(PSPW_ERR_ARG, "kerker_prec: null argument");
  if ((rc = kerker_prec_dev(s, d_x, beta, q0))) return rc;
  PSPW_CUDA(cudaStreamSynchronize(s->cell->stream));
  return device_status(s->cell);
}

int pspw_kerker_prec(pspw_scf *s, double *x, double beta, double q0) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (!x) return fail(PSPW_ERR_ARG, "kerker_prec: null argument");
  double *d;
  if ((rc = host_vec(s, kSlotScfA, &d)) || (rc = up(s, d, x)) ||
      (rc = kerker_prec_dev(s, d, beta, q0)))
    return rc;
  return down(s, x, d);
}

int pspw_mix_init(pspw_scf *s, int kind, int mixdim, double beta, double q0,
                  const double *rho_old) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (kind < PSPW_MIX_SIMPLE || kind > PSPW_MIX_BROYDEN ||
      ((kind == PSPW_MIX_PULAY || kind == PSPW_MIX_BROYDEN) && mixdim < 2))
    return fail(PSPW_ERR_ARG, "mix_init: unknown mixer or MIXDIM < 2");
  const size_t n = s->cell->basis.nnr;
  const int ncol = kind == PSPW_MIX_PULAY ? mixdim
                   : kind == PSPW_MIX_ANDERSON ? 3
                   : kind == PSPW_MIX_BROYDEN ? 2 : 1;
  const int ngm = kind == PSPW_MIX_BROYDEN ? 2 * mixdim : 2;
  for (double **p : {&s->d_hist, &s->d_f, &s->d_gm})
    if (*p) {
      cudaFree(*p);
      *p = nullptr;
    }
  if (cudaMalloc(&s->d_hist, sizeof(double) * n * ncol) != cudaSuccess ||
      cudaMalloc(&s->d_f, sizeof(double) * n * ncol) != cudaSuccess ||
      cudaMalloc(&s->d_gm, sizeof(double) * n * ngm) != cudaSuccess)
    return fail(PSPW_ERR_OOM, "mix_init: device memory");
  s->mix_a.assign((size_t)std::max(mixdim, 1) * std::max(mixdim, 1), 0.0);
  // the reference's history arrays start at zero (ChebySCFLoop.cpp:123-148)
  PSPW_CUDA(cudaMemsetAsync(s->d_hist, 0, sizeof(double) * n * ncol, s->cell->stream));
  PSPW_CUDA(cudaMemsetAsync(s->d_f, 0, sizeof(double) * n * ncol, s->cell->stream));
  PSPW_CUDA(cudaMemsetAsync(s->d_gm, 0, sizeof(double) * n * ngm, s->cell->stream));
  if (rho_old && (rc = up(s, s->d_hist, rho_old))) return rc;
  s->mix_kind = kind;
  s->mixdim = mixdim;
  s->mix_beta = beta;
  s->mix_q0 = q0;
  PSPW_CUDA(cudaStreamSynchronize(s->cell->stream));
  return PSPW_OK;
}

int pspw_mix_dev(pspw_scf *s, int iter, double *d_rhoe, double *d) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (!d_rhoe || iter < 1) return fail(PSPW_ERR_ARG, "mix: bad argument");
  return mix_dev(s, iter, d_rhoe, d);
}

int pspw_mix(pspw_scf *s, int iter, double *rhoe, double *d) {
  int rc = scf_enter(s);
  if (rc) return rc;
  if (!rhoe || iter < 1) return fail(PSPW_ERR_ARG, "mix: bad argument");
  double *dv;
  if ((rc = host_vec(s, kSlotScfA, &dv)) || (rc = up(s, dv, rhoe)) ||
      (rc = mix_dev(s, iter, dv, d)))
    return rc;
  return down(s, rhoe, dv);
}

}  // extern "C"
