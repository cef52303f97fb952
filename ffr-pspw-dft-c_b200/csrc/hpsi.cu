// Block H*psi on the device (the work of ApplyHam_block.cpp:5-172).
//
// Local part: the scatter -> inverse 3D FFT -> V_eff -> forward 3D FFT ->
// gather chain of ApplyHam_block.cpp:33-61, done as five passes that only
// touch the part of the grid the wavefunction sphere can reach:
//   1 sticks_inv   gather psi(G) of each stick (an (i1,i2) column holding
//                  sphere G's) into shared memory, inverse FFT along z,
//                  write the stick buffer S[band][z][stick]
//   2 planes_inv   for each z and a tile of active x: read the y line from S
//                  (zero where no stick), inverse FFT along y, write the
//                  plane buffer P[band][z][y][active x]
//   3 xlines       for each (y,z): expand the active x into the full x line,
//                  inverse FFT along x, multiply by V_eff/NNR, forward FFT
//                  along x, keep the active x -- V_eff is applied between the
//                  last inverse and the first forward pass
//   4 planes_fwd   forward FFT along y, keep the stick positions, write S
//   5 sticks_fwd   forward FFT along z, pick the sphere G's, add the kinetic
//                  term 0.5*XKG*TPIBA2*psi
// The 1/NNR of the forward transform (fft_fftw3.cpp:27) is folded into V.
//
// Nonlocal part (ApplyHam_block.cpp:68-165): with beta_p(G) =
// EIGR(G,a_p)*PKG_A(lm_p,G), the reference adds beta W beta^H psi (zdotu
// against conj(EIGR)*PKG_A, back-projection with EIGR*PKG_A).  Here that is
// two complex GEMMs.  FP32: on the tensor cores (nl_tc.cu) for one species,
// otherwise SIMT kernels whose beta operand is generated from EIGR and PKG_A
// while it is loaded, never stored: projection (split over G, partial sums
// reduced in a fixed order, so results are deterministic) and
// back-projection, whose epilogue also applies out = a*(H psi) + b*psi + g*x,
// the update of the Chebyshev three-term recurrence (chebyfilt.cpp:36-59).
// FP64: beta stored once per cell (NGW x nproj) and both products on the
// engine's FP64 tensor-core GEMM (gemm.cu, DMMA), the recurrence as a
// separate pass; the allocation-free entry point keeps the SIMT kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "common.cuh"
#include "dense.h"
#include "engine.h"
#include "fft.cuh"
#include "fftpath.h"
#include "gemm.h"
#include "nl_tc.h"

namespace pspw {

namespace {

constexpr int kNT = 256;        // threads per FFT-pass block
constexpr int kTileElems = 2048;  // complex elements per FFT-pass tile

struct Geo {
  int n1, n2, n3, ncol, nxa, ngw;
  const int *col_start, *sg_ig, *sg_z, *sg_col, *col_of_xy, *xa_list, *xa_of_x;
};

__host__ __device__ __forceinline__ int pad(int n) { return n + 1; }

FftArg fft_arg(const FftDim &d) {
  FftArg a;
  a.n = d.n;
  a.nf = d.nf;
  for (int i = 0; i < kMaxStages; i++) a.rad[i] = d.rad[i];
  return a;
}

template <typename T>
const T *tw(const FftDim &d);
template <>
const double2 *tw<double2>(const FftDim &d) {
  return d.d_w64;
}
template <>
const float2 *tw<float2>(const FftDim &d) {
  return d.d_w32;
}

// ---------------------------------------------------------------- pass 1
template <typename T>
__global__ void __launch_bounds__(kNT) k_sticks_inv(Geo g, FftArg fz, const T *__restrict__ wz,
                                                    const T *__restrict__ psi, int ld, int ngw_call,
                                                    T *__restrict__ S, int T1) {
  extern __shared__ unsigned char smem_raw[];
  T *a = reinterpret_cast<T *>(smem_raw);
  const int ls = pad(g.n3);
  T *b = a + T1 * ls;
  const int c0 = blockIdx.x * T1;
  const int band = blockIdx.y;
  const int nc = min(T1, g.ncol - c0);
  for (int e = threadIdx.x; e < T1 * ls; e += blockDim.x) a[e] = czero<T>();
  __syncthreads();
  const T *pb = psi + (size_t)band * ld;
  const int k0 = g.col_start[c0], k1 = g.col_start[c0 + nc];
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    const int ig = g.sg_ig[k];
    if (ig < ngw_call) a[(g.sg_col[k] - c0) * ls + g.sg_z[k]] = pb[ig];
  }
  __syncthreads();
  T *r = fft_lines(a, b, T1, ls, fz, wz, +1);
  T *Sb = S + (size_t)band * g.n3 * g.ncol;
  for (int e = threadIdx.x; e < T1 * g.n3; e += blockDim.x) {
    const int z = e / T1, t = e - z * T1;
    if (t < nc) Sb[(size_t)z * g.ncol + c0 + t] = r[t * ls + z];
  }
}

// ---------------------------------------------------------------- pass 2
template <typename T>
__global__ void __launch_bounds__(kNT) k_planes_inv(Geo g, FftArg fy, const T *__restrict__ wy,
                                                    const T *__restrict__ S, T *__restrict__ P,
                                                    int T2) {
  extern __shared__ unsigned char smem_raw[];
  T *a = reinterpret_cast<T *>(smem_raw);
  const int ls = pad(g.n2);
  T *b = a + T2 * ls;
  const int x0 = blockIdx.x * T2;
  const int z = blockIdx.y;
  const int band = blockIdx.z;
  const int nx = min(T2, g.nxa - x0);
  const T *Sz = S + ((size_t)band * g.n3 + z) * g.ncol;
  for (int e = threadIdx.x; e < T2 * g.n2; e += blockDim.x) {
    const int y = e / T2, t = e - y * T2;
    T v = czero<T>();
    if (t < nx) {
      const int c = g.col_of_xy[g.xa_list[x0 + t] + g.n1 * y];
      if (c >= 0) v = Sz[c];
    }
    a[t * ls + y] = v;
  }
  __syncthreads();
  T *r = fft_lines(a, b, T2, ls, fy, wy, +1);
  T *Pz = P + ((size_t)band * g.n3 + z) * g.n2 * g.nxa;
  for (int e = threadIdx.x; e < T2 * g.n2; e += blockDim.x) {
    const int y = e / T2, t = e - y * T2;
    if (t < nx) Pz[(size_t)y * g.nxa + x0 + t] = r[t * ls + y];
  }
}

// ---------------------------------------------------------------- pass 3
template <typename T, typename R>
__global__ void __launch_bounds__(kNT) k_xlines(Geo g, FftArg fx, const T *__restrict__ wx,
                                                const R *__restrict__ vs, T *__restrict__ P,
                                                int L3) {
  extern __shared__ unsigned char smem_raw[];
  T *a = reinterpret_cast<T *>(smem_raw);
  const int ls = pad(g.n1);
  T *b = a + L3 * ls;
  const int l0 = blockIdx.x * L3;
  const int band = blockIdx.y;
  const int nlines = g.n2 * g.n3;
  const int nl = min(L3, nlines - l0);
  T *Pb = P + (size_t)band * nlines * g.nxa;
  for (int e = threadIdx.x; e < L3 * g.n1; e += blockDim.x) {
    const int l = e / g.n1, x = e - l * g.n1;
    T v = czero<T>();
    if (l < nl) {
      const int xa = g.xa_of_x[x];
      if (xa >= 0) v = Pb[(size_t)(l0 + l) * g.nxa + xa];
    }
    a[l * ls + x] = v;
  }
  __syncthreads();
  T *r = fft_lines(a, b, L3, ls, fx, wx, +1);
  T *o = (r == a) ? b : a;
  for (int e = threadIdx.x; e < L3 * g.n1; e += blockDim.x) {
    const int l = e / g.n1, x = e - l * g.n1;
    const R v = (l < nl) ? vs[(size_t)(l0 + l) * g.n1 + x] : (R)0;
    const T u = r[l * ls + x];
    r[l * ls + x] = mk<T>(v * u.x, v * u.y);
  }
  __syncthreads();
  r = fft_lines(r, o, L3, ls, fx, wx, -1);
  for (int e = threadIdx.x; e < L3 * g.nxa; e += blockDim.x) {
    const int l = e / g.nxa, xa = e - l * g.nxa;
    if (l < nl) Pb[(size_t)(l0 + l) * g.nxa + xa] = r[l * ls + g.xa_list[xa]];
  }
}

// ---------------------------------------------------------------- density
// EvalRhoPsi on the generic path: after the stick and plane passes, each
// block takes L3 x-lines of every band of the batch in band order, inverse-
// transforms them and accumulates w_b |psi_b(r)|^2 in FP64; one block owns
// each line, so rho is updated band after band in the reference's order
// (EvalRhoPsi.cpp:136-149) with no atomics.
template <typename T>
__global__ void __launch_bounds__(kNT) k_xlines_rho(Geo g, FftArg fx, const T *__restrict__ wx,
                                                    const T *__restrict__ P, int nbb,
                                                    const double *__restrict__ wband,
                                                    double *__restrict__ rho, int L3) {
  extern __shared__ unsigned char smem_raw[];
  T *a = reinterpret_cast<T *>(smem_raw);
  const int ls = pad(g.n1);
  T *b = a + L3 * ls;
  double *acc = reinterpret_cast<double *>(b + L3 * ls);
  const int l0 = blockIdx.x * L3;
  const int nlines = g.n2 * g.n3;
  const int nl = min(L3, nlines - l0);
  for (int e = threadIdx.x; e < L3 * g.n1; e += blockDim.x) acc[e] = 0.0;
  for (int band = 0; band < nbb; band++) {
    const T *Pb = P + (size_t)band * nlines * g.nxa;
    __syncthreads();
    for (int e = threadIdx.x; e < L3 * g.n1; e += blockDim.x) {
      const int l = e / g.n1, x = e - l * g.n1;
      T v = czero<T>();
      if (l < nl) {
        const int xa = g.xa_of_x[x];
        if (xa >= 0) v = Pb[(size_t)(l0 + l) * g.nxa + xa];
      }
      a[l * ls + x] = v;
    }
    __syncthreads();
    const T *r = fft_lines(a, b, L3, ls, fx, wx, +1);
    const double w = wband[band];
    for (int e = threadIdx.x; e < L3 * g.n1; e += blockDim.x) {
      const int l = e / g.n1, x = e - l * g.n1;
      const T v = r[l * ls + x];
      acc[e] += w * ((double)v.x * (double)v.x + (double)v.y * (double)v.y);
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < L3 * g.n1; e += blockDim.x) {
    const int l = e / g.n1, x = e - l * g.n1;
    if (l < nl) rho[(size_t)(l0 + l) * g.n1 + x] += acc[e];
  }
}

// ---------------------------------------------------------------- pass 4
template <typename T>
__global__ void __launch_bounds__(kNT) k_planes_fwd(Geo g, FftArg fy, const T *__restrict__ wy,
                                                    const T *__restrict__ P, T *__restrict__ S,
                                                    int T2) {
  extern __shared__ unsigned char smem_raw[];
  T *a = reinterpret_cast<T *>(smem_raw);
  const int ls = pad(g.n2);
  T *b = a + T2 * ls;
  const int x0 = blockIdx.x * T2;
  const int z = blockIdx.y;
  const int band = blockIdx.z;
  const int nx = min(T2, g.nxa - x0);
  const T *Pz = P + ((size_t)band * g.n3 + z) * g.n2 * g.nxa;
  for (int e = threadIdx.x; e < T2 * g.n2; e += blockDim.x) {
    const int y = e / T2, t = e - y * T2;
    a[t * ls + y] = (t < nx) ? Pz[(size_t)y * g.nxa + x0 + t] : czero<T>();
  }
  __syncthreads();
  T *r = fft_lines(a, b, T2, ls, fy, wy, -1);
  T *Sz = S + ((size_t)band * g.n3 + z) * g.ncol;
  for (int e = threadIdx.x; e < T2 * g.n2; e += blockDim.x) {
    const int y = e / T2, t = e - y * T2;
    if (t < nx) {
      const int c = g.col_of_xy[g.xa_list[x0 + t] + g.n1 * y];
      if (c >= 0) Sz[c] = r[t * ls + y];
    }
  }
}

// ---------------------------------------------------------------- pass 5
template <typename T, typename R>
__global__ void __launch_bounds__(kNT) k_sticks_fwd(Geo g, FftArg fz, const T *__restrict__ wz,
                                                    const T *__restrict__ S,
                                                    const R *__restrict__ kin,
                                                    const T *__restrict__ psi, int ld,
                                                    T *__restrict__ out, int ldo, int ngw_call,
                                                    int T1) {
  extern __shared__ unsigned char smem_raw[];
  T *a = reinterpret_cast<T *>(smem_raw);
  const int ls = pad(g.n3);
  T *b = a + T1 * ls;
  const int c0 = blockIdx.x * T1;
  const int band = blockIdx.y;
  const int nc = min(T1, g.ncol - c0);
  const T *Sb = S + (size_t)band * g.n3 * g.ncol;
  for (int e = threadIdx.x; e < T1 * g.n3; e += blockDim.x) {
    const int z = e / T1, t = e - z * T1;
    a[t * ls + z] = (t < nc) ? Sb[(size_t)z * g.ncol + c0 + t] : czero<T>();
  }
  __syncthreads();
  T *r = fft_lines(a, b, T1, ls, fz, wz, -1);
  const T *pb = psi + (size_t)band * ld;
  T *ob = out + (size_t)band * ldo;
  const int k0 = g.col_start[c0], k1 = g.col_start[c0 + nc];
  for (int k = k0 + threadIdx.x; k < k1; k += blockDim.x) {
    const int ig = g.sg_ig[k];
    if (ig < ngw_call) {
      const R kk = kin[ig];
      const T p = pb[ig];
      const T f = r[(g.sg_col[k] - c0) * ls + g.sg_z[k]];
      ob[ig] = mk<T>(kk * p.x + f.x, kk * p.y + f.y);
    }
  }
}

// ---------------------------------------------------------------- nonlocal
constexpr int kBM = 64, kBN = 64;

struct ProjArg {
  const void *eigr;  // cx<R>[nat][ngw]
  const void *pkga;  // R[nsp][ngw][4]
  const int *patom, *psp, *plm;
  const void *pw;  // R[nproj]
  int ngw_cell, nproj;
};

template <typename R>
__device__ __forceinline__ cx<R> beta_at(const ProjArg &pa, int ig, int p) {
  const cx<R> e = reinterpret_cast<const cx<R> *>(pa.eigr)[(size_t)pa.patom[p] * pa.ngw_cell + ig];
  const R f = reinterpret_cast<const R *>(pa.pkga)[((size_t)pa.psp[p] * pa.ngw_cell + ig) * 4 + pa.plm[p]];
  return mk<cx<R>>(e.x * f, e.y * f);
}

// part[(split*nb + b)*nproj + p] = sum_{ig in split} conj(beta_p(ig)) psi_b(ig)
template <typename R, int BK>
__global__ void __launch_bounds__(256) k_proj(ProjArg pa, const cx<R> *__restrict__ psi, int ld,
                                              int ngw, int nb, int kchunk, cx<R> *__restrict__ part) {
  using T = cx<R>;
  __shared__ T As[BK][kBM + 1];
  __shared__ T Bs[BK][kBN + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int p0 = blockIdx.x * kBM, b0 = blockIdx.y * kBN;
  const int kb = blockIdx.z * kchunk;
  const int ke = min(ngw, kb + kchunk);
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = czero<T>();
  for (int k0 = kb; k0 < ke; k0 += BK) {
    for (int e = threadIdx.x; e < BK * kBM; e += 256) {
      const int kk = e % BK, m = e / BK;
      const int ig = k0 + kk, p = p0 + m;
      As[kk][m] = (ig < ke && p < pa.nproj) ? beta_at<R>(pa, ig, p) : czero<T>();
    }
    for (int e = threadIdx.x; e < BK * kBN; e += 256) {
      const int kk = e % BK, n = e / BK;
      const int ig = k0 + kk, bb = b0 + n;
      Bs[kk][n] = (ig < ke && bb < nb) ? psi[(size_t)bb * ld + ig] : czero<T>();
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < BK; kk++) {
      T av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; i++) av[i] = As[kk][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) bv[j] = Bs[kk][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) cfmac(acc[i][j], av[i], bv[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int p = p0 + tx + 16 * i, bb = b0 + ty + 16 * j;
      if (p < pa.nproj && bb < nb) part[((size_t)blockIdx.z * nb + bb) * pa.nproj + p] = acc[i][j];
    }
}

// wp[b*nproj + p] = W_p * sum_s part[(s*nb + b)*nproj + p]   (fixed order in s)
template <typename R>
__global__ void k_proj_reduce(const cx<R> *__restrict__ part, const R *__restrict__ w, int nsplit,
                              int nb, int nproj, cx<R> *__restrict__ wp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb * nproj) return;
  const int p = i % nproj;
  cx<R> s = part[i];
  for (int k = 1; k < nsplit; k++) s = s + part[(size_t)k * nb * nproj + i];
  const R wl = w ? w[p] : R(1);  // null: the projections themselves
  wp[i] = mk<cx<R>>(wl * s.x, wl * s.y);
}

// out = a*(out + sum_p beta_p(ig) wp[b][p]) + bc*in + g*xm2
template <typename R, int BK>
__global__ void __launch_bounds__(256) k_backproj(ProjArg pa, const cx<R> *__restrict__ wp, int ngw,
                                                  int nb, cx<R> *out, int ldo,
                                                  const cx<R> *__restrict__ in, int ldi,
                                                  const cx<R> *__restrict__ xm2, int ldx, R a,
                                                  R bc, R gc, bool pre) {
  using T = cx<R>;
  __shared__ T As[BK][kBM + 1];
  __shared__ T Bs[BK][kBN + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int g0 = blockIdx.x * kBM, b0 = blockIdx.y * kBN;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = czero<T>();
  for (int k0 = 0; k0 < pa.nproj; k0 += BK) {
    for (int e = threadIdx.x; e < BK * kBM; e += 256) {
      const int m = e % kBM, kk = e / kBM;
      const int ig = g0 + m, p = k0 + kk;
      As[kk][m] = (ig < ngw && p < pa.nproj) ? beta_at<R>(pa, ig, p) : czero<T>();
    }
    for (int e = threadIdx.x; e < BK * kBN; e += 256) {
      const int kk = e % BK, n = e / BK;
      const int p = k0 + kk, bb = b0 + n;
      Bs[kk][n] = (p < pa.nproj && bb < nb) ? wp[(size_t)bb * pa.nproj + p] : czero<T>();
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < BK; kk++) {
      T av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; i++) av[i] = As[kk][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; j++) bv[j] = Bs[kk][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) cfma(acc[i][j], av[i], bv[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < 4; j++) {
    const int bb = b0 + ty + 16 * j;
    if (bb >= nb) continue;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int ig = g0 + tx + 16 * i;
      if (ig >= ngw) continue;
      if (pre) {  // out holds a*(H_loc psi) + bc*in + gc*xm2 already
        const T o = out[(size_t)bb * ldo + ig];
        out[(size_t)bb * ldo + ig] = mk<T>(o.x + a * acc[i][j].x, o.y + a * acc[i][j].y);
        continue;
      }
      T h = out[(size_t)bb * ldo + ig] + acc[i][j];
      T v = mk<T>(a * h.x, a * h.y);
      if (bc != (R)0) {
        const T u = in[(size_t)bb * ldi + ig];
        v.x += bc * u.x;
        v.y += bc * u.y;
      }
      if (gc != (R)0) {
        const T u = xm2[(size_t)bb * ldx + ig];
        v.x += gc * u.x;
        v.y += gc * u.y;
      }
      out[(size_t)bb * ldo + ig] = v;
    }
  }
}

// Narrow tiles for blocks of at most 8 bands (the single vectors of Lanczos,
// small batches): 64 rows x 8 bands per block, thread (r = t & 63,
// c = t >> 6) owns row r and bands c and c + 4.  Within a K slice every
// output accumulates the same products in the same order as in the 64 x 64
// kernels above; only the wasted columns are gone.
constexpr int kNN = 8;

template <typename R, int BK>
__global__ void __launch_bounds__(256) k_proj_n8(ProjArg pa, const cx<R> *__restrict__ psi,
                                                 int ld, int ngw, int nb, int kchunk,
                                                 cx<R> *__restrict__ part) {
  using T = cx<R>;
  __shared__ T As[BK][kBM + 1];
  __shared__ T Bs[BK][kNN + 1];
  const int r = threadIdx.x & 63, cc = threadIdx.x >> 6;
  const int p0 = blockIdx.x * kBM;
  const int kb = blockIdx.z * kchunk;
  const int ke = min(ngw, kb + kchunk);
  T acc0 = czero<T>(), acc1 = czero<T>();
  for (int k0 = kb; k0 < ke; k0 += BK) {
    for (int e = threadIdx.x; e < BK * kBM; e += 256) {
      const int kk = e % BK, m = e / BK;
      const int ig = k0 + kk, p = p0 + m;
      As[kk][m] = (ig < ke && p < pa.nproj) ? beta_at<R>(pa, ig, p) : czero<T>();
    }
    for (int e = threadIdx.x; e < BK * kNN; e += 256) {
      const int kk = e % BK, n = e / BK;
      const int ig = k0 + kk;
      Bs[kk][n] = (ig < ke && n < nb) ? psi[(size_t)n * ld + ig] : czero<T>();
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < BK; kk++) {
      const T av = As[kk][r];
      cfmac(acc0, av, Bs[kk][cc]);
      cfmac(acc1, av, Bs[kk][cc + 4]);
    }
    __syncthreads();
  }
  const int p = p0 + r;
  if (p < pa.nproj) {
    if (cc < nb) part[((size_t)blockIdx.z * nb + cc) * pa.nproj + p] = acc0;
    if (cc + 4 < nb) part[((size_t)blockIdx.z * nb + cc + 4) * pa.nproj + p] = acc1;
  }
}

template <typename R, int BK>
__global__ void __launch_bounds__(256) k_backproj_n8(ProjArg pa, const cx<R> *__restrict__ wp,
                                                     int ngw, int nb, cx<R> *out, int ldo,
                                                     const cx<R> *__restrict__ in, int ldi,
                                                     const cx<R> *__restrict__ xm2, int ldx, R a,
                                                     R bc, R gc, bool pre) {
  using T = cx<R>;
  __shared__ T As[BK][kBM + 1];
  __shared__ T Bs[BK][kNN + 1];
  const int r = threadIdx.x & 63, cc = threadIdx.x >> 6;
  const int g0 = blockIdx.x * kBM;
  T acc[2] = {czero<T>(), czero<T>()};
  for (int k0 = 0; k0 < pa.nproj; k0 += BK) {
    for (int e = threadIdx.x; e < BK * kBM; e += 256) {
      const int m = e % kBM, kk = e / kBM;
      const int ig = g0 + m, p = k0 + kk;
      As[kk][m] = (ig < ngw && p < pa.nproj) ? beta_at<R>(pa, ig, p) : czero<T>();
    }
    for (int e = threadIdx.x; e < BK * kNN; e += 256) {
      const int kk = e % BK, n = e / BK;
      const int p = k0 + kk;
      Bs[kk][n] = (p < pa.nproj && n < nb) ? wp[(size_t)n * pa.nproj + p] : czero<T>();
    }
    __syncthreads();
#pragma unroll 4
    for (int kk = 0; kk < BK; kk++) {
      const T av = As[kk][r];
      cfma(acc[0], av, Bs[kk][cc]);
      cfma(acc[1], av, Bs[kk][cc + 4]);
    }
    __syncthreads();
  }
  const int ig = g0 + r;
  if (ig >= ngw) return;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const int bb = cc + 4 * j;
    if (bb >= nb) continue;
    if (pre) {
      const T o = out[(size_t)bb * ldo + ig];
      out[(size_t)bb * ldo + ig] = mk<T>(o.x + a * acc[j].x, o.y + a * acc[j].y);
      continue;
    }
    T h = out[(size_t)bb * ldo + ig] + acc[j];
    T v = mk<T>(a * h.x, a * h.y);
    if (bc != (R)0) {
      const T u = in[(size_t)bb * ldi + ig];
      v.x += bc * u.x;
      v.y += bc * u.y;
    }
    if (gc != (R)0) {
      const T u = xm2[(size_t)bb * ldx + ig];
      v.x += gc * u.x;
      v.y += gc * u.y;
    }
    out[(size_t)bb * ldo + ig] = v;
  }
}

// The split-K reduction of the narrow projection: one warp per output,
// lanes over the slices in a fixed order, then a fixed shuffle tree.
template <typename R>
__global__ void k_proj_reduce_warp(const cx<R> *__restrict__ part, const R *__restrict__ w,
                                   int nsplit, int nb, int nproj, cx<R> *__restrict__ wp) {
  const int o = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (o >= nb * nproj) return;  // uniform per warp
  cx<R> s = czero<cx<R>>();
  for (int k = lane; k < nsplit; k += 32) s = s + part[(size_t)k * nb * nproj + o];
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    s.x += __shfl_xor_sync(0xffffffffu, s.x, d);
    s.y += __shfl_xor_sync(0xffffffffu, s.y, d);
  }
  if (lane == 0) {
    const R wl = w ? w[o % nproj] : R(1);
    wp[o] = mk<cx<R>>(wl * s.x, wl * s.y);
  }
}

// split-K slices for the projection of nb bands over ngw plane waves: about
// two waves of the GPU for full tiles; for narrow blocks (nb <= 8) slices of
// 64 G so enough blocks are in flight to hide the latency of building beta
inline int proj_split(int ngw, int nb, int mt, int nt) {
  if (nb <= kNN) return std::max(1, std::min((ngw + 63) / 64, (8 * 148 + mt - 1) / mt));
  return std::max(1, std::min((ngw + 255) / 256, (2 * 148 + mt * nt - 1) / (mt * nt)));
}

// out = a*out + bc*in + g*xm2 (no projectors)
template <typename R>
__global__ void k_axpby3(int ngw, int nb, cx<R> *out, int ldo, const cx<R> *__restrict__ in,
                         int ldi, const cx<R> *__restrict__ xm2, int ldx, R a, R bc, R gc) {
  const size_t n = (size_t)ngw * nb;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    const int bb = (int)(i / ngw), ig = (int)(i - (size_t)bb * ngw);
    cx<R> h = out[(size_t)bb * ldo + ig];
    cx<R> v = mk<cx<R>>(a * h.x, a * h.y);
    if (bc != (R)0) {
      const cx<R> u = in[(size_t)bb * ldi + ig];
      v.x += bc * u.x;
      v.y += bc * u.y;
    }
    if (gc != (R)0) {
      const cx<R> u = xm2[(size_t)bb * ldx + ig];
      v.x += gc * u.x;
      v.y += gc * u.y;
    }
    out[(size_t)bb * ldo + ig] = v;
  }
}

template <typename R>
struct Prec;
template <>
struct Prec<double> {
  static const double *vperm(const pspw_cell *c) { return c->d_vperm64; }
  static const double *veff(const pspw_cell *c) { return c->d_veff64; }
  static const double *kin(const pspw_cell *c) { return c->basis.d_kin64; }
  static const void *eigr(const pspw_cell *c) { return c->proj.d_eigr64; }
  static const void *pkga(const pspw_cell *c) { return c->proj.d_pkga64; }
  static const double *pw(const pspw_cell *c) { return c->proj.d_pw64; }
};
template <>
struct Prec<float> {
  static const float *vperm(const pspw_cell *c) { return c->d_vperm32; }
  static const float *veff(const pspw_cell *c) { return c->d_veff32; }
  static const float *kin(const pspw_cell *c) { return c->basis.d_kin32; }
  static const void *eigr(const pspw_cell *c) { return c->proj.d_eigr32; }
  static const void *pkga(const pspw_cell *c) { return c->proj.d_pkga32; }
  static const float *pw(const pspw_cell *c) { return c->proj.d_pw32; }
};

int tile_lines(int n) { return std::max(1, std::min(64, kTileElems / n)); }

template <typename T>
size_t pass_smem(int lines, int n) {
  return (size_t)2 * lines * pad(n) * sizeof(T);
}

template <typename T, typename K>
int set_smem(K kernel, size_t bytes) {
  return bytes > 48 * 1024 ? smem_allow_max(kernel) : PSPW_OK;
}

}  // namespace

// ---------------------------------------------------------------- FP64 projectors
// beta(G, p) = EIGR(G, atom_p) PKG_A(lm_p, G), column-major NGW x nproj
__global__ void k_build_beta64(ProjArg pa, int nproj, double2 *beta) {
  const long long n = (long long)nproj * pa.ngw_cell;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(i / pa.ngw_cell), ig = (int)(i % pa.ngw_cell);
    beta[i] = beta_at<double>(pa, ig, p);
  }
}

// wp(p, b) = W_p P(p, b) (nproj x nb column-major)
__global__ void k_scale_proj(const double2 *__restrict__ P, const double *__restrict__ w,
                             int nproj, int nb, double2 *wp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nproj * nb) return;
  const double wl = w[i % nproj];
  wp[i] = make_double2(wl * P[i].x, wl * P[i].y);
}

int ensure_beta64(pspw_cell *c, const ProjArg &pa) {
  if (c->proj.d_beta64) return PSPW_OK;
  const size_t n = (size_t)c->proj.nproj * c->basis.ngw;
  if (cudaMalloc(&c->proj.d_beta64, n * sizeof(double2)) != cudaSuccess)
    return fail(PSPW_ERR_OOM, "FP64 projector matrix");
  k_build_beta64<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, c->stream>>>(
      pa, c->proj.nproj, c->proj.d_beta64);
  c->kernel_launches++;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

// P (nproj x nb) = beta^H psi over the first ngw plane waves (the engine's
// complex GEMM: DMMA tiles for more than 8 bands, matrix-vector for one)
int project_beta64(pspw_cell *c, const double2 *psi, int ld, int ngw, int nb, double2 *P) {
  const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
  return zgemm<double>(c, 'C', c->proj.nproj, nb, ngw, one, c->proj.d_beta64, c->basis.ngw, psi,
                       ld, zero, P, c->proj.nproj);
}

// out(:, b) += alpha beta wp(:, b) over the first ngw plane waves
int backproject_beta64(pspw_cell *c, const double2 *wp, int ngw, int nb, double2 *out, int ldo,
                       double alpha) {
  const double2 one = make_double2(1.0, 0.0), al = make_double2(alpha, 0.0);
  return zgemm<double>(c, 'N', ngw, nb, c->proj.nproj, al, c->proj.d_beta64, c->basis.ngw, wp,
                       c->proj.nproj, one, out, ldo);
}

// rho += sum_b wband[b] |psi_b(r)|^2 for any grid the generic FFT handles;
// psi scattered for ig < ngw_scatter (EvalRhoPsi.cpp:117).
int rho_generic(pspw_cell *c, const double2 *psi, int ld, int ngw_scatter, int nb,
                const double *d_wband, double *d_rho) {
  using T = double2;
  const Basis &B = c->basis;
  cudaStream_t st = c->stream;
  Geo geo{B.n1, B.n2, B.n3, B.ncol, B.nxa, B.ngw, B.d_col_start, B.d_sg_ig, B.d_sg_z,
          B.d_sg_col, B.d_col_of_xy, B.d_xa_list, B.d_xa_of_x};
  const size_t s_band = (size_t)B.n3 * B.ncol, p_band = (size_t)B.n3 * B.n2 * B.nxa;
  int nbatch = c->band_batch;
  if (nbatch <= 0) nbatch = (int)std::max<size_t>(1, (48u << 20) / ((s_band + p_band) * sizeof(T)));
  nbatch = std::min(nbatch, nb);
  T *S = nullptr, *P = nullptr;
  int rc;
  if ((rc = ws_reserve(c, kWsSticks, sizeof(T) * s_band * nbatch, (void **)&S)) ||
      (rc = ws_reserve(c, kWsPlanes, sizeof(T) * p_band * nbatch, (void **)&P)))
    return rc;
  const int T1 = tile_lines(B.n3), T2 = tile_lines(B.n2), L3 = tile_lines(B.n1);
  const size_t sm1 = pass_smem<T>(T1, B.n3), sm2 = pass_smem<T>(T2, B.n2),
               sm3 = pass_smem<T>(L3, B.n1) + sizeof(double) * (size_t)L3 * B.n1;
  if ((rc = set_smem<T>(k_sticks_inv<T>, sm1)) || (rc = set_smem<T>(k_planes_inv<T>, sm2)) ||
      (rc = set_smem<T>(k_xlines_rho<T>, sm3)))
    return rc;
  const FftArg fx = fft_arg(B.dim[0]), fy = fft_arg(B.dim[1]), fz = fft_arg(B.dim[2]);
  const T *wx = tw<T>(B.dim[0]), *wy = tw<T>(B.dim[1]), *wz = tw<T>(B.dim[2]);
  for (int b0 = 0; b0 < nb; b0 += nbatch) {
    const int nbb = std::min(nbatch, nb - b0);
    k_sticks_inv<T><<<dim3((B.ncol + T1 - 1) / T1, nbb), kNT, sm1, st>>>(
        geo, fz, wz, psi + (size_t)b0 * ld, ld, ngw_scatter, S, T1);
    k_planes_inv<T><<<dim3((B.nxa + T2 - 1) / T2, B.n3, nbb), kNT, sm2, st>>>(geo, fy, wy, S, P,
                                                                              T2);
    k_xlines_rho<T><<<(B.n2 * B.n3 + L3 - 1) / L3, kNT, sm3, st>>>(geo, fx, wx, P, nbb,
                                                                   d_wband + b0, d_rho, L3);
    c->kernel_launches += 3;
  }
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

template <typename R>
int hpsi_apply(pspw_cell *c, const void *in_v, int ld_in, void *out_v, int ld_out, int ngw, int nb,
               double a, double b, double g, const void *xm2_v, int ld_xm2,
               const ScratchPlan *plan) {
  using T = cx<R>;
  const Basis &B = c->basis;
  if (nb <= 0) return PSPW_OK;
  if (!in_v || !out_v) return fail(PSPW_ERR_ARG, "hpsi: null block");
  if (in_v == out_v) return fail(PSPW_ERR_ARG, "hpsi: input and output blocks must differ");
  if (ngw <= 0 || ngw > B.ngw) return fail(PSPW_ERR_SHAPE, "hpsi: ngw exceeds the cell's sphere");
  if (ld_in < ngw || ld_out < ngw) return fail(PSPW_ERR_SHAPE, "hpsi: leading dimension < ngw");
  if (g != 0.0 && (!xm2_v || ld_xm2 < ngw)) return fail(PSPW_ERR_ARG, "hpsi: missing x(d-2)");
  if (!c->veff_set) return fail(PSPW_ERR_ARG, "hpsi: V_eff not set (pspw_cell_set_veff)");
  const T *in = static_cast<const T *>(in_v);
  T *out = static_cast<T *>(out_v);
  const T *xm2 = static_cast<const T *>(xm2_v);
  cudaStream_t st = c->stream;

  // ---- projection
  const int nproj = c->proj.nproj;
  ProjArg pa;
  pa.eigr = Prec<R>::eigr(c);
  pa.pkga = Prec<R>::pkga(c);
  pa.patom = c->proj.d_patom;
  pa.psp = c->proj.d_psp;
  pa.plm = c->proj.d_plm;
  pa.pw = Prec<R>::pw(c);
  pa.ngw_cell = B.ngw;
  pa.nproj = nproj;
  constexpr int BK = sizeof(R) == 8 ? 16 : 32;
  T *wp = nullptr;
  cudaEvent_t ev = nullptr;
  // enqueue one kernel, with optional event timing of its family
  auto run = [&](int fam, auto &&launch) {
    cudaEvent_t e;
    timing_begin(c, fam, &e);
    launch();
    timing_end(c, fam, e);
    c->kernel_launches++;
  };
  // FP32 with one species: projector GEMMs on the tensor cores
  bool use_tc = false;
  if constexpr (sizeof(R) == 4) use_tc = nproj > 0 && nl_tc_usable(c);
  float *tc_part = nullptr, *tc_wt = nullptr;
  int tc_split = 0;
  // The projection reads psi only: it runs on the cell's second stream,
  // concurrently with the local part, and the back-projection waits for it
  // (unless the cell's overlap mode is PSPW_OVERLAP_OFF; on Si64 the
  // concurrent form is 6 % faster in FP32 and 8 % in FP64).  Callers with a
  // scratch plan, i.e. the allocation-free entry point, keep one stream.
  // c->stream is switched for the projection's launches and switched back
  // on every exit from this block.
  const cudaStream_t main_st = c->stream;
  const bool overlap = c->nl_overlap != PSPW_OVERLAP_OFF && nproj > 0 && !plan &&
                       c->stream2 != nullptr;
  struct StreamSwitch {
    pspw_cell *c;
    cudaStream_t main;
    ~StreamSwitch() { c->stream = main; }
  };
  if (nproj > 0) {
    StreamSwitch restore{c, main_st};
    if (overlap) {
      PSPW_CUDA(cudaEventRecord(c->ev_fork, main_st));
      PSPW_CUDA(cudaStreamWaitEvent(c->stream2, c->ev_fork, 0));
      c->stream = c->stream2;
      st = c->stream2;
    }
    const int mt = (nproj + kBM - 1) / kBM, nt = (nb + kBN - 1) / kBN;
    int nsplit = proj_split(ngw, nb, mt, nt);
    if (plan) nsplit = std::max(1, std::min(nsplit, plan->max_split));
    int kchunk = (ngw + nsplit - 1) / nsplit;
    kchunk = (kchunk + BK - 1) / BK * BK;
    nsplit = (ngw + kchunk - 1) / kchunk;
    T *part = nullptr;
    if (plan) {
      part = static_cast<T *>(plan->part);
      wp = static_cast<T *>(plan->wp);
    } else {
      if (!use_tc) {
        int rc = ws_reserve(c, 2, sizeof(T) * (size_t)nsplit * nb * nproj, (void **)&part);
        if (rc) return rc;
        rc = ws_reserve(c, 3, sizeof(T) * (size_t)nb * nproj, (void **)&wp);
        if (rc) return rc;
      }
    }
    timing_begin(c, kFamNonlocal, &ev);
    bool done = false;
    if constexpr (sizeof(R) == 8) {
      // FP64 without a scratch plan: beta materialised once, complex GEMMs
      if (!plan) {
        int rc = ensure_beta64(c, pa);
        if (rc) return rc;
        cudaEvent_t e;
        timing_begin(c, kFamProj, &e);
        rc = project_beta64(c, reinterpret_cast<const double2 *>(in), ld_in, ngw, nb,
                            reinterpret_cast<double2 *>(part));
        if (rc) return rc;
        k_scale_proj<<<(nb * nproj + 255) / 256, 256, 0, st>>>(
            reinterpret_cast<const double2 *>(part), c->proj.d_pw64, nproj, nb,
            reinterpret_cast<double2 *>(wp));
        c->kernel_launches++;
        timing_end(c, kFamProj, e);
        done = true;
      }
    }
    if (done) {
    } else if (use_tc) {
      if (plan) {
        tc_part = static_cast<float *>(plan->part);
        tc_wt = static_cast<float *>(plan->wt);
        tc_split = plan->max_split;
      } else {
        const int rc = nl_tc_reserve(c, ngw, nb, &tc_part, &tc_split, &tc_wt);
        if (rc) return rc;
      }
      cudaEvent_t e;
      timing_begin(c, kFamProj, &e);
      const int rc = nl_tc_project(c, reinterpret_cast<const float2 *>(in), ld_in, ngw, nb,
                                   tc_part, tc_split, tc_wt);
      timing_end(c, kFamProj, e);
      if (rc) return rc;
    } else {
      run(kFamProj, [&] {
        if (nb <= kNN)
          k_proj_n8<R, BK><<<dim3(mt, 1, nsplit), 256, 0, st>>>(pa, in, ld_in, ngw, nb, kchunk,
                                                                part);
        else
          k_proj<R, BK><<<dim3(mt, nt, nsplit), 256, 0, st>>>(pa, in, ld_in, ngw, nb, kchunk,
                                                              part);
      });
      run(kFamProj, [&] {
        if (nb <= kNN)
          k_proj_reduce_warp<R><<<(nb * nproj * 32 + 255) / 256, 256, 0, st>>>(
              part, Prec<R>::pw(c), nsplit, nb, nproj, wp);
        else
          k_proj_reduce<R><<<(nb * nproj + 255) / 256, 256, 0, st>>>(part, Prec<R>::pw(c), nsplit,
                                                                    nb, nproj, wp);
      });
    }
    timing_end(c, kFamNonlocal, ev);
    PSPW_CUDA(cudaGetLastError());
    if (overlap) PSPW_CUDA(cudaEventRecord(c->ev_join, c->stream2));
    st = main_st;
  }

  // ---- local part, in batches of bands
  Geo geo{B.n1, B.n2, B.n3, B.ncol, B.nxa, B.ngw, B.d_col_start, B.d_sg_ig, B.d_sg_z,
          B.d_sg_col, B.d_col_of_xy, B.d_xa_list, B.d_xa_of_x};
  if (B.fast) {
    const FastGeo fg{B.ncol,    B.nxa,       B.d_col_start, B.d_sg_ig,
                     B.d_sg_z,  B.d_sg_col,  B.d_xa_list,   B.d_col_x,
                     B.d_col_y, B.d_xa_of_x, c->stick.active, B.d_sg_off};
    RecArg<T, R> ra;
    ra.on = true;
    ra.ca = (R)a;
    ra.cb = (R)b;
    ra.cg = (R)g;
    ra.xm2 = xm2;
    ra.ldx = ld_xm2;
    int rc = local_fast<R>(c, fg, in, ld_in, out, ld_out, ngw, nb, plan, ra);
    if (rc) return rc;
  } else {
  const size_t s_band = (size_t)B.n3 * B.ncol, p_band = (size_t)B.n3 * B.n2 * B.nxa;
  int nbatch = c->band_batch;
  if (nbatch <= 0) {
    // keep a batch's stick and plane buffers within ~48 MB so they stay in L2
    nbatch = (int)std::max<size_t>(1, (48u << 20) / ((s_band + p_band) * sizeof(T)));
  }
  if (plan) nbatch = plan->nbatch;
  nbatch = std::min(nbatch, nb);
  T *S = nullptr, *P = nullptr;
  int rc = PSPW_OK;
  if (plan) {
    S = static_cast<T *>(plan->S);
    P = static_cast<T *>(plan->P);
  } else {
    rc = ws_reserve(c, 0, sizeof(T) * s_band * nbatch, (void **)&S);
    if (rc) return rc;
    rc = ws_reserve(c, 1, sizeof(T) * p_band * nbatch, (void **)&P);
    if (rc) return rc;
  }
  const int T1 = tile_lines(B.n3), T2 = tile_lines(B.n2), L3 = tile_lines(B.n1);
  const size_t sm1 = pass_smem<T>(T1, B.n3), sm2 = pass_smem<T>(T2, B.n2),
               sm3 = pass_smem<T>(L3, B.n1);
  if ((rc = set_smem<T>(k_sticks_inv<T>, sm1)) || (rc = set_smem<T>(k_sticks_fwd<T, R>, sm1)) ||
      (rc = set_smem<T>(k_planes_inv<T>, sm2)) || (rc = set_smem<T>(k_planes_fwd<T>, sm2)) ||
      (rc = set_smem<T>(k_xlines<T, R>, sm3)))
    return rc;
  const FftArg fx = fft_arg(B.dim[0]), fy = fft_arg(B.dim[1]), fz = fft_arg(B.dim[2]);
  const T *wx = tw<T>(B.dim[0]), *wy = tw<T>(B.dim[1]), *wz = tw<T>(B.dim[2]);
  timing_begin(c, kFamLocal, &ev);
  for (int b0 = 0; b0 < nb; b0 += nbatch) {
    const int nbb = std::min(nbatch, nb - b0);
    const T *inb = in + (size_t)b0 * ld_in;
    T *outb = out + (size_t)b0 * ld_out;
    run(kFamSticksInv, [&] {
      k_sticks_inv<T><<<dim3((B.ncol + T1 - 1) / T1, nbb), kNT, sm1, st>>>(geo, fz, wz, inb, ld_in,
                                                                            ngw, S, T1);
    });
    run(kFamPlanesInv, [&] {
      k_planes_inv<T><<<dim3((B.nxa + T2 - 1) / T2, B.n3, nbb), kNT, sm2, st>>>(geo, fy, wy, S, P,
                                                                                T2);
    });
    run(kFamXlines, [&] {
      k_xlines<T, R><<<dim3((B.n2 * B.n3 + L3 - 1) / L3, nbb), kNT, sm3, st>>>(
          geo, fx, wx, Prec<R>::veff(c), P, L3);
    });
    run(kFamPlanesFwd, [&] {
      k_planes_fwd<T><<<dim3((B.nxa + T2 - 1) / T2, B.n3, nbb), kNT, sm2, st>>>(geo, fy, wy, P, S,
                                                                                T2);
    });
    run(kFamSticksFwd, [&] {
      k_sticks_fwd<T, R><<<dim3((B.ncol + T1 - 1) / T1, nbb), kNT, sm1, st>>>(
          geo, fz, wz, S, Prec<R>::kin(c), inb, ld_in, outb, ld_out, ngw, T1);
    });
  }
  timing_end(c, kFamLocal, ev);
  }
  PSPW_CUDA(cudaGetLastError());

  // ---- back-projection + recurrence epilogue.  On the register-FFT path the
  // forward stick pass has applied the recurrence to the local part already
  // (out = a H_loc in + b in + g xm2), so the back-projection only adds
  // a * beta W beta^H in.
  const bool pre = B.fast;
  if (nproj > 0) {
    if (overlap) PSPW_CUDA(cudaStreamWaitEvent(st, c->ev_join, 0));
    timing_begin(c, kFamNonlocal, &ev);
    if (use_tc) {
      cudaEvent_t e;
      timing_begin(c, kFamBackproj, &e);
      const int rc = nl_tc_backproject(
          c, tc_wt, ngw, nb, reinterpret_cast<float2 *>(out), ld_out,
          reinterpret_cast<const float2 *>(in), ld_in, reinterpret_cast<const float2 *>(xm2),
          ld_xm2, (float)a, pre ? 0.f : (float)b, pre ? 0.f : (float)g, pre);
      timing_end(c, kFamBackproj, e);
      if (rc) return rc;
    } else {
      dim3 grid((ngw + kBM - 1) / kBM, (nb + kBN - 1) / kBN);
      bool done = false;
      if constexpr (sizeof(R) == 8) {
        if (!plan) {
          cudaEvent_t e;
          timing_begin(c, kFamBackproj, &e);
          int rc = backproject_beta64(c, reinterpret_cast<const double2 *>(wp), ngw, nb,
                                      reinterpret_cast<double2 *>(out), ld_out, pre ? a : 1.0);
          if (rc) return rc;
          if (!pre && (a != 1.0 || b != 0.0 || g != 0.0)) {
            k_axpby3<R><<<4 * 148, 256, 0, st>>>(ngw, nb, out, ld_out, in, ld_in, xm2, ld_xm2,
                                                (R)a, (R)b, (R)g);
            c->kernel_launches++;
          }
          timing_end(c, kFamBackproj, e);
          done = true;
        }
      }
      if (!done) run(kFamBackproj, [&] {
        if (nb <= kNN)
          k_backproj_n8<R, BK><<<grid.x, 256, 0, st>>>(pa, wp, ngw, nb, out, ld_out, in, ld_in,
                                                       xm2, ld_xm2, (R)a, (R)b, (R)g, pre);
        else
          k_backproj<R, BK><<<grid, 256, 0, st>>>(pa, wp, ngw, nb, out, ld_out, in, ld_in, xm2,
                                                  ld_xm2, (R)a, (R)b, (R)g, pre);
      });
    }
    timing_end(c, kFamNonlocal, ev);
  } else if (!pre && (a != 1.0 || b != 0.0 || g != 0.0)) {
    run(kFamBackproj, [&] {
      k_axpby3<R><<<4 * 148, 256, 0, st>>>(ngw, nb, out, ld_out, in, ld_in, xm2, ld_xm2, (R)a,
                                          (R)b, (R)g);
    });
  }
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

// P[b*nproj + p] = sum_{G < ngw} conj(beta_p(G)) psi_b(G), FP64, without the
// weights WNL (the projections FNL of EvalENL.cpp:27-33).
int project_fp64(pspw_cell *c, const double2 *psi, int ld, int ngw, int nb, double2 *P) {
  using R = double;
  const int nproj = c->proj.nproj;
  if (nproj <= 0 || nb <= 0) return PSPW_OK;
  ProjArg pa;
  pa.eigr = Prec<R>::eigr(c);
  pa.pkga = Prec<R>::pkga(c);
  pa.patom = c->proj.d_patom;
  pa.psp = c->proj.d_psp;
  pa.plm = c->proj.d_plm;
  pa.pw = Prec<R>::pw(c);
  pa.ngw_cell = c->basis.ngw;
  pa.nproj = nproj;
  int rc = ensure_beta64(c, pa);
  if (rc) return rc;
  // beta materialised: one complex GEMM (projections without the weights)
  if ((rc = project_beta64(c, psi, ld, ngw, nb, P))) return rc;
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

template int hpsi_apply<double>(pspw_cell *, const void *, int, void *, int, int, int, double,
                                double, double, const void *, int, const ScratchPlan *);
template int hpsi_apply<float>(pspw_cell *, const void *, int, void *, int, int, int, double,
                               double, double, const void *, int, const ScratchPlan *);

}  // namespace pspw
