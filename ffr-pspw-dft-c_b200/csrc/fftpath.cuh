// Register-FFT local part of block H*psi: three kernels per band batch.
//
//   k_sticks_inv<NZ>    gather psi(G) of T1 sticks into shared memory, inverse
//                       z FFT, write the stick buffer S[band][zpos][stick]
//   k_plane<NX,NY>      one z-plane of one band in shared memory: inverse y
//                       FFT on the active-x columns, inverse x FFT, times
//                       V_eff/NNR, forward x FFT, forward y FFT
//   k_sticks_fwd<NZ>    forward z FFT of each stick, pick the sphere G's, add
//                       the kinetic term
//
// Lengths are template parameters so every kernel holds only its own
// unrolled register DFTs (fft2.cuh).  Along each axis the inverse transform
// leaves the digit-permuted order of fft2.cuh; S holds z in that order and
// V_eff is stored permuted in (z, x, y), so no reordering pass exists.
#pragma once

#include <algorithm>

#include "fft2.cuh"
#include "fftpath.h"

namespace pspw {
namespace fastpath {

template <int NZ>
struct StickCfg {
  static constexpr int T1 = stick_tile(NZ);
  static constexpr int LS = NZ + 1;
};

template <int NZ, typename T>
__global__ void __launch_bounds__(256) k_sticks_inv(FastGeo g, const T *__restrict__ wz_g,
                                                    const T *__restrict__ psi, int ld,
                                                    int ngw_call, T *__restrict__ S) {
  constexpr int T1 = StickCfg<NZ>::T1, LS = StickCfg<NZ>::LS;
  constexpr int A = nsplit_for(NZ).n1, B = nsplit_for(NZ).n2;
  __shared__ T tile[T1 * LS];
  __shared__ T wz[NZ];
  const int c0 = blockIdx.x * T1;
  const int band = blockIdx.y;
  const int nc = min(T1, g.ncol - c0);
  for (int e = threadIdx.x; e < T1 * LS; e += blockDim.x) tile[e] = czero<T>();
  for (int t = threadIdx.x; t < NZ; t += blockDim.x) wz[t] = wz_g[t];
  __syncthreads();
  const T *pb = psi + (size_t)band * ld;
  const int k0 = g.col_start[c0], k1 = g.col_start[c0 + nc];
  // the gather in groups of four elements per thread: all index loads, then
  // all psi loads, then the shared-memory stores, so each thread has four
  // independent chains in flight instead of one
  constexpr int U = 4;
  for (int kb = k0 + threadIdx.x; kb < k1; kb += U * 256) {
    int ig[U], off[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int k = kb + u * 256;
      ig[u] = k < k1 ? (g.ig_iota ? k : g.sg_ig[k]) : ngw_call;
      off[u] = k < k1 ? g.sg_off[k] : 0;  // (sg_col[k] - c0) * LS + sg_z[k]
    }
    T v[U];
#pragma unroll
    for (int u = 0; u < U; u++) v[u] = ig[u] < ngw_call ? pb[ig[u]] : czero<T>();
#pragma unroll
    for (int u = 0; u < U; u++)
      if (ig[u] < ngw_call) tile[off[u]] = v[u];
  }
  __syncthreads();
  const Lines L{nullptr, LS, nc};
  inv_stepS<A, B>(tile, L, 1, wz);
  __syncthreads();
  inv_stepB<A, B>(tile, L, 1, wz);
  __syncthreads();
  T *Sb = S + (size_t)band * NZ * g.ncol;
  for (int e = threadIdx.x; e < T1 * NZ; e += blockDim.x) {
    const int p = e / T1, t = e - p * T1;
    if (t < nc) Sb[(size_t)p * g.ncol + c0 + t] = tile[t * LS + p];
  }
}

// out = kin psi + FFT part; with rec, out = ca (kin psi + FFT part) + cb psi
// + cg x (the Chebyshev recurrence, whose projector term ca W beta^H psi the
// back-projection then adds)
template <int NZ, typename T, typename R>
__global__ void __launch_bounds__(256) k_sticks_fwd(FastGeo g, const T *__restrict__ wz_g,
                                                    const T *__restrict__ S,
                                                    const R *__restrict__ kin,
                                                    const T *__restrict__ psi, int ld,
                                                    T *__restrict__ out, int ldo, int ngw_call,
                                                    bool rec, R ca, R cb, R cg,
                                                    const T *__restrict__ xm2, int ldx) {
  constexpr int T1 = StickCfg<NZ>::T1, LS = StickCfg<NZ>::LS;
  constexpr int A = nsplit_for(NZ).n1, B = nsplit_for(NZ).n2;
  __shared__ T tile[T1 * LS];
  __shared__ T wz[NZ];
  const int c0 = blockIdx.x * T1;
  const int band = blockIdx.y;
  const int nc = min(T1, g.ncol - c0);
  for (int t = threadIdx.x; t < NZ; t += blockDim.x) wz[t] = wz_g[t];
  const T *Sb = S + (size_t)band * NZ * g.ncol;
  // the transposing read of the stick buffer, four loads per thread in
  // flight before their shared-memory stores
  constexpr int U = 4;
  for (int eb = threadIdx.x; eb < T1 * NZ; eb += U * 256) {
    T v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int e = eb + u * 256, p = e / T1, t = e - p * T1;
      v[u] = (e < T1 * NZ && t < nc) ? Sb[(size_t)p * g.ncol + c0 + t] : czero<T>();
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int e = eb + u * 256, p = e / T1, t = e - p * T1;
      if (e < T1 * NZ) tile[t * LS + p] = v[u];
    }
  }
  __syncthreads();
  const Lines L{nullptr, LS, nc};
  fwd_stepB<A, B>(tile, L, 1, wz);
  __syncthreads();
  fwd_stepS<A, B>(tile, L, 1, wz);
  __syncthreads();
  const T *pb = psi + (size_t)band * ld;
  T *ob = out + (size_t)band * ldo;
  const T *xb = (rec && cg != (R)0) ? xm2 + (size_t)band * ldx : nullptr;
  const int k0 = g.col_start[c0], k1 = g.col_start[c0 + nc];
  // four elements per thread in flight, as in the inverse gather
  for (int kb = k0 + threadIdx.x; kb < k1; kb += U * 256) {
    int ig[U], off[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int k = kb + u * 256;
      ig[u] = k < k1 ? (g.ig_iota ? k : g.sg_ig[k]) : ngw_call;
      off[u] = k < k1 ? (g.sg_col[k] - c0) * LS + g.sg_z[k] : 0;
    }
    R kk[U];
    T p[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const bool on = ig[u] < ngw_call;
      kk[u] = on ? kin[ig[u]] : (R)0;
      p[u] = on ? pb[ig[u]] : czero<T>();
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      if (ig[u] < ngw_call) {
        const T f = tile[off[u]];
        T v = mk<T>(kk[u] * p[u].x + f.x, kk[u] * p[u].y + f.y);
        if (rec) {
          v = mk<T>(ca * v.x + cb * p[u].x, ca * v.y + cb * p[u].y);
          if (xb) {
            const T x = xb[ig[u]];
            v.x += cg * x.x;
            v.y += cg * x.y;
          }
        }
        ob[ig[u]] = v;
      }
    }
  }
}

template <int NX, int NY>
struct PlaneCfg {
  static constexpr int LS = NX + 1;
  static constexpr int NT = (NX * NY >= 6000) ? 512 : 256;
};

template <int NX, int NY, typename T>
constexpr size_t plane_smem() {
  return sizeof(T) * ((size_t)NY * PlaneCfg<NX, NY>::LS + NX + NY) + sizeof(int) * NX;
}

// One z-plane of one band.  The y transforms and the stick scatter/gather
// work on the compact view [y][xa] (active x only, odd row stride la), the x
// transforms on full rows [y][x] (stride LS); the two x steps at the ends of
// the x sandwich convert between the views (x_inv_expand / x_fwd_compact).
// Only the compact view needs clearing.
template <int NX, int NY, typename T, typename R>
__global__ void __launch_bounds__(PlaneCfg<NX, NY>::NT) k_plane(FastGeo g, int n3,
                                                                const T *__restrict__ wx_g,
                                                                const T *__restrict__ wy_g,
                                                                const R *__restrict__ vperm,
                                                                T *__restrict__ S) {
  constexpr int LS = PlaneCfg<NX, NY>::LS, NT = PlaneCfg<NX, NY>::NT;
  constexpr int AX = nsplit_for(NX).n1, BX = nsplit_for(NX).n2;
  constexpr int AY = nsplit_for(NY).n1, BY = nsplit_for(NY).n2;
  extern __shared__ unsigned char smem_raw[];
  T *plane = reinterpret_cast<T *>(smem_raw);
  T *wx = plane + NY * LS;
  T *wy = wx + NX;
  int *xa = reinterpret_cast<int *>(wy + NY);  // x -> active index or -1
  const int la = g.nxa | 1;
  const int zp = blockIdx.x, band = blockIdx.y;
  T *Sz = S + ((size_t)band * n3 + zp) * g.ncol;
  for (int e = threadIdx.x; e < NY * la; e += NT) plane[e] = czero<T>();
  for (int t = threadIdx.x; t < NX; t += NT) {
    wx[t] = wx_g[t];
    xa[t] = g.xa_of_x[t];
  }
  for (int t = threadIdx.x; t < NY; t += NT) wy[t] = wy_g[t];
  __syncthreads();
  for (int c = threadIdx.x; c < g.ncol; c += NT) plane[g.col_y[c] * la + xa[g.col_x[c]]] = Sz[c];
  __syncthreads();
  const Lines cols{nullptr, 1, g.nxa};
  const Lines rows{nullptr, LS, NY};
  inv_stepS<AY, BY>(plane, cols, la, wy);
  __syncthreads();
  inv_stepB<AY, BY>(plane, cols, la, wy);
  __syncthreads();
  x_inv_expand<NY, AX, BX, NT>(plane, la, LS, xa, wx);
  __syncthreads();
  inv_fwd_stepB_v<AX, BX>(plane, rows, wx, vperm + (size_t)zp * NY * NX, NY);
  __syncthreads();
  x_fwd_compact<NY, AX, BX, NT>(plane, la, LS, xa);
  __syncthreads();
  fwd_stepB<AY, BY>(plane, cols, la, wy);
  __syncthreads();
  fwd_stepS<AY, BY>(plane, cols, la, wy);
  __syncthreads();
  for (int c = threadIdx.x; c < g.ncol; c += NT) Sz[c] = plane[g.col_y[c] * la + xa[g.col_x[c]]];
}

// Density accumulation (EvalRhoPsi.cpp:139-150): inverse y and x FFTs of one
// z-plane for each band of a group, acc += w_b |psi_b(r)|^2 in FP64; the
// group's plane goes to part[group][zpos][ypos][xpos] (permuted order).
// the FP64 accumulator plane starts on a 16-byte boundary after the plane
// kernel's layout (whose int table leaves it 4 bytes off for odd NX)
template <int NX, int NY, typename T>
constexpr size_t plane_rho_acc_off() {
  return (plane_smem<NX, NY, T>() + 15) / 16 * 16;
}

template <int NX, int NY, typename T>
constexpr size_t plane_rho_smem() {
  return plane_rho_acc_off<NX, NY, T>() + sizeof(double) * (size_t)NX * NY;
}

template <int NX, int NY, typename T>
__global__ void __launch_bounds__(PlaneCfg<NX, NY>::NT) k_plane_rho(
    FastGeo g, int n3, const T *__restrict__ wx_g, const T *__restrict__ wy_g,
    const T *__restrict__ S, int nbb, int bands_per_group, const double *__restrict__ wband,
    double *__restrict__ part) {
  constexpr int LS = PlaneCfg<NX, NY>::LS;
  constexpr int AX = nsplit_for(NX).n1, BX = nsplit_for(NX).n2;
  constexpr int AY = nsplit_for(NY).n1, BY = nsplit_for(NY).n2;
  extern __shared__ unsigned char smem_raw[];
  T *plane = reinterpret_cast<T *>(smem_raw);
  T *wx = plane + NY * LS;
  T *wy = wx + NX;
  int *xoff = reinterpret_cast<int *>(wy + NY);
  double *acc = reinterpret_cast<double *>(smem_raw + plane_rho_acc_off<NX, NY, T>());
  const int zp = blockIdx.x, grp = blockIdx.y;
  for (int t = threadIdx.x; t < NX; t += blockDim.x) wx[t] = wx_g[t];
  for (int t = threadIdx.x; t < NY; t += blockDim.x) wy[t] = wy_g[t];
  for (int t = threadIdx.x; t < g.nxa; t += blockDim.x) xoff[t] = g.xa_list[t];
  for (int e = threadIdx.x; e < NX * NY; e += blockDim.x) acc[e] = 0.0;
  const Lines cols{xoff, 0, g.nxa};
  const Lines rows{nullptr, LS, NY};
  const int b0 = grp * bands_per_group, b1 = min(nbb, b0 + bands_per_group);
  for (int band = b0; band < b1; band++) {
    const T *Sz = S + ((size_t)band * n3 + zp) * g.ncol;
    __syncthreads();
    for (int e = threadIdx.x; e < NY * LS; e += blockDim.x) plane[e] = czero<T>();
    __syncthreads();
    for (int c = threadIdx.x; c < g.ncol; c += blockDim.x)
      plane[g.col_y[c] * LS + g.col_x[c]] = Sz[c];
    __syncthreads();
    inv_stepS<AY, BY>(plane, cols, LS, wy);
    __syncthreads();
    inv_stepB<AY, BY>(plane, cols, LS, wy);
    __syncthreads();
    inv_stepS<AX, BX>(plane, rows, 1, wx);
    __syncthreads();
    inv_stepB<AX, BX>(plane, rows, 1, wx);
    __syncthreads();
    const double w = wband[band];
    for (int e = threadIdx.x; e < NX * NY; e += blockDim.x) {
      const int y = e / NX, x = e - y * NX;
      const T v = plane[y * LS + x];
      acc[e] += w * ((double)v.x * (double)v.x + (double)v.y * (double)v.y);
    }
  }
  __syncthreads();
  double *pp = part + ((size_t)grp * n3 + zp) * NX * NY;
  for (int e = threadIdx.x; e < NX * NY; e += blockDim.x) pp[e] = acc[e];
}

// ---- host-side launchers
template <int NZ, typename T>
int launch_sticks_inv(const FastGeo &g, cudaStream_t st, int nbb, const T *wz, const T *in, int ld,
                      int ngw, T *S) {
  constexpr int T1 = StickCfg<NZ>::T1;
  k_sticks_inv<NZ, T><<<dim3((g.ncol + T1 - 1) / T1, nbb), 256, 0, st>>>(g, wz, in, ld, ngw, S);
  return PSPW_OK;
}

template <int NZ, typename T, typename R>
int launch_sticks_fwd(const FastGeo &g, cudaStream_t st, int nbb, const T *wz, const T *S,
                      const R *kin, const T *in, int ld, T *out, int ldo, int ngw,
                      const RecArg<T, R> &ra) {
  constexpr int T1 = StickCfg<NZ>::T1;
  k_sticks_fwd<NZ, T, R><<<dim3((g.ncol + T1 - 1) / T1, nbb), 256, 0, st>>>(
      g, wz, S, kin, in, ld, out, ldo, ngw, ra.on, ra.ca, ra.cb, ra.cg, ra.xm2, ra.ldx);
  return PSPW_OK;
}

template <int NX, int NY, typename T, typename R>
int launch_plane(const FastGeo &g, cudaStream_t st, int nbb, int n3, const T *wx, const T *wy,
                 const R *vperm, T *S) {
  constexpr size_t sm = plane_smem<NX, NY, T>();
  if (sm > 48 * 1024)
    PSPW_CUDA(cudaFuncSetAttribute(k_plane<NX, NY, T, R>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_plane<NX, NY, T, R><<<dim3(n3, nbb), PlaneCfg<NX, NY>::NT, sm, st>>>(g, n3, wx, wy, vperm, S);
  return PSPW_OK;
}

// dispatch over the compiled lengths; -1 if not compiled
template <typename T>
int dispatch_sticks_inv(int n3, const FastGeo &g, cudaStream_t st, int nbb, const T *wz,
                        const T *in, int ld, int ngw, T *S) {
  switch (n3) {
#define PSPW_CASE(NN) \
  case NN: return launch_sticks_inv<NN, T>(g, st, nbb, wz, in, ld, ngw, S);
    PSPW_FOR_EACH_SPLIT(PSPW_CASE)
#undef PSPW_CASE
    default: return -1;
  }
}

template <typename T, typename R>
int dispatch_sticks_fwd(int n3, const FastGeo &g, cudaStream_t st, int nbb, const T *wz,
                        const T *S, const R *kin, const T *in, int ld, T *out, int ldo, int ngw,
                        const RecArg<T, R> &ra) {
  switch (n3) {
#define PSPW_CASE(NN) \
  case NN: return launch_sticks_fwd<NN, T, R>(g, st, nbb, wz, S, kin, in, ld, out, ldo, ngw, ra);
    PSPW_FOR_EACH_SPLIT(PSPW_CASE)
#undef PSPW_CASE
    default: return -1;
  }
}

// plane kernels compiled for square planes (n1 == n2)
template <typename T, typename R>
int dispatch_plane(int n1, int n2, const FastGeo &g, cudaStream_t st, int nbb, int n3, const T *wx,
                   const T *wy, const R *vperm, T *S) {
  if (n1 != n2) return -1;
  switch (n1) {
#define PSPW_CASE(NN) \
  case NN: return launch_plane<NN, NN, T, R>(g, st, nbb, n3, wx, wy, vperm, S);
    PSPW_FOR_EACH_SPLIT(PSPW_CASE)
#undef PSPW_CASE
    default: return -1;
  }
}


template <int NX, int NY, typename T>
int launch_plane_rho(const FastGeo &g, cudaStream_t st, int n3, int ngroups, const T *wx,
                     const T *wy, const T *S, int nbb, int bpg, const double *wband, double *part) {
  constexpr size_t sm = plane_rho_smem<NX, NY, T>();
  if (sm > 48 * 1024)
    PSPW_CUDA(cudaFuncSetAttribute(k_plane_rho<NX, NY, T>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  k_plane_rho<NX, NY, T><<<dim3(n3, ngroups), PlaneCfg<NX, NY>::NT, sm, st>>>(g, n3, wx, wy, S, nbb,
                                                                             bpg, wband, part);
  return PSPW_OK;
}

template <typename T>
int dispatch_plane_rho(int n1, int n2, const FastGeo &g, cudaStream_t st, int n3, int ngroups,
                       const T *wx, const T *wy, const T *S, int nbb, int bpg,
                       const double *wband, double *part) {
  if (n1 != n2) return -1;
  switch (n1) {
#define PSPW_CASE(NN) \
  case NN: return launch_plane_rho<NN, NN, T>(g, st, n3, ngroups, wx, wy, S, nbb, bpg, wband, part);
    PSPW_FOR_EACH_SPLIT(PSPW_CASE)
#undef PSPW_CASE
    default: return -1;
  }
}

template <typename R>
struct PrecF;
template <>
struct PrecF<double> {
  static const double *vperm(const pspw_cell *c) { return c->d_vperm64; }
  static const double *kin(const pspw_cell *c) { return c->basis.d_kin64; }
  static const double2 *w(const FftDim &d) { return d.d_w64; }
};
template <>
struct PrecF<float> {
  static const float *vperm(const pspw_cell *c) { return c->d_vperm32; }
  static const float *kin(const pspw_cell *c) { return c->basis.d_kin32; }
  static const float2 *w(const FftDim &d) { return d.d_w32; }
};

}  // namespace fastpath

// sum of the group planes in fixed order, added to rho in natural order
static __global__ void k_rho_reduce(const double *__restrict__ part, int ngroups, int n1, int n2, int n3,
                             const int *__restrict__ px, const int *__restrict__ py,
                             const int *__restrict__ pz, double *rho) {
  const int n = n1 * n2 * n3;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double s = part[i];
    for (int gI = 1; gI < ngroups; gI++) s += part[(size_t)gI * n + i];
    const int a = i % n1, b = (i / n1) % n2, cz = i / (n1 * n2);
    rho[((size_t)pz[cz] * n2 + py[b]) * n1 + px[a]] += s;
  }
}

template <typename R>
int rho_fast(pspw_cell *c, const FastGeo &g, const cx<R> *psi, int ld, int ngw_scatter, int nb,
             const double *d_wband, double *d_rho) {
  using namespace fastpath;
  using T = cx<R>;
  const Basis &B = c->basis;
  cudaStream_t st = c->stream;
  const size_t s_band = (size_t)B.n3 * B.ncol;
  int nbatch = c->band_batch;
  if (nbatch <= 0) nbatch = (int)std::max<size_t>(1, (48u << 20) / (s_band * sizeof(T)));
  nbatch = std::min(nbatch, nb);
  const int ngroups = std::max(1, std::min(nbatch, (2 * 148 + B.n3 - 1) / B.n3));
  T *S = nullptr;
  double *part = nullptr;
  int rc;
  if ((rc = ws_reserve(c, kWsSticks, sizeof(T) * s_band * nbatch, (void **)&S)) ||
      (rc = ws_reserve(c, kWsRhoPart, sizeof(double) * (size_t)ngroups * B.nnr, (void **)&part)))
    return rc;
  const T *wx = PrecF<R>::w(B.dim[0]), *wy = PrecF<R>::w(B.dim[1]), *wz = PrecF<R>::w(B.dim[2]);
  for (int b0 = 0; b0 < nb; b0 += nbatch) {
    const int nbb = std::min(nbatch, nb - b0);
    const int bpg = (nbb + ngroups - 1) / ngroups;
    const int ng = (nbb + bpg - 1) / bpg;
    rc = dispatch_sticks_inv<T>(B.n3, g, st, nbb, wz, psi + (size_t)b0 * ld, ld, ngw_scatter, S);
    if (rc) return rc < 0 ? fail(PSPW_ERR_NOT_IMPL, "density: length not compiled") : rc;
    rc = dispatch_plane_rho<T>(B.n1, B.n2, g, st, B.n3, ng, wx, wy, S, nbb, bpg, d_wband + b0, part);
    if (rc) return rc < 0 ? fail(PSPW_ERR_NOT_IMPL, "density: plane not compiled") : rc;
    k_rho_reduce<<<2 * 148, 256, 0, st>>>(part, ng, B.n1, B.n2, B.n3, B.d_pinv[0], B.d_pinv[1],
                                           B.d_pinv[2], d_rho);
    c->kernel_launches += 3;
  }
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

template <typename R>
int local_fast(pspw_cell *c, const FastGeo &g, const cx<R> *in, int ld_in, cx<R> *out,
               int ld_out, int ngw, int nb, const ScratchPlan *plan, const RecArg<cx<R>, R> &ra) {
  using namespace fastpath;
  using T = cx<R>;
  const Basis &B = c->basis;
  cudaStream_t st = c->stream;
  const size_t s_band = (size_t)B.n3 * B.ncol;
  int nbatch = c->band_batch;
  if (nbatch <= 0) {
    // at most ~96 MB of stick buffer per batch (it stays in the 126 MB L2
    // between the three passes; on Si64 one batch of 144 bands, 73 MB, runs
    // the filter 4 % faster than two of 72), batches of equal size so no
    // launch runs with a small tail batch
    const int cap = (int)std::max<size_t>(1, (96u << 20) / (s_band * sizeof(T)));
    const int nbatches = (nb + cap - 1) / cap;
    nbatch = (nb + nbatches - 1) / nbatches;
  }
  if (plan) nbatch = plan->nbatch;
  nbatch = std::min(nbatch, nb);
  T *S = nullptr;
  if (plan) {
    S = static_cast<T *>(plan->S);
  } else {
    int rc = ws_reserve(c, 0, sizeof(T) * s_band * nbatch, (void **)&S);
    if (rc) return rc;
  }
  const T *wx = PrecF<R>::w(B.dim[0]), *wy = PrecF<R>::w(B.dim[1]), *wz = PrecF<R>::w(B.dim[2]);
  cudaEvent_t ev, e2;
  timing_begin(c, kFamLocal, &ev);
  for (int b0 = 0; b0 < nb; b0 += nbatch) {
    const int nbb = std::min(nbatch, nb - b0);
    const T *inb = in + (size_t)b0 * ld_in;
    T *outb = out + (size_t)b0 * ld_out;
    int rc;
    timing_begin(c, kFamSticksInv, &e2);
    rc = dispatch_sticks_inv<T>(B.n3, g, st, nbb, wz, inb, ld_in, ngw, S);
    timing_end(c, kFamSticksInv, e2);
    c->kernel_launches++;
    if (rc) return rc < 0 ? fail(PSPW_ERR_NOT_IMPL, "register-FFT path: length not compiled") : rc;
    timing_begin(c, kFamXlines, &e2);
    rc = dispatch_plane<T, R>(B.n1, B.n2, g, st, nbb, B.n3, wx, wy, PrecF<R>::vperm(c), S);
    timing_end(c, kFamXlines, e2);
    c->kernel_launches++;
    if (rc) return rc < 0 ? fail(PSPW_ERR_NOT_IMPL, "register-FFT path: plane not compiled") : rc;
    timing_begin(c, kFamSticksFwd, &e2);
    RecArg<T, R> rab = ra;
    if (rab.xm2) rab.xm2 += (size_t)b0 * rab.ldx;
    rc = dispatch_sticks_fwd<T, R>(B.n3, g, st, nbb, wz, S, PrecF<R>::kin(c), inb, ld_in, outb,
                                   ld_out, ngw, rab);
    timing_end(c, kFamSticksFwd, e2);
    c->kernel_launches++;
    if (rc) return rc < 0 ? fail(PSPW_ERR_NOT_IMPL, "register-FFT path: length not compiled") : rc;
  }
  timing_end(c, kFamLocal, ev);
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

}  // namespace pspw
