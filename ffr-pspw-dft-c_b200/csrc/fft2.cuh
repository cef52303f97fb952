// Two-step in-place line FFTs over shared memory, built on register DFTs.
//
// A line of length n = N1*N2 is transformed in two steps, each of which
// reads and writes the same n/NITEMS positions per work item, so a step needs
// no scratch and a single barrier separates the steps:
//
//   inverse-type (natural input -> digit-permuted output)
//     stepS<N2, N1>: item j (0<=j<N1) gathers positions j + N1*i (i<N2),
//                    DFT-N2, multiplies output k by w_n^{j*k}, writes back;
//     stepB<N1, N2>: item k (0<=k<N2) takes the block i + N1*k (i<N1),
//                    DFT-N1, writes back.
//     Result: X[k2 + N2*k1] sits at position k1 + N1*k2.
//   forward-type (digit-permuted input -> natural output)
//     stepB<N1, N2> with twiddle w_n^{k*j} on output j, then stepS<N2, N1>
//     without twiddle: X[j1 + N1*j2] lands at position j1 + N1*j2.
//
// This is Cooley-Tukey in two factors (the "four-step" decomposition) with
// the transposition left implicit in the index order; the permutation of the
// intermediate data is absorbed by indexing V_eff and the stick buffer in the
// same permuted order.  Lines are addressed as base + off(l) + pos*es, with
// the line index fastest across threads so a warp touches 32 lines at one
// position (conflict-free for unit-stride line offsets with odd padding).
#pragma once

#include "common.cuh"
#include "rdft.cuh"

namespace pspw {

// Line-length table: n -> (N1, N2).  N1 is the block (contiguous) factor.
struct NSplit {
  int n, n1, n2;
};

__host__ __device__ constexpr NSplit nsplit_for(int n) {
  switch (n) {
    case 12: return {12, 4, 3};
    case 16: return {16, 4, 4};
    case 18: return {18, 6, 3};
    case 20: return {20, 5, 4};
    case 24: return {24, 6, 4};
    case 25: return {25, 5, 5};
    case 27: return {27, 9, 3};
    case 30: return {30, 6, 5};
    case 32: return {32, 8, 4};
    case 36: return {36, 6, 6};
    case 40: return {40, 8, 5};
    case 45: return {45, 9, 5};
    case 48: return {48, 8, 6};
    case 50: return {50, 10, 5};
    case 54: return {54, 9, 6};
    case 60: return {60, 10, 6};
    case 64: return {64, 8, 8};
    case 72: return {72, 9, 8};
    case 75: return {75, 15, 5};
    case 80: return {80, 10, 8};
    case 81: return {81, 9, 9};
    case 90: return {90, 10, 9};
    case 96: return {96, 12, 8};
    case 100: return {100, 10, 10};
    case 108: return {108, 12, 9};
    case 120: return {120, 12, 10};
    case 128: return {128, 16, 8};
    default: return {n, 0, 0};
  }
}

template <typename T>
__device__ __forceinline__ T twv(const T *__restrict__ w, int t, int sign) {
  T v = w[t];
  if (sign < 0) v.y = -v.y;
  return v;
}

// Strided step: items j in [0, NB), gathers NS elements j + NB*i.
template <int NS, int NB, int S, bool TW, typename T>
__device__ __forceinline__ void stepS_item(T *line, int es, int j, const T *__restrict__ w) {
  T v[NS];
#pragma unroll
  for (int i = 0; i < NS; i++) v[i] = line[(j + NB * i) * es];
  RDft<NS, S>::run(v);
  if (TW && j) {
#pragma unroll
    for (int k = 1; k < NS; k++) v[k] = cmul(v[k], twv(w, j * k, S));
  }
#pragma unroll
  for (int i = 0; i < NS; i++) line[(j + NB * i) * es] = v[i];
}

// Block step: items k in [0, NS), block i + NB*k (i < NB).
template <int NB, int S, bool TW, typename T>
__device__ __forceinline__ void stepB_item(T *line, int es, int k, const T *__restrict__ w) {
  T v[NB];
#pragma unroll
  for (int i = 0; i < NB; i++) v[i] = line[(i + NB * k) * es];
  RDft<NB, S>::run(v);
  if (TW && k) {
#pragma unroll
    for (int j = 1; j < NB; j++) v[j] = cmul(v[j], twv(w, k * j, S));
  }
#pragma unroll
  for (int i = 0; i < NB; i++) line[(i + NB * k) * es] = v[i];
}

// Line offsets: explicit table, or l * ls.
struct Lines {
  const int *off;  // may be null
  int ls;
  int nl;
  __device__ __forceinline__ int operator()(int l) const { return off ? off[l] : l * ls; }
};

// The four step kinds over all lines of a block (no trailing barrier).
template <int N1, int N2, typename T>
__device__ __forceinline__ void inv_stepS(T *base, Lines L, int es, const T *w) {
  for (int it = threadIdx.x; it < L.nl * N1; it += blockDim.x) {
    const int l = it % L.nl, j = it / L.nl;
    stepS_item<N2, N1, +1, true>(base + L(l), es, j, w);
  }
}
template <int N1, int N2, typename T>
__device__ __forceinline__ void inv_stepB(T *base, Lines L, int es, const T *w) {
  for (int it = threadIdx.x; it < L.nl * N2; it += blockDim.x) {
    const int l = it % L.nl, k = it / L.nl;
    stepB_item<N1, +1, false>(base + L(l), es, k, w);
  }
}
template <int N1, int N2, typename T>
__device__ __forceinline__ void fwd_stepB(T *base, Lines L, int es, const T *w) {
  for (int it = threadIdx.x; it < L.nl * N2; it += blockDim.x) {
    const int l = it % L.nl, k = it / L.nl;
    stepB_item<N1, -1, true>(base + L(l), es, k, w);
  }
}
template <int N1, int N2, typename T>
__device__ __forceinline__ void fwd_stepS(T *base, Lines L, int es, const T *w) {
  for (int it = threadIdx.x; it < L.nl * N1; it += blockDim.x) {
    const int l = it % L.nl, j = it / L.nl;
    stepS_item<N2, N1, -1, false>(base + L(l), es, j, w);
  }
}

// The fused middle of an x-line sandwich: inverse block step, multiply by
// the (permuted) potential, forward block step with its twiddles.  The
// potential plane is stored x-major (vplane[x * ny + y]), so for each of the
// N1 positions of a block the lines (rows y, fastest across threads) of a
// warp read consecutive values: one coalesced load per position.
template <int N1, int N2, typename T, typename R>
__device__ __forceinline__ void inv_fwd_stepB_v(T *base, Lines L, const T *w,
                                                const R *__restrict__ vplane, int ny) {
  for (int it = threadIdx.x; it < L.nl * N2; it += blockDim.x) {
    const int l = it % L.nl, k = it / L.nl;
    T *line = base + L(l);
    R s[N1];
#pragma unroll
    for (int i = 0; i < N1; i++) s[i] = __ldg(vplane + (size_t)(N1 * k + i) * ny + l);
    T v[N1];
#pragma unroll
    for (int i = 0; i < N1; i++) v[i] = line[i + N1 * k];
    RDft<N1, +1>::run(v);
#pragma unroll
    for (int i = 0; i < N1; i++) v[i] = mk<T>(s[i] * v[i].x, s[i] * v[i].y);
    RDft<N1, -1>::run(v);
    if (k) {
#pragma unroll
      for (int j = 1; j < N1; j++) v[j] = cmul(v[j], twv(w, k * j, -1));
    }
#pragma unroll
    for (int i = 0; i < N1; i++) line[i + N1 * k] = v[i];
  }
}

// The first (inverse) and last (forward) x steps of the plane kernel, which
// move between two views of one shared buffer: the compact view holds only
// the active x positions of each row (row stride la), the full view all NX
// positions (row stride lb).  Every item first loads its inputs, the block
// synchronises, then the items write; so the views may overlap.  Items are
// (row l, j) with the row fastest; NY rows, NT threads.
//
// inverse: compact -> full, stepS<N2, N1> with twiddles; inactive x are zero.
template <int NY, int N1, int N2, int NT, typename T>
__device__ __forceinline__ void x_inv_expand(T *buf, int la, int lb, const int *xa_of_x,
                                             const T *w) {
  constexpr int NI = NY * N1, NR = (NI + NT - 1) / NT;
  T v[NR][N2];
#pragma unroll
  for (int r = 0; r < NR; r++) {
    const int it = threadIdx.x + r * NT;
    if (it < NI) {
      const int l = it % NY, j = it / NY;
#pragma unroll
      for (int i = 0; i < N2; i++) {
        const int q = xa_of_x[j + N1 * i];
        v[r][i] = q >= 0 ? buf[l * la + q] : czero<T>();
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < NR; r++) {
    const int it = threadIdx.x + r * NT;
    if (it < NI) {
      const int l = it % NY, j = it / NY;
      RDft<N2, +1>::run(v[r]);
      if (j) {
#pragma unroll
        for (int k = 1; k < N2; k++) v[r][k] = cmul(v[r][k], twv(w, j * k, +1));
      }
#pragma unroll
      for (int i = 0; i < N2; i++) buf[l * lb + j + N1 * i] = v[r][i];
    }
  }
}
// forward: full -> compact, stepS<N2, N1> without twiddles; only the active
// x positions are stored.
template <int NY, int N1, int N2, int NT, typename T>
__device__ __forceinline__ void x_fwd_compact(T *buf, int la, int lb, const int *xa_of_x) {
  constexpr int NI = NY * N1, NR = (NI + NT - 1) / NT;
  T v[NR][N2];
#pragma unroll
  for (int r = 0; r < NR; r++) {
    const int it = threadIdx.x + r * NT;
    if (it < NI) {
      const int l = it % NY, j = it / NY;
#pragma unroll
      for (int i = 0; i < N2; i++) v[r][i] = buf[l * lb + j + N1 * i];
    }
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < NR; r++) {
    const int it = threadIdx.x + r * NT;
    if (it < NI) {
      const int l = it % NY, j = it / NY;
      RDft<N2, -1>::run(v[r]);
#pragma unroll
      for (int i = 0; i < N2; i++) {
        const int q = xa_of_x[j + N1 * i];
        if (q >= 0) buf[l * la + q] = v[r][i];
      }
    }
  }
}

// Runtime dispatch over the supported lengths.  Returns false if n has no
// register split (the caller then uses the generic path).
#define PSPW_FOR_EACH_SPLIT(X) \
  X(12) X(16) X(18) X(20) X(24) X(25) X(27) X(30) X(32) X(36) X(40) X(45) X(48) X(50) X(54) \
  X(60) X(64) X(72) X(75) X(80) X(81) X(90) X(96) X(100) X(108) X(120) X(128)

enum StepKind { kInvS = 0, kInvB = 1, kFwdB = 2, kFwdS = 3 };

template <typename T>
__device__ __forceinline__ void line_step(int kind, int n, T *base, Lines L, int es, const T *w) {
  switch (n) {
#define PSPW_CASE(NN)                                                    \
  case NN: {                                                             \
    constexpr int A = nsplit_for(NN).n1, B = nsplit_for(NN).n2;          \
    if (kind == kInvS) inv_stepS<A, B>(base, L, es, w);                  \
    else if (kind == kInvB) inv_stepB<A, B>(base, L, es, w);             \
    else if (kind == kFwdB) fwd_stepB<A, B>(base, L, es, w);             \
    else fwd_stepS<A, B>(base, L, es, w);                                \
    break;                                                               \
  }
    PSPW_FOR_EACH_SPLIT(PSPW_CASE)
#undef PSPW_CASE
    default:
      break;
  }
}

}  // namespace pspw
