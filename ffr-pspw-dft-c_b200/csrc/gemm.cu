// Complex GEMM for the subspace steps of the eigensolvers (zgemm_ calls of
// davidson_cpu.cpp, lobpcg_cpu.cpp, eig_zhegv.cpp, ChebySCFLoop.cpp):
//   C = alpha * op(A) * B + beta * C,  op(A) = A or A^H,
// column-major with leading dimensions, FP64 or FP32 complex.  FP64 products
// with more than 8 columns go to cuBLAS ZGEMM (a plain library GEMM); the
// rest use the kernels below.
//
// Tiles of 64 x 64 outputs, 256 threads, 4 x 4 outputs per thread, the K loop
// staged through shared memory.  When K is long and the output small (the
// Gram matrices X^H Y over NGW plane waves) K is split across blocks; the
// slices are reduced in a fixed order, so results do not depend on timing.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "dense.h"
#include "engine.h"
#include "gemm.h"

namespace pspw {
namespace {

constexpr int kGM = 64, kGN = 64;

template <typename T>
__device__ __forceinline__ T cj(T a) {
  return mk<T>(a.x, -a.y);
}

// part = op(A)[m0:, k-slice] * B[k-slice, n0:]  (alpha/beta applied later
// unless nsplit == 1)
template <typename R, int BK, bool CONJ_A>
__global__ void __launch_bounds__(256) k_zgemm(int m, int n, int k, cx<R> alpha,
                                               const cx<R> *__restrict__ A, int lda,
                                               const cx<R> *__restrict__ B, int ldb, cx<R> beta,
                                               cx<R> *C, int ldc, int kchunk,
                                               cx<R> *__restrict__ part) {
  using T = cx<R>;
  __shared__ T As[BK][kGM + 1];
  __shared__ T Bs[BK][kGN + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int m0 = blockIdx.x * kGM, n0 = blockIdx.y * kGN;
  const int kb = blockIdx.z * kchunk;
  const int ke = min(k, kb + kchunk);
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = czero<T>();
  for (int k0 = kb; k0 < ke; k0 += BK) {
    if (CONJ_A) {
      // A^H: element (mm, kk) is conj(A[kk + mm*lda]); contiguous in kk
      for (int e = threadIdx.x; e < BK * kGM; e += 256) {
        const int kk = e % BK, mm = e / BK;
        const int gk = k0 + kk, gm = m0 + mm;
        As[kk][mm] = (gk < ke && gm < m) ? cj(A[(size_t)gm * lda + gk]) : czero<T>();
      }
    } else {
      // A: element (mm, kk) is A[mm + kk*lda]; contiguous in mm
      for (int e = threadIdx.x; e < BK * kGM; e += 256) {
        const int mm = e % kGM, kk = e / kGM;
        const int gk = k0 + kk, gm = m0 + mm;
        As[kk][mm] = (gk < ke && gm < m) ? A[(size_t)gk * lda + gm] : czero<T>();
      }
    }
    for (int e = threadIdx.x; e < BK * kGN; e += 256) {
      const int kk = e % BK, nn = e / BK;
      const int gk = k0 + kk, gn = n0 + nn;
      Bs[kk][nn] = (gk < ke && gn < n) ? B[(size_t)gn * ldb + gk] : czero<T>();
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
    const int gn = n0 + ty + 16 * j;
    if (gn >= n) continue;
#pragma unroll
    for (int i = 0; i < 4; i++) {
      const int gm = m0 + tx + 16 * i;
      if (gm >= m) continue;
      if (part) {
        part[((size_t)blockIdx.z * n + gn) * m + gm] = acc[i][j];
      } else {
        T r = cmul(alpha, acc[i][j]);
        if (beta.x != (R)0 || beta.y != (R)0) r = r + cmul(beta, C[(size_t)gn * ldc + gm]);
        C[(size_t)gn * ldc + gm] = r;
      }
    }
  }
}

// The same for n <= 8 columns: 64 rows x 8 columns per block, thread
// (r = t & 63, c = t >> 6) owns row r and columns c and c + 4; within a K
// slice each output accumulates the same products in the same order as
// k_zgemm.
template <typename R, int BK, bool CONJ_A>
__global__ void __launch_bounds__(256) k_zgemm_n8(int m, int n, int k, cx<R> alpha,
                                                  const cx<R> *__restrict__ A, int lda,
                                                  const cx<R> *__restrict__ B, int ldb,
                                                  cx<R> beta, cx<R> *C, int ldc, int kchunk,
                                                  cx<R> *__restrict__ part) {
  using T = cx<R>;
  __shared__ T As[BK][kGM + 1];
  __shared__ T Bs[BK][8 + 1];
  const int r = threadIdx.x & 63, cc = threadIdx.x >> 6;
  const int m0 = blockIdx.x * kGM;
  const int kb = blockIdx.z * kchunk;
  const int ke = min(k, kb + kchunk);
  T acc[2] = {czero<T>(), czero<T>()};
  for (int k0 = kb; k0 < ke; k0 += BK) {
    if (CONJ_A) {
      for (int e = threadIdx.x; e < BK * kGM; e += 256) {
        const int kk = e % BK, mm = e / BK;
        const int gk = k0 + kk, gm = m0 + mm;
        As[kk][mm] = (gk < ke && gm < m) ? cj(A[(size_t)gm * lda + gk]) : czero<T>();
      }
    } else {
      for (int e = threadIdx.x; e < BK * kGM; e += 256) {
        const int mm = e % kGM, kk = e / kGM;
        const int gk = k0 + kk, gm = m0 + mm;
        As[kk][mm] = (gk < ke && gm < m) ? A[(size_t)gk * lda + gm] : czero<T>();
      }
    }
    for (int e = threadIdx.x; e < BK * 8; e += 256) {
      const int kk = e % BK, nn = e / BK;
      const int gk = k0 + kk;
      Bs[kk][nn] = (gk < ke && nn < n) ? B[(size_t)nn * ldb + gk] : czero<T>();
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
  const int gm = m0 + r;
  if (gm >= m) return;
#pragma unroll
  for (int j = 0; j < 2; j++) {
    const int gn = cc + 4 * j;
    if (gn >= n) continue;
    if (part) {
      part[((size_t)blockIdx.z * n + gn) * m + gm] = acc[j];
    } else {
      T r2 = cmul(alpha, acc[j]);
      if (beta.x != (R)0 || beta.y != (R)0) r2 = r2 + cmul(beta, C[(size_t)gn * ldc + gm]);
      C[(size_t)gn * ldc + gm] = r2;
    }
  }
}

// Single-column products (the Lanczos recurrence: V^H v and v - V h with a
// few columns V).  y = A^H x: one block per output, each thread sums a
// strided slice of the k products with four partial sums, then a fixed-order
// warp and block reduction.
template <typename R>
__global__ void __launch_bounds__(512) k_gemv_c(int k, cx<R> alpha, const cx<R> *__restrict__ A,
                                                int lda, const cx<R> *__restrict__ x, cx<R> beta,
                                                cx<R> *y) {
  using T = cx<R>;
  __shared__ T red[16];
  const int j = blockIdx.x, nt = blockDim.x;
  const T *a = A + (size_t)j * lda;
  T s0 = czero<T>(), s1 = czero<T>(), s2 = czero<T>(), s3 = czero<T>();
  int i = threadIdx.x;
  for (; i + 3 * nt < k; i += 4 * nt) {
    cfmac(s0, a[i], x[i]);
    cfmac(s1, a[i + nt], x[i + nt]);
    cfmac(s2, a[i + 2 * nt], x[i + 2 * nt]);
    cfmac(s3, a[i + 3 * nt], x[i + 3 * nt]);
  }
  for (; i < k; i += nt) cfmac(s0, a[i], x[i]);
  T t = (s0 + s1) + (s2 + s3);
  for (int o = 16; o > 0; o >>= 1) {
    t.x += __shfl_down_sync(0xffffffffu, t.x, o);
    t.y += __shfl_down_sync(0xffffffffu, t.y, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) red[warp] = t;
  __syncthreads();
  if (warp == 0) {
    t = lane < (nt >> 5) ? red[lane] : czero<T>();
    for (int o = 16; o > 0; o >>= 1) {
      t.x += __shfl_down_sync(0xffffffffu, t.x, o);
      t.y += __shfl_down_sync(0xffffffffu, t.y, o);
    }
    if (lane == 0) {
      T r = cmul(alpha, t);
      if (beta.x != (R)0 || beta.y != (R)0) r = r + cmul(beta, y[j]);
      y[j] = r;
    }
  }
}

// y = alpha A x + beta y for A with few columns: one thread per row, the
// columns summed in order
template <typename R>
__global__ void k_gemv_n(int m, int k, cx<R> alpha, const cx<R> *__restrict__ A, int lda,
                         const cx<R> *__restrict__ x, cx<R> beta, cx<R> *y) {
  using T = cx<R>;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    T s = czero<T>();
    for (int j = 0; j < k; j++) cfma(s, A[(size_t)j * lda + i], x[j]);
    T r = cmul(alpha, s);
    if (beta.x != (R)0 || beta.y != (R)0) r = r + cmul(beta, y[i]);
    y[i] = r;
  }
}

template <typename R>
__global__ void k_zgemm_reduce(int m, int n, int nsplit, const cx<R> *__restrict__ part,
                               cx<R> alpha, cx<R> beta, cx<R> *C, int ldc) {
  using T = cx<R>;
  const size_t tot = (size_t)m * n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < tot;
       i += (size_t)gridDim.x * blockDim.x) {
    T s = part[i];
    for (int p = 1; p < nsplit; p++) s = s + part[(size_t)p * tot + i];
    const int gn = (int)(i / m), gm = (int)(i - (size_t)gn * m);
    T r = cmul(alpha, s);
    if (beta.x != (R)0 || beta.y != (R)0) r = r + cmul(beta, C[(size_t)gn * ldc + gm]);
    C[(size_t)gn * ldc + gm] = r;
  }
}

// split-K reduction for narrow products: one warp per output, lanes over
// the slices in a fixed order, then a fixed shuffle tree
template <typename R>
__global__ void k_zgemm_reduce_warp(int m, int n, int nsplit, const cx<R> *__restrict__ part,
                                    cx<R> alpha, cx<R> beta, cx<R> *C, int ldc) {
  using T = cx<R>;
  const size_t tot = (size_t)m * n;
  const size_t o = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (o >= tot) return;  // uniform per warp
  T s = czero<T>();
  for (int p = lane; p < nsplit; p += 32) s = s + part[(size_t)p * tot + o];
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    s.x += __shfl_xor_sync(0xffffffffu, s.x, d);
    s.y += __shfl_xor_sync(0xffffffffu, s.y, d);
  }
  if (lane == 0) {
    const int gn = (int)(o / m), gm = (int)(o - (size_t)gn * m);
    T r = cmul(alpha, s);
    if (beta.x != (R)0 || beta.y != (R)0) r = r + cmul(beta, C[(size_t)gn * ldc + gm]);
    C[(size_t)gn * ldc + gm] = r;
  }
}

}  // namespace

template <typename R>
int zgemm(pspw_cell *c, char opa, int m, int n, int k, cx<R> alpha, const cx<R> *A, int lda,
          const cx<R> *B, int ldb, cx<R> beta, cx<R> *C, int ldc) {
  using T = cx<R>;
  if (m <= 0 || n <= 0) return PSPW_OK;
  if constexpr (sizeof(R) == 8) {
    // FP64 with more than 8 columns: a plain library GEMM on the FP64 pipe
    // (cuBLAS ZGEMM, deterministic); narrow products (the Lanczos vectors)
    // stay on the split-K kernels below, which are faster at that shape
    if (k > 0 && n > 8) {
      cublasHandle_t h;
      int rc = cublas_handle(c, &h);
      if (rc) return rc;
      cudaEvent_t ev;
      timing_begin(c, kFamGemm, &ev);
      const cublasOperation_t ta = (opa == 'C' || opa == 'c') ? CUBLAS_OP_C : CUBLAS_OP_N;
      if (cublasZgemm(h, ta, CUBLAS_OP_N, m, n, k,
                      reinterpret_cast<const cuDoubleComplex *>(&alpha),
                      reinterpret_cast<const cuDoubleComplex *>(A), lda,
                      reinterpret_cast<const cuDoubleComplex *>(B), ldb,
                      reinterpret_cast<const cuDoubleComplex *>(&beta),
                      reinterpret_cast<cuDoubleComplex *>(C), ldc) != CUBLAS_STATUS_SUCCESS)
        return fail(PSPW_ERR_CUDA, "cublasZgemm");
      timing_end(c, kFamGemm, ev);
      c->kernel_launches++;
      return PSPW_OK;
    }
  }
  cudaStream_t st = c->stream;
  if (n == 1 && k > 0) {
    // one column: matrix-vector kernels (the Lanczos recurrence)
    cudaEvent_t ev;
    timing_begin(c, kFamGemm, &ev);
    if (opa == 'C' || opa == 'c')
      k_gemv_c<R><<<m, 512, 0, st>>>(k, alpha, A, lda, B, beta, C);
    else
      k_gemv_n<R><<<(unsigned)std::min<long long>(((long long)m + 255) / 256, 4 * 148), 256, 0,
                    st>>>(m, k, alpha, A, lda, B, beta, C);
    c->kernel_launches++;
    timing_end(c, kFamGemm, ev);
    PSPW_CUDA(cudaGetLastError());
    return PSPW_OK;
  }
  constexpr int BK = sizeof(R) == 8 ? 16 : 32;
  const bool conj = (opa == 'C' || opa == 'c');
  const int mt = (m + kGM - 1) / kGM, nt = (n + kGN - 1) / kGN;
  int nsplit = 1;
  const bool narrow = n <= 8;
  if (narrow && k > 4 * BK && mt < 8 * 148) {
    // narrow products (Lanczos, single columns): short slices, many blocks
    nsplit = std::max(1, std::min((k + 63) / 64, (8 * 148 + mt - 1) / mt));
  } else if (k > 4 * BK && mt * nt < 2 * 148) {
    nsplit = std::min((k + 255) / 256, (2 * 148 + mt * nt - 1) / (mt * nt));
    nsplit = std::max(1, nsplit);
  }
  int kchunk = (k + nsplit - 1) / nsplit;
  kchunk = (kchunk + BK - 1) / BK * BK;
  if (k <= 0) kchunk = BK;
  nsplit = std::max(1, (k + kchunk - 1) / kchunk);
  T *part = nullptr;
  if (nsplit > 1) {
    int rc = ws_reserve(c, 9, sizeof(T) * (size_t)nsplit * m * n, (void **)&part);
    if (rc) return rc;
  }
  dim3 grid(mt, nt, nsplit);
  cudaEvent_t ev;
  timing_begin(c, kFamGemm, &ev);
  if (n <= 8) {
    const dim3 g8(mt, 1, nsplit);
    if (conj)
      k_zgemm_n8<R, BK, true><<<g8, 256, 0, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                  kchunk, part);
    else
      k_zgemm_n8<R, BK, false><<<g8, 256, 0, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                   kchunk, part);
  } else if (conj) {
    k_zgemm<R, BK, true><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                               kchunk, part);
  } else {
    k_zgemm<R, BK, false><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                kchunk, part);
  }
  c->kernel_launches++;
  if (nsplit > 1) {
    if (narrow)
      k_zgemm_reduce_warp<R><<<(unsigned)(((size_t)m * n * 32 + 255) / 256), 256, 0, st>>>(
          m, n, nsplit, part, alpha, beta, C, ldc);
    else
      k_zgemm_reduce<R><<<std::min<size_t>(4 * 148, ((size_t)m * n + 255) / 256), 256, 0, st>>>(
          m, n, nsplit, part, alpha, beta, C, ldc);
    c->kernel_launches++;
  }
  timing_end(c, kFamGemm, ev);
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

template int zgemm<double>(pspw_cell *, char, int, int, int, double2, const double2 *, int,
                           const double2 *, int, double2, double2 *, int);
template int zgemm<float>(pspw_cell *, char, int, int, int, float2, const float2 *, int,
                          const float2 *, int, float2, float2 *, int);

}  // namespace pspw
