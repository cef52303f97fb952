// Complex GEMM for the subspace steps of the eigensolvers (zgemm_ calls of
// davidson_cpu.cpp, lobpcg_cpu.cpp, eig_zhegv.cpp, ChebySCFLoop.cpp) and the
// FP64 projector products of H*psi (ApplyHam_block.cpp:86-117):
//   C = alpha * op(A) * B + beta * C,  op(A) = A or A^H,
// column-major with leading dimensions, FP64 or FP32 complex.
//
// FP64 products with more than 8 columns run on the FP64 tensor-core
// instruction (DMMA: mma.sync m16n8k4 .f64, the only tensor-core form of
// FP64 arithmetic on sm_100a; tcgen05 has no FP64 kind).  A complex product
// is four real products on split real/imaginary fragments:
//   Cr += Ar Br - Ai Bi,  Ci += Ar Bi + Ai Br   (A^H: Ai -> -Ai).
// Warps of 32 x 16 outputs in blocks of 64 x 64, 64 x 32 or 32 x 32 (the
// shape that pads the output least), K staged through a four-deep cp.async
// ring of 8-wide complex tiles.  Operands whose K index
// is contiguous in memory (A^H, B) are staged [row][k]; A in the 'N' form is
// staged [k][m] (its M index is contiguous), both padded so that the 16-byte
// fragment loads of a quarter warp hit distinct banks.
//
// FP32 products and FP64 products of at most 8 columns use the SIMT kernels
// below: tiles of 64 x 64 outputs, 256 threads, 4 x 4 outputs per thread,
// and a narrow 64 x 8 form.  Single columns use matrix-vector kernels.
//
// When K is long and the output small (the Gram matrices X^H Y over NGW
// plane waves) K is split across blocks; the slices are reduced in a fixed
// order, so results do not depend on timing.
#include <cuda_runtime.h>

#include <algorithm>

#include "common.cuh"
#include "dense.h"
#include "engine.h"
#include "gemm.h"
#include "tc.cuh"

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

// ---------------------------------------------------------------- FP64 DMMA
// Block tiles of (32 WM) x (16 WN) outputs, WM x WN warps of 32 x 16 each:
// 64 x 64 (8 warps), 64 x 32 (4 warps) or 32 x 32 (2 warps); the host picks
// the tile that pads the output least (e.g. 146 columns: 160 with 32-wide
// tiles against 192 with 64-wide ones).
template <int WM, int WN>
struct Dm {
  static constexpr int BM = 32 * WM, BN = 16 * WN, BK = 8, STAGES = 4;
  static constexpr int THREADS = 32 * WM * WN;
  // [row][k] tiles: BK + 4 = 12 complex per row (12 = 4 mod 8): the fragment
  // loads of a quarter warp (rows g, g+1; k = t..t+3) cover 8 distinct
  // 16-byte bank groups.  [k][m] tiles: BM + 2 per k (= 2 mod 8), likewise.
  static constexpr int LDK = BK + 4, LDM = BM + 2;
  static constexpr int A_ELEMS = BM * LDK > BK * LDM ? BM * LDK : BK * LDM;
  static constexpr int B_ELEMS = BN * LDK;
  static constexpr int STAGE = A_ELEMS + B_ELEMS;  // complex elements per ring slot
  static constexpr size_t SMEM = sizeof(double2) * STAGE * STAGES;
  static constexpr int MIN_BLOCKS = 16 / (WM * WN);  // 2, 4 or 8 blocks of registers per SM
};

// d(16 x 8) += a(16 x 4) b(4 x 8), FP64: lane (g = lane / 4, t = lane % 4)
// holds a = A[g][t], A[g+8][t]; b = B[t][g]; d = D[g][2t], D[g][2t+1],
// D[g+8][2t], D[g+8][2t+1]
__device__ __forceinline__ void dmma(double (&d)[4], double a0, double a1, double b) {
  asm volatile(
      "mma.sync.aligned.m16n8k4.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
      "{%0,%1,%2,%3};"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a0), "d"(a1), "d"(b));
}

// part or C over the block's K slice [blockIdx.z * kchunk, +kchunk)
template <bool CONJ_A, int WM, int WN>
__global__ void __launch_bounds__(Dm<WM, WN>::THREADS, Dm<WM, WN>::MIN_BLOCKS)
    k_zgemm_dmma(int m, int n, int k, double2 alpha, const double2 *__restrict__ A, int lda,
                 const double2 *__restrict__ B, int ldb, double2 beta, double2 *C, int ldc,
                 int kchunk, double2 *__restrict__ part, int tri) {
  using D = Dm<WM, WN>;
  constexpr int BM = D::BM, BN = D::BN, BK = D::BK, STAGES = D::STAGES, THREADS = D::THREADS;
  constexpr int LDK = D::LDK, LDM = D::LDM, A_ELEMS = D::A_ELEMS, STAGE = D::STAGE;
  extern __shared__ __align__(16) double2 sm[];
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
  const int kb = blockIdx.z * kchunk;
  // kZgemmUpperB: rows of B past n0 + BN - 1 are zero in this column tile
  const int ke = min(min(k, kb + kchunk), tri == kZgemmUpperB ? n0 + BN : k);
  // kZgemmUpperC: a tile wholly below the diagonal keeps a zero product
  const bool skip = tri == kZgemmUpperC && m0 >= n0 + BN;
  const int nkt = ke > kb && !skip ? (ke - kb + BK - 1) / BK : 0;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wm = (warp % WM) * 32, wn = (warp / WM) * 16;
  const int g = lane >> 2, t = lane & 3;

  // one ring slot of 16-byte copies, zero-filled outside the matrices
  auto load = [&](int kt, int slot) {
    double2 *As = sm + slot * STAGE, *Bs = As + A_ELEMS;
    const int k0 = kb + kt * BK;
#pragma unroll
    for (int e = tid; e < BN * BK; e += THREADS) {
      const int r = e / BK, kk = e % BK;
      const int gn = n0 + r, gk = k0 + kk;
      const bool ok = gn < n && gk < ke;
      tc::cp_async16(Bs + r * LDK + kk, ok ? B + (size_t)gn * ldb + gk : B, ok);
    }
    if (CONJ_A) {  // A is k x m; A^H(mm, kk) = conj(A[mm * lda + kk]), K contiguous
#pragma unroll
      for (int e = tid; e < BM * BK; e += THREADS) {
        const int r = e / BK, kk = e % BK;
        const int gm = m0 + r, gk = k0 + kk;
        const bool ok = gm < m && gk < ke;
        tc::cp_async16(As + r * LDK + kk, ok ? A + (size_t)gm * lda + gk : A, ok);
      }
    } else {  // A is m x k; A(mm, kk) = A[kk * lda + mm], M contiguous
#pragma unroll
      for (int e = tid; e < BM * BK; e += THREADS) {
        const int kk = e / BM, r = e % BM;
        const int gm = m0 + r, gk = k0 + kk;
        const bool ok = gm < m && gk < ke;
        tc::cp_async16(As + kk * LDM + r, ok ? A + (size_t)gk * lda + gm : A, ok);
      }
    }
  };

  double cr[2][2][4], ci[2][2][4];  // [m16 sub-tile][n8 sub-tile][fragment]
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) cr[i][j][q] = ci[i][j][q] = 0.0;

#pragma unroll
  for (int s = 0; s < STAGES - 1; s++) {
    if (s < nkt) load(s, s);
    tc::cp_async_commit();
  }
  for (int kt = 0; kt < nkt; kt++) {
    tc::cp_async_wait<STAGES - 2>();
    __syncthreads();  // slot kt % STAGES landed for all; slot (kt-1) % STAGES free
    if (kt + STAGES - 1 < nkt) load(kt + STAGES - 1, (kt + STAGES - 1) % STAGES);
    tc::cp_async_commit();
    const double2 *As = sm + (kt % STAGES) * STAGE, *Bs = As + A_ELEMS;
#pragma unroll
    for (int ks = 0; ks < BK; ks += 4) {
      double ar[2][2], ai[2][2], an[2][2], br[2], bi[2];
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int h = 0; h < 2; h++) {
          const int row = wm + i * 16 + g + 8 * h;
          const double2 v = CONJ_A ? As[row * LDK + ks + t] : As[(ks + t) * LDM + row];
          ar[i][h] = v.x;
          ai[i][h] = CONJ_A ? -v.y : v.y;  // imaginary part of op(A)
          an[i][h] = -ai[i][h];
        }
#pragma unroll
      for (int j = 0; j < 2; j++) {
        const double2 v = Bs[(wn + j * 8 + g) * LDK + ks + t];
        br[j] = v.x;
        bi[j] = v.y;
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
          dmma(cr[i][j], ar[i][0], ar[i][1], br[j]);
          dmma(cr[i][j], an[i][0], an[i][1], bi[j]);
          dmma(ci[i][j], ar[i][0], ar[i][1], bi[j]);
          dmma(ci[i][j], ai[i][0], ai[i][1], br[j]);
        }
    }
  }
  tc::cp_async_wait<0>();

#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
      for (int q = 0; q < 4; q++) {
        const int gm = m0 + wm + i * 16 + g + 8 * (q >> 1);
        const int gn = n0 + wn + j * 8 + 2 * t + (q & 1);
        if (gm >= m || gn >= n) continue;
        const double2 acc = make_double2(cr[i][j][q], ci[i][j][q]);
        if (part) {
          part[((size_t)blockIdx.z * n + gn) * m + gm] = acc;
        } else {
          double2 r = cmul(alpha, acc);
          if (beta.x != 0.0 || beta.y != 0.0) r = r + cmul(beta, C[(size_t)gn * ldc + gm]);
          C[(size_t)gn * ldc + gm] = r;
        }
      }
}

}  // namespace

static int sm_count_now() {
  static const int n = [] {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
  }();
  return n;
}

template <int WM, int WN>
static int launch_dmma(pspw_cell *c, bool conj, int m, int n, int k, double2 alpha,
                       const double2 *A, int lda, const double2 *B, int ldb, double2 beta,
                       double2 *C, int ldc, int tri) {
  using D = Dm<WM, WN>;
  cudaStream_t st = c->stream;
  const int mt = (m + D::BM - 1) / D::BM, nt = (n + D::BN - 1) / D::BN;
  // K split over blocks when the output has fewer blocks than the SMs hold
  const int target = D::MIN_BLOCKS * sm_count_now();
  int nsplit = 1;
  if (k > 8 * D::BK && mt * nt < target)
    nsplit = std::max(1, std::min((k + 255) / 256, (target + mt * nt - 1) / (mt * nt)));
  int kchunk = k > 0 ? (k + nsplit - 1) / nsplit : D::BK;
  kchunk = (kchunk + D::BK - 1) / D::BK * D::BK;
  nsplit = k > 0 ? (k + kchunk - 1) / kchunk : 1;
  double2 *part = nullptr;
  if (nsplit > 1) {
    int rc = ws_reserve(c, kWsGemmPart, sizeof(double2) * (size_t)nsplit * m * n, (void **)&part);
    if (rc) return rc;
  }
  auto kern = conj ? k_zgemm_dmma<true, WM, WN> : k_zgemm_dmma<false, WM, WN>;
  if (D::SMEM > 48 * 1024) {
    const int rc = smem_allow_max(kern);
    if (rc) return rc;
  }
  cudaEvent_t ev;
  timing_begin(c, kFamGemm, &ev);
  kern<<<dim3(mt, nt, nsplit), D::THREADS, D::SMEM, st>>>(m, n, k, alpha, A, lda, B, ldb, beta,
                                                          C, ldc, kchunk, part, tri);
  c->kernel_launches++;
  if (nsplit > 1) {
    k_zgemm_reduce<double><<<std::min<size_t>(4 * 148, ((size_t)m * n + 255) / 256), 256, 0,
                             st>>>(m, n, nsplit, part, alpha, beta, C, ldc);
    c->kernel_launches++;
  }
  timing_end(c, kFamGemm, ev);
  PSPW_CUDA(cudaGetLastError());
  return PSPW_OK;
}

// FP64, more than 8 columns: DMMA tiles of the shape that pads the output
// least (ties go to the larger tile, which re-reads its operands less)
static int zgemm_dmma(pspw_cell *c, bool conj, int m, int n, int k, double2 alpha,
                      const double2 *A, int lda, const double2 *B, int ldb, double2 beta,
                      double2 *C, int ldc, int tri = 0) {
  auto padded = [&](int bm, int bn) {
    return (double)((m + bm - 1) / bm * bm) * (double)((n + bn - 1) / bn * bn);
  };
  const double a64 = padded(64, 64), a6432 = padded(64, 32), a32 = padded(32, 32);
  if (a64 <= a6432 && a64 <= a32)
    return launch_dmma<2, 4>(c, conj, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri);
  if (a6432 <= a32)
    return launch_dmma<2, 2>(c, conj, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri);
  return launch_dmma<1, 2>(c, conj, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, tri);
}

int zgemm_tri(pspw_cell *c, char opa, int tri, int m, int n, int k, double2 alpha,
              const double2 *A, int lda, const double2 *B, int ldb, double2 beta, double2 *C,
              int ldc) {
  if (opa != 'N' && opa != 'n' && opa != 'C' && opa != 'c')
    return fail(PSPW_ERR_ARG, "zgemm_tri: op(A) must be 'N' or 'C'");
  if (tri == kZgemmUpperC && m != n) return fail(PSPW_ERR_ARG, "zgemm_tri: C must be square");
  if (n <= 8 || m <= 0 || k <= 0)  // the narrow kernels: the full product
    return zgemm<double>(c, opa, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
  return zgemm_dmma(c, opa == 'C' || opa == 'c', m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                    tri);
}

template <typename R>
int zgemm(pspw_cell *c, char opa, int m, int n, int k, cx<R> alpha, const cx<R> *A, int lda,
          const cx<R> *B, int ldb, cx<R> beta, cx<R> *C, int ldc) {
  using T = cx<R>;
  if (opa != 'N' && opa != 'n' && opa != 'C' && opa != 'c')
    return fail(PSPW_ERR_ARG, "zgemm: op(A) must be 'N' or 'C'");
  if (m <= 0 || n <= 0) return PSPW_OK;
  if constexpr (sizeof(R) == 8) {
    // FP64 with more than 8 columns: the DMMA kernel
    if (n > 8) return zgemm_dmma(c, opa == 'C' || opa == 'c', m, n, k, alpha, A, lda, B, ldb,
                                 beta, C, ldc);
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
