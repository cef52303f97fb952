// Device complex GEMM used by the eigensolvers (gemm.cu).
#pragma once

#include "common.cuh"
#include "engine.h"

namespace pspw {

// C = alpha * op(A) * B + beta * C on the cell stream; op(A) = A ('N') or
// A^H ('C').  Column-major, A is m x k ('N') or k x m ('C').
template <typename R>
int zgemm(pspw_cell *c, char opa, int m, int n, int k, cx<R> alpha, const cx<R> *A, int lda,
          const cx<R> *B, int ldb, cx<R> beta, cx<R> *C, int ldc);

// FP64 zgemm with triangular structure the tiles can skip (the CholeskyQR
// products):
//   kZgemmUpperC: only the upper triangle of C (m == n) is wanted; output
//                 tiles wholly below the diagonal are written as beta * C
//                 (alpha times a zero product) without their K loop;
//   kZgemmUpperB: B (k x n) is upper triangular (zero below the diagonal,
//                 stored as zeros), so column tile [n0, n0 + BN) stops its K
//                 loop at row n0 + BN; the result is the full product's.
// Every element the caller reads is the one zgemm gives.
constexpr int kZgemmUpperC = 1, kZgemmUpperB = 2;
int zgemm_tri(pspw_cell *c, char opa, int tri, int m, int n, int k, double2 alpha,
              const double2 *A, int lda, const double2 *B, int ldb, double2 beta, double2 *C,
              int ldc);

}  // namespace pspw
