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

}  // namespace pspw
