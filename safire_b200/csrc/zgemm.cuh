// Batched complex128 GEMM on the FP64 tensor path (DMMA, mma.sync m8n8k4 f64).
//
//   C[b] = alpha * op(A[b]) * op(B[b]) + beta * C[b]        (row-major, C-ordered like nda views)
//   D[b] (+)= alpha * op(A[b]) * op(B[b])                     (optional second output)
//
// op(A) is A (stored m x k), A^T (stored k x m), optionally conjugated; either operand may be a
// real (float64) matrix, in which case the complex product needs only 2 (or 1) real DMMAs per
// k-step instead of 4.  This is the plain complex128 path of every dense product of the walker
// step (the reference routes these through nda -> cuBLAS / cuTENSOR, numerics/operations/
// product.hpp:125-323 and HamiltonianOperations/Real3IndexFactorization.hpp:321,384,571).
#pragma once

#include "common.cuh"

namespace afqmc {

struct GemmParams {
  int m, n, k;
  const void* A; long lda, strideA;
  const void* B; long ldb, strideB;
  c128* C; long ldc, strideC;
  c128 alpha, beta;
  c128* D; long ldd, strideD;  // optional second output (nullptr: none)
  bool d_store;                 // D = result (true) or D += result (false)
};

// op codes for the C++ launcher
enum GemmTrans : int { GN = 0, GT = 1, GC = 2, GH = 3 };  // N, T, conj, conj-transpose

// Launch C = alpha*op(A)*op(B) + beta*C over `batch` problems on `stream`.
// a_real / b_real: the operand is float64 instead of complex128.
int zgemm(cudaStream_t stream, int batch, GemmTrans ta, bool a_real, GemmTrans tb, bool b_real,
          const GemmParams& p);

}  // namespace afqmc
