// FP64 GEMM on the FP64 tensor cores (mma.sync m8n8k4 f64), written for
// sm_100a; used by the QR stage, the re-orthogonalisation of the mixed
// engine and the products that assemble U and V.
#pragma once

#include <cuda_runtime.h>

namespace jsvd {

// C = alpha op(A) op(B) + beta C, column-major, op = 'N' or 'T'.  op(A) is
// m x k, op(B) k x n.  lower != 0 writes only the elements on or below the
// diagonal of C (the DSYRK-lower contract) and skips tiles above it.  beta == 0
// never reads C.  Leading dimensions are in elements.  Returns JSVD_OK or a
// JSVD_ERR_* code (launch failure).
int dgemm(cudaStream_t st, char opA, char opB, int m, int n, int k, double alpha, const double *A, long lda,
          const double *B, long ldb, double beta, double *C, long ldc, int lower = 0);

// Launches issued by dgemm on this thread (cumulative).
unsigned long long dgemm_launches();

}  // namespace jsvd
