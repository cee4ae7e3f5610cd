// Launch interface of the dense linear algebra kernels (k_linalg.cu).
#pragma once

#include <cuda_runtime.h>

namespace pa {

// Column-major C := beta C + alpha op(A) op(B). Returns the number of launches.
int gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double* A, long long lda,
         const double* B, long long ldb, double beta, double* C, long long ldc, bool lower_only,
         cudaStream_t s);
// In-place lower Cholesky factor of the n x n matrix A (lda = n). *d_info
// (device) receives 0 or the 1-based column of the first non-positive pivot.
int cholesky_lower(double* A, int n, int* d_info, cudaStream_t s);
// B := L^-1 B for the lower factor L (n x n, ldl = n) and nrhs columns of B.
int trsm_lower_left(const double* L, int n, double* B, long long ldb, int nrhs, cudaStream_t s);
// Coulomb tensor R[ns,ns,ns,ns] (column-major) from df[naux, ndens].
int coulomb_4d(const double* df, int naux, int ndens, int nstates, double* gram_scratch,
               double* R, cudaStream_t s);

}  // namespace pa
