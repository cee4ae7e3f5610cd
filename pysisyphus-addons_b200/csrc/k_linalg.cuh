// Launch interface of the dense linear algebra kernels (k_linalg.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace pa {

// Column-major C := beta C + alpha op(A) op(B). Returns the number of launches.
int gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double* A, long long lda,
         const double* B, long long ldb, double beta, double* C, long long ldc, bool lower_only,
         cudaStream_t s);
// Doubles of scratch cholesky_lower needs for an n x n matrix (the inverted
// 64 x 64 diagonal blocks, kept for trsm_lower_left).
size_t linalg_workspace_doubles(int n);
// Second stream of the Cholesky factorization: with it, the trailing update
// beyond the next block column runs there while the next diagonal block is
// factorized on the main stream (one step of lookahead). The events order the
// two streams; all three are owned by the caller.
struct CholLookahead {
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_panel = nullptr, ev_rest = nullptr;
};
// In place: the lower triangle of A (n x n, lda = n) becomes L with A = L L^T
// (dpotrf); work receives the inverses of L's diagonal blocks. *d_info
// (device) receives 0 or the 1-based column of the first non-positive pivot.
// Without la every launch goes to s; with it the work is complete on s when
// the last launch enqueued on s completes.
int cholesky_lower(double* A, int n, int* d_info, double* work, cudaStream_t s,
                   const CholLookahead* la = nullptr);
// C := L^-1 B (n x nrhs) for the factor and work of cholesky_lower. B is
// overwritten (used as scratch).
int trsm_lower_left(const double* L, int n, const double* dinv, double* B, long long ldb, int nrhs,
                    double* C, long long ldc, cudaStream_t s);
// A[i + n i] += shift for i < n (no launch when shift == 0).
int add_diagonal(double* A, int n, double shift, cudaStream_t s);
// Coulomb tensor R[ns,ns,ns,ns] (column-major) from df[naux, ndens].
int coulomb_4d(const double* df, int naux, int ndens, int nstates, double* gram_scratch,
               double* R, cudaStream_t s);

}  // namespace pa
