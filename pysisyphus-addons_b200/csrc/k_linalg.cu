// Dense FP64 linear algebra of the density-fitting path (column-major):
//  * blocked right-looking Cholesky of the metric, lower triangle
//    (replaces dpotrf("L"), common/linalg.f90:78);
//  * blocked forward substitution B := L^-1 B, which replaces the reference's
//    dtrtri("L","N") + dtrmm("L","L","N","N") pair (common/linalg.f90:81,
//    diabatization/intor.f90:198) by the same product computed without
//    forming L^-1;
//  * a tiled FP64 GEMM C := beta C + alpha op(A) op(B) used by the trailing
//    updates and by the Coulomb-tensor Gram matrix;
//  * the 8-fold-symmetric scatter of the Coulomb tensor
//    (diabatization/intor.f90:241-269).
#include <algorithm>

#include "k_linalg.cuh"

namespace pa {

namespace {

constexpr int NB = 64;

// Unblocked Cholesky of the nb x nb diagonal block at (j0, j0) in shared memory.
__global__ void __launch_bounds__(256) k_potrf_diag(double* A, long long lda, int j0, int nb,
                                                    int* info) {
  __shared__ double S[NB][NB + 1];
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int i = idx % nb, j = idx / nb;
    S[i][j] = (i >= j) ? A[(j0 + i) + lda * (j0 + j)] : 0.0;
  }
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    if (threadIdx.x == 0) {
      const double d = S[k][k];
      if (!(d > 0.0)) {
        if (*info == 0) *info = j0 + k + 1;
        S[k][k] = 1.0;  // keep the factorization finite; the error is reported
      } else {
        S[k][k] = sqrt(d);
      }
    }
    __syncthreads();
    const double dkk = S[k][k];
    for (int i = k + 1 + threadIdx.x; i < nb; i += blockDim.x) S[i][k] /= dkk;
    __syncthreads();
    const int m = nb - k - 1;
    for (int idx = threadIdx.x; idx < m * m; idx += blockDim.x) {
      const int i = k + 1 + idx % m, j = k + 1 + idx / m;
      if (i >= j) S[i][j] -= S[i][k] * S[j][k];
    }
    __syncthreads();
  }
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int i = idx % nb, j = idx / nb;
    if (i >= j) A[(j0 + i) + lda * (j0 + j)] = S[i][j];
  }
}

// Panel solve: rows r in [r0, n) of columns j0..j0+nb: A[r, j0:] := A[r, j0:] L_kk^-T.
constexpr int kPanelRows = 128;
__global__ void __launch_bounds__(kPanelRows) k_trsm_panel(double* A, long long lda, int n, int j0,
                                                           int nb) {
  extern __shared__ double dsm[];
  double(*Lk)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm);
  double(*X)[kPanelRows + 1] = reinterpret_cast<double(*)[kPanelRows + 1]>(dsm + NB * (NB + 1));
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int i = idx % nb, j = idx / nb;
    Lk[i][j] = (i >= j) ? A[(j0 + i) + lda * (j0 + j)] : 0.0;
  }
  const int r = j0 + nb + blockIdx.x * kPanelRows + threadIdx.x;
  const bool ok = r < n;
  for (int j = 0; j < nb; ++j) X[j][threadIdx.x] = ok ? A[r + lda * (j0 + j)] : 0.0;
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    double x = X[j][threadIdx.x];
    for (int l = 0; l < j; ++l) x -= X[l][threadIdx.x] * Lk[j][l];
    X[j][threadIdx.x] = x / Lk[j][j];
  }
  if (ok)
    for (int j = 0; j < nb; ++j) A[r + lda * (j0 + j)] = X[j][threadIdx.x];
}

// Diagonal-block forward substitution for a block of right-hand sides:
// B[j0:j0+nb, c] := L_kk^-1 B[j0:j0+nb, c].
constexpr int kRhsCols = 64;
__global__ void __launch_bounds__(kRhsCols) k_trsm_diag(const double* L, long long ldl, double* B,
                                                        long long ldb, int nrhs, int j0, int nb) {
  extern __shared__ double dsm[];
  double(*Lk)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm);
  double(*X)[kRhsCols + 1] = reinterpret_cast<double(*)[kRhsCols + 1]>(dsm + NB * (NB + 1));
  for (int idx = threadIdx.x; idx < nb * nb; idx += blockDim.x) {
    const int i = idx % nb, j = idx / nb;
    Lk[i][j] = (i >= j) ? L[(j0 + i) + ldl * (j0 + j)] : 0.0;
  }
  const int c = blockIdx.x * kRhsCols + threadIdx.x;
  const bool ok = c < nrhs;
  for (int j = 0; j < nb; ++j) X[j][threadIdx.x] = ok ? B[(j0 + j) + ldb * c] : 0.0;
  __syncthreads();
  for (int j = 0; j < nb; ++j) {
    double x = X[j][threadIdx.x];
    for (int l = 0; l < j; ++l) x -= Lk[j][l] * X[l][threadIdx.x];
    X[j][threadIdx.x] = x / Lk[j][j];
  }
  if (ok)
    for (int j = 0; j < nb; ++j) B[(j0 + j) + ldb * c] = X[j][threadIdx.x];
}

// C[m x n] := beta C + alpha op(A) op(B); op(A) is m x k, op(B) is k x n.
// 64 x 64 tiles, k-steps of 16, 256 threads with 4 x 4 outputs each.
// lower_only: skip tiles strictly above the diagonal (and entries above it).
constexpr int TM = 64, TN = 64, TK = 16;
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_gemm(int m, int n, int k, double alpha,
                                              const double* __restrict__ A, long long lda,
                                              const double* __restrict__ B, long long ldb,
                                              double beta, double* C, long long ldc,
                                              int lower_only) {
  const int bi = blockIdx.x, bj = blockIdx.y;
  if (lower_only && bj > bi) return;
  __shared__ double As[TK][TM + 1];
  __shared__ double Bs[TK][TN + 1];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int i0 = bi * TM, j0 = bj * TN;
  double acc[4][4] = {};
  for (int kk = 0; kk < k; kk += TK) {
    for (int idx = threadIdx.x; idx < TK * TM; idx += 256) {
      int r, c;  // r in tile rows (m), c in k
      if (TA) {  // A stored k x m: op(A)(r, c) = A[c + lda * r]; read along c fastest
        c = idx % TK;
        r = idx / TK;
      } else {
        r = idx % TM;
        c = idx / TM;
      }
      const int gi = i0 + r, gk = kk + c;
      double v = 0.0;
      if (gi < m && gk < k) v = TA ? A[gk + lda * gi] : A[gi + lda * gk];
      As[c][r] = v;
    }
    for (int idx = threadIdx.x; idx < TK * TN; idx += 256) {
      int r, c;  // r in k, c in tile cols (n)
      if (TB) {  // B stored n x k: op(B)(r, c) = B[c + ldb * r]
        c = idx % TN;
        r = idx / TN;
      } else {
        r = idx % TK;
        c = idx / TK;
      }
      const int gk = kk + r, gj = j0 + c;
      double v = 0.0;
      if (gk < k && gj < n) v = TB ? B[gj + ldb * gk] : B[gk + ldb * gj];
      Bs[r][c] = v;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < TK; ++q) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[q][tx + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = Bs[q][ty + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gi = i0 + tx + 16 * i, gj = j0 + ty + 16 * j;
      if (gi < m && gj < n && (!lower_only || gi >= gj)) {
        double* c = C + gi + ldc * gj;
        *c = (beta == 0.0 ? 0.0 : beta * *c) + alpha * acc[i][j];
      }
    }
}

// R(i,j,k,l) = Gram[pair(i,j)][pair(k,l)], pair(i,j) = max(max+1)/2 + min.
__global__ void k_coulomb4d(const double* __restrict__ gram, int ndens, int ns, double* R) {
  const long long total = static_cast<long long>(ns) * ns * ns * ns;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    long long t = idx;
    const int i = t % ns;
    t /= ns;
    const int j = t % ns;
    t /= ns;
    const int k = t % ns;
    const int l = static_cast<int>(t / ns);
    const int a = max(i, j), b = min(i, j), c = max(k, l), d = min(k, l);
    const int p1 = a * (a + 1) / 2 + b, p2 = c * (c + 1) / 2 + d;
    R[idx] = gram[p1 + static_cast<long long>(ndens) * p2];
  }
}

}  // namespace

int gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double* A, long long lda,
         const double* B, long long ldb, double beta, double* C, long long ldc, bool lower_only,
         cudaStream_t s) {
  if (m <= 0 || n <= 0) return 0;
  dim3 grid((m + TM - 1) / TM, (n + TN - 1) / TN);
  const int lo = lower_only ? 1 : 0;
  if (!ta && !tb)
    k_gemm<false, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lo);
  else if (!ta && tb)
    k_gemm<false, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lo);
  else if (ta && !tb)
    k_gemm<true, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lo);
  else
    k_gemm<true, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lo);
  return 1;
}

constexpr size_t kPanelSmem = sizeof(double) * (NB * (NB + 1) + NB * (kPanelRows + 1));
constexpr size_t kDiagSmem = sizeof(double) * (NB * (NB + 1) + NB * (kRhsCols + 1));

int cholesky_lower(double* A, int n, int* d_info, cudaStream_t s) {
  int launches = 0;
  cudaFuncSetAttribute(k_trsm_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmem);
  cudaMemsetAsync(d_info, 0, sizeof(int), s);
  for (int j0 = 0; j0 < n; j0 += NB) {
    const int nb = std::min(NB, n - j0);
    k_potrf_diag<<<1, 256, 0, s>>>(A, n, j0, nb, d_info);
    ++launches;
    const int rest = n - j0 - nb;
    if (rest > 0) {
      k_trsm_panel<<<(rest + kPanelRows - 1) / kPanelRows, kPanelRows, kPanelSmem, s>>>(A, n, n, j0, nb);
      ++launches;
      // trailing lower update: A22 -= P P^T
      double* P = A + (j0 + nb) + static_cast<long long>(n) * j0;
      double* A22 = A + (j0 + nb) + static_cast<long long>(n) * (j0 + nb);
      launches += gemm(false, true, rest, rest, nb, -1.0, P, n, P, n, 1.0, A22, n, true, s);
    }
  }
  return launches;
}

int trsm_lower_left(const double* L, int n, double* B, long long ldb, int nrhs, cudaStream_t s) {
  int launches = 0;
  if (nrhs <= 0) return 0;
  cudaFuncSetAttribute(k_trsm_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiagSmem);
  for (int j0 = 0; j0 < n; j0 += NB) {
    const int nb = std::min(NB, n - j0);
    k_trsm_diag<<<(nrhs + kRhsCols - 1) / kRhsCols, kRhsCols, kDiagSmem, s>>>(L, n, B, ldb, nrhs, j0, nb);
    ++launches;
    const int rest = n - j0 - nb;
    if (rest > 0) {
      const double* Lp = L + (j0 + nb) + static_cast<long long>(n) * j0;
      launches += gemm(false, false, rest, nrhs, nb, -1.0, Lp, n, B + j0, ldb, 1.0,
                       B + j0 + nb, ldb, false, s);
    }
  }
  return launches;
}

int coulomb_4d(const double* df, int naux, int ndens, int nstates, double* gram_scratch,
               double* R, cudaStream_t s) {
  int launches = gemm(true, false, ndens, ndens, naux, 1.0, df, naux, df, naux, 0.0, gram_scratch,
                      ndens, false, s);
  const long long total = static_cast<long long>(nstates) * nstates * nstates * nstates;
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 4096));
  k_coulomb4d<<<std::max(blocks, 1), 256, 0, s>>>(gram_scratch, ndens, nstates, R);
  return launches + 1;
}

}  // namespace pa
