// Dense FP64 linear algebra of the density-fitting path (column-major):
//  * blocked right-looking Cholesky of the metric, lower triangle
//    (replaces dpotrf("L"), common/linalg.f90:78); each 64 x 64 diagonal block is
//    factorized and inverted by one thread block, the panel below it is
//    scaled in place and the trailing matrix updated by a lower GEMM;
//  * L^-1 df as a blocked forward substitution on the density columns, using
//    the inverted diagonal blocks (replaces dtrtri("L","N"), common/linalg.f90:81,
//    followed by dtrmm("L","L","N","N"), diabatization/intor.f90:198: the
//    explicit inverse is never formed);
//  * a tiled FP64 GEMM C := beta C + alpha op(A) op(B) on the FP64 tensor
//    cores with optional lower triangular A, used by all of the above and by
//    the Coulomb-tensor Gram matrix;
//  * the 8-fold-symmetric scatter of the Coulomb tensor
//    (diabatization/intor.f90:241-269).
#include <algorithm>

#include "k_linalg.cuh"

#include <cstdint>

namespace pa {

namespace {

constexpr int NB = 64;

// Factorize the nb x nb diagonal block at (j0, j0) in place (lower) and write
// its inverse (lower, zeros above the diagonal, NB x NB) to dinv. The serial
// part is kept short: one square root and one reciprocal per pivot, the
// columns scaled by the reciprocal (as dpotf2 does), rows held in registers.
//  * Cholesky, per 16-column sub-block: warp 0 factors the 16 x 16 diagonal
//    sub-block (lane r holds row r, pivots and L(j, k) move by shuffles); one
//    thread per row below solves x L11^T = a in registers; all threads update
//    the trailing lower triangle;
//  * inverse: four warps invert the diagonal sub-blocks (lane c holds column c
//    in registers), then block rows i = 1..3 follow from
//    X_ij = -X_ii sum_(j <= k < i) L_ik X_kj.
constexpr int SB = 16;
__global__ void __launch_bounds__(256) k_potrf_diag_inv(double* A, long long lda, int j0, int nb,
                                                        double* dinv, int* info) {
  extern __shared__ double dsm[];
  double(*S)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm);                       // the block, then L
  double(*Xs)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm + NB * (NB + 1));      // L^-1
  double(*Ts)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(dsm + 2 * NB * (NB + 1));  // block-row sums
  __shared__ double invd[NB];                                                           // 1 / L(j, j)
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int idx = tid; idx < NB * NB; idx += 256) {
    const int r = idx & (NB - 1), c = idx >> 6;
    S[r][c] = (r < nb && c < nb) ? (c <= r ? A[(j0 + r) + lda * (j0 + c)] : 0.0) : (r == c ? 1.0 : 0.0);
    Xs[r][c] = 0.0;
  }
  __syncthreads();
  for (int k0 = 0; k0 < NB; k0 += SB) {
    if (warp == 0) {
      // lanes 16..31 repeat lanes 0..15 (they only feed the shuffles)
      const int r = lane & (SB - 1);
      double v[SB];
#pragma unroll
      for (int j = 0; j < SB; ++j) v[j] = (j <= r) ? S[k0 + r][k0 + j] : 0.0;
#pragma unroll
      for (int k = 0; k < SB; ++k) {
        double dkk = __shfl_sync(0xffffffffu, v[k], k);
        if (!(dkk > 0.0)) {
          if (lane == 0 && k0 + k < nb) atomicCAS(info, 0, j0 + k0 + k + 1);
          dkk = 1.0;  // keep the factor finite; the error is reported through info
        }
        const double d = sqrt(dkk);
        const double id = 1.0 / d;
        if (r == k) v[k] = d;
        if (r > k) v[k] *= id;  // L(r, k)
#pragma unroll
        for (int j = 1; j < SB; ++j) {  // fixed trip count: j > k folds once k is unrolled
          if (j <= k) continue;
          const double ljk = __shfl_sync(0xffffffffu, v[k], j);  // L(j, k) from lane j
          if (r >= j) v[j] = fma(-v[k], ljk, v[j]);
        }
        if (lane == k) invd[k0 + k] = id;
      }
      if (lane < SB) {
#pragma unroll
        for (int j = 0; j < SB; ++j)
          if (j <= r) S[k0 + r][k0 + j] = v[j];
      }
    }
    __syncthreads();
    // panel rows below: x L11^T = a, right-looking in registers, one thread per row
    const int pr = k0 + SB + tid;
    if (pr < NB) {
      double v[SB];
#pragma unroll
      for (int j = 0; j < SB; ++j) v[j] = S[pr][k0 + j];
#pragma unroll
      for (int j = 0; j < SB; ++j) {
        v[j] *= invd[k0 + j];
#pragma unroll
        for (int jj = 1; jj < SB; ++jj)
          if (jj > j) v[jj] = fma(-v[j], S[k0 + jj][k0 + j], v[jj]);
      }
#pragma unroll
      for (int j = 0; j < SB; ++j) S[pr][k0 + j] = v[j];
    }
    __syncthreads();
    // trailing lower triangle: S[r][c] -= sum_k S[r][k] S[c][k], k in the sub-block
    const int m = NB - k0 - SB;
    for (int e = tid; e < m * m; e += 256) {
      const int rr = k0 + SB + e / m, cc = k0 + SB + e % m;
      if (cc > rr) continue;
      double v = S[rr][cc];
#pragma unroll
      for (int k = 0; k < SB; ++k) v = fma(-S[rr][k0 + k], S[cc][k0 + k], v);
      S[rr][cc] = v;
    }
    __syncthreads();
  }
  // write the factor back
  for (int idx = tid; idx < NB * NB; idx += 256) {
    const int r = idx & (NB - 1), c = idx >> 6;
    if (r < nb && c <= r) A[(j0 + r) + lda * (j0 + c)] = S[r][c];
  }
  // diagonal sub-blocks of the inverse: warp w < 4 inverts sub-block w by
  // forward substitution, lane c holding column c
  if (warp < NB / SB) {
    const int o = warp * SB, c = lane & (SB - 1);
    double x[SB];
#pragma unroll
    for (int i = 0; i < SB; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
#pragma unroll
      for (int k = 0; k < SB - 1; ++k)
        if (k < i) v = fma(-S[o + i][o + k], x[k], v);
      x[i] = (i >= c) ? v * invd[o + i] : 0.0;
    }
    if (lane < SB) {
#pragma unroll
      for (int i = 0; i < SB; ++i) Xs[o + i][o + c] = x[i];
    }
  }
  __syncthreads();
  // block rows i = 1..3: T_j = sum_(j <= k < i) L_ik X_kj, then X_ij = -X_ii T_j
  for (int bi = 1; bi < NB / SB; ++bi) {
    const int ro = bi * SB, ncol = bi * SB;  // columns 0 .. ro - 1
    for (int e = tid; e < SB * ncol; e += 256) {
      const int i = e / ncol, c = e % ncol;
      const int bj = c / SB;
      double v = 0.0;
      for (int k = bj * SB; k < ro; ++k) v = fma(S[ro + i][k], Xs[k][c], v);
      Ts[ro + i][c] = v;
    }
    __syncthreads();
    for (int e = tid; e < SB * ncol; e += 256) {
      const int i = e / ncol, c = e % ncol;
      double v = 0.0;
      for (int k = 0; k <= i; ++k) v = fma(Xs[ro + i][ro + k], Ts[ro + k][c], v);
      Xs[ro + i][c] = -v;
    }
    __syncthreads();
  }
  for (int idx = tid; idx < NB * NB; idx += 256) {
    const int r = idx & (NB - 1), c = idx >> 6;
    dinv[r + NB * c] = (r < nb && c <= r) ? Xs[r][c] : 0.0;
  }
}

// Panel below the diagonal block (rows j0 + NB.., columns j0..j0 + nb):
// P := P Dinv^T in place. One block per 64 rows; the whole row slice is read
// into shared memory before it is overwritten.
__global__ void __launch_bounds__(256) k_panel_inplace(double* A, long long lda, int j0, int nb,
                                                       int rows, const double* __restrict__ dinv) {
  extern __shared__ double psm[];
  double(*P)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(psm);           // [row][p]
  double(*D)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(psm + NB * (NB + 1));  // [j][p]
  const int tid = threadIdx.x;
  const int i0 = blockIdx.x * NB;
  double* base = A + (j0 + nb) + lda * j0;
#pragma unroll
  for (int idx = tid; idx < NB * NB; idx += 256) {
    const int i = idx & (NB - 1), p = idx >> 6;
    P[i][p] = (i0 + i < rows && p < nb) ? base[(i0 + i) + lda * p] : 0.0;
    D[i][p] = dinv[i + NB * p];
  }
  __syncthreads();
  const int tx = tid & 15, ty = tid >> 4;
  double acc[4][4] = {};
  for (int p = 0; p < NB; ++p) {
    double x[4], y[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      x[u] = P[tx + 16 * u][p];
      y[u] = D[ty + 16 * u][p];
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] = fma(x[u], y[v], acc[u][v]);
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = i0 + tx + 16 * u, j = ty + 16 * v;
      if (i < rows && j < nb) base[i + lda * j] = acc[u][v];
    }
}

// Super-step of the blocked forward substitution B := L^-1 B (right-looking)
// over the diagonal blocks k0 .. k0 + ns - 1 (ns <= kTrsmSuper). Block
// (it, jt), it = k0.., jt over 16-column tiles of B, first solves the
// super-step's blocks itself, in the order of the one-block-per-launch scheme:
// for j = 0 .. ns-1, B_(k0+j) -= L_(k0+j, k0+l) X_l for l < j, then
// X_j = Dinv_(k0+j) B_(k0+j). Every product is sum_p M[r][p] X[p][c] with p
// ascending and each update one subtraction, so the results are those of one
// launch per diagonal block, in a quarter of the launches. Blocks with it in
// the super-step store X_(it-k0) in C; the others update
// B_it -= L_(it, k0+j) X_j for j = 0 .. ns-1 (B itself is only written by
// these, and B_(k0..) is read before any block of this launch writes). Thread
// (r, g) = (tid % 64, tid / 64) owns row r, columns 4 g .. 4 g + 3 of the tile.
constexpr int kTrsmCols = 16;
constexpr int kTrsmSuper = 4;
constexpr size_t kTrsmSmem = sizeof(double) * (NB * (NB + 1) + kTrsmSuper * NB * (kTrsmCols + 1));
__global__ void __launch_bounds__(256) k_trsm_super(const double* __restrict__ L, long long lda, int n,
                                                    int k0, int ns, const double* __restrict__ dinv,
                                                    const double* B, long long ldb, int nrhs, double* Bw,
                                                    double* C, long long ldc) {
  extern __shared__ double tsm[];
  double(*M)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(tsm);  // Dinv or an L block   [i][p]
  double(*Xs)[NB][kTrsmCols + 1] =
      reinterpret_cast<double(*)[NB][kTrsmCols + 1]>(tsm + NB * (NB + 1));  // X_j     [j][p][c]
  const int tid = threadIdx.x, r = tid & (NB - 1), g = tid >> 6;
  const int it = k0 + blockIdx.x, c0 = blockIdx.y * kTrsmCols;
  auto load_M = [&](const double* src, long long ld, int rows, int cols) {
    __syncthreads();  // every thread is done with M
#pragma unroll
    for (int idx = tid; idx < NB * NB; idx += 256) {
      const int i = idx & (NB - 1), q = idx >> 6;
      M[i][q] = (i < rows && q < cols) ? src[i + ld * q] : 0.0;
    }
    __syncthreads();
  };
  // the super-step's solutions X_0 .. X_(ns-1), kept in shared memory
  for (int j = 0; j < ns; ++j) {
    const int rj = (k0 + j) * NB, nbj = min(NB, n - rj);
    double t[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int col = c0 + 4 * g + c;
      t[c] = (r < nbj && col < nrhs) ? B[(rj + r) + ldb * col] : 0.0;
    }
    for (int l = 0; l < j; ++l) {
      const int rl = (k0 + l) * NB, nbl = min(NB, n - rl);
      load_M(L + rj + lda * rl, lda, nbj, nbl);
      double upd[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
      for (int p = 0; p < NB; ++p) {
        const double m = M[r][p];
#pragma unroll
        for (int c = 0; c < 4; ++c) upd[c] = fma(m, Xs[l][p][4 * g + c], upd[c]);
      }
#pragma unroll
      for (int c = 0; c < 4; ++c) t[c] -= upd[c];
    }
    // X_j = Dinv_j t: t goes through shared memory (row r of the tile)
#pragma unroll
    for (int c = 0; c < 4; ++c) Xs[j][r][4 * g + c] = (r < nbj) ? t[c] : 0.0;
    load_M(dinv + static_cast<size_t>(k0 + j) * NB * NB, NB, NB, NB);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
    for (int p = 0; p < NB; ++p) {
      const double m = M[r][p];
#pragma unroll
      for (int c = 0; c < 4; ++c) acc[c] = fma(m, Xs[j][p][4 * g + c], acc[c]);
    }
    __syncthreads();  // every thread has read Xs[j] as B_j
#pragma unroll
    for (int c = 0; c < 4; ++c) Xs[j][r][4 * g + c] = acc[c];
  }
  if (it < k0 + ns) {
    __syncthreads();
    const int j = it - k0, rj = it * NB, nbj = min(NB, n - rj);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const int col = c0 + 4 * g + c;
      if (r < nbj && col < nrhs) C[(rj + r) + ldc * col] = Xs[j][r][4 * g + c];
    }
    return;
  }
  const int ri = it * NB, nbi = min(NB, n - ri);
  double bv[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int col = c0 + 4 * g + c;
    bv[c] = (r < nbi && col < nrhs) ? B[(ri + r) + ldb * col] : 0.0;
  }
  for (int j = 0; j < ns; ++j) {
    const int rj = (k0 + j) * NB, nbj = min(NB, n - rj);
    load_M(L + ri + lda * rj, lda, nbi, nbj);
    double upd[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 8
    for (int p = 0; p < NB; ++p) {
      const double m = M[r][p];
#pragma unroll
      for (int c = 0; c < 4; ++c) upd[c] = fma(m, Xs[j][p][4 * g + c], upd[c]);
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) bv[c] -= upd[c];
  }
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const int col = c0 + 4 * g + c;
    if (r < nbi && col < nrhs) Bw[(ri + r) + ldb * col] = bv[c];
  }
}

__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// C[m x n] := beta C + alpha op(A) op(B); op(A) is m x k, op(B) is k x n.
// 64 x 64 tiles, k-steps of 16 staged in shared memory, products on the FP64
// tensor cores (mma.sync m8n8k4): warp w owns rows 16 (w % 4) .. + 16 and
// columns 32 (w / 4) .. + 32 of the tile.
// lower_c: skip output tiles strictly above the diagonal (and entries above it).
// lower_a: A (not transposed) is lower triangular; entries above its diagonal
//          are treated as zero whatever the storage holds.
constexpr int TM = 64, TN = 64, TK = 16;
template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_gemm(int m, int n, int k, double alpha,
                                              const double* __restrict__ A, long long lda,
                                              const double* __restrict__ B, long long ldb,
                                              double beta, double* C, long long ldc,
                                              int lower_c, int lower_a) {
  const int bi = blockIdx.x, bj = blockIdx.y;
  if (lower_c && bj > bi) return;
  __shared__ double As[TK][TM + 1];
  __shared__ double Bs[TK][TN + 1];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int wm = (warp & 3) * 16, wn = (warp >> 2) * 32;
  const int i0 = bi * TM, j0 = bj * TN;
  double acc[2][4][2] = {};
  // with a lower triangular A, columns k > i0 + TM - 1 contribute nothing
  const int kend = (lower_a && !TA) ? min(k, i0 + TM) : k;
  for (int kk = 0; kk < kend; kk += TK) {
    for (int idx = threadIdx.x; idx < TK * TM; idx += 256) {
      int r, c;  // r in tile rows (m), c in k
      if (TA) {  // A stored k x m: op(A)(r, c) = A[c + lda * r]
        c = idx % TK;
        r = idx / TK;
      } else {
        r = idx % TM;
        c = idx / TM;
      }
      const int gi = i0 + r, gk = kk + c;
      double v = 0.0;
      if (gi < m && gk < k && (!lower_a || TA || gi >= gk)) v = TA ? A[gk + lda * gi] : A[gi + lda * gk];
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
    for (int q = 0; q < TK; q += 4) {
      double a[2], b[4];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt) a[mt] = As[q + t4][wm + 8 * mt + g];
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) b[nt] = Bs[q + t4][wn + 8 * nt + g];
#pragma unroll
      for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) dmma_m8n8k4(acc[mt][nt][0], acc[mt][nt][1], a[mt], b[nt]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int gi = i0 + wm + 8 * mt + g, gj = j0 + wn + 8 * nt + 2 * t4 + i;
        if (gi < m && gj < n && (!lower_c || gi >= gj)) {
          double* c = C + gi + ldc * gj;
          *c = (beta == 0.0 ? 0.0 : beta * *c) + alpha * acc[mt][nt][i];
        }
      }
}

// Trailing update of the Cholesky factorization: C -= P P^T on the lower part
// (i >= j) of C (m x ncols, ncols <= m, column-major, ldc), P (m x k,
// column-major, ldp, k <= NB). One block per 64 x 64 tile of that lower part:
// blockIdx.x enumerates the triangle of the first ncols tile rows, then the
// full tile rows below. Both panels of a tile are staged whole (every k at
// once) by cp.async copies (16 bytes when the columns are 16-byte aligned,
// else 8 bytes: ldp may be odd), in rows of 68 doubles
// (4 mod 16: conflict-free m8n8k4 fragment loads); two blocks per SM (128
// registers: the C prefetch spills at three) keep one block's copies in
// flight during another's products (standalone 13400 x 13400 factor: 66.0 ms
// with three blocks and 8-byte copies, 49.2 ms now). The products run
// in k_gemm's order (k ascending, four at a time, zeros up to a multiple of
// 16), so the factor is the same bit for bit.
constexpr int kSyrkLd = TM + 4;
constexpr size_t kSyrkSmem = sizeof(double) * 2 * NB * kSyrkLd;

__device__ __forceinline__ void cp_async8(double* smem_dst, const double* gmem_src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(gmem_src));
}

__device__ __forceinline__ void cp_async16_ld(double* smem_dst, const double* gmem_src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gmem_src));
}

// V16: the panel columns start on 16-byte boundaries (ldp even, P aligned), so
// pairs of rows are copied 16 bytes at a time. The block's entries of C are
// loaded into registers before the panels arrive, so their latency overlaps
// the copies and the products.
template <bool V16>
__global__ void __launch_bounds__(256, 2) k_syrk_update(int m, int ncols, int k, const double* __restrict__ P,
                                                        long long ldp, double* C, long long ldc) {
  extern __shared__ __align__(16) double sm[];
  double* As = sm;                  // As[c * kSyrkLd + r] = P[i0 + r, c]
  double* Bs = sm + NB * kSyrkLd;   // Bs[c * kSyrkLd + r] = P[j0 + r, c]
  const int nbc = (ncols + TN - 1) / TN;
  const int t = blockIdx.x, ntri = nbc * (nbc + 1) / 2;
  int bi, bj;
  if (t < ntri) {
    bi = static_cast<int>((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
    while ((bi + 1) * (bi + 2) / 2 <= t) ++bi;
    while (bi * (bi + 1) / 2 > t) --bi;
    bj = t - bi * (bi + 1) / 2;
  } else {
    bi = nbc + (t - ntri) / nbc;
    bj = (t - ntri) % nbc;
  }
  const int i0 = bi * TM, j0 = bj * TN;
  const int kq = (k + TK - 1) / TK * TK;
  if constexpr (V16) {
    for (int idx = threadIdx.x; idx < kq * (TM / 2); idx += 256) {
      const int r = 2 * (idx % (TM / 2)), c = idx / (TM / 2);
      double* da = As + c * kSyrkLd + r;
      double* db = Bs + c * kSyrkLd + r;
      if (c < k && i0 + r + 1 < m) {
        cp_async16_ld(da, P + (i0 + r) + ldp * c);
      } else {
        da[0] = (c < k && i0 + r < m) ? P[(i0 + r) + ldp * c] : 0.0;
        da[1] = 0.0;
      }
      if (c < k && j0 + r + 1 < ncols) {
        cp_async16_ld(db, P + (j0 + r) + ldp * c);
      } else {
        db[0] = (c < k && j0 + r < ncols) ? P[(j0 + r) + ldp * c] : 0.0;
        db[1] = 0.0;
      }
    }
  } else {
    for (int idx = threadIdx.x; idx < kq * TM; idx += 256) {
      const int r = idx % TM, c = idx / TM;
      double* da = As + c * kSyrkLd + r;
      double* db = Bs + c * kSyrkLd + r;
      if (c < k && i0 + r < m)
        cp_async8(da, P + (i0 + r) + ldp * c);
      else
        *da = 0.0;
      if (c < k && j0 + r < ncols)
        cp_async8(db, P + (j0 + r) + ldp * c);
      else
        *db = 0.0;
    }
  }
  asm volatile("cp.async.commit_group;\n" ::);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane >> 2, t4 = lane & 3;
  const int wm = (warp & 3) * 16, wn = (warp >> 2) * 32;
  // this thread's entries of C, in flight while the panels arrive
  double cv[2][4][2];
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int gi = i0 + wm + 8 * mt + g, gj = j0 + wn + 8 * nt + 2 * t4 + i;
        cv[mt][nt][i] = (gi < m && gj < ncols && gi >= gj) ? C[gi + ldc * gj] : 0.0;
      }
  asm volatile("cp.async.wait_group 0;\n" ::);
  __syncthreads();
  double acc[2][4][2] = {};
#pragma unroll 4
  for (int q = 0; q < kq; q += 4) {
    double a[2], b[4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) a[mt] = As[(q + t4) * kSyrkLd + wm + 8 * mt + g];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) b[nt] = Bs[(q + t4) * kSyrkLd + wn + 8 * nt + g];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) dmma_m8n8k4(acc[mt][nt][0], acc[mt][nt][1], a[mt], b[nt]);
  }
#pragma unroll
  for (int mt = 0; mt < 2; ++mt)
#pragma unroll
    for (int nt = 0; nt < 4; ++nt)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int gi = i0 + wm + 8 * mt + g, gj = j0 + wn + 8 * nt + 2 * t4 + i;
        if (gi < m && gj < ncols && gi >= gj) C[gi + ldc * gj] = cv[mt][nt][i] + -1.0 * acc[mt][nt][i];
      }
}

// Gram matrix G[i + nd j] = sum_k df[k + naux i] df[k + naux j] of the fitted
// densities, one warp per entry: lanes stride over k (contiguous columns),
// then a fixed-order shuffle reduction. Used for nd <= kGramWarpMax, where the
// tiled GEMM would run as a single block over the whole k range.
constexpr int kGramWarpMax = 128;
__global__ void __launch_bounds__(256) k_gram_warp(const double* __restrict__ df, int naux, int nd,
                                                   double* G) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nd * nd) return;
  const int i = w % nd, j = w / nd;
  const double* a = df + static_cast<long long>(naux) * i;
  const double* b = df + static_cast<long long>(naux) * j;
  double s = 0.0;
  for (int k = lane; k < naux; k += 32) s = fma(a[k], b[k], s);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0) G[i + static_cast<long long>(nd) * j] = s;
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

__global__ void k_add_diagonal(double* A, int n, double shift) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[i + static_cast<long long>(n) * i] += shift;
}

constexpr size_t kTileSmem = sizeof(double) * NB * (NB + 1);

int gemm_impl(bool ta, bool tb, int m, int n, int k, double alpha, const double* A, long long lda,
              const double* B, long long ldb, double beta, double* C, long long ldc, bool lower_c,
              bool lower_a, cudaStream_t s) {
  if (m <= 0 || n <= 0) return 0;
  dim3 grid((m + TM - 1) / TM, (n + TN - 1) / TN);
  const int lc = lower_c ? 1 : 0, la = lower_a ? 1 : 0;
  if (!ta && !tb)
    k_gemm<false, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lc, la);
  else if (!ta && tb)
    k_gemm<false, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lc, la);
  else if (ta && !tb)
    k_gemm<true, false><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lc, la);
  else
    k_gemm<true, true><<<grid, 256, 0, s>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lc, la);
  return 1;
}

// C -= P P^T on the lower part of C (m x ncols), P m x k (k <= NB).
int syrk_update(int m, int ncols, int k, const double* P, long long ldp, double* C, long long ldc,
                cudaStream_t s) {
  if (m <= 0 || ncols <= 0) return 0;
  const long long nbr = (m + TM - 1) / TM, nbc = (ncols + TN - 1) / TN;
  const long long tiles = nbc * (nbc + 1) / 2 + (nbr - nbc) * nbc;
  if (ldp % 2 == 0 && reinterpret_cast<uintptr_t>(P) % 16 == 0)
    k_syrk_update<true><<<static_cast<unsigned>(tiles), 256, kSyrkSmem, s>>>(m, ncols, k, P, ldp, C, ldc);
  else
    k_syrk_update<false><<<static_cast<unsigned>(tiles), 256, kSyrkSmem, s>>>(m, ncols, k, P, ldp, C, ldc);
  return 1;
}

}  // namespace

int gemm(bool ta, bool tb, int m, int n, int k, double alpha, const double* A, long long lda,
         const double* B, long long ldb, double beta, double* C, long long ldc, bool lower_only,
         cudaStream_t s) {
  return gemm_impl(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lower_only, false, s);
}

size_t linalg_workspace_doubles(int n) {
  const int nblk = (n + NB - 1) / NB;
  return static_cast<size_t>(nblk) * NB * NB;
}

int cholesky_lower(double* A, int n, int* d_info, double* work, cudaStream_t s,
                   const CholLookahead* la) {
  int launches = 0;
  cudaFuncSetAttribute(k_panel_inplace, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(2 * kTileSmem));
  cudaFuncSetAttribute(k_potrf_diag_inv, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(3 * kTileSmem));
  cudaFuncSetAttribute(k_syrk_update<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSyrkSmem));
  cudaFuncSetAttribute(k_syrk_update<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kSyrkSmem));
  cudaMemsetAsync(d_info, 0, sizeof(int), s);
  const int nblk = (n + NB - 1) / NB;
  bool rest_pending = false;  // a trailing update of the previous step is queued on la->aux
  // per block column b: diagonal factor + inverse, panel P := P L_bb^-T, then
  // A22 -= P P^T, split (with lookahead) into the next block column (main
  // stream, on the path to the next diagonal block) and the rest (aux stream)
  for (int b = 0; b < nblk; ++b) {
    const int j0 = b * NB, nb = std::min(NB, n - j0);
    double* Db = work + static_cast<size_t>(b) * NB * NB;
    k_potrf_diag_inv<<<1, 256, 3 * kTileSmem, s>>>(A, n, j0, nb, Db, d_info);
    ++launches;
    const int rest = n - j0 - nb;
    if (rest <= 0) continue;
    k_panel_inplace<<<(rest + NB - 1) / NB, 256, 2 * kTileSmem, s>>>(A, n, j0, nb, rest, Db);
    ++launches;
    double* P = A + (j0 + nb) + static_cast<long long>(n) * j0;
    double* A22 = A + (j0 + nb) + static_cast<long long>(n) * (j0 + nb);
    if (!la) {
      launches += syrk_update(rest, rest, nb, P, n, A22, n, s);
      continue;
    }
    const int nb1 = std::min(NB, rest), rest2 = rest - nb1;
    cudaEventRecord(la->ev_panel, s);
    // the previous step's remainder also updated this next block column
    if (rest_pending) cudaStreamWaitEvent(s, la->ev_rest, 0);
    launches += syrk_update(rest, nb1, nb, P, n, A22, n, s);
    rest_pending = rest2 > 0;
    if (rest_pending) {
      cudaStreamWaitEvent(la->aux, la->ev_panel, 0);
      launches += syrk_update(rest2, rest2, nb, P + nb1, n, A22 + nb1 + static_cast<long long>(n) * nb1, n,
                              la->aux);
      cudaEventRecord(la->ev_rest, la->aux);
    }
  }
  if (rest_pending) cudaStreamWaitEvent(s, la->ev_rest, 0);
  return launches;
}

int trsm_lower_left(const double* L, int n, const double* dinv, double* B, long long ldb, int nrhs,
                    double* C, long long ldc, cudaStream_t s) {
  if (n <= 0 || nrhs <= 0) return 0;
  cudaFuncSetAttribute(k_trsm_super, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kTrsmSmem));
  const int nblk = (n + NB - 1) / NB, ct = (nrhs + kTrsmCols - 1) / kTrsmCols;
  int launches = 0;
  for (int k0 = 0; k0 < nblk; k0 += kTrsmSuper, ++launches) {
    const int ns = std::min(kTrsmSuper, nblk - k0);
    k_trsm_super<<<dim3(nblk - k0, ct), 256, kTrsmSmem, s>>>(L, n, n, k0, ns, dinv, B, ldb, nrhs, B, C, ldc);
  }
  return launches;
}

int add_diagonal(double* A, int n, double shift, cudaStream_t s) {
  if (shift == 0.0 || n <= 0) return 0;
  k_add_diagonal<<<(n + 255) / 256, 256, 0, s>>>(A, n, shift);
  return 1;
}

int coulomb_4d(const double* df, int naux, int ndens, int nstates, double* gram_scratch,
               double* R, cudaStream_t s) {
  int launches = 0;
  if (ndens <= kGramWarpMax) {
    const long long threads = 32LL * ndens * ndens;
    k_gram_warp<<<static_cast<int>((threads + 255) / 256), 256, 0, s>>>(df, naux, ndens, gram_scratch);
    launches = 1;
  } else {
    launches = gemm(true, false, ndens, ndens, naux, 1.0, df, naux, df, naux, 0.0, gram_scratch, ndens,
                    false, s);
  }
  const long long total = static_cast<long long>(nstates) * nstates * nstates * nstates;
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 4096));
  k_coulomb4d<<<std::max(blocks, 1), 256, 0, s>>>(gram_scratch, ndens, nstates, R);
  return launches + 1;
}

}  // namespace pa
