// Kernels of the sTDDFT ("std") density-fitting tensors (std/intor.f90):
//  * k_std_df1c       (mu mu|P) for every orbital function mu: the diagonal of
//                     the (aa|c) blocks, screened by Q_aa * Q_c
//                     (intor_df1c, std/intor.f90:66-111);
//  * k_std_df2c_half  the first half-transformation of intor_df2c_mo
//                     (std/intor.f90:207-261) with the reference's two value
//                     skips, summed over the partner shell a for every target
//                     shell b and auxiliary shell c; the second half
//                     (std/intor.f90:263-279) is then one GEMM per batch of
//                     auxiliary functions, followed by k_std_pack;
//  * k_transpose      column-major transposition of the L^-1-applied results.
//
// Both integral kernels evaluate explicit spherical (ab|c) blocks, because the
// reference drops individual integrals |(ab|c)| <= 1e-10 (REAL(4) literal) and
// individual half-transformed values <= 1e-10 before summing; at the 8-atom
// workload these skips move intor_df2c_mo by ~4e-9, so they are reproduced
// triple by triple. A block of (ab|c) is built by McMurchie-Davidson like the
// other kernels of the library:
//   (ab|c)[(ma,mb)][m] = sum_(units u of ab) sum_(prims of c) sum_tuv
//                        E_sph,u[(ma,mb)][tuv] X_(u,c)[tuv][m]
// with X = pref sum_tau S_lc,m[tau] R_(tuv+tau)(alpha, P_u - C).
#include "boys.cuh"
#include "k_std.cuh"
#include "md.cuh"

namespace pa {

namespace {

struct BlockSync {
  __device__ void operator()() const { __syncthreads(); }
};

constexpr int kStdThreads = 128;
// k_std_df2c_half: two blocks per SM (its shared memory: the integral
// scratch and the half-transformed accumulator), so eight warps each
constexpr int kStdHalfThreads = 256;
constexpr int kLtot = 2 * PA_LMAX + PA_LAUXMAX;           // highest la + lb + lc
constexpr int kNR = ncum(kLtot);                           // R entries of one build
constexpr int kNHMax = ncum(2 * PA_LMAX);                  // Hermite components of a bra
constexpr int kNCMax = 2 * PA_LAUXMAX + 1;                 // spherical aux functions
constexpr int kNSMax = 2 * PA_LMAX + 1;                    // spherical orbital functions
constexpr int kNabMax = kNSMax * kNSMax;
constexpr int kMoChunk = 64;                               // MOs per df2c block
constexpr double kSkip1 = static_cast<double>(1e-10f);     // std/intor.f90:247 (REAL(4))
constexpr double kSkip2 = 1e-10;                           // std/intor.f90:269

// Shared scratch of block_3c.
struct Blk3cScratch {
  double* Rn;  // 32
  double* R0;  // kNR
  double* R1;  // kNR
  double* Xs;  // kNHMax * kNCMax
  double* I;   // kNabMax * kNCMax
};
constexpr int kBlk3cDoubles = 32 + 2 * kNR + kNHMax * kNCMax + kNabMax * kNCMax;

__device__ __forceinline__ Blk3cScratch blk3c_scratch(double* base) {
  Blk3cScratch s;
  s.Rn = base;
  s.R0 = s.Rn + 32;
  s.R1 = s.R0 + kNR;
  s.Xs = s.R1 + kNR;
  s.I = s.Xs + kNHMax * kNCMax;
  return s;
}

__device__ __forceinline__ int cidx_sum(const IndexTables* __restrict__ it, int i, int j) {
  const uchar4 a = *reinterpret_cast<const uchar4*>(it->xyz[i]);
  const uchar4 b = *reinterpret_cast<const uchar4*>(it->xyz[j]);
  return cidx(a.x + b.x, a.y + b.y, a.z + b.z);
}

// I[(ma * nsb + mb) * NC + m] = (a_ma b_mb | c_m) for pair = (a, b), a >= b, by
// the whole block. Starts and ends with a block barrier.
__device__ void block_3c(const StdArgs& a, int pair, int c, Blk3cScratch s) {
  const IndexTables* it = a.dt.idx;
  const int tid = threadIdx.x, nthr = blockDim.x;
  const int2 ab = a.pair_ab[pair];
  const int4 sa = a.B.shell[ab.x], sb = a.B.shell[ab.y];
  const int nab = (2 * sa.x + 1) * (2 * sb.x + 1);
  const int NH = ncum(sa.x + sb.x);
  const int4 sc = a.X.shell[c];
  const int lc = sc.x, NC = 2 * lc + 1;
  const int L = sa.x + sb.x + lc;
  const int offc = ncum(lc - 1);
  const double4 C = a.X.center[c];
  __syncthreads();  // previous readers of I are done
  for (int i = tid; i < nab * NC; i += nthr) s.I[i] = 0.0;
  const int u0 = a.pair_unit0[pair], nu = sa.y * sb.y;
  for (int u = u0; u < u0 + nu; ++u) {
    const double4 up = a.unit_pP[u];
    const double* E = a.esph + a.unit_esph[u];
    const double p = up.x;
    const double X = up.y - C.x, Y = up.z - C.y, Z = up.w - C.z;
    const double RPC2 = X * X + Y * Y + Z * Z;
    for (int kc = 0; kc < sc.y; ++kc) {
      const double2 gp = a.X.prim[sc.z + kc];
      const double gam = gp.x, pg = p + gam, alpha = p * gam / pg;
      double pref = kTwoPi52 / (p * gam * sqrt(pg)) * gp.y;
      for (int l = 0; l < lc; ++l) pref *= -0.5 / gam;  // (-1)^lc (2 gam)^-lc
      __syncthreads();  // previous users of Rn / R / Xs are done
      if (tid <= L) {
        double f = pref;
        for (int k = 0; k < tid; ++k) f *= -2.0 * alpha;
        s.Rn[tid] = f * boys_n(a.dt, a.boys_mode, tid, alpha * RPC2);
      }
      __syncthreads();
      hermite_R(a.dt.rdesc, L, s.Rn, X, Y, Z, s.R0, s.R1, tid, nthr, BlockSync());
      for (int idx = tid; idx < NH * NC; idx += nthr) {
        const int t = idx / NC, m = idx - t * NC;
        const int row = lc * lc + m;
        double y = 0.0;
        for (int k = a.dt.sph_start[row]; k < a.dt.sph_start[row + 1]; ++k)
          y = fma(a.dt.sph_val[k], s.R0[cidx_sum(it, t, offc + a.dt.sph_col[k])], y);
        s.Xs[idx] = y;
      }
      __syncthreads();
      for (int idx = tid; idx < nab * NC; idx += nthr) {
        const int r = idx / NC, m = idx - r * NC;
        const double* e = E + static_cast<long long>(r) * NH;
        double v = 0.0;
        for (int t = 0; t < NH; ++t) v = fma(__ldg(e + t), s.Xs[t * NC + m], v);
        s.I[idx] += v;
      }
    }
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kStdThreads) k_std_df1c(StdArgs a, double* __restrict__ Tt,
                                                          int naux) {
  __shared__ double scratch[kBlk3cDoubles];
  const int c = blockIdx.x, sh = blockIdx.y;
  const int pair = sh * (sh + 1) / 2 + sh;
  if (a.Qab[pair] * a.Qc[c] < a.thresh) return;  // schwarz_estimate(a, a, c) < 1e-10
  Blk3cScratch s = blk3c_scratch(scratch);
  block_3c(a, pair, c, s);
  const int4 sa = a.B.shell[sh], sc = a.X.shell[c];
  const int na = 2 * sa.x + 1, NC = 2 * sc.x + 1;
  for (int idx = threadIdx.x; idx < na * NC; idx += blockDim.x) {
    const int i = idx / NC, m = idx - i * NC;
    Tt[(sc.w + m) + static_cast<long long>(naux) * (sa.w + i)] = s.I[(i * na + i) * NC + m];
  }
}

// ||(ab|c)||_2 of the block of pair rec_pair[blockIdx.y] and auxiliary shell
// blockIdx.x (the estimator study of intor/benchmark.f90:96-118).
__global__ void __launch_bounds__(kStdThreads) k_std_block_norm(StdArgs a, const int* __restrict__ rec_pair,
                                                                int nx, double* __restrict__ out) {
  __shared__ double scratch[kBlk3cDoubles];
  __shared__ double s_red[kStdThreads / 32];
  const int c = blockIdx.x, kp = blockIdx.y;
  const int pair = rec_pair[kp];
  Blk3cScratch s = blk3c_scratch(scratch);
  block_3c(a, pair, c, s);
  const int2 ab = a.pair_ab[pair];
  const int n = (2 * a.B.shell[ab.x].x + 1) * (2 * a.B.shell[ab.y].x + 1) * (2 * a.X.shell[c].x + 1);
  double ss = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) ss = fma(s.I[i], s.I[i], ss);
  for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = ss;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kStdThreads / 32; ++w) t += s_red[w];
    out[static_cast<long long>(kp) * nx + c] = sqrt(t);
  }
}

// One block per (aux shell c, target shell b, chunk of MOs).
__global__ void __launch_bounds__(kStdHalfThreads) k_std_df2c_half(StdArgs a, int c0, int k0, int nmos,
                                                               const double* __restrict__ mo,
                                                               double* __restrict__ W, int moc) {
  extern __shared__ double sm[];
  Blk3cScratch s = blk3c_scratch(sm);
  double* Cs = sm + kBlk3cDoubles;     // [kNSMax][moc]
  double* Wacc = Cs + kNSMax * moc;    // [moc][nb][NC]
  const int c = c0 + blockIdx.x, b = blockIdx.y;
  const int mo0 = blockIdx.z * moc, nm = min(moc, nmos - mo0);
  const int tid = threadIdx.x;
  const int nbf = a.B.nsph;
  const int4 sb = a.B.shell[b], sc = a.X.shell[c];
  const int nb = 2 * sb.x + 1, NC = 2 * sc.x + 1;
  const int nw = nm * nb * NC;
  for (int i = tid; i < nw; i += blockDim.x) Wacc[i] = 0.0;
  const double qc = a.Qc[c];
  // partners in ascending order (the reference's loop order), tested
  // kStdHalfThreads at a time: each thread tests one partner, the warps'
  // ballots go to shared memory, and the block walks the surviving partners
  // of the chunk bit by bit (warp by warp)
  __shared__ unsigned s_alive[kStdHalfThreads / 32];
  for (int sh0 = 0; sh0 < a.B.nshells; sh0 += kStdHalfThreads) {
    {
      const int sh = sh0 + tid;
      bool alive = false;
      if (sh < a.B.nshells) {
        const int hi = max(sh, b), lo = min(sh, b);
        alive = !(a.Qab[hi * (hi + 1) / 2 + lo] * qc < a.thresh);  // schwarz_estimate(a, b, c) >= 1e-10
      }
      const unsigned m = __ballot_sync(0xffffffffu, alive);
      if ((tid & 31) == 0) s_alive[tid >> 5] = m;
    }
    __syncthreads();
    for (int wi = 0; wi < kStdHalfThreads / 32; ++wi) {
      unsigned m = s_alive[wi];
      while (m) {
        const int sh = sh0 + 32 * wi + __ffs(m) - 1;
        m &= m - 1;
        const int hi = max(sh, b), lo = min(sh, b);
        const int pair = hi * (hi + 1) / 2 + lo;
        block_3c(a, pair, c, s);
        const int4 sa = a.B.shell[sh];
        const int na = 2 * sa.x + 1;
        for (int i = tid; i < na * nm; i += blockDim.x) {
          const int ii = i / nm, mm = i - ii * nm;
          Cs[ii * moc + mm] = mo[(sa.w + ii) + static_cast<long long>(nbf) * (mo0 + mm)];
        }
        for (int i = tid; i < na * nb * NC; i += blockDim.x)
          if (fabs(s.I[i]) <= kSkip1) s.I[i] = 0.0;
        __syncthreads();
        // h[mo][j][m] = sum_(i in a) C[i, mo] (a_i b_j | c_m); the stored block is
        // (hi lo | c), so (a b|c) is its transpose when a < b
        const bool a_first = sh >= b;
        for (int idx = tid; idx < nw; idx += blockDim.x) {
          const int mm = idx / (nb * NC), rem = idx - mm * (nb * NC);
          const int j = rem / NC, m = rem - j * NC;
          double h = 0.0;
          for (int i = 0; i < na; ++i) {
            const double iv = a_first ? s.I[(i * nb + j) * NC + m] : s.I[(j * na + i) * NC + m];
            h = fma(Cs[i * moc + mm], iv, h);
          }
          if (fabs(h) > kSkip2) Wacc[idx] += h;
        }
      }
    }
    __syncthreads();  // s_alive is rewritten by the next chunk
  }
  __syncthreads();
  for (int idx = tid; idx < nw; idx += blockDim.x) {
    const int mm = idx / (nb * NC), rem = idx - mm * (nb * NC);
    const int j = rem / NC, m = rem - j * NC;
    const long long k = sc.w + m - k0;
    W[(k * nmos + mo0 + mm) * nbf + sb.w + j] = Wacc[idx];
  }
}

__global__ void k_std_pack(const double* __restrict__ Res, int nk, int nmos, int k0, int naux,
                           double* __restrict__ Raw) {
  const long long npack = static_cast<long long>(nmos) * (nmos + 1) / 2;
  const long long total = npack * nk;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long pk = idx / nk;
    const int kk = static_cast<int>(idx - pk * nk);
    int p = static_cast<int>((sqrt(8.0 * static_cast<double>(pk) + 1.0) - 1.0) * 0.5);
    while (static_cast<long long>(p) * (p + 1) / 2 > pk) --p;
    while (static_cast<long long>(p + 1) * (p + 2) / 2 <= pk) ++p;
    const int q = static_cast<int>(pk - static_cast<long long>(p) * (p + 1) / 2);
    Raw[(k0 + kk) + static_cast<long long>(naux) * pk] =
        Res[(static_cast<long long>(kk) * nmos + p) + static_cast<long long>(nk) * nmos * q];
  }
}

__global__ void k_transpose(const double* __restrict__ in, int rows, int cols, double* __restrict__ out) {
  // out (rows x cols) = in^T, in (cols x rows); a block moves one 32 x 32 tile,
  // reading along in's leading dimension and writing along out's
  __shared__ double tile[32][33];  // [out row][out col] within the tile
  const int j0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int j = j0 + threadIdx.x, i = i0 + k;
    if (i < rows && j < cols) tile[k][threadIdx.x] = in[j + static_cast<long long>(cols) * i];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + k;
    if (i < rows && j < cols) out[i + static_cast<long long>(rows) * j] = tile[threadIdx.x][k];
  }
}

}  // namespace

int launch_std_df1c(const StdArgs& a, double* Tt, cudaStream_t s) {
  if (a.B.nshells == 0 || a.X.nshells == 0) return 0;
  dim3 grid(a.X.nshells, a.B.nshells);
  k_std_df1c<<<grid, kStdThreads, 0, s>>>(a, Tt, a.X.nsph);
  return 1;
}

int launch_std_df2c_half(const StdArgs& a, int c0, int c1, int k0, int nmos, const double* mo,
                         double* W, cudaStream_t s) {
  if (c1 <= c0 || a.B.nshells == 0 || nmos == 0) return 0;
  const int moc = nmos < kMoChunk ? nmos : kMoChunk;
  const size_t smem = sizeof(double) * (kBlk3cDoubles + kNSMax * moc + static_cast<size_t>(moc) * kNSMax * kNCMax);
  cudaFuncSetAttribute(k_std_df2c_half, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  dim3 grid(c1 - c0, a.B.nshells, (nmos + moc - 1) / moc);
  k_std_df2c_half<<<grid, kStdHalfThreads, smem, s>>>(a, c0, k0, nmos, mo, W, moc);
  return 1;
}

int launch_std_block_norms(const StdArgs& a, const int* rec_pair, int npairs, double* out, cudaStream_t s) {
  if (npairs <= 0 || a.X.nshells == 0) return 0;
  int done = 0;
  for (int p0 = 0; p0 < npairs; p0 += 65535) {  // grid y limit
    dim3 grid(a.X.nshells, std::min(65535, npairs - p0));
    k_std_block_norm<<<grid, kStdThreads, 0, s>>>(a, rec_pair + p0, a.X.nshells,
                                                 out + static_cast<long long>(p0) * a.X.nshells);
    ++done;
  }
  return done;
}

int launch_std_pack(const double* Res, int nk, int nmos, int k0, int naux, double* Raw, cudaStream_t s) {
  const long long total = static_cast<long long>(nmos) * (nmos + 1) / 2 * nk;
  if (total == 0) return 0;
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148 * 16));
  k_std_pack<<<blocks, 256, 0, s>>>(Res, nk, nmos, k0, naux, Raw);
  return 1;
}

int launch_transpose(const double* in, int rows, int cols, double* out, cudaStream_t s) {
  if (rows <= 0 || cols <= 0) return 0;
  dim3 grid((cols + 31) / 32, (rows + 31) / 32);
  k_transpose<<<grid, dim3(32, 8), 0, s>>>(in, rows, cols, out);
  return 1;
}

}  // namespace pa
