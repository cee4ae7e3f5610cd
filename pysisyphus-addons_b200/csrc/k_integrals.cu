// Integral kernels of the density-fitting path (McMurchie-Davidson, FP64):
//  * k_unit_setup_warp / k_unit_setup   per primitive pair of an orbital shell
//                   pair ("bra unit"): Gaussian-product data and the spherical
//                   Hermite expansion E_sph[(ma,mb)][tuv] (contraction
//                   coefficients folded in);
//  * k_schwarz_bra_warp / k_schwarz_bra_dmma<LAB> / k_schwarz_bra<LAB>
//                   sqrt(||(ab|ab)||_F) per shell pair
//                   (common/integrals/intor.f90:131-160);
//  * k_schwarz_aux  sqrt(||(c|c)||_F) per auxiliary shell (intor.f90:97-129);
//  * k_metric       the symmetric (P|Q) matrix (intor.f90:40-95);
//  * k_bra_prep     density folding G_d[tuv] = sum_(ma,mb) Dsym_d[ma,mb] E_sph[(ma,mb)][tuv]
//                   with Dsym = D + (a != b) D^T as in diabatization/intor.f90:155-177.
#include <algorithm>

#include "boys.cuh"
#include "k_integrals.cuh"
#include "md.cuh"

namespace pa {

namespace {

struct WarpSync {
  __device__ void operator()() const { __syncwarp(); }
};
struct BlockSync {
  __device__ void operator()() const { __syncthreads(); }
};

__device__ __forceinline__ int sph_row(int l, int m_plus_l) { return l * l + m_plus_l; }

// Index of the sum of two Hermite/Cartesian multi-indices given by table index.
__device__ __forceinline__ int cidx_sum(const IndexTables* __restrict__ it, int i, int j) {
  const uchar4 a = *reinterpret_cast<const uchar4*>(it->xyz[i]);
  const uchar4 b = *reinterpret_cast<const uchar4*>(it->xyz[j]);
  return cidx(a.x + b.x, a.y + b.y, a.z + b.z);
}

// ---------------------------------------------------------------------------
// One block per unit (higher L_ab classes; units: the class's slice of the
// class-ordered unit list).
__global__ void __launch_bounds__(128) k_unit_setup(DevBasis B, const int2* __restrict__ pair_ab,
                                                    UnitArrays U, const int* __restrict__ units, int nunits,
                                                    DeviceTables dt) {
  if (static_cast<int>(blockIdx.x) >= nunits) return;
  const int u = units[blockIdx.x];
  __shared__ double E[3][(PA_LMAX + 1) * (PA_LMAX + 1) * (2 * PA_LMAX + 1)];
  __shared__ double sh[8];
  const int pair = U.unit_pair[u];
  const int2 ab = pair_ab[pair];
  const int4 sa = B.shell[ab.x], sb = B.shell[ab.y];
  const int la = sa.x, lb = sb.x;
  const int2 pr = U.unit_prims[u];
  if (threadIdx.x == 0) {
    const double4 A = B.center[ab.x], Bc = B.center[ab.y];
    const double2 pa_ = B.prim[pr.x], pb_ = B.prim[pr.y];
    const double p = pa_.x + pb_.x;
    const double Px = (pa_.x * A.x + pb_.x * Bc.x) / p;
    const double Py = (pa_.x * A.y + pb_.x * Bc.y) / p;
    const double Pz = (pa_.x * A.z + pb_.x * Bc.z) / p;
    const double ABx = A.x - Bc.x, ABy = A.y - Bc.y, ABz = A.z - Bc.z;
    const double K = exp(-pa_.x * pb_.x / p * (ABx * ABx + ABy * ABy + ABz * ABz));
    sh[0] = p;
    sh[1] = Px;
    sh[2] = Py;
    sh[3] = Pz;
    sh[4] = pa_.y * pb_.y * K;
    sh[5] = Px - A.x;
    sh[6] = Py - A.y;
    sh[7] = Pz - A.z;
    U.unit_pP[u] = make_double4(p, Px, Py, Pz);
  }
  __syncthreads();
  if (threadIdx.x < 3) {
    const int d = threadIdx.x;
    const double4 Bc = B.center[ab.y];
    const double Pd = sh[1 + d];
    const double PB = Pd - (d == 0 ? Bc.x : (d == 1 ? Bc.y : Bc.z));
    hermite_E_1d(la, lb, sh[5 + d], PB, 0.5 / sh[0], E[d]);
  }
  __syncthreads();
  const IndexTables* it = dt.idx;
  const int nsa = 2 * la + 1, nsb = 2 * lb + 1;
  const int nab = nsa * nsb;
  const int NH = ncum(la + lb);
  const int nt = la + lb + 1, nj = lb + 1;
  const int offa = ncum(la - 1 < 0 ? -1 : la - 1), offb = ncum(lb - 1 < 0 ? -1 : lb - 1);
  const double pref = sh[4];
  double* out = U.esph + U.unit_esph[u];
  // the sparse solid-harmonic rows of both shells (coefficients and decoded
  // Cartesian powers) in shared memory: the inner loop below reads no table
  // from global memory; same terms in the same order as the table rows
  constexpr int kRowMax = ncart(PA_LMAX);
  __shared__ double rv[2][2 * PA_LMAX + 1][kRowMax];
  __shared__ uchar4 rx[2][2 * PA_LMAX + 1][kRowMax];
  __shared__ int rn[2][2 * PA_LMAX + 1];
  for (int i = threadIdx.x; i < nsa + nsb; i += blockDim.x) {
    const int side = i < nsa ? 0 : 1, m = side ? i - nsa : i;
    const int l = side ? lb : la, off = side ? offb : offa;
    const int row = sph_row(l, m);
    const int k0 = dt.sph_start[row], k1 = dt.sph_start[row + 1];
    rn[side][m] = k1 - k0;
    for (int k = k0; k < k1; ++k) {
      rv[side][m][k - k0] = dt.sph_val[k];
      rx[side][m][k - k0] = *reinterpret_cast<const uchar4*>(it->xyz[off + dt.sph_col[k]]);
    }
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < nab * NH; idx += blockDim.x) {
    const int r = idx / NH, t = idx - r * NH;
    const int ma = r / nsb, mb = r - ma * nsb;
    const uchar4 tt = *reinterpret_cast<const uchar4*>(it->xyz[t]);
    const int na = rn[0][ma], nbk = rn[1][mb];
    double v = 0.0;
    for (int ka = 0; ka < na; ++ka) {
      const uchar4 ea = rx[0][ma][ka];
      const double ca = rv[0][ma][ka];
      for (int kb = 0; kb < nbk; ++kb) {
        const uchar4 eb = rx[1][mb][kb];
        if (tt.x > ea.x + eb.x || tt.y > ea.y + eb.y || tt.z > ea.z + eb.z) continue;
        v += ca * rv[1][mb][kb] * E[0][(ea.x * nj + eb.x) * nt + tt.x] *
             E[1][(ea.y * nj + eb.y) * nt + tt.y] * E[2][(ea.z * nj + eb.z) * nt + tt.z];
      }
    }
    out[idx] = pref * v;
  }
}

// One warp per unit for the low classes (L_a + L_b <= kUsLab, at most 90
// E_sph entries, where a block per unit mostly idles): every lane forms the
// Gaussian-product data itself, lanes 0-2 the 1D Hermite coefficients.
constexpr int kUsLab = 2;
constexpr int kUsE = 12;  // largest (la+1)(lb+1)(la+lb+1) with la + lb <= kUsLab
constexpr int kUsWarps = 8;

__global__ void __launch_bounds__(32 * kUsWarps) k_unit_setup_warp(DevBasis B, const int2* __restrict__ pair_ab,
                                                                 UnitArrays U, const int* __restrict__ units,
                                                                 int nunits, DeviceTables dt) {
  __shared__ double E[kUsWarps][3][kUsE];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kUsWarps + warp;
  if (i >= nunits) return;  // warp-uniform
  const int u = units[i];
  const int pair = U.unit_pair[u];
  const int2 ab = pair_ab[pair];
  const int4 sa = B.shell[ab.x], sb = B.shell[ab.y];
  const int la = sa.x, lb = sb.x;
  const int2 pr = U.unit_prims[u];
  const double4 A = B.center[ab.x], Bc = B.center[ab.y];
  const double2 pa_ = B.prim[pr.x], pb_ = B.prim[pr.y];
  const double p = pa_.x + pb_.x;
  const double Px = (pa_.x * A.x + pb_.x * Bc.x) / p;
  const double Py = (pa_.x * A.y + pb_.x * Bc.y) / p;
  const double Pz = (pa_.x * A.z + pb_.x * Bc.z) / p;
  if (lane == 0) U.unit_pP[u] = make_double4(p, Px, Py, Pz);
  if (lane < 3) {
    const double Pd = lane == 0 ? Px : (lane == 1 ? Py : Pz);
    const double Ad = lane == 0 ? A.x : (lane == 1 ? A.y : A.z);
    const double Bd = lane == 0 ? Bc.x : (lane == 1 ? Bc.y : Bc.z);
    hermite_E_1d(la, lb, Pd - Ad, Pd - Bd, 0.5 / p, E[warp][lane]);
  }
  const double ABx = A.x - Bc.x, ABy = A.y - Bc.y, ABz = A.z - Bc.z;
  const double pref = pa_.y * pb_.y * exp(-pa_.x * pb_.x / p * (ABx * ABx + ABy * ABy + ABz * ABz));
  __syncwarp();
  const IndexTables* it = dt.idx;
  const int nsb = 2 * lb + 1;
  const int nab = (2 * la + 1) * nsb;
  const int NH = ncum(la + lb);
  const int nt = la + lb + 1, nj = lb + 1;
  const int offa = ncum(la - 1 < 0 ? -1 : la - 1), offb = ncum(lb - 1 < 0 ? -1 : lb - 1);
  const double* E0 = E[warp][0];
  const double* E1 = E[warp][1];
  const double* E2 = E[warp][2];
  double* out = U.esph + U.unit_esph[u];
  for (int idx = lane; idx < nab * NH; idx += 32) {
    const int r = idx / NH, t = idx - r * NH;
    const int ma = r / nsb, mb = r - ma * nsb;
    const uchar4 tt = *reinterpret_cast<const uchar4*>(it->xyz[t]);
    const int rowa = sph_row(la, ma), rowb = sph_row(lb, mb);
    double v = 0.0;
    for (int ka = dt.sph_start[rowa]; ka < dt.sph_start[rowa + 1]; ++ka) {
      const uchar4 ea = *reinterpret_cast<const uchar4*>(it->xyz[offa + dt.sph_col[ka]]);
      const double ca = dt.sph_val[ka];
      for (int kb = dt.sph_start[rowb]; kb < dt.sph_start[rowb + 1]; ++kb) {
        const uchar4 eb = *reinterpret_cast<const uchar4*>(it->xyz[offb + dt.sph_col[kb]]);
        if (tt.x > ea.x + eb.x || tt.y > ea.y + eb.y || tt.z > ea.z + eb.z) continue;
        v += ca * dt.sph_val[kb] * E0[(ea.x * nj + eb.x) * nt + tt.x] * E1[(ea.y * nj + eb.y) * nt + tt.y] *
             E2[(ea.z * nj + eb.z) * nt + tt.z];
      }
    }
    out[idx] = pref * v;
  }
}

// ---------------------------------------------------------------------------
// Schwarz values sqrt(||(ab|ab)||_F) of the bra pairs. For every pair of bra
// units (iu, ku) the block of the pair is
//   M_ik[r][s] = sum_(t,t') E_iu[r][t] (-1)^|t'| R[t + t'] E_ku[s][t'].
// Swapping the units negates P - Q, R_tau(-d) = (-1)^|tau| R_tau(d), so
// M_ki = M_ik^T and (ab|ab) = sum_(i,k) M_ik = A + A^T with
// A = sum_(i<k) M_ik + 1/2 sum_i M_ii: only the unordered unit pairs are
// computed. R is built for the displacement Q - P (R~ = (-1)^|tau| R), so that
// H[t][t'] = (-1)^|t| R~[t + t'] carries the sign on the output row, and the
// products are reassociated:
//   Z_i = sum_(k>=i) w_ik H_ik E_ku^T   (NH x nab, w_ii = 1/2)
//   A  += E_iu Z_i                       (once per iu, not per unit pair).
// Three kernels: k_schwarz_bra_warp (L_ab <= 2, one warp per pair, FP64 FMA),
// k_schwarz_bra_dmma<LAB> (L_ab 3, 4, one warp per pair) and
// k_schwarz_bra<LAB> (L_ab >= 5, one block per pair), the last two on the
// FP64 tensor cores (DMMA m8n8k4).
__device__ __forceinline__ void sw_dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Low-L pairs, one warp per pair, with warp barriers instead of block
// barriers (most pairs of a basis are low-L, and for them a block mostly waits
// at its barriers). Launches per group of L_ab classes, each warp's scratch sized for the
// group's largest class (sw_nr R entries, sw_nh x sw_nab Z, sw_nab^2 A, stride
// sw_stride doubles), so low-L classes keep many more warps resident.
constexpr int kSwLab = 4;
constexpr int kSwNR = ncum(2 * kSwLab);
constexpr int kSwNH = ncum(kSwLab);
constexpr int kSwNab = 25;  // largest (2la+1)(2lb+1) with la + lb <= 4, la, lb <= PA_LMAX
constexpr int kSwScratch = 32 + 2 * kSwNR + kSwNab * kSwNH + kSwNab * kSwNab;
constexpr int kSwWarps = 4;

__global__ void __launch_bounds__(32 * kSwWarps) k_schwarz_bra_warp(
    DevBasis B, const int2* __restrict__ pair_ab, const int* __restrict__ pair_unit0,
    const int* __restrict__ pair_list, UnitArrays U, int npairs, DeviceTables dt, int boys_mode,
    double* __restrict__ Qab, int sw_nr, int sw_nab, int sw_nh, int sw_stride) {
  extern __shared__ double sw_smem[];  // [kSwWarps][sw_stride]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.x * kSwWarps + warp;
  if (i >= npairs) return;  // warp-uniform
  const int pair = pair_list[i];
  const int2 ab = pair_ab[pair];
  const int4 sa = B.shell[ab.x], sb = B.shell[ab.y];
  const int la = sa.x, lb = sb.x;
  const int nab = (2 * la + 1) * (2 * lb + 1);
  const int NH = ncum(la + lb);
  const int L4 = 2 * (la + lb);
  double* Rn = sw_smem + warp * sw_stride;
  double* R0 = Rn + 32;
  double* R1 = R0 + sw_nr;
  double* Zs = R1 + sw_nr;            // Z_i [NH][nab]
  double* out = Zs + sw_nab * sw_nh;  // A [nab][nab]
  const IndexTables* it = dt.idx;
  for (int k = lane; k < nab * nab; k += 32) out[k] = 0.0;
  const int u0 = pair_unit0[pair];
  const int nu = sa.y * sb.y;
  for (int iu = 0; iu < nu; ++iu) {
    const double4 P = U.unit_pP[u0 + iu];
    __syncwarp();  // the previous A update has read Z
    for (int k = lane; k < NH * nab; k += 32) Zs[k] = 0.0;
    for (int ku = iu; ku < nu; ++ku) {
      const double4 Q = U.unit_pP[u0 + ku];
      const double p = P.x, q = Q.x, pq = p + q, alpha = p * q / pq;
      const double X = Q.y - P.y, Yd = Q.z - P.z, Z = Q.w - P.w;
      const double T = alpha * (X * X + Yd * Yd + Z * Z);
      const double pref = kTwoPi52 / (p * q * sqrt(pq));
      const double w = ku == iu ? 0.5 : 1.0;
      __syncwarp();  // previous users of Rn / R are done
      if (lane <= L4) {
        double f = pref;
        for (int k = 0; k < lane; ++k) f *= -2.0 * alpha;
        Rn[lane] = f * boys_n(dt, boys_mode, lane, T);
      }
      __syncwarp();
      hermite_R(dt.rdesc, L4, Rn, X, Yd, Z, R0, R1, lane, 32, WarpSync());
      const double* Ek = U.esph + U.unit_esph[u0 + ku];
      // each lane updates its own entries of Z (the same ones it zeroed)
      for (int idx = lane; idx < NH * nab; idx += 32) {
        const int t = idx / nab, sc = idx - t * nab;
        const double* e = Ek + sc * NH;
        const int16_t* sidx = dt.sum_idx + t * kNSum;
        double z = 0.0;
        for (int tp = 0; tp < NH; ++tp) z = fma(R0[__ldg(sidx + tp)], e[tp], z);
        Zs[idx] = fma((it->xyz[t][3] & 1) ? -w : w, z, Zs[idx]);
      }
    }
    __syncwarp();
    const double* Ei = U.esph + U.unit_esph[u0 + iu];
    for (int idx = lane; idx < nab * nab; idx += 32) {
      const int rr = idx / nab, sc = idx - rr * nab;
      const double* e = Ei + rr * NH;
      double v = 0.0;
      for (int t = 0; t < NH; ++t) v = fma(e[t], Zs[t * nab + sc], v);
      out[idx] += v;
    }
  }
  __syncwarp();
  double s2 = 0.0;
  for (int k = lane; k < nab * nab; k += 32) {
    const int rr = k / nab, sc = k - rr * nab;
    const double v = out[k] + out[sc * nab + rr];
    s2 = fma(v, v, s2);
  }
  for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  if (lane == 0) Qab[pair] = sqrt(sqrt(s2));
}

// Schwarz values of the classes L_ab = LAB (3 and 4), one warp per pair, with
// both products of k_schwarz_bra_warp on the FP64 tensor cores (DMMA
// m8n8k4): Z_i (NH x nab, in registers across the unit pairs k >= i) gets
// the tiles H_ik E_ku^T with H gathered from R~ through the multi-index sum
// table, and A (nab x nab, in registers across the whole pair) gets E_iu Z_i.
// Fragments: lane (g = lane / 4, t4 = lane % 4) holds A-row g / k-column t4,
// B-column g / k-row t4, and accumulator row g, columns 2 t4 and 2 t4 + 1.
constexpr int sw_nab_max(int lab) {
  int m = 1;
  for (int la = 0; la <= PA_LMAX; ++la) {
    const int lb = lab - la;
    if (lb < 0 || lb > PA_LMAX) continue;
    const int v = (2 * la + 1) * (2 * lb + 1);
    m = v > m ? v : m;
  }
  return m;
}

template <int LAB>
struct SwDmma {
  static constexpr int NH = ncum(LAB);
  static constexpr int NR = ncum(2 * LAB);
  static constexpr int NABM = sw_nab_max(LAB);
  static constexpr int MT = (NH + 7) / 8;    // row tiles of Z
  static constexpr int KT = (NH + 3) / 4;    // k steps of both products
  static constexpr int NT = (NABM + 7) / 8;  // column tiles of Z, row and column tiles of A
  static constexpr int STRIDE = 32 + 2 * NR + NH * NABM + NABM * NABM;  // doubles per warp
};

template <int LAB>
__global__ void __launch_bounds__(32 * kSwWarps) k_schwarz_bra_dmma(
    DevBasis B, const int2* __restrict__ pair_ab, const int* __restrict__ pair_unit0,
    const int* __restrict__ pair_list, UnitArrays U, int npairs, DeviceTables dt, int boys_mode,
    double* __restrict__ Qab) {
  using C = SwDmma<LAB>;
  constexpr int NH = C::NH, MT = C::MT, KT = C::KT, NT = C::NT;
  extern __shared__ double sw_smem[];  // [kSwWarps][STRIDE]
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t4 = lane & 3;
  const int i = blockIdx.x * kSwWarps + warp;
  if (i >= npairs) return;  // warp-uniform
  const int pair = pair_list[i];
  const int2 ab = pair_ab[pair];
  const int4 sa = B.shell[ab.x], sb = B.shell[ab.y];
  const int nab = (2 * sa.x + 1) * (2 * sb.x + 1);
  const int ntr = (nab + 7) / 8;  // column tiles in use (warp-uniform)
  double* Rn = sw_smem + warp * C::STRIDE;
  double* R0 = Rn + 32;
  double* R1 = R0 + C::NR;
  double* Zs = R1 + C::NR;            // Z_i [NH][nab]
  double* out = Zs + NH * C::NABM;    // A [nab][nab]
  const IndexTables* it = dt.idx;
  const int u0 = pair_unit0[pair];
  const int nu = sa.y * sb.y;
  double aacc[NT][NT][2];
#pragma unroll
  for (int mt = 0; mt < NT; ++mt)
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) aacc[mt][nt][0] = aacc[mt][nt][1] = 0.0;
  for (int iu = 0; iu < nu; ++iu) {
    const double4 P = U.unit_pP[u0 + iu];
    double zacc[MT][NT][2];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) zacc[mt][nt][0] = zacc[mt][nt][1] = 0.0;
    for (int ku = iu; ku < nu; ++ku) {
      const double4 Q = U.unit_pP[u0 + ku];
      const double p = P.x, q = Q.x, pq = p + q, alpha = p * q / pq;
      const double X = Q.y - P.y, Yd = Q.z - P.z, Z = Q.w - P.w;
      const double T = alpha * (X * X + Yd * Yd + Z * Z);
      const double pref = kTwoPi52 / (p * q * sqrt(pq));
      __syncwarp();  // previous readers of Rn / R are done
      if (lane <= 2 * LAB) {
        double f = pref;
        for (int k = 0; k < lane; ++k) f *= -2.0 * alpha;
        Rn[lane] = f * boys_n(dt, boys_mode, lane, T);
      }
      __syncwarp();
      hermite_R(dt.rdesc, 2 * LAB, Rn, X, Yd, Z, R0, R1, lane, 32, WarpSync());
      const double* Ek = U.esph + U.unit_esph[u0 + ku];
#pragma unroll
      for (int k4 = 0; k4 < KT; ++k4) {
        const int tp = 4 * k4 + t4;
        double af[MT], bf[NT];
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
          const int t = 8 * mt + g;
          af[mt] = (t < NH && tp < NH) ? R0[__ldg(dt.sum_idx + t * kNSum + tp)] : 0.0;
        }
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
          const int c = 8 * nt + g;
          bf[nt] = (nt < ntr && tp < NH && c < nab) ? Ek[c * NH + tp] : 0.0;
        }
#pragma unroll
        for (int mt = 0; mt < MT; ++mt)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt)
            if (nt < ntr) sw_dmma(zacc[mt][nt][0], zacc[mt][nt][1], af[mt], bf[nt]);
      }
      if (ku == iu) {  // weight 1/2 of the diagonal unit pair (exact scaling)
#pragma unroll
        for (int mt = 0; mt < MT; ++mt)
#pragma unroll
          for (int nt = 0; nt < NT; ++nt) {
            zacc[mt][nt][0] *= 0.5;
            zacc[mt][nt][1] *= 0.5;
          }
      }
    }
    __syncwarp();  // the previous A step has read Zs
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
      const int t = 8 * mt + g;
      if (t >= NH) continue;
      const double sg = (it->xyz[t][3] & 1) ? -1.0 : 1.0;  // (-1)^|t| of H = (-1)^|t| R~
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int c = 8 * nt + 2 * t4;
        if (c < nab) Zs[t * nab + c] = sg * zacc[mt][nt][0];
        if (c + 1 < nab) Zs[t * nab + c + 1] = sg * zacc[mt][nt][1];
      }
    }
    __syncwarp();
    const double* Ei = U.esph + U.unit_esph[u0 + iu];
#pragma unroll
    for (int k4 = 0; k4 < KT; ++k4) {
      const int t = 4 * k4 + t4;
      double af[NT], bf[NT];
#pragma unroll
      for (int mt = 0; mt < NT; ++mt) {
        const int r = 8 * mt + g;
        af[mt] = (mt < ntr && r < nab && t < NH) ? Ei[r * NH + t] : 0.0;
      }
#pragma unroll
      for (int nt = 0; nt < NT; ++nt) {
        const int c = 8 * nt + g;
        bf[nt] = (nt < ntr && t < NH && c < nab) ? Zs[t * nab + c] : 0.0;
      }
#pragma unroll
      for (int mt = 0; mt < NT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
          if (mt < ntr && nt < ntr) sw_dmma(aacc[mt][nt][0], aacc[mt][nt][1], af[mt], bf[nt]);
    }
  }
#pragma unroll
  for (int mt = 0; mt < NT; ++mt) {
    const int r = 8 * mt + g;
    if (r >= nab) continue;
#pragma unroll
    for (int nt = 0; nt < NT; ++nt) {
      const int c = 8 * nt + 2 * t4;
      if (c < nab) out[r * nab + c] = aacc[mt][nt][0];
      if (c + 1 < nab) out[r * nab + c + 1] = aacc[mt][nt][1];
    }
  }
  __syncwarp();
  double s2 = 0.0;
  for (int k = lane; k < nab * nab; k += 32) {
    const int rr = k / nab, sc = k - rr * nab;
    const double v = out[k] + out[sc * nab + rr];
    s2 = fma(v, v, s2);
  }
  for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  if (lane == 0) Qab[pair] = sqrt(sqrt(s2));
}

// High-L pairs (L_ab = LAB >= 5), one block of kSbWarps warps per pair. Each
// warp takes whole 8 x 8 tiles (the K reduction in two registers, so many
// blocks stay resident): the tiles of H_ik E_ku^T are added into Z_i in shared
// memory after every unit pair, the tiles of E_iu Z_i into A once per bra unit.
constexpr int kSbWarps = 8;

template <int LAB>
struct SwBlk {
  static constexpr int NH = ncum(LAB);
  static constexpr int NR = ncum(2 * LAB);
  static constexpr int NABM = sw_nab_max(LAB);
  static constexpr int MT = (NH + 7) / 8;
  static constexpr int KT = (NH + 3) / 4;
  // Rn, R0, R1, Z_i [NH][nab], A [nab][nab]
  static constexpr int SMEM = 32 + 2 * NR + NH * NABM + NABM * NABM;
  // blocks per SM that the shared memory allows (at most 4): the register
  // budget of the launch follows from it
  static constexpr int fit = (227 * 1024) / (SMEM * 8 + 1024);
  static constexpr int kMinBlocks = fit < 1 ? 1 : (fit > 4 ? 4 : fit);
};

template <int LAB>
__global__ void __launch_bounds__(32 * kSbWarps, SwBlk<LAB>::kMinBlocks) k_schwarz_bra(DevBasis B, const int2* __restrict__ pair_ab,
                                                            const int* __restrict__ pair_unit0,
                                                            const int* __restrict__ pair_list, UnitArrays U,
                                                            int npairs, DeviceTables dt, int boys_mode,
                                                            double* __restrict__ Qab) {
  using C = SwBlk<LAB>;
  constexpr int NH = C::NH, KT = C::KT, MT = C::MT;
  extern __shared__ double smem[];
  __shared__ double red[kSbWarps];
  if (static_cast<int>(blockIdx.x) >= npairs) return;
  const int pair = pair_list[blockIdx.x];
  const int2 ab = pair_ab[pair];
  const int4 sa = B.shell[ab.x], sb = B.shell[ab.y];
  const int nab = (2 * sa.x + 1) * (2 * sb.x + 1);
  const int ntr = (nab + 7) / 8;  // column tiles in use
  double* Rn = smem;
  double* R0 = Rn + 32;
  double* R1 = R0 + C::NR;
  double* Zs = R1 + C::NR;        // Z_i [NH][nab]
  double* out = Zs + NH * C::NABM;  // A [nab][nab]
  const IndexTables* it = dt.idx;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, t4 = lane & 3;
  for (int i = tid; i < nab * nab; i += blockDim.x) out[i] = 0.0;
  const int u0 = pair_unit0[pair];
  const int nu = sa.y * sb.y;
  for (int iu = 0; iu < nu; ++iu) {
    const double4 P = U.unit_pP[u0 + iu];
    for (int ku = iu; ku < nu; ++ku) {
      const double4 Q = U.unit_pP[u0 + ku];
      const double p = P.x, q = Q.x, pq = p + q, alpha = p * q / pq;
      const double X = Q.y - P.y, Yd = Q.z - P.z, Z = Q.w - P.w;
      const double T = alpha * (X * X + Yd * Yd + Z * Z);
      const double pref = kTwoPi52 / (p * q * sqrt(pq));
      const double w = ku == iu ? 0.5 : 1.0;
      __syncthreads();  // previous readers of Rn / R / Zs are done
      if (tid <= 2 * LAB) {
        double f = pref;
        for (int k = 0; k < tid; ++k) f *= -2.0 * alpha;
        Rn[tid] = f * boys_n(dt, boys_mode, tid, T);
      }
      __syncthreads();
      hermite_R(dt.rdesc, 2 * LAB, Rn, X, Yd, Z, R0, R1, tid, blockDim.x, BlockSync());
      const double* Ek = U.esph + U.unit_esph[u0 + ku];
      for (int tile = warp; tile < MT * ntr; tile += kSbWarps) {
        const int mt = tile / ntr, nt = tile - mt * ntr;
        const int t = 8 * mt + g, c = 8 * nt + g;
        double z0 = 0.0, z1 = 0.0;
        // unrolled: the index, R and E loads of several k steps in flight
        // ahead of the products (same k order, same results)
#pragma unroll 7
        for (int k4 = 0; k4 < KT; ++k4) {
          const int tp = 4 * k4 + t4;
          const double a = (t < NH && tp < NH) ? R0[__ldg(dt.sum_idx + t * kNSum + tp)] : 0.0;
          const double b = (tp < NH && c < nab) ? Ek[c * NH + tp] : 0.0;
          sw_dmma(z0, z1, a, b);
        }
        const int tr = 8 * mt + g, cc = 8 * nt + 2 * t4;
        if (tr < NH) {
          const double ws = (it->xyz[tr][3] & 1) ? -w : w;  // (-1)^|t| of H = (-1)^|t| R~
          double* zr = Zs + tr * nab;
          if (cc < nab) zr[cc] = ku == iu ? ws * z0 : fma(ws, z0, zr[cc]);
          if (cc + 1 < nab) zr[cc + 1] = ku == iu ? ws * z1 : fma(ws, z1, zr[cc + 1]);
        }
      }
    }
    __syncthreads();  // Z_i complete
    const double* Ei = U.esph + U.unit_esph[u0 + iu];
    for (int tile = warp; tile < ntr * ntr; tile += kSbWarps) {
      const int mt = tile / ntr, nt = tile - mt * ntr;
      const int r = 8 * mt + g, c = 8 * nt + g;
      double o0 = 0.0, o1 = 0.0;
#pragma unroll 7
      for (int k4 = 0; k4 < KT; ++k4) {
        const int t = 4 * k4 + t4;
        const double a = (r < nab && t < NH) ? Ei[r * NH + t] : 0.0;
        const double b = (t < NH && c < nab) ? Zs[t * nab + c] : 0.0;
        sw_dmma(o0, o1, a, b);
      }
      const int cc = 8 * nt + 2 * t4;
      if (r < nab && cc < nab) out[r * nab + cc] += o0;
      if (r < nab && cc + 1 < nab) out[r * nab + cc + 1] += o1;
    }
  }
  __syncthreads();
  double s2 = 0.0;
  for (int i = tid; i < nab * nab; i += blockDim.x) {
    const int r = i / nab, c = i - r * nab;
    const double v = out[i] + out[c * nab + r];
    s2 = fma(v, v, s2);
  }
  for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  if (lane == 0) red[warp] = s2;
  __syncthreads();
  if (tid == 0) {
    double tot = 0.0;
    for (int w = 0; w < kSbWarps; ++w) tot += red[w];
    Qab[pair] = sqrt(sqrt(tot));
  }
}

// ---------------------------------------------------------------------------
// Two-center block (P|Q)[mP][mQ] of two auxiliary shells, computed by one warp.
// Scratch (per warp): Rn[16], R0/R1[ncum(lP+lQ)], Y[nsP * ncart(lQ)], out[nsP * nsQ].
struct TwoCScratch {
  double* Rn;
  double* R0;
  double* R1;
  double* Y;
  double* out;
};

__device__ void twoc_block_warp(const DevBasis& X, int P, int Q, const DeviceTables& dt,
                                int boys_mode, TwoCScratch s, int lane) {
  const IndexTables* it = dt.idx;
  const int4 sP = X.shell[P], sQ = X.shell[Q];
  const int lP = sP.x, lQ = sQ.x;
  const int nsP = 2 * lP + 1, nsQ = 2 * lQ + 1, ncQ = ncart(lQ);
  const int L = lP + lQ;
  const int offP = ncum(lP - 1 < 0 ? -1 : lP - 1), offQ = ncum(lQ - 1 < 0 ? -1 : lQ - 1);
  const double4 CP = X.center[P], CQ = X.center[Q];
  const double Xd = CP.x - CQ.x, Yd = CP.y - CQ.y, Zd = CP.z - CQ.z;
  const double RPQ2 = Xd * Xd + Yd * Yd + Zd * Zd;
  for (int i = lane; i < nsP * nsQ; i += 32) s.out[i] = 0.0;
  for (int kp = 0; kp < sP.y; ++kp)
    for (int kq = 0; kq < sQ.y; ++kq) {
      const double2 gp = X.prim[sP.z + kp], gq = X.prim[sQ.z + kq];
      const double g = gp.x, h = gq.x, gh = g + h, alpha = g * h / gh;
      double pref = kTwoPi52 / (g * h * sqrt(gh)) * gp.y * gq.y * pow(2.0 * g, -lP) *
                    pow(2.0 * h, -lQ);
      if (lQ & 1) pref = -pref;
      const double T = alpha * RPQ2;
      __syncwarp();
      if (lane <= L) {
        double f = pref;
        for (int k = 0; k < lane; ++k) f *= -2.0 * alpha;
        s.Rn[lane] = f * boys_n(dt, boys_mode, lane, T);
      }
      __syncwarp();
      hermite_R(dt.rdesc, L, s.Rn, Xd, Yd, Zd, s.R0, s.R1, lane, 32, WarpSync());
      for (int idx = lane; idx < nsP * ncQ; idx += 32) {
        const int m = idx / ncQ, sg = idx - m * ncQ;
        const int row = sph_row(lP, m);
        double y = 0.0;
        for (int k = dt.sph_start[row]; k < dt.sph_start[row + 1]; ++k)
          y = fma(dt.sph_val[k], s.R0[cidx_sum(it, offP + dt.sph_col[k], offQ + sg)], y);
        s.Y[idx] = y;
      }
      __syncwarp();
      for (int idx = lane; idx < nsP * nsQ; idx += 32) {
        const int m = idx / nsQ, mq = idx - m * nsQ;
        const int row = sph_row(lQ, mq);
        double v = 0.0;
        for (int k = dt.sph_start[row]; k < dt.sph_start[row + 1]; ++k)
          v = fma(dt.sph_val[k], s.Y[m * ncQ + dt.sph_col[k]], v);
        s.out[idx] += v;
      }
      __syncwarp();
    }
}

constexpr int kTwoCWarps = 4;
constexpr int kTwoCScratch = 32 + 2 * ncum(2 * PA_LAUXMAX) + (2 * PA_LAUXMAX + 1) * ncart(PA_LAUXMAX) +
                             (2 * PA_LAUXMAX + 1) * (2 * PA_LAUXMAX + 1);

__device__ __forceinline__ TwoCScratch twoc_scratch(double* base) {
  TwoCScratch s;
  s.Rn = base;
  s.R0 = s.Rn + 32;
  s.R1 = s.R0 + ncum(2 * PA_LAUXMAX);
  s.Y = s.R1 + ncum(2 * PA_LAUXMAX);
  s.out = s.Y + (2 * PA_LAUXMAX + 1) * ncart(PA_LAUXMAX);
  return s;
}

__global__ void __launch_bounds__(32 * kTwoCWarps) k_schwarz_aux(DevBasis X, DeviceTables dt,
                                                                 int boys_mode,
                                                                 double* __restrict__ Qc) {
  __shared__ double scratch[kTwoCWarps][kTwoCScratch];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c = blockIdx.x * kTwoCWarps + warp;
  if (c >= X.nshells) return;
  TwoCScratch s = twoc_scratch(scratch[warp]);
  twoc_block_warp(X, c, c, dt, boys_mode, s, lane);
  const int ns = 2 * X.shell[c].x + 1;
  double s2 = 0.0;
  for (int i = lane; i < ns * ns; i += 32) s2 += s.out[i] * s.out[i];
  for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
  if (lane == 0) Qc[c] = sqrt(sqrt(s2));
}

__global__ void __launch_bounds__(32 * kTwoCWarps) k_metric(DevBasis X, DeviceTables dt,
                                                            int boys_mode, long long npairs,
                                                            double* __restrict__ M) {
  __shared__ double scratch[kTwoCWarps][kTwoCScratch];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long long pr = static_cast<long long>(blockIdx.x) * kTwoCWarps + warp;
  if (pr >= npairs) return;
  // pr = a (a + 1) / 2 + b, b <= a
  long long a = static_cast<long long>((sqrt(8.0 * static_cast<double>(pr) + 1.0) - 1.0) * 0.5);
  while (a * (a + 1) / 2 > pr) --a;
  while ((a + 1) * (a + 2) / 2 <= pr) ++a;
  const long long b = pr - a * (a + 1) / 2;
  TwoCScratch s = twoc_scratch(scratch[warp]);
  twoc_block_warp(X, static_cast<int>(a), static_cast<int>(b), dt, boys_mode, s, lane);
  const int4 sA = X.shell[a], sB = X.shell[b];
  const int nsA = 2 * sA.x + 1, nsB = 2 * sB.x + 1;
  const long long N = X.nsph;
  for (int i = lane; i < nsA * nsB; i += 32) {
    const int ia = i / nsB, ib = i - ia * nsB;
    const long long r = sA.w + ia, c = sB.w + ib;
    const double v = s.out[i];
    M[r + N * c] = v;
    M[c + N * r] = v;
  }
}

// ---------------------------------------------------------------------------
constexpr int kBraTChunk = 16;

__global__ void __launch_bounds__(256) k_bra_prep(DevBasis B, const int2* __restrict__ pair_ab,
                                                  UnitArrays U, BraPrepArgs a) {
  extern __shared__ double smem[];
  const int slot = a.slot0 + blockIdx.x;
  if (slot >= a.slot_end) return;
  const double q = a.slot_Q[slot];
  if (q * (*a.qmax_aux) < a.thresh) return;  // never reached by any surviving triple
  const int u = a.sorted_unit[slot];
  const int2 ab = pair_ab[U.unit_pair[u]];
  const int4 sa = B.shell[ab.x], sb = B.shell[ab.y];
  const int la = sa.x, lb = sb.x;
  const int nsb = 2 * lb + 1, nab = (2 * la + 1) * nsb;
  const int NH = ncum(la + lb);
  const int nd = a.nd;
  double* Ds = smem;            // [nab][nd]
  double* Es = Ds + nab * nd;   // [nab][kBraTChunk]
  for (int idx = threadIdx.x; idx < nab * nd; idx += blockDim.x) {
    const int r = idx / nd, d = idx - r * nd;
    const int ma = r / nsb, mb = r - ma * nsb;
    const long long i = sa.w + ma, j = sb.w + mb;
    double v = a.dens[d * a.sd + i * a.si + j * a.sj];
    if (ab.x != ab.y) v += a.dens[d * a.sd + j * a.si + i * a.sj];
    Ds[idx] = v;
  }
  if (threadIdx.x == 0) {
    a.slot_pP[slot] = U.unit_pP[u];
    if (a.slot_qvl) {
      const int pr = U.unit_pair[u];
      a.slot_qvl[slot] = a.pair_qvl[pr];
      a.slot_den[slot] = a.pair_den[pr];
    }
  }
  const double* E = U.esph + U.unit_esph[u];
  // G layout: [z][slot in class][t][dw], density d = z * dw + column, zero padded
  const int dw = a.dw;
  const int nz = (nd + dw - 1) / dw;
  const long long zstride = static_cast<long long>(a.n_class) * NH * dw;
  double* G = a.G + a.g_base + static_cast<long long>(slot - a.slot0) * NH * dw;
  for (int t0 = 0; t0 < NH; t0 += kBraTChunk) {
    const int tn = min(kBraTChunk, NH - t0);
    __syncthreads();
    for (int idx = threadIdx.x; idx < nab * kBraTChunk; idx += blockDim.x) {
      const int r = idx / kBraTChunk, tt = idx - r * kBraTChunk;
      Es[idx] = tt < tn ? E[r * NH + t0 + tt] : 0.0;
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < tn * nz * dw; idx += blockDim.x) {
      const int tt = idx / (nz * dw), dd = idx - tt * (nz * dw);
      const int z = dd / dw, c = dd - z * dw;
      double v = 0.0;
      if (dd < nd)
        for (int r = 0; r < nab; ++r) v = fma(Ds[r * nd + dd], Es[r * kBraTChunk + tt], v);
      G[z * zstride + (t0 + tt) * dw + c] = v;
    }
  }
}

}  // namespace

// ---------------------------------------------------------------------------
// Launchers.

int launch_unit_setup(const DevBasis& B, const int2* pair_ab, const int* class_unit, const PairLists& P,
                      UnitArrays U, const DeviceTables& dt, cudaStream_t s) {
  if (P.nunits == 0) return 0;
  int launches = 0;
  const int split = std::min(kUsLab, P.lab_max) + 1;  // classes [0, split) by warps
  const int nlow = P.class_off[split];
  if (nlow > 0) {
    k_unit_setup_warp<<<(nlow + kUsWarps - 1) / kUsWarps, 32 * kUsWarps, 0, s>>>(B, pair_ab, U, class_unit, nlow,
                                                                                 dt);
    ++launches;
  }
  const int nhigh = P.nunits - nlow;
  if (nhigh > 0) {
    k_unit_setup<<<nhigh, 128, 0, s>>>(B, pair_ab, U, class_unit + nlow, nhigh, dt);
    ++launches;
  }
  return launches;
}

template <int LAB>
int launch_schwarz_blk(const DevBasis& B, const int2* pair_ab, const int* pair_unit0, const int* pairs,
                       UnitArrays U, int n, const DeviceTables& dt, int boys_mode, double* Qab, cudaStream_t s) {
  const size_t smem = sizeof(double) * SwBlk<LAB>::SMEM;
  cudaFuncSetAttribute(k_schwarz_bra<LAB>, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  k_schwarz_bra<LAB><<<n, 32 * kSbWarps, smem, s>>>(B, pair_ab, pair_unit0, pairs, U, n, dt, boys_mode, Qab);
  return 1;
}

template <int LAB>
int launch_schwarz_dmma(const DevBasis& B, const int2* pair_ab, const int* pair_unit0, const int* pairs,
                        UnitArrays U, int n, const DeviceTables& dt, int boys_mode, double* Qab, cudaStream_t s) {
  const size_t smem = sizeof(double) * kSwWarps * SwDmma<LAB>::STRIDE;
  cudaFuncSetAttribute(k_schwarz_bra_dmma<LAB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  k_schwarz_bra_dmma<LAB><<<(n + kSwWarps - 1) / kSwWarps, 32 * kSwWarps, smem, s>>>(
      B, pair_ab, pair_unit0, pairs, U, n, dt, boys_mode, Qab);
  return 1;
}

int launch_schwarz_bra(const DevBasis& B, const int2* pair_ab, const int* pair_unit0,
                       const int* class_pair, const PairLists& P, UnitArrays U, const DeviceTables& dt,
                       int boys_mode, double* Qab, cudaStream_t s) {
  if (P.npairs == 0) return 0;
  int launches = 0;
  const int split = std::min(kSwLab, P.lab_max) + 1;  // classes [0, split) by warps
  const int nlow = P.pair_class_off[split];
  if (nlow > 0) {
    cudaFuncSetAttribute(k_schwarz_bra_warp, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         static_cast<int>(sizeof(double) * kSwWarps * kSwScratch));
    // classes L_ab 0..2 together (their scratch is small either way); 3 and 4
    // on their own, with both products on the tensor cores
    for (int g = 0; g < split;) {
      const int lab = g < 2 ? std::min(2, split - 1) : g;  // largest class of the group
      const int off = P.pair_class_off[g], n = P.pair_class_off[lab + 1] - off;
      g = lab + 1;
      if (n <= 0) continue;
      if (lab == 3 || lab == 4) {
        launches += lab == 3 ? launch_schwarz_dmma<3>(B, pair_ab, pair_unit0, class_pair + off, U, n, dt,
                                                      boys_mode, Qab, s)
                             : launch_schwarz_dmma<4>(B, pair_ab, pair_unit0, class_pair + off, U, n, dt,
                                                      boys_mode, Qab, s);
        continue;
      }
      int nab = 1;  // largest (2la+1)(2lb+1) with la + lb <= lab
      for (int l = 0; l <= lab; ++l)
        for (int la = std::max(0, l - PA_LMAX); la <= std::min(l, PA_LMAX); ++la)
          nab = std::max(nab, (2 * la + 1) * (2 * (l - la) + 1));
      const int nr = ncum(2 * lab), nh = ncum(lab);
      const int stride = 32 + 2 * nr + nab * nh + nab * nab;
      const size_t wsm = sizeof(double) * kSwWarps * stride;
      k_schwarz_bra_warp<<<(n + kSwWarps - 1) / kSwWarps, 32 * kSwWarps, wsm, s>>>(
          B, pair_ab, pair_unit0, class_pair + off, U, n, dt, boys_mode, Qab, nr, nab, nh, stride);
      ++launches;
    }
  }
  // one block per pair for the higher classes, one launch per class
  for (int lab = split; lab <= P.lab_max; ++lab) {
    const int off = P.pair_class_off[lab], n = P.pair_class_off[lab + 1] - off;
    if (n <= 0) continue;
    const int* pl = class_pair + off;
    switch (lab) {
      case 5: launches += launch_schwarz_blk<5>(B, pair_ab, pair_unit0, pl, U, n, dt, boys_mode, Qab, s); break;
      case 6: launches += launch_schwarz_blk<6>(B, pair_ab, pair_unit0, pl, U, n, dt, boys_mode, Qab, s); break;
      case 7: launches += launch_schwarz_blk<7>(B, pair_ab, pair_unit0, pl, U, n, dt, boys_mode, Qab, s); break;
      case 8: launches += launch_schwarz_blk<8>(B, pair_ab, pair_unit0, pl, U, n, dt, boys_mode, Qab, s); break;
      default: break;
    }
  }
  return launches;
}

int launch_schwarz_aux(const DevBasis& X, const DeviceTables& dt, int boys_mode, double* Qc,
                       cudaStream_t s) {
  if (X.nshells == 0) return 0;
  const int blocks = (X.nshells + kTwoCWarps - 1) / kTwoCWarps;
  k_schwarz_aux<<<blocks, 32 * kTwoCWarps, 0, s>>>(X, dt, boys_mode, Qc);
  return 1;
}

int launch_metric(const DevBasis& X, const DeviceTables& dt, int boys_mode, double* M,
                  cudaStream_t s) {
  const long long npairs = static_cast<long long>(X.nshells) * (X.nshells + 1) / 2;
  if (npairs == 0) return 0;
  const long long blocks = (npairs + kTwoCWarps - 1) / kTwoCWarps;
  k_metric<<<static_cast<unsigned>(blocks), 32 * kTwoCWarps, 0, s>>>(X, dt, boys_mode, npairs, M);
  return 1;
}

int launch_bra_prep(const DevBasis& B, const int2* pair_ab, UnitArrays U, const BraPrepArgs& a,
                    int lab, cudaStream_t s) {
  const int n = a.slot_end - a.slot0;
  if (n <= 0) return 0;
  int nab_max = 1;
  for (int la = 0; la <= PA_LMAX; ++la)
    for (int lb = 0; lb <= la; ++lb)
      if (la + lb == lab) nab_max = max(nab_max, (2 * la + 1) * (2 * lb + 1));
  const size_t smem = sizeof(double) * nab_max * (a.nd + kBraTChunk);
  cudaFuncSetAttribute(k_bra_prep, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  k_bra_prep<<<n, 256, smem, s>>>(B, pair_ab, U, a);
  return 1;
}

}  // namespace pa
