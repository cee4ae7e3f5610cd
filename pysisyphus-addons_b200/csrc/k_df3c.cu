// Screened three-center contraction df[P][d] = sum_(a>=b) sum_(i in a, j in b)
// (ij|P) [D_d(i,j) + (a != b) D_d(j,i)]  -- the hot loop of
// contract_coulomb_densities_2d (diabatization/intor.f90:108-183).
//
// Formulation (McMurchie-Davidson with the density folded into the bra):
//   df[P,m][d] += sum_tuv G_u[tuv][d] * X_(u,P)[tuv][m]
//   X_(u,P)[tuv][m] = pref(u,P) sum_(|tau|=lc) S_lc,m[tau] R_(tuv+tau)(alpha, P_u - C_P)
// where u is a primitive pair ("bra unit") of a surviving shell pair, G_u the
// density-folded Hermite expansion of the pair (k_bra_prep) and S the solid
// harmonic coefficients of the auxiliary shell (Hobson's theorem: only Hermite
// components of degree exactly lc appear on the auxiliary side).
//
// One kernel instance per class (LAB = la + lb, LC = l_aux). Bra units and
// auxiliary shells are sorted by Schwarz value (descending) within their class,
// so the surviving triples Q_ab * Q_c >= threshold form a staircase: a block
// stops at the first unit failing against the largest auxiliary shell of its
// tile, and individual triples below the threshold are skipped exactly as in
// the reference (schwarz_estimate < 1e-10 -> cycle).
//
// A block owns a tile of TC auxiliary shells x (density chunk) and loops over a
// chunk of bra units, UB units per step:
//   1. stage G of the UB units into shared memory;
//   2. build X for the UB x TC triples (Boys function, Hermite R recurrence,
//      solid-harmonic contraction) into shared memory;
//   3. register-tiled FP64 update acc[aux fn][d] += X^T G.
// Each block writes its partial sums to a per-chunk slab; k_df3c_reduce sums
// the slabs in a fixed order (deterministic results, no atomics).
#include "boys.cuh"
#include "k_df3c.cuh"
#include "md.cuh"

namespace pa {

namespace {

struct BlockSync {
  __device__ void operator()() const { __syncthreads(); }
};

constexpr int kThreads = 256;
constexpr int kSmemBudget = 200 * 1024 / 8;  // doubles

template <int LAB, int LC>
struct Cfg {
  static constexpr int NH = ncum(LAB);
  static constexpr int NC = 2 * LC + 1;
  static constexpr int NCC = ncart(LC);
  static constexpr int L = LAB + LC;
  static constexpr int NR = ncum(L);
  static constexpr bool kPerThread = (L <= 3);
  static constexpr int UB = NH >= 32 ? 1 : (32 / NH < 16 ? 32 / NH : 16);
  static constexpr int smem_for(int tc, int ndc) {
    const int mp = ((tc * NC + 15) / 16) * 16;
    const int k = UB * NH;
    const int ntrip = UB * tc;
    const int team = kPerThread ? 0 : ntrip * (2 * NR + 16);
    return k * mp + k * ndc + team + ((NC * NCC + 3) / 4) * 4 + 8 * 64;
  }
  static constexpr int pick_tc() {
    int tc = 128 / NC;
    if (tc > 64) tc = 64;
    if (!kPerThread && UB * tc > kThreads) tc = kThreads / UB;
    while (tc > 1 && smem_for(tc, 32) > kSmemBudget) --tc;
    return tc;
  }
  static constexpr int TC = pick_tc();
  static constexpr int M = TC * NC;
  static constexpr int MP = ((M + 15) / 16) * 16;
  static constexpr int RM = MP / 16;
  static constexpr int pick_ndc() {
    int ndc = 64;
    while (ndc > 16 && smem_for(TC, ndc) > kSmemBudget) ndc -= 16;
    return ndc;
  }
  static constexpr int NDC = pick_ndc();  // max densities per block
  static constexpr int RN = NDC / 16;
  static constexpr int K = UB * NH;
  static constexpr int NTRIP = UB * TC;
  static constexpr int TS = kPerThread ? 1 : (kThreads / NTRIP >= 32 ? 32 : kThreads / NTRIP);
  static constexpr int SMEM = smem_for(TC, NDC);
};

// Per-thread Hermite R (small L): in-place level recursion in registers.
template <int L>
__device__ __forceinline__ void hermite_R_thread(const double* Rn, double X, double Y, double Z,
                                                 double* R) {
  R[0] = Rn[L];
#pragma unroll
  for (int n = L - 1; n >= 0; --n) {
#pragma unroll
    for (int deg = L - n; deg >= 1; --deg) {
#pragma unroll
      for (int t = deg; t >= 0; --t) {
#pragma unroll
        for (int u = deg - t; u >= 0; --u) {
          const int v = deg - t - u;
          double val;
          if (t > 0) {
            val = X * R[cidx(t - 1, u, v)];
            if (t > 1) val += (t - 1) * R[cidx(t - 2, u, v)];
          } else if (u > 0) {
            val = Y * R[cidx(0, u - 1, v)];
            if (u > 1) val += (u - 1) * R[cidx(0, u - 2, v)];
          } else {
            val = Z * R[cidx(0, 0, v - 1)];
            if (v > 1) val += (v - 1) * R[cidx(0, 0, v - 2)];
          }
          R[cidx(t, u, v)] = val;
        }
      }
    }
    R[0] = Rn[n];
  }
}

__constant__ double c_sph_dense[1024];  // dense solid harmonics, row (l, m) at c_sph_off[l] + m * ncart(l)
__constant__ int c_sph_off[PA_LAUXMAX + 2];

template <int LAB, int LC>
__global__ void __launch_bounds__(kThreads) k_df3c(Df3cArgs a) {
  using C = Cfg<LAB, LC>;
  extern __shared__ double smem[];
  double* Xs = smem;                    // [K][MP]
  double* Gs = Xs + C::K * C::MP;       // [K][NDC]
  double* Ts = Gs + C::K * C::NDC;      // [NC][NCC] solid harmonics
  double* misc = Ts + ((C::NC * C::NCC + 3) / 4) * 4;  // unit / aux parameters (32-byte aligned)
  double* Rteam = misc + 8 * 64;        // team scratch
  double4* u_pP = reinterpret_cast<double4*>(misc);         // [UB]      (4 doubles each)
  double* u_Q = misc + 4 * 16;                              // [UB]
  double4* c_C = reinterpret_cast<double4*>(misc + 4 * 16 + 16);  // [TC] center (x,y,z,Q)
  int* c_info = reinterpret_cast<int*>(misc + 4 * 16 + 16 + 4 * 64);  // [TC] (nprim, prim_off)

  const int tid = threadIdx.x;
  const int c0 = blockIdx.x * C::TC;
  const int tile_n = min(C::TC, a.n_aux - c0);
  const int d0 = blockIdx.z * C::NDC;
  const int ndc = min(C::NDC, a.nd - d0);
  const int ub = blockIdx.y * a.units_per_chunk;
  const int ue = min(a.n_units, ub + a.units_per_chunk);

  // auxiliary tile
  int maxprim = 0;
  if (tid < C::TC) {
    if (tid < tile_n) {
      const int sh = a.sorted_aux[a.aux_slot0 + c0 + tid];
      const int4 info = a.X.shell[sh];
      const double4 cen = a.X.center[sh];
      c_C[tid] = make_double4(cen.x, cen.y, cen.z, a.aux_Q[a.aux_slot0 + c0 + tid]);
      c_info[2 * tid] = info.y;
      c_info[2 * tid + 1] = info.z;
    } else {
      c_C[tid] = make_double4(0.0, 0.0, 0.0, 0.0);
      c_info[2 * tid] = 0;
      c_info[2 * tid + 1] = 0;
    }
  }
  for (int i = tid; i < C::NC * C::NCC; i += kThreads) Ts[i] = c_sph_dense[c_sph_off[LC] + i];
  __syncthreads();
  for (int i = 0; i < tile_n; ++i) maxprim = max(maxprim, c_info[2 * i]);
  const double qc_max = tile_n > 0 ? c_C[0].w : 0.0;

  double acc[C::RM][C::RN];
#pragma unroll
  for (int i = 0; i < C::RM; ++i)
#pragma unroll
    for (int j = 0; j < C::RN; ++j) acc[i][j] = 0.0;
  const int tx = tid & 15, ty = tid >> 4;
  const double thr = a.thresh;
  const IndexTables* it = a.dt.idx;

  for (int u0 = ub; u0 < ue && tile_n > 0; u0 += C::UB) {
    if (a.unit_Q[a.unit_slot0 + u0] * qc_max < thr) break;  // sorted: nothing below survives
    __syncthreads();
    if (tid < C::UB) {
      const int s = u0 + tid;
      if (s < ue) {
        u_pP[tid] = a.slot_pP[a.unit_slot0 + s];
        u_Q[tid] = a.unit_Q[a.unit_slot0 + s];
      } else {
        u_pP[tid] = make_double4(1.0, 0.0, 0.0, 0.0);
        u_Q[tid] = 0.0;
      }
    }
    // stage G
    for (int idx = tid; idx < C::K * C::NDC; idx += kThreads) {
      const int k = idx / C::NDC, col = idx - k * C::NDC;
      const int ui = k / C::NH, t = k - ui * C::NH;
      const int s = u0 + ui;
      double v = 0.0;
      // Units failing against the tile's largest auxiliary shell were skipped by
      // k_bra_prep (their G is not written) and contribute nothing here.
      if (s < ue && col < ndc && a.unit_Q[a.unit_slot0 + s] * qc_max >= thr)
        v = a.G[static_cast<long long>(s) * C::NH * a.nd + t * a.nd + d0 + col];
      Gs[idx] = v;
    }
    for (int idx = tid; idx < C::K * C::MP; idx += kThreads) Xs[idx] = 0.0;
    __syncthreads();

    // build X
    if constexpr (C::kPerThread) {
      for (int trip = tid; trip < C::NTRIP; trip += kThreads) {
        const int ui = trip / C::TC, ci = trip - ui * C::TC;
        if (ci >= tile_n || u0 + ui >= ue) continue;
        const double4 cc = c_C[ci];
        if (u_Q[ui] * cc.w < thr) continue;
        const double4 up = u_pP[ui];
        const double p = up.x;
        const double X = up.y - cc.x, Y = up.z - cc.y, Z = up.w - cc.z;
        const double RPC2 = X * X + Y * Y + Z * Z;
        double xacc[C::NH][C::NC];
#pragma unroll
        for (int t = 0; t < C::NH; ++t)
#pragma unroll
          for (int m = 0; m < C::NC; ++m) xacc[t][m] = 0.0;
        const int np = c_info[2 * ci], po = c_info[2 * ci + 1];
        for (int kp = 0; kp < np; ++kp) {
          const double2 g = a.X.prim[po + kp];
          const double gam = g.x, pg = p + gam, alpha = p * gam / pg;
          double pref = kTwoPi52 / (p * gam * sqrt(pg)) * g.y;
#pragma unroll
          for (int l = 0; l < LC; ++l) pref *= -0.5 / gam;  // (-1)^LC (2 gam)^-LC
          double F[C::L + 1];
          boys_all(a.dt, a.boys_mode, C::L, alpha * RPC2, F);
          double Rn[C::L + 1];
          double f = pref;
#pragma unroll
          for (int n = 0; n <= C::L; ++n) {
            Rn[n] = f * F[n];
            f *= -2.0 * alpha;
          }
          double R[C::NR];
          hermite_R_thread<C::L>(Rn, X, Y, Z, R);
#pragma unroll
          for (int t = 0; t <= LAB; ++t)
#pragma unroll
            for (int tt = t; tt >= 0; --tt)
#pragma unroll
              for (int uu = t - tt; uu >= 0; --uu) {
                const int vv = t - tt - uu;
                const int th = cidx(tt, uu, vv);
#pragma unroll
                for (int m = 0; m < C::NC; ++m) {
                  double s = 0.0;
#pragma unroll
                  for (int ta = LC; ta >= 0; --ta)
#pragma unroll
                    for (int ua = LC - ta; ua >= 0; --ua) {
                      const int va = LC - ta - ua;
                      const int cl = cidx(ta, ua, va) - ncum(LC - 1);
                      s += Ts[m * C::NCC + cl] * R[cidx(tt + ta, uu + ua, vv + va)];
                    }
                  xacc[th][m] += s;
                }
              }
        }
#pragma unroll
        for (int t = 0; t < C::NH; ++t)
#pragma unroll
          for (int m = 0; m < C::NC; ++m) Xs[(ui * C::NH + t) * C::MP + ci * C::NC + m] = xacc[t][m];
      }
    } else {
      const int team = tid / C::TS, lane = tid - team * C::TS;
      const bool in_team = team < C::NTRIP;
      const int ui = in_team ? team / C::TC : 0, ci = in_team ? team - ui * C::TC : 0;
      double* Rn = Rteam + (in_team ? team : 0) * (2 * C::NR + 16);
      double* b0 = Rn + 16;
      double* b1 = b0 + C::NR;
      bool active = in_team && ci < tile_n && (u0 + ui) < ue;
      double4 cc = c_C[ci];
      active = active && (u_Q[ui] * cc.w >= thr);
      const double4 up = u_pP[ui];
      const double p = up.x;
      const double X = up.y - cc.x, Y = up.z - cc.y, Z = up.w - cc.z;
      const double RPC2 = X * X + Y * Y + Z * Z;
      const int np = active ? c_info[2 * ci] : 0, po = c_info[2 * ci + 1];
      for (int kp = 0; kp < maxprim; ++kp) {
        const bool has = active && kp < np;
        if (has) {
          const double2 g = a.X.prim[po + kp];
          const double gam = g.x, pg = p + gam, alpha = p * gam / pg;
          double pref = kTwoPi52 / (p * gam * sqrt(pg)) * g.y;
          for (int l = 0; l < LC; ++l) pref *= -0.5 / gam;
          // orders n = lane, lane + TS, ...: a team may have fewer lanes than L + 1
          for (int n = lane; n <= C::L; n += C::TS) {
            double f = pref;
            for (int k = 0; k < n; ++k) f *= -2.0 * alpha;
            Rn[n] = f * boys_n(a.dt, a.boys_mode, n, alpha * RPC2);
          }
        }
        __syncthreads();
        hermite_R(it, C::L, Rn, X, Y, Z, b0, b1, in_team ? lane : C::TS, has ? C::TS : 0,
                  BlockSync());
        if (has) {
          for (int idx = lane; idx < C::NH * C::NC; idx += C::TS) {
            const int t = idx / C::NC, m = idx - t * C::NC;
            double s = 0.0;
#pragma unroll
            for (int cl = 0; cl < C::NCC; ++cl) {
              const double w = Ts[m * C::NCC + cl];
              if (w != 0.0) {
                const uchar4 e = *reinterpret_cast<const uchar4*>(it->xyz[t]);
                const uchar4 f = *reinterpret_cast<const uchar4*>(it->xyz[ncum(LC - 1) + cl]);
                s = fma(w, b0[cidx(e.x + f.x, e.y + f.y, e.z + f.z)], s);
              }
            }
            Xs[(ui * C::NH + t) * C::MP + ci * C::NC + m] += s;
          }
        }
        __syncthreads();
      }
    }
    __syncthreads();

    // acc[row][col] += sum_k Xs[k][row] Gs[k][col]
#pragma unroll 4
    for (int k = 0; k < C::K; ++k) {
      double xr[C::RM], gc[C::RN];
#pragma unroll
      for (int i = 0; i < C::RM; ++i) xr[i] = Xs[k * C::MP + ty + 16 * i];
#pragma unroll
      for (int j = 0; j < C::RN; ++j) gc[j] = Gs[k * C::NDC + tx + 16 * j];
#pragma unroll
      for (int i = 0; i < C::RM; ++i)
#pragma unroll
        for (int j = 0; j < C::RN; ++j) acc[i][j] = fma(xr[i], gc[j], acc[i][j]);
    }
  }

  // partial[y][fn][d]
  double* out = a.partial + static_cast<long long>(blockIdx.y) * a.n_aux * C::NC * a.nd;
#pragma unroll
  for (int i = 0; i < C::RM; ++i) {
    const int row = ty + 16 * i;
    if (row >= C::M || row / C::NC >= tile_n) continue;
    const long long fn = static_cast<long long>(c0) * C::NC + row;
#pragma unroll
    for (int j = 0; j < C::RN; ++j) {
      const int col = tx + 16 * j;
      if (col < ndc) out[fn * a.nd + d0 + col] = acc[i][j];
    }
  }
}

// df_raw[sph_off(P) + m][d] (column-major, naux rows) = sum over LAB classes and
// bra chunks of the partial slabs of class LC.
__global__ void k_df3c_reduce(Df3cReduceArgs r) {
  const long long total = static_cast<long long>(r.n_aux) * r.nc * r.nd;
  for (long long idx = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; idx < total;
       idx += static_cast<long long>(gridDim.x) * blockDim.x) {
    const long long fn = idx / r.nd;
    const int d = static_cast<int>(idx - fn * r.nd);
    double s = 0.0;
    for (int c = 0; c < r.nclasses; ++c) {
      const double* p = r.part[c];
      if (!p) continue;
      const long long slab = static_cast<long long>(r.n_aux) * r.nc * r.nd;
      for (int y = 0; y < r.ny[c]; ++y) s += p[y * slab + fn * r.nd + d];
    }
    const int pos = static_cast<int>(fn / r.nc), m = static_cast<int>(fn - pos * r.nc);
    const int sh = r.sorted_aux[r.aux_slot0 + pos];
    const long long row = r.X.shell[sh].w + m;
    r.df[row + static_cast<long long>(r.naux) * d] = s;
  }
}

template <int LAB, int LC>
int launch_class(const Df3cArgs& a, int ny, cudaStream_t s) {
  using C = Cfg<LAB, LC>;
  const size_t smem = sizeof(double) * C::SMEM;
  cudaFuncSetAttribute(k_df3c<LAB, LC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       static_cast<int>(smem));
  dim3 grid((a.n_aux + C::TC - 1) / C::TC, ny, (a.nd + C::NDC - 1) / C::NDC);
  k_df3c<LAB, LC><<<grid, kThreads, smem, s>>>(a);
  return 1;
}

template <int LAB, int LC>
void class_info(Df3cClassInfo* ci) {
  using C = Cfg<LAB, LC>;
  ci->tc = C::TC;
  ci->ub = C::UB;
  ci->ndc = C::NDC;
  ci->smem = sizeof(double) * C::SMEM;
}

using LaunchFn = int (*)(const Df3cArgs&, int, cudaStream_t);
using InfoFn = void (*)(Df3cClassInfo*);

template <int LAB, int LC>
struct Entry {
  static constexpr LaunchFn launch = &launch_class<LAB, LC>;
  static constexpr InfoFn info = &class_info<LAB, LC>;
};

#define PA_ROW(LAB)                                                                    \
  {Entry<LAB, 0>::launch, Entry<LAB, 1>::launch, Entry<LAB, 2>::launch, Entry<LAB, 3>::launch, \
   Entry<LAB, 4>::launch, Entry<LAB, 5>::launch}
#define PA_IROW(LAB)                                                                 \
  {Entry<LAB, 0>::info, Entry<LAB, 1>::info, Entry<LAB, 2>::info, Entry<LAB, 3>::info, \
   Entry<LAB, 4>::info, Entry<LAB, 5>::info}

const LaunchFn kLaunch[2 * PA_LMAX + 1][PA_LAUXMAX + 1] = {
    PA_ROW(0), PA_ROW(1), PA_ROW(2), PA_ROW(3), PA_ROW(4), PA_ROW(5), PA_ROW(6), PA_ROW(7), PA_ROW(8)};
const InfoFn kInfo[2 * PA_LMAX + 1][PA_LAUXMAX + 1] = {
    PA_IROW(0), PA_IROW(1), PA_IROW(2), PA_IROW(3), PA_IROW(4),
    PA_IROW(5), PA_IROW(6), PA_IROW(7), PA_IROW(8)};

}  // namespace

void df3c_class_info(int lab, int lc, Df3cClassInfo* ci) { kInfo[lab][lc](ci); }

int launch_df3c_class(int lab, int lc, const Df3cArgs& a, int ny, cudaStream_t s) {
  return kLaunch[lab][lc](a, ny, s);
}

int launch_df3c_reduce(const Df3cReduceArgs& r, cudaStream_t s) {
  const long long total = static_cast<long long>(r.n_aux) * r.nc * r.nd;
  if (total == 0) return 0;
  const int blocks = static_cast<int>(std::min<long long>((total + 255) / 256, 148 * 16));
  k_df3c_reduce<<<blocks, 256, 0, s>>>(r);
  return 1;
}

cudaError_t upload_sph_dense(const double* vals, int n, const int* offs, cudaStream_t s) {
  cudaError_t e = cudaMemcpyToSymbolAsync(c_sph_dense, vals, sizeof(double) * n, 0,
                                          cudaMemcpyHostToDevice, s);
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbolAsync(c_sph_off, offs, sizeof(int) * (PA_LAUXMAX + 2), 0,
                                 cudaMemcpyHostToDevice, s);
}

}  // namespace pa
