// Screened three-center contraction df[P][d] = sum_(a>=b) sum_(i in a, j in b)
// (ij|P) [D_d(i,j) + (a != b) D_d(j,i)]  -- the hot loop of
// contract_coulomb_densities_2d (diabatization/intor.f90:108-183).
//
// Formulation (McMurchie-Davidson with the density folded into the bra):
//   df[P,m][d] += sum_tuv X_(u,P)[tuv][m] G_u[tuv][d]
//   X_(u,P)[tuv][m] = pref(u,P) sum_(|tau|=lc) S_lc,m[tau] R_(tuv+tau)(alpha, P_u - C_P)
// where u is a primitive pair ("bra unit") of a surviving shell pair, G_u its
// density-folded Hermite expansion (k_bra_prep) and S the solid harmonic
// coefficients of the auxiliary shell (Hobson's theorem: only Hermite
// components of degree exactly lc appear on the auxiliary side).
//
// One kernel instance per class (LAB = la + lb, LC = l_aux) and tile-shape
// variant V (Cfg below); each k_df3c_l<LAB>.cu instantiates the classes of one
// LAB, and k_df3c.cu dispatches on (LAB, LC, V) at run time. Bra units and
// auxiliary shells are sorted by Schwarz value (descending) within their class,
// so the surviving triplets Q_ab * Q_c >= threshold form a staircase: a block
// stops at the first unit failing against the largest auxiliary shell of its
// tile, and individual triplets below the threshold contribute exactly zero, as
// the reference skips them (schwarz_estimate < 1e-10 -> cycle).
//
// A block (8 warps; two blocks per SM) owns a tile of TC auxiliary shells and a density chunk of
// up to 40 columns, and walks a range of bra units, UB units per step:
//   1. cp.async stages G of the UB units (one contiguous range) into shared
//      memory while
//   2. X of the UB x TC triplets is built into shared memory: the Boys function,
//      the Hermite recurrence for R and the solid-harmonic contraction --
//      per thread with R in registers and compile-time indices for L <= 5, by
//      thread teams with R in shared memory above;
//   3. the update acc[aux fn][d] += X^T G runs on the FP64 tensor cores
//      (mma.sync m8n8k4 f64), accumulators in registers.
// Each block writes its partial sums to a per-chunk slab; k_df3c_reduce sums the
// slabs in a fixed order (deterministic results, no atomics).
#pragma once

#include "boys.cuh"
#include "k_df3c.cuh"
#include "md.cuh"
#include "sph_raw.cuh"
#include "umma.cuh"

#include <algorithm>
#include <utility>

namespace pa {

namespace {


struct BlockSync {
  __device__ void operator()() const { __syncthreads(); }
};

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kSmemBudget = 110 * 1024 / 8;  // doubles (two blocks per SM)
constexpr int kSmemBudget3 = 72 * 1024 / 8;  // doubles (three blocks per SM)
constexpr int kGStride = 44;                 // shared-memory row stride of G (>= 40, = 4 mod 16)

__constant__ double c_sph_rownorm[(PA_LAUXMAX + 1) * (PA_LAUXMAX + 1)];  // [l*l + m + l]

constexpr int round_up(int x, int m) { return (x + m - 1) / m * m; }
// row stride = 4 (mod 16) doubles: conflict-free m8n8k4 fragment loads
constexpr int pad_stride(int mp) { return mp + ((20 - mp % 16) % 16); }

// Shape of class (LAB, LC) in tile-shape variant V:
//   0: the largest auxiliary tile (TC shells) that fits two blocks per SM;
//   1: the tile, at least half as large, that keeps the most lanes busy in the
//      X build (triplets x lanes per triplet, up to the block's 256 threads);
//   2: team classes (L > 5) at three blocks per SM: 72 KB of shared memory and
//      80 registers per thread (variant 0 where even one shell does not fit).
// k_df3c.cu picks the variant per class at run time (default 0).
template <int LAB, int LC, int V>
struct Cfg {
  static constexpr int NH = ncum(LAB);
  static constexpr int NC = 2 * LC + 1;
  static constexpr int NCC = ncart(LC);
  static constexpr int L = LAB + LC;
  static constexpr int NR = ncum(L);
  static constexpr bool kPerThread = (L <= 5);
  static constexpr int pick_ub(int tc) {
    if (kPerThread) {
      int ub = 64 / NH;
      if (ub < 1) ub = 1;
      if (ub * tc > 512) ub = 512 / tc;
      return ub < 1 ? 1 : ub;
    }
    int ub = 40 / NH;
    if (ub < 1) ub = 1;
    if (ub * tc > 64) ub = 64 / tc;
    return ub < 1 ? 1 : ub;
  }
  static constexpr int smem_for(int tc) {
    const int ub = pick_ub(tc);
    const int kp = round_up(ub * NH, 4);
    const int mpad = pad_stride(round_up(tc * NC, 8));
    const int team = kPerThread ? 0 : ub * tc * (2 * NR + 16) + 2 * NR;
    return kp * mpad + kp * kGStride + team + 1024;
  }
  static constexpr int kMinBlocks = (V == 2 && !kPerThread && smem_for(1) <= kSmemBudget3) ? 3 : 2;
  static constexpr int kBudget = kMinBlocks == 3 ? kSmemBudget3 : kSmemBudget;
  // lanes per triplet in the X build: threads per triplet (per-thread mode,
  // up to 8) or the team size (team mode), a power of two
  static constexpr int width_for(int tc) {
    const int n = pick_ub(tc) * tc;
    int t = 1;
    if (kPerThread) {
      while (t < 8 && 2 * t * n <= kThreads) t *= 2;
    } else {
      while (t < kThreads && 2 * t * n <= kThreads) t *= 2;
    }
    return t;
  }
  static constexpr int lanes_for(int tc) {
    const int u = pick_ub(tc) * tc * width_for(tc);
    return u < kThreads ? u : kThreads;
  }
  static constexpr int pick_tc() {
    int tc = 128 / NC;
    if (tc > 128) tc = 128;
    if (!kPerThread && tc > 32) tc = 32;
    while (tc > 1 && smem_for(tc) > kBudget) --tc;
    if (V != 1) return tc;
    int best = tc;
    for (int t = tc - 1; t >= 1 && 2 * t >= tc; --t)
      if (lanes_for(t) > lanes_for(best)) best = t;
    return best;
  }
  static constexpr int TC = pick_tc();
  static constexpr int UB = pick_ub(TC);
  static constexpr int M = TC * NC;
  static constexpr int MP = round_up(M, 8);
  static constexpr int MPAD = pad_stride(MP);
  static constexpr int MT = MP / 8;                 // m8n8k4 row tiles
  static constexpr int MTW = (MT + kWarps - 1) / kWarps;
  static constexpr int K = UB * NH;
  static constexpr int KP = round_up(K, 4);
  static constexpr int NTRIP = UB * TC;
  // per-thread mode: threads per triplet (warp-uniform split of t); team
  // mode: teams of up to 32 lanes share a warp, larger ones are whole warps
  // synchronized by a named barrier
  static constexpr int TPT = kPerThread ? width_for(TC) : 1;
  static constexpr int TS = kPerThread ? 1 : width_for(TC);
  static_assert(TS <= 32 || TS % 32 == 0, "multi-warp teams are whole warps");
  static_assert(TS <= 32 || kThreads / TS < 16, "named barrier ids 1..15");
  // DMMA product: with fewer row tiles than warps, KSPLIT warps share a row
  // tile and split its k range; their accumulators are summed once per item
  static constexpr int KSPLIT = MT >= kWarps ? 1 : kWarps / MT;
  // team scratch stride (doubles): the teams of a warp read and write their
  // components at the same offsets, so a stride of TS (mod 16) doubles puts
  // their TS-wide chunks in different banks (when it fits the budget)
  static constexpr int kPadWanted = (!kPerThread && TS <= 8) ? (TS - (2 * NR + 16) % 16 + 16) % 16 : 0;
  static constexpr int kPad = smem_for(TC) + NTRIP * kPadWanted <= kBudget ? kPadWanted : 0;
  static constexpr int kTeamStride = 2 * NR + 16 + kPad;
  static constexpr int SMEM = smem_for(TC) + (kPerThread ? 0 : NTRIP * kPad);
  static_assert(KSPLIT == 1 || KSPLIT * MT * 320 <= KP * (MPAD + kGStride),
                "k-split reduction fits in the X and G tiles");
};

// Barrier of one team of TS threads (team mode): the warp for teams of up to
// 32 lanes, a named barrier (ids 1..15; 0 is __syncthreads) for larger teams.
template <int TS>
__device__ __forceinline__ void team_sync(int team) {
  if constexpr (TS <= 32)
    __syncwarp();
  else
    asm volatile("bar.sync %0, %1;\n" ::"r"(1 + team), "r"(TS) : "memory");
}

__device__ __forceinline__ void dmma_m8n8k4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src));
}
__device__ __forceinline__ void cp_async_commit_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::);
}

// Per-thread Hermite R (small L): in-place level recursion in registers.
template <int L, class Real>
__device__ __forceinline__ void hermite_R_thread(const Real* Rn, Real X, Real Y, Real Z, Real* R) {
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
          Real val;
          if (t > 0) {
            val = X * R[cidx(t - 1, u, v)];
            if (t > 1) val = fma(static_cast<Real>(t - 1), R[cidx(t - 2, u, v)], val);
          } else if (u > 0) {
            val = Y * R[cidx(0, u - 1, v)];
            if (u > 1) val = fma(static_cast<Real>(u - 1), R[cidx(0, u - 2, v)], val);
          } else {
            val = Z * R[cidx(0, 0, v - 1)];
            if (v > 1) val = fma(static_cast<Real>(v - 1), R[cidx(0, 0, v - 2)], val);
          }
          R[cidx(t, u, v)] = val;
        }
      }
    }
    R[0] = Rn[n];
  }
}

// Decoded local Cartesian index c of degree l (x^l, x^(l-1) y, ...), compile time.
__host__ __device__ constexpr int cart_x(int l, int c) {
  int i = l, k = c;
  while (k > l - i) {
    k -= l - i + 1;
    --i;
  }
  return i;
}
__host__ __device__ constexpr int cart_y(int l, int c) {
  int i = l, k = c;
  while (k > l - i) {
    k -= l - i + 1;
    --i;
  }
  return l - i - k;
}

// One solid-harmonic term w * R[t + tau] with w a compile-time constant (the
// term vanishes at compile time when w == 0). Real is double, or float for the
// FP32 recurrences of weak triplets.
template <int LC, int M, int C, class Real>
__device__ __forceinline__ Real sph_term(const Real* R, int tx, int ty, int tz) {
  constexpr int ax = cart_x(LC, C), ay = cart_y(LC, C), az = LC - ax - ay;
  constexpr double w = sph_raw(LC, M - LC, ax, ay, az);
  if constexpr (w != 0.0)
    return static_cast<Real>(w) * R[cidx(tx + ax, ty + ay, tz + az)];
  else
    return static_cast<Real>(-0.0);  // x + (-0.0) == x exactly, so the compiler drops the term
}

template <int LC, int M, class Real, int... Cs>
__device__ __forceinline__ Real sph_row(const Real* R, int tx, int ty, int tz,
                                        std::integer_sequence<int, Cs...>) {
  return (static_cast<Real>(-0.0) + ... + sph_term<LC, M, Cs, Real>(R, tx, ty, tz));
}

// xr[m] (+)= N_lc,m * sum_tau S_lc,m[tau] R[t + tau] (in FP64). The first
// auxiliary primitive stores (ACC = false), later ones accumulate: the X tile
// needs no zeroing pass (fma(a, b, 0) and a * b round alike).
template <int LC, class Real, bool ACC, int... Ms>
__device__ __forceinline__ void sph_rows(const Real* R, int tx, int ty, int tz, double* xr,
                                         std::integer_sequence<int, Ms...>) {
  if constexpr (ACC)
    ((xr[Ms] = fma(c_sph_rownorm[LC * LC + Ms],
                   static_cast<double>(sph_row<LC, Ms, Real>(R, tx, ty, tz,
                                                             std::make_integer_sequence<int, ncart(LC)>{})),
                   xr[Ms])),
     ...);
  else
    ((xr[Ms] = c_sph_rownorm[LC * LC + Ms] *
               static_cast<double>(sph_row<LC, Ms, Real>(R, tx, ty, tz, std::make_integer_sequence<int, ncart(LC)>{}))),
     ...);
}

// X rows of one triplet, per thread: rows t with t % TPT == part.
template <int LAB, int LC, int TPT, class Real, bool ACC>
__device__ __forceinline__ void x_rows_thread(const Real* R, double* xrow0, int mpad, int part) {
#pragma unroll
  for (int tl = 0; tl <= LAB; ++tl)
#pragma unroll
    for (int tx = tl; tx >= 0; --tx)
#pragma unroll
      for (int ty = tl - tx; ty >= 0; --ty) {
        const int tz = tl - tx - ty;
        const int th = cidx(tx, ty, tz);
        if (th % TPT != part) continue;
        sph_rows<LC, Real, ACC>(R, tx, ty, tz, xrow0 + th * mpad, std::make_integer_sequence<int, 2 * LC + 1>{});
      }
}

// Zeros the X rows of a screened triplet (per thread: rows t % TPT == part).
template <int LAB, int LC, int TPT>
__device__ __forceinline__ void x_rows_zero(double* xrow0, int mpad, int part) {
#pragma unroll
  for (int th = part; th < ncum(LAB); th += TPT)
#pragma unroll
    for (int m = 0; m < 2 * LC + 1; ++m) xrow0[th * mpad + m] = 0.0;
}

// X of one triplet by one thread (L <= 5): Boys, R in registers, solid harmonics.
template <int LAB, int LC, int NR, int MPAD, int TPT, class Real>
__device__ __forceinline__ void x_triplet_thread(const Df3cArgs& a, double p, double X, double Y,
                                                 double Z, int np, int po, double* xrow0, int part) {
  constexpr int L = LAB + LC;
  const double RPC2 = X * X + Y * Y + Z * Z;
  for (int kp = 0; kp < np; ++kp) {
    const double2 gp = a.X.prim[po + kp];
    const double gam = gp.x, pg = p + gam, alpha = p * gam / pg;
    double pref = kTwoPi52 / (p * gam * sqrt(pg)) * gp.y;
#pragma unroll
    for (int l = 0; l < LC; ++l) pref *= -0.5 / gam;  // (-1)^LC (2 gam)^-LC
    Real F[L + 1];
    boys_all(a.dt, a.boys_mode, L, alpha * RPC2, F);
    Real Rn[L + 1];
    double f = pref;
#pragma unroll
    for (int n = 0; n <= L; ++n) {
      Rn[n] = static_cast<Real>(f) * F[n];
      f *= -2.0 * alpha;
    }
    Real R[NR];
    hermite_R_thread<L, Real>(Rn, static_cast<Real>(X), static_cast<Real>(Y), static_cast<Real>(Z), R);
    if (kp == 0)
      x_rows_thread<LAB, LC, TPT, Real, false>(R, xrow0, MPAD, part);
    else
      x_rows_thread<LAB, LC, TPT, Real, true>(R, xrow0, MPAD, part);
  }
}

// X of one triplet by a team of TS threads (L > 5): orders of the Boys
// function across lanes, R level by level in shared memory, X rows across the
// lanes. Every thread of a warp (of a team, for teams larger than a warp)
// calls this with the same Real (the caller makes the precision choice
// uniform), so the team barriers pair up.
template <int LAB, int LC, int TS, class Real>
__device__ __forceinline__ void x_triplet_team(const Df3cArgs& a, const uchar4* txyz, const int* rdesc,
                                               double* rbuf, int team, int tl, bool active, int np, int po,
                                               int maxprim, double p, double X, double Y, double Z,
                                               double* xrow, int mpad) {
  constexpr int L = LAB + LC;
  constexpr int NR = ncum(L);
  constexpr int NH = ncum(LAB);
  Real* Rn = reinterpret_cast<Real*>(rbuf);
  Real* b0 = Rn + 16;
  Real* b1 = b0 + NR;
  const double RPC2 = X * X + Y * Y + Z * Z;
  const Real Xr = static_cast<Real>(X), Yr = static_cast<Real>(Y), Zr = static_cast<Real>(Z);
  for (int kp = 0; kp < maxprim; ++kp) {
    const bool has = active && kp < np;
    if (has) {
      const double2 gp = a.X.prim[po + kp];
      const double gam = gp.x, pg = p + gam, alpha = p * gam / pg;
      double pref = kTwoPi52 / (p * gam * sqrt(pg)) * gp.y;
      for (int l = 0; l < LC; ++l) pref *= -0.5 / gam;
      // orders n = tl, tl + TS, ...: a team may have fewer lanes than L + 1
      const typename BoysAtT<Real>::type F(a.boys_mode, alpha * RPC2);
      for (int n = tl; n <= L; n += TS) {
        double f = pref;
        for (int k = 0; k < n; ++k) f *= -2.0 * alpha;
        Rn[n] = static_cast<Real>(f) * F(a.dt, n);
      }
    }
    team_sync<TS>(team);
    // Hermite R, level by level. The loops have compile-time trip counts and
    // are unrolled: the components of one level are independent, so their
    // descriptor and operand loads are issued back to back instead of one
    // dependent load chain per component.
    {
      Real* top = (L & 1) ? b1 : b0;
      if (has && tl == 0) top[0] = Rn[L];
      team_sync<TS>(team);
#pragma unroll
      for (int n = L - 1; n >= 0; --n) {
        Real* dst = (n & 1) ? b1 : b0;
        const Real* src = (n & 1) ? b0 : b1;
        const int cnt = ncum(L - n);
#pragma unroll
        for (int it = 0; it < (cnt + TS - 1) / TS; ++it) {
          const int idx = tl + it * TS;
          if (has && idx < cnt) {
            Real v;
            if (idx == 0) {
              v = Rn[n];
            } else {
              const int dsc = rdesc[idx];
              const int d = rdesc_d(dsc), c = rdesc_c(dsc);
              const Real xd = d == 0 ? Xr : (d == 1 ? Yr : Zr);
              v = xd * src[rdesc_s1(dsc)];
              if (c) v = fma(static_cast<Real>(c), src[rdesc_s2(dsc)], v);
            }
            dst[idx] = v;
          }
        }
        team_sync<TS>(team);
      }
    }
    // X rows: lanes over the Hermite components t of the bra, compile-time
    // solid-harmonic terms of the auxiliary shell (the first primitive stores)
#pragma unroll
    for (int it = 0; it < (NH + TS - 1) / TS; ++it) {
      const int t = tl + it * TS;
      if (has && t < NH) {
        const uchar4 e = txyz[t];
        if (kp == 0)
          sph_rows<LC, Real, false>(b0, e.x, e.y, e.z, xrow + t * mpad, std::make_integer_sequence<int, 2 * LC + 1>{});
        else
          sph_rows<LC, Real, true>(b0, e.x, e.y, e.z, xrow + t * mpad, std::make_integer_sequence<int, 2 * LC + 1>{});
      }
    }
    team_sync<TS>(team);
  }
}

// Screening estimate of triplet (unit slot us, auxiliary slot cs), unit Schwarz
// value uq, auxiliary center cc.xyz: schwarz_estimate Q_ab Q_c
// (common/screening.f90:301-313; cc.w = Q_c) or, with QVL screening,
// qvl_estimate (:267-299): Q_ab Q_c within the sum of the extents, beyond it
// Q_ab pi sqrt(2) beta_c / ((zeta_a + zeta_b)^(1/4) R^(L_c + 1)).
template <int LC>
__device__ __forceinline__ double triplet_estimate(const Df3cArgs& a, int us, int cs, double uq,
                                                   const double4& cc) {
  if (!a.qvl) return uq * cc.w;
  const double4 aq = a.aux_qvl[a.aux_slot0 + cs];   // (Q_c, extent, beta, 0)
  const double4 pq = a.slot_qvl[a.unit_slot0 + us];  // (contracted center, extent)
  const double dx = pq.x - cc.x, dy = pq.y - cc.y, dz = pq.z - cc.z;
  const double R = sqrt(dx * dx + dy * dy + dz * dz);
  if (R <= pq.w + aq.y) return uq * aq.x;
  double RL = R;
#pragma unroll
  for (int l = 0; l < LC; ++l) RL *= R;
  return uq * kPi * 1.4142135623730951 * aq.z / (a.slot_den[a.unit_slot0 + us] * RL);
}

// First unit slot i (class-relative, 0..n_units) with unit_Q[i] * q < bound:
// the unit Schwarz values are sorted in descending order, so the products are
// non-increasing. Evaluated alike by every thread (the same loads, in order).
__device__ __forceinline__ int first_unit_below(const Df3cArgs& a, double bound, double q) {
  int lo = 0, hi = a.n_units;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (a.unit_Q[a.unit_slot0 + mid] * q < bound)
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

// One work item: aux tile bx (TC shells), bra-unit chunk by, density chunk bz.
template <int LAB, int LC, int V>
__device__ __forceinline__ void df3c_item(const Df3cArgs& a, int bx, int by, int bz, double* smem) {
  using C = Cfg<LAB, LC, V>;
  double* Xs = smem;                               // [KP][MPAD]
  double* Gs = Xs + C::KP * C::MPAD;               // [KP][kGStride]
  double* misc = Gs + C::KP * kGStride;            // unit / aux parameters
  double* Rteam = misc + 1024;                     // team scratch
  double4* u_pP = reinterpret_cast<double4*>(misc);                   // [UB <= 64]
  double* u_Q = misc + 256;                                           // [UB]
  double4* c_C = reinterpret_cast<double4*>(misc + 320);              // [TC <= 128] (x, y, z, Q)
  int* c_info = reinterpret_cast<int*>(misc + 320 + 512);             // [TC] (nprim, prim_off)

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int c0 = bx * C::TC;
  const int tile_n = min(C::TC, a.n_aux - c0);
  const int z = bz;
  const int d0 = z * a.dw;
  const int ndc = min(a.dw, a.nd - d0);
  const int nt_rt = a.dw / 8;  // n-tiles of this launch (dw multiple of 8, <= 40)

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
  __syncthreads();
  int maxprim = 0;
  for (int i = 0; i < tile_n; ++i) maxprim = max(maxprim, c_info[2 * i]);
  const double qc_max = tile_n > 0 ? c_C[0].w : 0.0;
  const double thr = a.thresh;
  const IndexTables* it = a.dt.idx;
  // the units that can meet the tile form a prefix of the sorted class (the
  // staircase); the item takes chunk `by` of nby equal chunks of that prefix,
  // so every item of a tile has the same number of steps
  const int ue0 = first_unit_below(a, thr, qc_max);
  const int cs = (ue0 + a.nby - 1) / a.nby;
  const int ub = by * cs;
  const int ue = min(ue0, ub + cs);
  const int g = lane >> 2, t4 = lane & 3;
  // DMMA work of this warp: its first row tile and its k slice (warps past
  // MT * KSPLIT get slice KSPLIT, which has no k steps)
  const int mt0 = C::KSPLIT > 1 ? warp % C::MT : warp;
  const int ks = C::KSPLIT > 1 ? warp / C::MT : 0;

  double acc[C::MTW][5][2];
#pragma unroll
  for (int j = 0; j < C::MTW; ++j)
#pragma unroll
    for (int n = 0; n < 5; ++n) acc[j][n][0] = acc[j][n][1] = 0.0;

  // unit data of the next step, loaded one step ahead by threads tid < UB
  double nq = 0.0;
  double4 npP = make_double4(1.0, 0.0, 0.0, 0.0);
  if (tid < C::UB && ub + tid < ue) {
    nq = a.unit_Q[a.unit_slot0 + ub + tid];
    npP = a.slot_pP[a.unit_slot0 + ub + tid];
  }
  for (int u0 = ub; u0 < ue && tile_n > 0; u0 += C::UB) {
    // units of this step that can meet the tile: a prefix, units are sorted.
    // The unit data written here were last read by the previous step's X
    // build (before its closing barrier); the barrier of the count below
    // orders the previous step's product before this step's writes to Xs / Gs.
    bool valid = false;
    if (tid < C::UB) {
      valid = u0 + tid < ue && nq * qc_max >= thr;
      u_pP[tid] = valid ? npP : make_double4(1.0, 0.0, 0.0, 0.0);
      u_Q[tid] = valid ? nq : 0.0;
    }
    const int nvalid = __syncthreads_count(valid);
    if (nvalid == 0) break;  // sorted: nothing below survives
    if (tid < C::UB) {
      const int s = u0 + C::UB + tid;
      nq = 0.0;
      if (s < ue) {
        nq = a.unit_Q[a.unit_slot0 + s];
        npP = a.slot_pP[a.unit_slot0 + s];
      }
    }
    // 1. G of the valid units: rows k = ui * NH + t, dw doubles each (16-byte chunks)
    {
      const double* gsrc = a.G + (static_cast<long long>(z) * a.n_units + u0) * C::NH * a.dw;
      const int rows = nvalid * C::NH;
      const int chunks_per_row = a.dw / 2;
      for (int i = tid; i < rows * chunks_per_row; i += kThreads) {
        const int r = i / chunks_per_row, c = i - r * chunks_per_row;
        cp_async16(Gs + r * kGStride + 2 * c, gsrc + static_cast<long long>(r) * a.dw + 2 * c);
      }
      for (int i = tid; i < (C::KP - rows) * 40; i += kThreads) {
        const int r = rows + i / 40, c = i % 40;
        Gs[r * kGStride + c] = 0.0;
      }
      for (int i = tid; i < rows * (40 - a.dw); i += kThreads) {
        const int r = i / (40 - a.dw), c = a.dw + i % (40 - a.dw);
        Gs[r * kGStride + c] = 0.0;
      }
    }
    // (no zeroing pass over X: every triplet of a valid unit and auxiliary
    // shell writes its rows below -- values, or zeros when screened; rows of
    // invalid units meet zero G rows, and columns of shells past the tile end
    // feed accumulator rows that are not written out)
    __syncthreads();

    // 2. X
    if constexpr (C::kPerThread) {
      const int part = warp % C::TPT;
      for (int tr = lane + 32 * (warp / C::TPT); tr < C::NTRIP; tr += 32 * (kWarps / C::TPT)) {
        const int ui = tr / C::TC, ci = tr - ui * C::TC;
        if (ci >= tile_n || ui >= nvalid) continue;
        const double4 cc = c_C[ci];
        const double est = triplet_estimate<LC>(a, u0 + ui, c0 + ci, u_Q[ui], cc);
        double* xrow0 = Xs + (ui * C::NH) * C::MPAD + ci * C::NC;
        if (est < thr) {
          x_rows_zero<LAB, LC, C::TPT>(xrow0, C::MPAD, part);
          continue;
        }
        const double4 up = u_pP[ui];
        const double p = up.x;
        const double X = up.y - cc.x, Y = up.z - cc.y, Z = up.w - cc.z;
        const int np = c_info[2 * ci], po = c_info[2 * ci + 1];
        if (est < a.thr32)
          x_triplet_thread<LAB, LC, C::NR, C::MPAD, C::TPT, float>(a, p, X, Y, Z, np, po, xrow0, part);
        else
          x_triplet_thread<LAB, LC, C::NR, C::MPAD, C::TPT, double>(a, p, X, Y, Z, np, po, xrow0, part);
      }
    } else {
      // team index tables (shared memory copies of the decoded multi-indices)
      uchar4* txyz = reinterpret_cast<uchar4*>(Rteam + C::NTRIP * C::kTeamStride);
      int* rdesc = reinterpret_cast<int*>(txyz + C::NR);
      if (u0 == ub) {
        for (int i = tid; i < C::NR; i += kThreads) {
          txyz[i] = *reinterpret_cast<const uchar4*>(it->xyz[i]);
          rdesc[i] = a.dt.rdesc[i];
        }
        __syncthreads();
      }
      const int team = tid / C::TS, tl = tid - team * C::TS;
      const bool in_team = team < C::NTRIP;
      const int ui = in_team ? team / C::TC : 0, ci = in_team ? team - ui * C::TC : 0;
      double* rbuf = Rteam + (in_team ? team : 0) * C::kTeamStride;
      const double4 cc = c_C[ci];
      const bool valid = in_team && ci < tile_n && ui < nvalid;
      const double est = valid ? triplet_estimate<LC>(a, u0 + ui, c0 + ci, u_Q[ui], cc) : 0.0;
      const bool active = valid && est >= thr;
      const double4 up = u_pP[ui];
      const double X = up.y - cc.x, Y = up.z - cc.y, Z = up.w - cc.z;
      const int np = active ? c_info[2 * ci] : 0, po = c_info[2 * ci + 1];
      double* xrow = Xs + (ui * C::NH) * C::MPAD + ci * C::NC;
      if (valid && !active)  // screened: its X rows are zero
        for (int t = tl; t < C::NH; t += C::TS)
#pragma unroll
          for (int m = 0; m < C::NC; ++m) xrow[t * C::MPAD + m] = 0.0;
      // FP32 recurrences only when every active team of the warp has a weak
      // triplet (a team larger than a warp has one triplet: uniform over it)
      const bool weak = !active || est < a.thr32;
      const bool f32 = __all_sync(0xffffffffu, weak) && __any_sync(0xffffffffu, active);
      if (f32)
        x_triplet_team<LAB, LC, C::TS, float>(a, txyz, rdesc, rbuf, team, tl, active, np, po, maxprim, up.x, X, Y,
                                              Z, xrow, C::MPAD);
      else
        x_triplet_team<LAB, LC, C::TS, double>(a, txyz, rdesc, rbuf, team, tl, active, np, po, maxprim, up.x, X,
                                               Y, Z, xrow, C::MPAD);
    }
    cp_async_commit_wait_all();
    __syncthreads();

    // 3. acc[aux fn][d] += X^T G on the FP64 tensor cores (warp w: row tiles
    //    w, w + 8, ...; with KSPLIT > 1 row tile w % MT, k steps w / MT + KSPLIT j)
#pragma unroll 2
    for (int k4 = ks < C::KSPLIT ? ks : C::KP / 4; k4 < C::KP / 4; k4 += C::KSPLIT) {
      const int kr = 4 * k4 + t4;
      double bf[5];
#pragma unroll
      for (int n = 0; n < 5; ++n) bf[n] = n < nt_rt ? Gs[kr * kGStride + 8 * n + g] : 0.0;
#pragma unroll
      for (int j = 0; j < C::MTW; ++j) {
        const int mt = mt0 + kWarps * j;
        if (mt < C::MT) {
          const double av = Xs[kr * C::MPAD + 8 * mt + g];
#pragma unroll
          for (int n = 0; n < 5; ++n)
            if (n < nt_rt) dmma_m8n8k4(acc[j][n][0], acc[j][n][1], av, bf[n]);
        }
      }
    }
  }

  if constexpr (C::KSPLIT > 1) {
    // sum the k slices of each row tile in a fixed order (slice 0 first),
    // through the X and G tiles (contiguous; free once every warp is past its
    // last product, and rewritten before they are read again)
    __syncthreads();
    if (ks < C::KSPLIT) {
      double* red = Xs + (ks * C::MT + mt0) * 320;
#pragma unroll
      for (int n = 0; n < 5; ++n)
#pragma unroll
        for (int i = 0; i < 2; ++i) red[(2 * n + i) * 32 + lane] = acc[0][n][i];
    }
    __syncthreads();
    if (ks == 0) {
#pragma unroll
      for (int n = 0; n < 5; ++n)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          double v = Xs[mt0 * 320 + (2 * n + i) * 32 + lane];
          for (int q = 1; q < C::KSPLIT; ++q) v += Xs[(q * C::MT + mt0) * 320 + (2 * n + i) * 32 + lane];
          acc[0][n][i] = v;
        }
    }
  }
  // partial[y][fn][d] (with KSPLIT > 1 only the warps of slice 0 hold sums)
  double* out = a.partial + static_cast<long long>(by) * a.n_aux * C::NC * a.nd;
#pragma unroll
  for (int j = 0; j < C::MTW; ++j) {
    const int mt = (ks == 0 ? mt0 : C::MT) + kWarps * j;
    const int row = 8 * mt + g;
    if (mt >= C::MT || row >= C::M || row / C::NC >= tile_n) continue;
    const long long fn = static_cast<long long>(c0) * C::NC + row;
#pragma unroll
    for (int n = 0; n < 5; ++n)
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        const int col = 8 * n + 2 * t4 + i;
        if (n < nt_rt && col < ndc) out[fn * a.nd + d0 + col] = acc[j][n][i];
      }
  }
}

// Persistent blocks: each pulls work items from the class's counter, heaviest
// first (items are numbered with the bra-unit chunk slowest; units and aux
// shells are sorted by Schwarz value, so early chunks and tiles carry the most
// surviving triplets).
// The X tile starts zeroed: entries that no step writes (padding rows and
// columns) must be finite.
template <int LAB, int LC, int V>
__device__ __forceinline__ void zero_x_tile(double* smem) {
  using C = Cfg<LAB, LC, V>;
  for (int i = threadIdx.x; i < C::KP * C::MPAD; i += blockDim.x) smem[i] = 0.0;
}

template <int LAB, int LC, int V>
__global__ void __launch_bounds__(kThreads, (Cfg<LAB, LC, V>::kMinBlocks)) k_df3c(Df3cArgs a) {
  extern __shared__ __align__(16) double smem[];
  __shared__ int s_item;
  zero_x_tile<LAB, LC, V>(smem);
  for (;;) {
    __syncthreads();  // the previous item is done with shared memory and s_item
    if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= a.n_items) return;
    const int bz = item % a.nbz;
    const int r = item / a.nbz;
    df3c_item<LAB, LC, V>(a, r % a.nbx, r / a.nbx, bz, smem);
  }
}

// Batched form: the work items of one class for many molecules in one
// persistent launch. Molecule m owns items [item_off[m], item_off[m + 1]) and
// its own descriptor args[m]; molecules are ordered by decreasing work, and a
// molecule's items heavy-first, so the queue drains with light items last.
template <int LAB, int LC, int V>
__global__ void __launch_bounds__(kThreads, (Cfg<LAB, LC, V>::kMinBlocks)) k_df3c_batch(const Df3cArgs* __restrict__ args,
                                                            const int* __restrict__ item_off, int nm,
                                                            int* counter) {
  extern __shared__ __align__(16) double smem[];
  __shared__ int s_item, s_m;
  __shared__ __align__(16) unsigned char s_raw[sizeof(Df3cArgs)];
  const Df3cArgs& sa = *reinterpret_cast<const Df3cArgs*>(s_raw);
  const int total = item_off[nm];
  zero_x_tile<LAB, LC, V>(smem);
  for (;;) {
    __syncthreads();  // the previous item is done with shared memory and the descriptor
    if (threadIdx.x == 0) {
      const int item = atomicAdd(counter, 1);
      int m = 0;
      if (item < total) {
        int lo = 0, hi = nm - 1;  // last m with item_off[m] <= item
        while (lo < hi) {
          const int mid = (lo + hi + 1) / 2;
          if (item_off[mid] <= item)
            lo = mid;
          else
            hi = mid - 1;
        }
        m = lo;
      }
      s_item = item;
      s_m = m;
    }
    __syncthreads();
    const int item = s_item;
    if (item >= total) return;
    const int m = s_m;
    static_assert(sizeof(Df3cArgs) % 4 == 0, "descriptor copied in 32-bit words");
    const unsigned* src = reinterpret_cast<const unsigned*>(args + m);
    unsigned* dst = reinterpret_cast<unsigned*>(s_raw);
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(Df3cArgs) / 4); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    const int local = item - item_off[m];
    const int bz = local % sa.nbz;
    const int r = local / sa.nbz;
    df3c_item<LAB, LC, V>(sa, r % sa.nbx, r / sa.nbx, bz, smem);
  }
}

// Resident blocks of a kernel on the current device (cached per device and
// kernel), after raising its dynamic shared-memory limit to smem.
template <class K>
int resident_blocks(K kernel, size_t smem, int* occ_cache) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (occ_cache[dev] == 0) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    int o = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, kernel, kThreads, smem);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    occ_cache[dev] = (o > 0 ? o : 1) * sms;
  }
  return occ_cache[dev];
}

template <int LAB, int LC, int V>
void fill_items(Df3cArgs* a, int ny) {
  using C = Cfg<LAB, LC, V>;
  a->nbx = (a->n_aux + C::TC - 1) / C::TC;
  a->nby = ny;
  a->nbz = (a->nd + a->dw - 1) / a->dw;
  a->n_items = a->nbx * a->nby * a->nbz;
}

template <int LAB, int LC, int V>
int launch_class(const Df3cArgs& a, int ny, cudaStream_t s) {
  using C = Cfg<LAB, LC, V>;
  const size_t smem = sizeof(double) * C::SMEM;
  static int occ[64] = {};
  const int resident = resident_blocks(k_df3c<LAB, LC, V>, smem, occ);
  Df3cArgs b = a;
  fill_items<LAB, LC, V>(&b, ny);
  if (b.n_items == 0) return 0;
  k_df3c<LAB, LC, V><<<df3c_grid(b.n_items, resident), kThreads, smem, s>>>(b);
  return 1;
}

template <int LAB, int LC, int V>
int launch_class_batch(const Df3cArgs* d_args, const int* d_item_off, int nm, int total_items,
                       int* counter, cudaStream_t s) {
  using C = Cfg<LAB, LC, V>;
  const size_t smem = sizeof(double) * C::SMEM;
  static int occ[64] = {};
  const int resident = resident_blocks(k_df3c_batch<LAB, LC, V>, smem, occ);
  if (total_items <= 0 || nm <= 0) return 0;
  k_df3c_batch<LAB, LC, V><<<df3c_grid(total_items, resident), kThreads, smem, s>>>(d_args, d_item_off, nm,
                                                                                     counter);
  return 1;
}

template <int LAB, int LC, int V>
void class_info(Df3cClassInfo* ci) {
  using C = Cfg<LAB, LC, V>;
  ci->tc = C::TC;
  ci->ub = C::UB;
  ci->ndc = 40;
  ci->lanes = C::kPerThread ? C::TPT : C::TS;
  ci->blocks_per_sm = C::kMinBlocks;
  ci->smem = sizeof(double) * C::SMEM;
}

// The dispatch row of one LAB: every LC and variant (variants with the shape
// of a lower one share its instantiation).
template <int LAB, int LC, int V>
constexpr int canonical_variant() {
  using A = Cfg<LAB, LC, V>;
  if constexpr (V == 0) {
    return 0;
  } else {
    using B = Cfg<LAB, LC, V - 1>;
    constexpr int prev = canonical_variant<LAB, LC, V - 1>();
    if constexpr (A::TC == B::TC && A::UB == B::UB && A::kMinBlocks == B::kMinBlocks) return prev;
    if constexpr (V >= 2) {
      using Z = Cfg<LAB, LC, 0>;
      if constexpr (A::TC == Z::TC && A::UB == Z::UB && A::kMinBlocks == Z::kMinBlocks) return 0;
    }
    return V;
  }
}

template <int LAB, int LC, int V>
void fill_entry(Df3cRow* row) {
  constexpr int W = canonical_variant<LAB, LC, V>();
  row->launch[V][LC] = &launch_class<LAB, LC, W>;
  row->info[V][LC] = &class_info<LAB, LC, W>;
  row->fill[V][LC] = &fill_items<LAB, LC, W>;
  row->batch[V][LC] = &launch_class_batch<LAB, LC, W>;
  if constexpr (V + 1 < kDf3cVariants) fill_entry<LAB, LC, V + 1>(row);
}

template <int LAB, int LC>
void fill_row(Df3cRow* row) {
  fill_entry<LAB, LC, 0>(row);
  if constexpr (LC < PA_LAUXMAX) fill_row<LAB, LC + 1>(row);
}

cudaError_t upload_rownorm(const double* rownorm, cudaStream_t s) {
  return cudaMemcpyToSymbolAsync(c_sph_rownorm, rownorm, sizeof(double) * (PA_LAUXMAX + 1) * (PA_LAUXMAX + 1), 0,
                                 cudaMemcpyHostToDevice, s);
}

}  // namespace

}  // namespace pa

#include "k_df3c_w.cuh"

// Defines df3c_row_<LAB>(): the dispatch row of this translation unit's LAB.
#define PA_DF3C_ROW(LAB)                       \
  namespace pa {                               \
  void df3c_row_##LAB(Df3cRow* row) {          \
    fill_row<LAB, 0>(row);                     \
    fill_row_w<LAB, 0>(row);                   \
    row->upload_rownorm = &upload_rownorm;     \
  }                                            \
  }
