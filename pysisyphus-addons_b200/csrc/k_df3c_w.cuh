// Weak-triplet three-center kernels of the precision form (included by
// k_df3c_impl.cuh, inside its namespace).
//
// In the mixed form every class (LAB, LC) runs twice: the FP64 kernel k_df3c
// takes the triplets whose Schwarz bound Q_ab Q_c is at least thr32 (its
// screening threshold raised to thr32), and k_df3c_w takes the weak ones,
// thresh <= Q_ab Q_c < thr32. For those:
//   * X is built in FP32 (Boys values, Hermite recurrence, solid harmonics;
//     the Boys function keeps its FP64 branches for large arguments) and
//     written as three BF16 slices into the K-major A operand (umma.cuh):
//     row = auxiliary function of the tile, k = (unit, Hermite component t)
//     with every unit padded to NHP = round_up(NH, 8) components;
//   * the density-folded bra G (FP64, from k_bra_prep) is split into three
//     BF16 slices while it is staged into the K-major B operand (row =
//     density);
//   * the product runs on the tensor cores (tcgen05.mma kind::f16, six slice
//     products, FP32 accumulator in tensor memory), issued by one thread per
//     step, and every step's accumulator is drained into FP64 registers, so FP32
//     accumulation spans one step (at most a few hundred k) only.
// Work items are (auxiliary tile, chunk, density chunk) as in k_df3c, but the
// chunks divide the tile's weak region of the sorted units (found by binary
// search) rather than all units; strong and screened triplets inside a step
// write zero X entries. The partial slabs are those of k_df3c.
#pragma once

namespace pa {

namespace {

template <int LAB, int LC>
struct CfgW {
  static constexpr int NH = ncum(LAB);
  static constexpr int NHP = round_up(NH, 8);
  static constexpr int NC = 2 * LC + 1;
  static constexpr int L = LAB + LC;
  static constexpr int NR = ncum(L);
  static constexpr bool kPerThread = (L <= 5);
  static constexpr int kN = 48;            // MMA N; the B operand has dw <= 40 real rows
  static constexpr int kPadA = 2048;       // virtual A rows (M = 128) past the last k column
  static constexpr int kPadB = 1024;       // virtual B rows (N = 48)
  static constexpr int kMiscBytes = 8192;  // unit and auxiliary parameters of the item
  static constexpr int kTeamBase = 2 * NR + 16;  // floats per team: Rn, two level buffers
  static constexpr int pick_ub(int tc) {
    int ub = 1;
    if (kPerThread) {
      ub = 64 / NHP;
      if (ub < 1) ub = 1;
      if (ub * tc > 512) ub = 512 / tc;
    } else {
      ub = 48 / NHP;
      if (ub < 1) ub = 1;
      if (ub * tc > 64) ub = 64 / tc;
    }
    return ub < 1 ? 1 : ub;
  }
  static constexpr int k_for(int tc) { return round_up(pick_ub(tc) * NHP, 16); }
  static constexpr int ar_for(int tc) { return round_up(tc * NC, 8); }
  static constexpr int zero_bytes(int tc) {
    return 3 * k_for(tc) * ar_for(tc) * 2 + kPadA + 3 * k_for(tc) * 40 * 2 + kPadB;
  }
  static constexpr int smem_for(int tc) {
    const int team = kPerThread ? 0 : pick_ub(tc) * tc * kTeamBase * 4 + NR * 8;
    return zero_bytes(tc) + kMiscBytes + team;
  }
  static constexpr int kBudget = 110 * 1024;
  static constexpr int pick_tc() {
    int tc = 128 / NC;
    if (!kPerThread && tc > 32) tc = 32;
    while (tc > 1 && smem_for(tc) > kBudget) --tc;
    return tc;
  }
  static constexpr int TC = pick_tc();
  static constexpr int UB = pick_ub(TC);
  static constexpr int K = k_for(TC);
  static constexpr int AR = ar_for(TC);
  static constexpr int NTRIP = UB * TC;
  static constexpr int ZERO = zero_bytes(TC);
  static constexpr int width_for() {
    int t = 1;
    if (kPerThread) {
      while (t < 8 && 2 * t * NTRIP <= kThreads) t *= 2;
    } else {
      while (t < kThreads && 2 * t * NTRIP <= kThreads) t *= 2;
    }
    return t;
  }
  static constexpr int TPT = kPerThread ? width_for() : 1;
  static constexpr int TS = kPerThread ? 1 : width_for();
  // team scratch stride (floats): the teams of a warp address their
  // components at the same offsets, so a stride of TS (mod 32) floats puts
  // their TS-wide chunks in different banks (when it fits the budget)
  static constexpr int kPadWanted = (!kPerThread && TS <= 16) ? (TS - kTeamBase % 32 + 32) % 32 : 0;
  static constexpr int kPad = smem_for(TC) + NTRIP * kPadWanted * 4 <= kBudget ? kPadWanted : 0;
  static constexpr int kTeamStride = kTeamBase + kPad;
  static constexpr int SMEM = smem_for(TC) + (kPerThread ? 0 : NTRIP * kPad * 4);
  static_assert(TS <= 32 || TS % 32 == 0, "multi-warp teams are whole warps");
  static_assert(TS <= 32 || kThreads / TS < 16, "named barrier ids 1..15");
  static_assert(K % 16 == 0 && AR <= 128 && TC * NC <= 128, "one MMA of M = 128 per k step");
  static_assert(SMEM <= 113 * 1024, "two blocks per SM");
  static_assert(ZERO % 16 == 0, "zeroed in 16-byte words");
};

// A operand of a step: three BF16 slices, element (m, k) at kmajor_off.
struct ASink {
  unsigned char* a0;
  uint32_t slice;
  int rows;
  __device__ __forceinline__ void put(int m, int k, float v) const {
    __nv_bfloat16 s0, s1, s2;
    umma::split3(v, s0, s1, s2);
    unsigned char* p = a0 + umma::kmajor_off(m, k, rows);
    *reinterpret_cast<__nv_bfloat16*>(p) = s0;
    *reinterpret_cast<__nv_bfloat16*>(p + slice) = s1;
    *reinterpret_cast<__nv_bfloat16*>(p + 2 * slice) = s2;
  }
  __device__ __forceinline__ float get(int m, int k) const {
    const unsigned char* p = a0 + umma::kmajor_off(m, k, rows);
    return __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(p)) +
           (__bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(p + slice)) +
            __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(p + 2 * slice)));
  }
  __device__ __forceinline__ void zero(int m, int k) const {
    unsigned char* p = a0 + umma::kmajor_off(m, k, rows);
    const __nv_bfloat16 z = __float2bfloat16_rn(0.f);
    *reinterpret_cast<__nv_bfloat16*>(p) = z;
    *reinterpret_cast<__nv_bfloat16*>(p + slice) = z;
    *reinterpret_cast<__nv_bfloat16*>(p + 2 * slice) = z;
  }
};

// X entry (m0 + M, k) = N_lc,M sum_tau S_lc,M[tau] R[t + tau] in FP32 (the first
// auxiliary primitive stores, later ones add).
template <int LC, int M, bool ACC>
__device__ __forceinline__ void sph_put_w(const float* R, int tx, int ty, int tz, const ASink& s, int m0, int k) {
  float v = static_cast<float>(c_sph_rownorm[LC * LC + M]) *
            sph_row<LC, M, float>(R, tx, ty, tz, std::make_integer_sequence<int, ncart(LC)>{});
  if constexpr (ACC) v += s.get(m0 + M, k);
  s.put(m0 + M, k, v);
}
template <int LC, bool ACC, int... Ms>
__device__ __forceinline__ void sph_rows_w(const float* R, int tx, int ty, int tz, const ASink& s, int m0, int k,
                                           std::integer_sequence<int, Ms...>) {
  (sph_put_w<LC, Ms, ACC>(R, tx, ty, tz, s, m0, k), ...);
}

// Rows t % TPT == part of one triplet (per-thread mode).
template <int LAB, int LC, int TPT, bool ACC>
__device__ __forceinline__ void x_rows_thread_w(const float* R, const ASink& s, int m0, int k0, int part) {
#pragma unroll
  for (int tl = 0; tl <= LAB; ++tl)
#pragma unroll
    for (int tx = tl; tx >= 0; --tx)
#pragma unroll
      for (int ty = tl - tx; ty >= 0; --ty) {
        const int tz = tl - tx - ty;
        const int th = cidx(tx, ty, tz);
        if (th % TPT != part) continue;
        sph_rows_w<LC, ACC>(R, tx, ty, tz, s, m0, k0 + th, std::make_integer_sequence<int, 2 * LC + 1>{});
      }
}

template <int LAB, int LC, int TPT>
__device__ __forceinline__ void x_rows_zero_w(const ASink& s, int m0, int k0, int part) {
  for (int th = part; th < ncum(LAB); th += TPT)
#pragma unroll
    for (int m = 0; m < 2 * LC + 1; ++m) s.zero(m0 + m, k0 + th);
}

// X of one weak triplet by one thread (L <= 5), FP32 throughout.
template <int LAB, int LC, int NR, int TPT>
__device__ __forceinline__ void x_triplet_thread_w(const Df3cArgs& a, double p, double X, double Y, double Z, int np,
                                                   int po, const ASink& s, int m0, int k0, int part) {
  constexpr int L = LAB + LC;
  const double RPC2 = X * X + Y * Y + Z * Z;
  for (int kp = 0; kp < np; ++kp) {
    const double2 gp = a.X.prim[po + kp];
    const double gam = gp.x, pg = p + gam, alpha = p * gam / pg;
    double pref = kTwoPi52 / (p * gam * sqrt(pg)) * gp.y;
#pragma unroll
    for (int l = 0; l < LC; ++l) pref *= -0.5 / gam;
    float F[L + 1];
    boys_all(a.dt, a.boys_mode, L, alpha * RPC2, F);
    float Rn[L + 1];
    double f = pref;
#pragma unroll
    for (int n = 0; n <= L; ++n) {
      Rn[n] = static_cast<float>(f) * F[n];
      f *= -2.0 * alpha;
    }
    float R[NR];
    hermite_R_thread<L, float>(Rn, static_cast<float>(X), static_cast<float>(Y), static_cast<float>(Z), R);
    if (kp == 0)
      x_rows_thread_w<LAB, LC, TPT, false>(R, s, m0, k0, part);
    else
      x_rows_thread_w<LAB, LC, TPT, true>(R, s, m0, k0, part);
  }
}

// X of one weak triplet by a team of TS threads (L > 5), FP32 throughout; the
// same level-by-level recurrence as x_triplet_team.
template <int LAB, int LC, int TS>
__device__ __forceinline__ void x_triplet_team_w(const Df3cArgs& a, const uchar4* txyz, const int* rdesc, float* rbuf,
                                                 int team, int tl, bool active, int np, int po, int maxprim, double p,
                                                 double X, double Y, double Z, const ASink& s, int m0, int k0) {
  constexpr int L = LAB + LC;
  constexpr int NR = ncum(L);
  constexpr int NH = ncum(LAB);
  float* Rn = rbuf;
  float* b0 = Rn + 16;
  float* b1 = b0 + NR;
  const double RPC2 = X * X + Y * Y + Z * Z;
  const float Xr = static_cast<float>(X), Yr = static_cast<float>(Y), Zr = static_cast<float>(Z);
  for (int kp = 0; kp < maxprim; ++kp) {
    const bool has = active && kp < np;
    if (has) {
      const double2 gp = a.X.prim[po + kp];
      const double gam = gp.x, pg = p + gam, alpha = p * gam / pg;
      double pref = kTwoPi52 / (p * gam * sqrt(pg)) * gp.y;
      for (int l = 0; l < LC; ++l) pref *= -0.5 / gam;
      const BoysAtF F(a.boys_mode, alpha * RPC2);
      for (int n = tl; n <= L; n += TS) {
        double f = pref;
        for (int k = 0; k < n; ++k) f *= -2.0 * alpha;
        Rn[n] = static_cast<float>(f) * F(a.dt, n);
      }
    }
    team_sync<TS>(team);
    {
      float* top = (L & 1) ? b1 : b0;
      if (has && tl == 0) top[0] = Rn[L];
      team_sync<TS>(team);
#pragma unroll
      for (int n = L - 1; n >= 0; --n) {
        float* dst = (n & 1) ? b1 : b0;
        const float* src = (n & 1) ? b0 : b1;
        const int cnt = ncum(L - n);
#pragma unroll
        for (int it = 0; it < (cnt + TS - 1) / TS; ++it) {
          const int idx = tl + it * TS;
          if (has && idx < cnt) {
            float v;
            if (idx == 0) {
              v = Rn[n];
            } else {
              const int dsc = rdesc[idx];
              const int d = rdesc_d(dsc), c = rdesc_c(dsc);
              const float xd = d == 0 ? Xr : (d == 1 ? Yr : Zr);
              v = xd * src[rdesc_s1(dsc)];
              if (c) v = fmaf(static_cast<float>(c), src[rdesc_s2(dsc)], v);
            }
            dst[idx] = v;
          }
        }
        team_sync<TS>(team);
      }
    }
#pragma unroll
    for (int it = 0; it < (NH + TS - 1) / TS; ++it) {
      const int t = tl + it * TS;
      if (has && t < NH) {
        const uchar4 e = txyz[t];
        if (kp == 0)
          sph_rows_w<LC, false>(b0, e.x, e.y, e.z, s, m0, k0 + t, std::make_integer_sequence<int, 2 * LC + 1>{});
        else
          sph_rows_w<LC, true>(b0, e.x, e.y, e.z, s, m0, k0 + t, std::make_integer_sequence<int, 2 * LC + 1>{});
      }
    }
    team_sync<TS>(team);
  }
}

// One work item of the weak kernel (same item decomposition as df3c_item).
// Returns false when a tensor-core completion wait gave up (uniform over the
// block).
template <int LAB, int LC>
__device__ __forceinline__ bool df3c_item_w(const Df3cArgs& a, int bx, int by, int bz, unsigned char* smem,
                                            uint32_t tmem, uint64_t* bar, uint32_t& phase) {
  using C = CfgW<LAB, LC>;
  unsigned char* a0 = smem;
  const uint32_t a_slice = static_cast<uint32_t>(C::K * C::AR * 2);
  unsigned char* b0 = a0 + 3 * a_slice + C::kPadA;
  unsigned char* mb = b0 + 3 * C::K * 40 * 2 + C::kPadB;
  double* misc = reinterpret_cast<double*>(mb);
  float* Rteam = reinterpret_cast<float*>(mb + C::kMiscBytes);
  double4* u_pP = reinterpret_cast<double4*>(misc);              // [UB <= 64]
  double* u_Q = misc + 256;                                      // [UB]
  double4* c_C = reinterpret_cast<double4*>(misc + 320);         // [TC <= 128] (x, y, z, Q)
  int* c_info = reinterpret_cast<int*>(misc + 320 + 512);        // [TC] (nprim, prim_off)
  const ASink sink{a0, a_slice, C::AR};

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int c0 = bx * C::TC;
  const int tile_n = min(C::TC, a.n_aux - c0);
  const int z = bz;
  const int dw = a.dw;
  const int d0 = z * dw;
  const int ndc = min(dw, a.nd - d0);
  const uint32_t b_slice = static_cast<uint32_t>(C::K * dw * 2);
  const double* Gz = a.G + static_cast<long long>(z) * a.n_units * C::NH * dw;

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
  // team index tables (shared-memory copies of the decoded multi-indices),
  // loaded before the first step (steps may be skipped)
  uchar4* txyz = reinterpret_cast<uchar4*>(Rteam + C::NTRIP * C::kTeamStride);
  int* rdesc = reinterpret_cast<int*>(txyz + C::NR);
  if constexpr (!C::kPerThread) {
    const IndexTables* it = a.dt.idx;
    for (int i = tid; i < C::NR; i += kThreads) {
      txyz[i] = *reinterpret_cast<const uchar4*>(it->xyz[i]);
      rdesc[i] = a.dt.rdesc[i];
    }
  }
  __syncthreads();
  int maxprim = 0;
  for (int i = 0; i < tile_n; ++i) maxprim = max(maxprim, c_info[2 * i]);
  const double qc_max = tile_n > 0 ? c_C[0].w : 0.0;
  const double qc_min = tile_n > 0 ? c_C[tile_n - 1].w : 0.0;
  const double thr = a.thresh, thr32 = a.thr32;
  // The tile's weak region of the sorted units: from the first unit that has a
  // weak triplet with the tile's smallest auxiliary shell (with QVL estimates,
  // which are not products, from the first unit) to the end of the staircase.
  // The item takes chunk `by` of nby equal chunks of it.
  const int ub0 = a.qvl ? 0 : first_unit_below(a, thr32, qc_min);
  const int ue0 = first_unit_below(a, thr, qc_max);
  const int cs = ue0 > ub0 ? (ue0 - ub0 + a.nby - 1) / a.nby : 0;
  const int ub = ub0 + by * cs;
  const int ue = min(ue0, ub + cs);

  double acc[24];
#pragma unroll
  for (int j = 0; j < 24; ++j) acc[j] = 0.0;
  bool ok = true;

  double nq = 0.0;
  double4 npP = make_double4(1.0, 0.0, 0.0, 0.0);
  if (tid < C::UB && ub + tid < ue) {
    nq = a.unit_Q[a.unit_slot0 + ub + tid];
    npP = a.slot_pP[a.unit_slot0 + ub + tid];
  }
  for (int u0 = ub; u0 < ue && tile_n > 0; u0 += C::UB) {
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
    // 1. BF16 slices of G of the valid units, split from the FP64 folded bra
    //    G[z][slot][t][n]: a warp takes 8 components t (fastest) of 4 densities,
    //    so its loads are 8 rows x 32 bytes and its stores 64 contiguous bytes
    //    of the K-major operand; components NH..NHP-1 of a unit are zero
    {
      const int per_unit = dw * C::NHP;
      for (int i = tid; i < nvalid * per_unit; i += kThreads) {
        const int ui = i / per_unit, r = i - ui * per_unit;
        const int t8 = r / (8 * dw), r2 = r - t8 * 8 * dw;
        const int n = r2 >> 3, t = 8 * t8 + (r2 & 7);
        const double v = t < C::NH ? Gz[(static_cast<long long>(u0 + ui) * C::NH + t) * dw + n] : 0.0;
        __nv_bfloat16 s0, s1, s2;
        umma::split3(v, s0, s1, s2);
        unsigned char* p = b0 + umma::kmajor_off(n, ui * C::NHP + t, dw);
        *reinterpret_cast<__nv_bfloat16*>(p) = s0;
        *reinterpret_cast<__nv_bfloat16*>(p + b_slice) = s1;
        *reinterpret_cast<__nv_bfloat16*>(p + 2 * b_slice) = s2;
      }
      // k columns past the valid units are zero
      const int kc0 = nvalid * C::NHP / 8, ncol = C::K / 8 - kc0;
      for (int i = tid; i < 3 * ncol * dw; i += kThreads) {
        const int j = i / (ncol * dw);
        const int r = i - j * ncol * dw;
        const int kc = kc0 + r / dw, n = r - (r / dw) * dw;
        *reinterpret_cast<uint4*>(b0 + j * b_slice + kc * dw * 16 + n * 16) = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    // 2. X (FP32) of the weak triplets; strong and screened ones write zeros
    if constexpr (C::kPerThread) {
      const int part = warp % C::TPT;
      for (int tr = lane + 32 * (warp / C::TPT); tr < C::NTRIP; tr += 32 * (kWarps / C::TPT)) {
        const int ui = tr / C::TC, ci = tr - ui * C::TC;
        if (ci >= tile_n || ui >= nvalid) continue;
        const double4 cc = c_C[ci];
        const double est = triplet_estimate<LC>(a, u0 + ui, c0 + ci, u_Q[ui], cc);
        const int m0 = ci * C::NC, k0 = ui * C::NHP;
        if (est < thr || est >= thr32) {
          x_rows_zero_w<LAB, LC, C::TPT>(sink, m0, k0, part);
          continue;
        }
        const double4 up = u_pP[ui];
        const int np = c_info[2 * ci], po = c_info[2 * ci + 1];
        x_triplet_thread_w<LAB, LC, C::NR, C::TPT>(a, up.x, up.y - cc.x, up.z - cc.y, up.w - cc.z, np, po, sink, m0,
                                                   k0, part);
      }
    } else {
      const int team = tid / C::TS, tl = tid - team * C::TS;
      const bool in_team = team < C::NTRIP;
      const int ui = in_team ? team / C::TC : 0, ci = in_team ? team - ui * C::TC : 0;
      float* rbuf = Rteam + (in_team ? team : 0) * C::kTeamStride;
      const double4 cc = c_C[ci];
      const bool valid_t = in_team && ci < tile_n && ui < nvalid;
      const double est = valid_t ? triplet_estimate<LC>(a, u0 + ui, c0 + ci, u_Q[ui], cc) : 0.0;
      const bool active = valid_t && est >= thr && est < thr32;
      const double4 up = u_pP[ui];
      const int np = active ? c_info[2 * ci] : 0, po = c_info[2 * ci + 1];
      const int m0 = ci * C::NC, k0 = ui * C::NHP;
      if (valid_t && !active)
        for (int t = tl; t < C::NH; t += C::TS)
#pragma unroll
          for (int m = 0; m < C::NC; ++m) sink.zero(m0 + m, k0 + t);
      x_triplet_team_w<LAB, LC, C::TS>(a, txyz, rdesc, rbuf, team, tl, active, np, po, maxprim, up.x, up.y - cc.x,
                                       up.z - cc.y, up.w - cc.z, sink, m0, k0);
    }
    umma::fence_async_smem();
    __syncthreads();
    // 3. acc[aux fn][d] += X^T G on the tensor cores, then into FP64
    if (tid == 0) {
      umma::fence_after();
      umma::issue_split_product(tmem, umma::smem_addr(a0), a_slice, C::AR, umma::smem_addr(b0), b_slice, dw, C::K,
                                umma::idesc_bf16(128, C::kN));
      umma::commit(umma::smem_addr(bar));
    }
    const bool done = umma::mbar_wait(bar, phase);
    phase ^= 1u;
    if (!__syncthreads_and(done)) {
      ok = false;
      break;
    }
    umma::fence_after();
    {
      const int q = warp & 3, h = warp >> 2;
      float v[24];
#pragma unroll
      for (int j = 0; j < 3; ++j)
        umma::tmem_ld8(tmem + (static_cast<uint32_t>(32 * q) << 16) + static_cast<uint32_t>(24 * h + 8 * j), v + 8 * j);
      umma::tmem_wait_ld();
#pragma unroll
      for (int j = 0; j < 24; ++j) acc[j] += static_cast<double>(v[j]);
    }
    umma::fence_before();
  }
  // partial[y][fn][d]: every item writes its whole block (zeros when no step ran)
  {
    double* out = a.partial + static_cast<long long>(by) * a.n_aux * C::NC * a.nd;
    const int q = warp & 3, h = warp >> 2;
    const int row = 32 * q + lane;
    if (row < tile_n * C::NC) {
      const long long fn = static_cast<long long>(c0) * C::NC + row;
#pragma unroll
      for (int j = 0; j < 24; ++j) {
        const int col = 24 * h + j;
        if (col < ndc) out[fn * a.nd + d0 + col] = acc[j];
      }
    }
  }
  return ok;
}

// Zeroes the operand buffers (virtual rows and padding read finite values),
// initializes the completion barrier and allocates the accumulator (64 TMEM
// columns; with at most eight blocks per SM every allocation succeeds at once).
template <int LAB, int LC>
__device__ __forceinline__ uint32_t weak_setup(unsigned char* smem, uint32_t* s_tmem, uint64_t* s_bar) {
  using C = CfgW<LAB, LC>;
  for (int i = threadIdx.x; i < C::ZERO / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(smem)[i] = make_uint4(0u, 0u, 0u, 0u);
  if (threadIdx.x == 0) umma::mbar_init(s_bar, 1);
  if (threadIdx.x < 32) umma::tmem_alloc(s_tmem, 64);
  umma::fence_async_smem();
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  return *s_tmem;
}

// Frees the accumulator. After a wait that gave up, waits once more (bounded)
// for the product in flight and flags the failure.
__device__ __forceinline__ void weak_teardown(uint32_t tmem, uint64_t* s_bar, uint32_t phase, bool ok, int* err) {
  if (!ok) {
    umma::mbar_wait(s_bar, phase ^ 1u);
    if (threadIdx.x == 0 && err) atomicOr(err, 1);
  }
  umma::fence_before();
  __syncthreads();
  if (threadIdx.x < 32) {
    umma::fence_after();
    umma::tmem_free(tmem, 64);
  }
}

template <int LAB, int LC>
__global__ void __launch_bounds__(kThreads, 2) k_df3c_w(Df3cArgs a) {
  extern __shared__ __align__(128) unsigned char smem_w[];
  __shared__ int s_item;
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_bar;
  const uint32_t tmem = weak_setup<LAB, LC>(smem_w, &s_tmem, &s_bar);
  uint32_t phase = 0;
  bool ok = true;
  for (;;) {
    __syncthreads();  // the previous item is done with shared memory and s_item
    if (threadIdx.x == 0) s_item = atomicAdd(a.counter, 1);
    __syncthreads();
    const int item = s_item;
    if (item >= a.n_items) break;
    const int bz = item % a.nbz;
    const int r = item / a.nbz;
    ok = df3c_item_w<LAB, LC>(a, r % a.nbx, r / a.nbx, bz, smem_w, tmem, &s_bar, phase);
    if (!ok) break;
  }
  weak_teardown(tmem, &s_bar, phase, ok, a.err);
}

// Batched form of the weak kernel (descriptor of the item's molecule copied to
// shared memory, as k_df3c_batch).
template <int LAB, int LC>
__global__ void __launch_bounds__(kThreads, 2) k_df3c_w_batch(const Df3cArgs* __restrict__ args,
                                                              const int* __restrict__ item_off, int nm, int* counter) {
  extern __shared__ __align__(128) unsigned char smem_w[];
  __shared__ int s_item, s_m;
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_bar;
  __shared__ __align__(16) unsigned char s_raw[sizeof(Df3cArgs)];
  const Df3cArgs& sa = *reinterpret_cast<const Df3cArgs*>(s_raw);
  const int total = item_off[nm];
  const uint32_t tmem = weak_setup<LAB, LC>(smem_w, &s_tmem, &s_bar);
  uint32_t phase = 0;
  bool ok = true;
  int* err = nullptr;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) {
      const int item = atomicAdd(counter, 1);
      int m = 0;
      if (item < total) {
        int lo = 0, hi = nm - 1;
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
    if (item >= total) break;
    const int m = s_m;
    const unsigned* src = reinterpret_cast<const unsigned*>(args + m);
    unsigned* dst = reinterpret_cast<unsigned*>(s_raw);
    for (int i = threadIdx.x; i < static_cast<int>(sizeof(Df3cArgs) / 4); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    err = sa.err;
    const int local = item - item_off[m];
    const int bz = local % sa.nbz;
    const int r = local / sa.nbz;
    ok = df3c_item_w<LAB, LC>(sa, r % sa.nbx, r / sa.nbx, bz, smem_w, tmem, &s_bar, phase);
    if (!ok) break;
  }
  weak_teardown(tmem, &s_bar, phase, ok, err);
}

template <int LAB, int LC>
void fill_items_w(Df3cArgs* a, int ny) {
  using C = CfgW<LAB, LC>;
  a->nbx = (a->n_aux + C::TC - 1) / C::TC;
  a->nby = ny;
  a->nbz = (a->nd + a->dw - 1) / a->dw;
  a->n_items = a->nbx * a->nby * a->nbz;
}

// Persistent blocks of a weak kernel: two per SM, as the shape is sized
// (shared memory <= 113 KB, 128 registers, 64 tensor-memory columns). The
// runtime's occupancy query answers one block per SM for kernels that use
// tensor memory, so it is not asked; the dynamic shared-memory limit is raised
// once per device.
template <int LAB, int LC, class K>
int weak_resident(K kernel) {
  static int cache[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (cache[dev] == 0) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, CfgW<LAB, LC>::SMEM);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cache[dev] = 2 * sms;
  }
  return cache[dev];
}

template <int LAB, int LC>
int launch_class_w(const Df3cArgs& a, int ny, cudaStream_t s) {
  using C = CfgW<LAB, LC>;
  const int resident = weak_resident<LAB, LC>(k_df3c_w<LAB, LC>);
  Df3cArgs b = a;
  fill_items_w<LAB, LC>(&b, ny);
  if (b.n_items == 0) return 0;
  k_df3c_w<LAB, LC><<<df3c_grid(b.n_items, resident), kThreads, C::SMEM, s>>>(b);
  return 1;
}

template <int LAB, int LC>
int launch_class_w_batch(const Df3cArgs* d_args, const int* d_item_off, int nm, int total_items, int* counter,
                         cudaStream_t s) {
  using C = CfgW<LAB, LC>;
  const int resident = weak_resident<LAB, LC>(k_df3c_w_batch<LAB, LC>);
  if (total_items <= 0 || nm <= 0) return 0;
  k_df3c_w_batch<LAB, LC><<<df3c_grid(total_items, resident), kThreads, C::SMEM, s>>>(d_args, d_item_off, nm,
                                                                                        counter);
  return 1;
}

template <int LAB, int LC>
void class_info_w(Df3cClassInfo* ci) {
  using C = CfgW<LAB, LC>;
  ci->tc = C::TC;
  ci->ub = C::UB;
  ci->ndc = 40;
  ci->lanes = C::kPerThread ? C::TPT : C::TS;
  ci->blocks_per_sm = 2;
  ci->smem = C::SMEM;
}

template <int LAB, int LC>
void fill_row_w(Df3cRow* row) {
  row->launch_w[LC] = &launch_class_w<LAB, LC>;
  row->info_w[LC] = &class_info_w<LAB, LC>;
  row->fill_w[LC] = &fill_items_w<LAB, LC>;
  row->batch_w[LC] = &launch_class_w_batch<LAB, LC>;
  if constexpr (LC < PA_LAUXMAX) fill_row_w<LAB, LC + 1>(row);
}

}  // namespace

}  // namespace pa
