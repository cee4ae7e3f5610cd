// Boys function F_n(T) = int_0^1 t^(2n) exp(-T t^2) dt on the device.
//
// Two modes (the mode is a runtime, block-uniform flag):
//  * exact: T < kBoysTSwitch: 8-term Taylor expansion around the nearest
//    point of a table with step 0.05 (tabulated values from a long-double
//    series evaluated on the host at start-up); T >= kBoysTSwitch:
//    F_0 = sqrt(pi/T)/2 and upward recursion F_(n+1) = ((2n+1) F_n - e^-T) / 2T.
//  * reference: the behaviour of the reference's Boys function
//    (common/integrals/boys.f90:88-97): 5-point polynomial interpolation on
//    the 0.01 grid (points i0..i0+4, i0 = int(100 T)) for T < 27 and the
//    asymptotic (2n-1)!!/2^(n+1) sqrt(pi/T^(2n+1)) for T >= 27. The
//    interpolating polynomial is evaluated in Lagrange form with weights shared
//    by all orders n.
#pragma once

#include "pa_common.cuh"

namespace pa {

constexpr double kBoysStep = 0.05;
constexpr double kBoysInvStep = 20.0;
constexpr double kBoysTSwitch = 40.0;
constexpr int kBoysTaylorTerms = 8;
constexpr int kBoysNOrd = PA_BOYS_NMAX + kBoysTaylorTerms;  // table columns
constexpr int kBoysNPts = 801;                              // 0 .. 40 step 0.05
constexpr int kBoysRefNPts = 2711;                          // 0 .. 27.10 step 0.01
constexpr int kBoysRefNOrd = PA_BOYS_NMAX + 1;

enum BoysMode : int { kBoysExact = 0, kBoysReference = 1 };

// 1 / (2n + 1), n = 0 .. PA_BOYS_NMAX (downward recursion of the exact mode).
__device__ __forceinline__ double inv_odd(int n) {
  constexpr double t[PA_BOYS_NMAX + 1] = {1.0,      1.0 / 3,  1.0 / 5,  1.0 / 7,  1.0 / 9,  1.0 / 11,
                                          1.0 / 13, 1.0 / 15, 1.0 / 17, 1.0 / 19, 1.0 / 21, 1.0 / 23,
                                          1.0 / 25, 1.0 / 27, 1.0 / 29, 1.0 / 31, 1.0 / 33};
  return t[n];
}

// Taylor coefficients 1/k!
__device__ __forceinline__ double inv_fact(int k) {
  constexpr double f[kBoysTaylorTerms] = {1.0,
                                          1.0,
                                          0.5,
                                          0.16666666666666666,
                                          0.041666666666666664,
                                          0.008333333333333333,
                                          0.001388888888888889,
                                          0.0001984126984126984};
  return f[k];
}

// Single order n (lane-parallel use). Exact mode.
__device__ __forceinline__ double boys_exact_n(const double* __restrict__ tab, int n, double T) {
  if (T < kBoysTSwitch) {
    const int i = __double2int_rn(T * kBoysInvStep);
    const double mdx = i * kBoysStep - T;  // -(T - T_i)
    const double* row = tab + i * kBoysNOrd + n;
    double s = __ldg(row + kBoysTaylorTerms - 1) * inv_fact(kBoysTaylorTerms - 1);
#pragma unroll
    for (int k = kBoysTaylorTerms - 2; k >= 0; --k) s = fma(s, mdx, __ldg(row + k) * inv_fact(k));
    // Horner in mdx with coefficients F_(n+k)/k!: sum_k F_(n+k) mdx^k / k!
    return s;
  }
  const double e = exp(-T);
  const double inv2T = 0.5 / T;
  double F = 0.5 * sqrt(kPi / T);
  for (int k = 0; k < n; ++k) F = ((2 * k + 1) * F - e) * inv2T;
  return F;
}

// Lagrange weights of the reference's 5-point interpolation at T (< 27).
// Numerators and denominators are products over the other four nodes; one
// reciprocal of the product of all denominators replaces five divisions.
__device__ __forceinline__ int boys_ref_weights(double T, double w[5]) {
  const int i0 = static_cast<int>(T * 100.0);
  double xs[5], d[5];
  // The grid points are the rounded doubles i * 0.01 (boys.f90:30); __dmul_rn
  // keeps the compiler from fusing the product into the later T - x subtraction.
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    xs[k] = __dmul_rn(static_cast<double>(i0 + k), 0.01);
    d[k] = T - xs[k];
  }
  double pre[5], suf[5], den[5], dpre[5], dsuf[5];
  pre[0] = 1.0;
#pragma unroll
  for (int k = 1; k < 5; ++k) pre[k] = pre[k - 1] * d[k - 1];
  suf[4] = 1.0;
#pragma unroll
  for (int k = 3; k >= 0; --k) suf[k] = suf[k + 1] * d[k + 1];
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double v = 1.0;
#pragma unroll
    for (int j = 0; j < 5; ++j)
      if (j != k) v *= xs[k] - xs[j];
    den[k] = v;
  }
  dpre[0] = 1.0;
#pragma unroll
  for (int k = 1; k < 5; ++k) dpre[k] = dpre[k - 1] * den[k - 1];
  dsuf[4] = 1.0;
#pragma unroll
  for (int k = 3; k >= 0; --k) dsuf[k] = dsuf[k + 1] * den[k + 1];
  const double inv_all = 1.0 / (dpre[4] * den[4]);
#pragma unroll
  for (int k = 0; k < 5; ++k) w[k] = pre[k] * suf[k] * (inv_all * dpre[k] * dsuf[k]);
  return i0;
}

__device__ __forceinline__ double boys_ref_asym(int n, double T) {
  double F = 0.5 * sqrt(kPi / T);
  const double inv2T = 0.5 / T;
  for (int k = 1; k <= n; ++k) F *= (2 * k - 1) * inv2T;
  return F;
}

__device__ __forceinline__ double boys_ref_n(const double* __restrict__ tab, int n, double T) {
  if (T >= 27.0) return boys_ref_asym(n, T);
  double w[5];
  const int i0 = boys_ref_weights(T, w);
  const double* row = tab + n * kBoysRefNPts + i0;
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 5; ++k) s = fma(w[k], __ldg(row + k), s);
  return s;
}

__device__ __forceinline__ double boys_n(const DeviceTables& dt, int mode, int n, double T) {
  return mode == kBoysReference ? boys_ref_n(dt.boys_ref, n, T) : boys_exact_n(dt.boys_taylor, n, T);
}

// F_n(T) for several orders n at one T: the interpolation weights (reference
// mode) or the table row (exact mode) are set up once.
struct BoysAt {
  int mode, i0;
  double T, w[5];
  __device__ __forceinline__ BoysAt(int mode_, double T_) : mode(mode_), i0(0), T(T_) {
    if (mode == kBoysReference && T < 27.0) i0 = boys_ref_weights(T, w);
  }
  __device__ __forceinline__ double operator()(const DeviceTables& dt, int n) const {
    if (mode != kBoysReference) return boys_exact_n(dt.boys_taylor, n, T);
    if (T >= 27.0) return boys_ref_asym(n, T);
    const double* row = dt.boys_ref + n * kBoysRefNPts + i0;
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 5; ++k) s = fma(w[k], __ldg(row + k), s);
    return s;
  }
};

// All orders 0..nmax by one thread.
__device__ __forceinline__ void boys_all(const DeviceTables& dt, int mode, int nmax, double T,
                                         double* F) {
  if (mode == kBoysReference) {
    if (T >= 27.0) {
      double f = 0.5 * sqrt(kPi / T);
      const double inv2T = 0.5 / T;
      F[0] = f;
      for (int k = 1; k <= nmax; ++k) {
        f *= (2 * k - 1) * inv2T;
        F[k] = f;
      }
      return;
    }
    double w[5];
    const int i0 = boys_ref_weights(T, w);
    for (int n = 0; n <= nmax; ++n) {
      const double* row = dt.boys_ref + n * kBoysRefNPts + i0;
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < 5; ++k) s = fma(w[k], __ldg(row + k), s);
      F[n] = s;
    }
    return;
  }
  const double e = exp(-T);
  if (T < kBoysTSwitch) {
    F[nmax] = boys_exact_n(dt.boys_taylor, nmax, T);
    const double twoT = 2.0 * T;
    for (int n = nmax - 1; n >= 0; --n) F[n] = fma(twoT, F[n + 1], e) * inv_odd(n);
    return;
  }
  const double inv2T = 0.5 / T;
  double f = 0.5 * sqrt(kPi / T);
  F[0] = f;
  for (int k = 0; k < nmax; ++k) {
    f = ((2 * k + 1) * f - e) * inv2T;
    F[k + 1] = f;
  }
}

// ---------------------------------------------------------------------------
// Single-precision Boys values for the FP32 recurrences of weakly coupled
// triplets (precision form). The large-T branches stay in FP64 and are rounded
// once: the reference-mode asymptotic formula (T >= 27) and, in exact mode,
// T >= 30 (upward recursion from the closed form F_0).
struct BoysAtF {
  int mode, i0;
  double T;
  float Tf, w[5], e;
  __device__ __forceinline__ BoysAtF(int mode_, double T_) : mode(mode_), i0(0), T(T_), Tf(static_cast<float>(T_)) {
    if (mode == kBoysReference) {
      if (T < 27.0) {
        i0 = static_cast<int>(T * 100.0);
        float d[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) d[k] = static_cast<float>(T - (i0 + k) * 0.01);
        // 5-point Lagrange weights on the uniform 0.01 grid
        constexpr float inv_den[5] = {1.0f / (24e-8f), -1.0f / (6e-8f), 1.0f / (4e-8f), -1.0f / (6e-8f),
                                      1.0f / (24e-8f)};
#pragma unroll
        for (int k = 0; k < 5; ++k) {
          float num = 1.0f;
#pragma unroll
          for (int j = 0; j < 5; ++j)
            if (j != k) num *= d[j];
          w[k] = num * inv_den[k];
        }
      }
    } else if (T < 30.0) {
      i0 = __double2int_rn(T * kBoysInvStep);
      e = static_cast<float>(i0 * kBoysStep - T);  // -(T - T_i)
    }
  }
  __device__ __forceinline__ float operator()(const DeviceTables& dt, int n) const {
    if (mode == kBoysReference) {
      if (T >= 27.0) return static_cast<float>(boys_ref_asym(n, T));
      const double* row = dt.boys_ref + n * kBoysRefNPts + i0;
      float s = 0.0f;
#pragma unroll
      for (int k = 0; k < 5; ++k) s = fmaf(w[k], static_cast<float>(__ldg(row + k)), s);
      return s;
    }
    if (T >= 30.0) return static_cast<float>(boys_exact_n(dt.boys_taylor, n, T));
    // Taylor series around the table point, 6 terms (|dx| <= 0.025)
    const double* row = dt.boys_taylor + i0 * kBoysNOrd + n;
    float s = static_cast<float>(__ldg(row + 5)) * (1.0f / 120.0f);
    s = fmaf(s, e, static_cast<float>(__ldg(row + 4)) * (1.0f / 24.0f));
    s = fmaf(s, e, static_cast<float>(__ldg(row + 3)) * (1.0f / 6.0f));
    s = fmaf(s, e, static_cast<float>(__ldg(row + 2)) * 0.5f);
    s = fmaf(s, e, static_cast<float>(__ldg(row + 1)));
    s = fmaf(s, e, static_cast<float>(__ldg(row)));
    return s;
  }
};

// F_0..F_nmax in single precision (one thread).
__device__ __forceinline__ void boys_all(const DeviceTables& dt, int mode, int nmax, double T, float* F) {
  if (mode == kBoysReference || T >= 30.0) {
    const BoysAtF B(mode, T);
    for (int n = 0; n <= nmax; ++n) F[n] = B(dt, n);
    return;
  }
  const BoysAtF B(mode, T);
  F[nmax] = B(dt, nmax);
  const float ex = expf(-static_cast<float>(T)), twoT = 2.0f * static_cast<float>(T);
  for (int n = nmax - 1; n >= 0; --n) F[n] = fmaf(twoT, F[n + 1], ex) * static_cast<float>(inv_odd(n));
}

template <class Real>
struct BoysAtT;
template <>
struct BoysAtT<double> {
  using type = BoysAt;
};
template <>
struct BoysAtT<float> {
  using type = BoysAtF;
};

}  // namespace pa

