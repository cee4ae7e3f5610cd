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
__device__ __forceinline__ int boys_ref_weights(double T, double w[5]) {
  const int i0 = static_cast<int>(T * 100.0);
  double xs[5];
  // The grid points are the rounded doubles i * 0.01 (boys.f90:221); __dmul_rn
  // keeps the compiler from fusing the product into the later T - x subtraction.
#pragma unroll
  for (int k = 0; k < 5; ++k) xs[k] = __dmul_rn(static_cast<double>(i0 + k), 0.01);
#pragma unroll
  for (int k = 0; k < 5; ++k) {
    double num = 1.0, den = 1.0;
#pragma unroll
    for (int j = 0; j < 5; ++j)
      if (j != k) {
        num *= (T - xs[j]);
        den *= (xs[k] - xs[j]);
      }
    w[k] = num / den;
  }
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
    for (int n = nmax - 1; n >= 0; --n) F[n] = (2.0 * T * F[n + 1] + e) / (2 * n + 1);
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

}  // namespace pa
