// McMurchie-Davidson building blocks on the device.
//
// Notation (Helgaker, Jorgensen, Olsen, "Molecular Electronic-Structure
// Theory", ch. 9):
//  * a Gaussian pair (exponents a, b at A, B) is expanded in Hermite Gaussians
//    Lambda_tuv(r; p, P), p = a + b, with coefficients E^ij_t per direction;
//  * a spherical single-center function S_lm(r - C) exp(-g |r - C|^2) equals
//    (2g)^-l sum_{|tau| = l} S_lm[tau] Lambda_tau(r; g, C) (Hobson's theorem),
//    so only Hermite components of degree exactly l appear on the auxiliary side;
//  * Coulomb integrals between Hermite Gaussians are
//    2 pi^(5/2) / (p q sqrt(p+q)) (-1)^|tau| R_(t+tau)(alpha, P - Q) with
//    R^n_000 = (-2 alpha)^n F_n(alpha |P-Q|^2) and the R recurrence.
#pragma once

#include "pa_common.cuh"

namespace pa {

// R^0_tuv for all |tuv| <= L, built level by level (n = L-1 .. 0) by `nlanes`
// cooperating threads with ping-pong buffers b0/b1 (each >= ncum(L) doubles).
// Rn[n] = prefactor * (-2 alpha)^n F_n(T). The result is left in b0. `sync`
// is called between levels by every participating thread (also by threads
// with no entries to compute in a level).
template <class Sync>
__device__ __forceinline__ void hermite_R(const int* __restrict__ rdesc, int L, const double* Rn,
                                          double X, double Y, double Z, double* b0, double* b1,
                                          int lane, int nlanes, Sync sync) {
  // Threads with lane >= nlanes (e.g. nlanes == 0 for an inactive team) only
  // take part in the synchronization.
  const bool works = lane < nlanes;
  double* top = (L & 1) ? b1 : b0;
  if (works && lane == 0) top[0] = Rn[L];
  sync();
  for (int n = L - 1; n >= 0; --n) {
    double* dst = (n & 1) ? b1 : b0;
    const double* src = (n & 1) ? b0 : b1;
    const int cnt = works ? ncum(L - n) : 0;
    for (int idx = lane; idx < cnt; idx += nlanes) {
      double v;
      if (idx == 0) {
        v = Rn[n];
      } else {
        const int dsc = __ldg(rdesc + idx);
        const int d = rdesc_d(dsc), c = rdesc_c(dsc);
        const double xd = d == 0 ? X : (d == 1 ? Y : Z);
        v = xd * src[rdesc_s1(dsc)];
        if (c) v = fma(static_cast<double>(c), src[rdesc_s2(dsc)], v);
      }
      dst[idx] = v;
    }
    sync();
  }
}

// Hermite expansion coefficients of one Cartesian direction for a primitive
// pair: E[(i * (lb+1) + j) * (la+lb+1) + t], i <= la, j <= lb, t <= i+j
// (E^00_0 = 1; the Gaussian-product exponential is applied separately).
__device__ __forceinline__ void hermite_E_1d(int la, int lb, double PA, double PB, double inv2p,
                                             double* E) {
  const int nt = la + lb + 1;
  const int nj = lb + 1;
  for (int k = 0; k < (la + 1) * nj * nt; ++k) E[k] = 0.0;
  E[0] = 1.0;
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j) {
      if (i == 0 && j == 0) continue;
      const double* src;
      double X;
      int smax;  // highest t of the source (i + j - 1)
      if (j == 0) {
        src = E + ((i - 1) * nj + 0) * nt;
        X = PA;
      } else {
        src = E + (i * nj + (j - 1)) * nt;
        X = PB;
      }
      smax = i + j - 1;
      double* dst = E + (i * nj + j) * nt;
      for (int t = 0; t <= i + j; ++t) {
        double v = 0.0;
        if (t >= 1 && t - 1 <= smax) v += inv2p * src[t - 1];
        if (t <= smax) v += X * src[t];
        if (t + 1 <= smax) v += (t + 1) * src[t + 1];
        dst[t] = v;
      }
    }
}

}  // namespace pa
