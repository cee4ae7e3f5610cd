// Real solid harmonics S_lm (m = -l..l) as constexpr arithmetic: the unnormalized
// coefficient of x^ax y^ay z^az from Helgaker, Jorgensen, Olsen,
// "Molecular Electronic-Structure Theory", eqs. 6.4.47-6.4.50, without the
// prefactor N_lm. All terms are small-integer ratios (exact in double). The
// normalized coefficient is sph_raw(...) * rownorm(l, m), with the row factor
// taken from pa_tables.cu. Being a function (not data), it folds to a constant
// when its arguments are compile-time constants and stays correct otherwise.
#pragma once

namespace pa {

__host__ __device__ constexpr long long sph_fact(int n) {
  long long r = 1;
  for (int k = 2; k <= n; ++k) r *= k;
  return r;
}

__host__ __device__ constexpr long long sph_binom(int n, int k) {
  return (k < 0 || k > n) ? 0 : sph_fact(n) / (sph_fact(k) * sph_fact(n - k));
}

__host__ __device__ constexpr double sph_raw(int l, int m, int ax, int ay, int az) {
  const int am = m < 0 ? -m : m;
  const int vm2 = m < 0 ? 1 : 0;
  const int v2max = 2 * ((am - vm2) / 2) + vm2;
  double s = 0.0;
  for (int t = 0; t <= (l - am) / 2; ++t) {
    double inv4t = 1.0;
    for (int k = 0; k < t; ++k) inv4t *= 0.25;
    for (int u = 0; u <= t; ++u)
      for (int v2 = vm2; v2 <= v2max; v2 += 2) {
        if (2 * t + am - 2 * u - v2 != ax || 2 * u + v2 != ay || l - 2 * t - am != az) continue;
        const double sign = ((t + (v2 - vm2) / 2) % 2) ? -1.0 : 1.0;
        s += sign * inv4t *
             static_cast<double>(sph_binom(l, t) * sph_binom(l - t, am + t) * sph_binom(t, u) *
                                 sph_binom(am, v2));
      }
  }
  return s;
}

}  // namespace pa
