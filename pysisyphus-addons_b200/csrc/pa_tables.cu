// Constant tables of the library, built on the host once per device and kept
// in device memory until the process exits:
//  * decoded Cartesian / Hermite multi-index tables;
//  * Boys-function tables (exact-mode Taylor table and the reference-mode 0.01
//    grid), evaluated in long double from the convergent series
//    F_n(x) = e^-x sum_k (2x)^k / ((2n+1)(2n+3)...(2n+2k+1)) with downward
//    recursion -- regenerated, not copied from the reference's boys_data.f90;
//  * real solid harmonics S_lm, m = -l..l (Helgaker, Jorgensen, Olsen,
//    "Molecular Electronic-Structure Theory", eqs. 6.4.47-6.4.50), normalized
//    so that a contracted shell normalized like common/normalization.f90 gives
//    unit-norm spherical functions.
#include <cmath>
#include <mutex>
#include <vector>

#include "boys.cuh"
#include "k_df3c.cuh"
#include "pa_internal.h"
#include "sph_raw.cuh"

namespace pa {

namespace {

void boys_series_ld(int nmax, long double x, long double* F) {
  if (x < 1e-30L) {
    for (int n = 0; n <= nmax; ++n) F[n] = 1.0L / (2 * n + 1);
    return;
  }
  const long double ex = expl(-x);
  long double term = 1.0L / (2 * nmax + 1), sum = term;
  for (int k = 1; k < 4000; ++k) {
    term *= 2.0L * x / (2 * nmax + 2 * k + 1);
    sum += term;
    if (term < 1e-24L * sum) break;
  }
  F[nmax] = ex * sum;
  for (int n = nmax - 1; n >= 0; --n) F[n] = (2.0L * x * F[n + 1] + ex) / (2 * n + 1);
}

double fact(int n) {
  double r = 1.0;
  for (int k = 2; k <= n; ++k) r *= k;
  return r;
}
double binom(int n, int k) { return (k < 0 || k > n) ? 0.0 : fact(n) / (fact(k) * fact(n - k)); }
double dfact(int n) {
  double r = 1.0;
  for (int k = n; k > 1; k -= 2) r *= k;
  return r;
}

// Dense normalized solid harmonics for l <= PA_LAUXMAX: rows m + l, columns =
// local Cartesian index within degree l.
std::vector<double> solid_harmonics(int l) {
  const int nc = ncart(l);
  std::vector<double> T(static_cast<size_t>(2 * l + 1) * nc, 0.0);
  auto local = [&](int i, int j, int k) { return cidx(i, j, k) - ncum(l - 1); };
  for (int m = -l; m <= l; ++m) {
    const int am = std::abs(m);
    const double N = 1.0 / (std::pow(2.0, am) * fact(l)) *
                     std::sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0));
    const int vm2 = m < 0 ? 1 : 0;
    const int v2max = 2 * static_cast<int>(std::floor(am / 2.0 - vm2 / 2.0)) + vm2;
    for (int t = 0; t <= (l - am) / 2; ++t)
      for (int u = 0; u <= t; ++u)
        for (int v2 = vm2; v2 <= v2max; v2 += 2) {
          const double sgn = ((t + (v2 - vm2) / 2) % 2) ? -1.0 : 1.0;
          const double c = sgn * std::pow(0.25, t) * binom(l, t) * binom(l - t, am + t) *
                           binom(t, u) * binom(am, v2);
          T[(m + l) * nc + local(2 * t + am - 2 * u - v2, 2 * u + v2, l - 2 * t - am)] += N * c;
        }
    // normalization: sum_cc' T_c T_c' (i+i'-1)!! (j+j'-1)!! (k+k'-1)!! = 1
    std::vector<int> ex(3 * nc);
    for (int i = l, q = 0; i >= 0; --i)
      for (int j = l - i; j >= 0; --j, ++q) {
        ex[3 * q] = i;
        ex[3 * q + 1] = j;
        ex[3 * q + 2] = l - i - j;
      }
    double s = 0.0;
    for (int c1 = 0; c1 < nc; ++c1)
      for (int c2 = 0; c2 < nc; ++c2) {
        double f = T[(m + l) * nc + c1] * T[(m + l) * nc + c2];
        for (int d = 0; d < 3; ++d) {
          const int n = ex[3 * c1 + d] + ex[3 * c2 + d];
          if (n & 1) {
            f = 0.0;
            break;
          }
          f *= dfact(n - 1);
        }
        s += f;
      }
    for (int c = 0; c < nc; ++c) T[(m + l) * nc + c] /= std::sqrt(s);
  }
  return T;
}

struct TablesOnDevice {
  bool ready = false;
  int status = PA_OK;
  std::string err;
  DeviceTables dt{};
};

std::mutex g_mu;
std::vector<TablesOnDevice> g_tables;

int build_tables(TablesOnDevice* out, std::string* err) {
  // index tables
  IndexTables h_idx{};
  for (int l = 0; l <= PA_LTOT_MAX; ++l)
    for (int i = l; i >= 0; --i)
      for (int j = l - i; j >= 0; --j) {
        const int k = l - i - j, g = cidx(i, j, k);
        h_idx.xyz[g][0] = static_cast<uint8_t>(i);
        h_idx.xyz[g][1] = static_cast<uint8_t>(j);
        h_idx.xyz[g][2] = static_cast<uint8_t>(k);
        h_idx.xyz[g][3] = static_cast<uint8_t>(l);
        const int e[3] = {i, j, k};
        for (int d = 0; d < 3; ++d) {
          int f[3] = {e[0], e[1], e[2]};
          if (f[d] == 0) {
            h_idx.minus[g][d] = -1;
          } else {
            f[d] -= 1;
            h_idx.minus[g][d] = static_cast<int16_t>(cidx(f[0], f[1], f[2]));
          }
        }
      }
  // Boys tables
  std::vector<double> taylor(static_cast<size_t>(kBoysNPts) * kBoysNOrd);
  long double F[kBoysNOrd + 1];
  for (int i = 0; i < kBoysNPts; ++i) {
    boys_series_ld(kBoysNOrd - 1, static_cast<long double>(i) * 0.05L, F);
    for (int n = 0; n < kBoysNOrd; ++n) taylor[static_cast<size_t>(i) * kBoysNOrd + n] = (double)F[n];
  }
  std::vector<double> ref(static_cast<size_t>(kBoysRefNOrd) * kBoysRefNPts);
  for (int i = 0; i < kBoysRefNPts; ++i) {
    const double xi = i * 0.01;  // the reference's grid points, i * 0.01 in double
    boys_series_ld(kBoysRefNOrd - 1, xi, F);
    for (int n = 0; n < kBoysRefNOrd; ++n) ref[static_cast<size_t>(n) * kBoysRefNPts + i] = (double)F[n];
  }
  // solid harmonics: sparse rows, and the row normalization of the auxiliary
  // shells' terms (the class kernels carry the raw coefficients)
  std::vector<int> start{0};
  std::vector<int16_t> col;
  std::vector<double> val;
  std::vector<double> rownorm((PA_LAUXMAX + 1) * (PA_LAUXMAX + 1), 0.0);
  const int lsph = std::max(PA_LMAX, PA_LAUXMAX);
  for (int l = 0; l <= lsph; ++l) {
    const std::vector<double> T = solid_harmonics(l);
    const int nc = ncart(l);
    if (l <= PA_LAUXMAX)
      for (int m = 0; m < 2 * l + 1; ++m)
        for (int i = l, c = 0; i >= 0; --i)
          for (int j = l - i; j >= 0; --j, ++c) {
            const double r = sph_raw(l, m - l, i, j, l - i - j);
            if (r != 0.0 && rownorm[l * l + m] == 0.0) rownorm[l * l + m] = T[m * nc + c] / r;
          }
    for (int m = 0; m < 2 * l + 1; ++m) {
      for (int c = 0; c < nc; ++c) {
        const double v = T[m * nc + c];
        if (v != 0.0) {
          col.push_back(static_cast<int16_t>(c));
          val.push_back(v);
        }
      }
      start.push_back(static_cast<int>(col.size()));
    }
  }
  // multi-index sums of two bra Hermite components
  std::vector<int16_t> sum_idx(static_cast<size_t>(kNSum) * kNSum);
  for (int i = 0; i < kNSum; ++i)
    for (int j = 0; j < kNSum; ++j)
      sum_idx[static_cast<size_t>(i) * kNSum + j] = static_cast<int16_t>(
          cidx(h_idx.xyz[i][0] + h_idx.xyz[j][0], h_idx.xyz[i][1] + h_idx.xyz[j][1], h_idx.xyz[i][2] + h_idx.xyz[j][2]));
  // Hermite recursion descriptors
  std::vector<int> rdesc(kNCumMax, 0);
  for (int idx = 1; idx < kNCumMax; ++idx) {
    const int e[3] = {h_idx.xyz[idx][0], h_idx.xyz[idx][1], h_idx.xyz[idx][2]};
    const int d = e[0] ? 0 : (e[1] ? 1 : 2);
    const int s1 = h_idx.minus[idx][d];
    const int c = e[d] - 1;
    const int s2 = c > 0 ? h_idx.minus[s1][d] : 0;
    rdesc[idx] = s1 | (s2 << 10) | (d << 20) | (c << 22);
  }
  // upload
  const size_t bytes = sizeof(IndexTables) + sizeof(double) * (taylor.size() + ref.size() + val.size()) +
                       sizeof(int) * start.size() + sizeof(int16_t) * col.size() +
                       sizeof(int16_t) * sum_idx.size() + sizeof(int) * rdesc.size() + 8 * 256;
  char* base = nullptr;
  cudaError_t e = cudaMalloc(&base, bytes);
  if (e != cudaSuccess) {
    *err = std::string("cudaMalloc(tables): ") + cudaGetErrorString(e);
    return PA_ERR_CUDA;
  }
  size_t off = 0;
  auto put = [&](const void* src, size_t n) {
    char* p = base + off;
    cudaMemcpy(p, src, n, cudaMemcpyHostToDevice);
    off += (n + 255) & ~size_t(255);
    return p;
  };
  DeviceTables dt{};
  dt.idx = reinterpret_cast<const IndexTables*>(put(&h_idx, sizeof(IndexTables)));
  dt.boys_taylor = reinterpret_cast<const double*>(put(taylor.data(), sizeof(double) * taylor.size()));
  dt.boys_ref = reinterpret_cast<const double*>(put(ref.data(), sizeof(double) * ref.size()));
  dt.sph_start = reinterpret_cast<const int*>(put(start.data(), sizeof(int) * start.size()));
  dt.sph_col = reinterpret_cast<const int16_t*>(put(col.data(), sizeof(int16_t) * col.size()));
  dt.sph_val = reinterpret_cast<const double*>(put(val.data(), sizeof(double) * val.size()));
  dt.sum_idx = reinterpret_cast<const int16_t*>(put(sum_idx.data(), sizeof(int16_t) * sum_idx.size()));
  dt.rdesc = reinterpret_cast<const int*>(put(rdesc.data(), sizeof(int) * rdesc.size()));
  e = upload_sph_rownorm(rownorm.data(), 0);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    *err = std::string("table upload: ") + cudaGetErrorString(e);
    return PA_ERR_CUDA;
  }
  out->dt = dt;
  return PA_OK;
}

}  // namespace

int get_device_tables(DeviceTables* out, std::string* err) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    *err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
    return PA_ERR_NO_DEVICE;
  }
  std::lock_guard<std::mutex> lock(g_mu);
  if (static_cast<int>(g_tables.size()) <= dev) g_tables.resize(dev + 1);
  TablesOnDevice& t = g_tables[dev];
  if (!t.ready) {
    t.status = build_tables(&t, &t.err);
    t.ready = true;
  }
  if (t.status != PA_OK) {
    *err = t.err;
    return t.status;
  }
  *out = t.dt;
  return PA_OK;
}

// Host copies for tests of the tables themselves.
void host_solid_harmonics(int l, std::vector<double>* out) { *out = solid_harmonics(l); }

}  // namespace pa
