// THE ORACLE -- test infrastructure, not product code (see oracle.h).
//
// CPU FP64 restatement of pysisyphus-addons' density-fitting path. Citations
// are file:line within the reference project (pysisyphus_addons/...).

#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

namespace {

constexpr double PI = 3.141592653589793238462643383279502884;
constexpr int MAXL = 6;             // per-center angular momentum supported by the oracle
constexpr int MAXLT = 4 * MAXL;     // total angular momentum of a quartet
constexpr int BOYS_NMAX = MAXLT + 1;

// Screening threshold of the reference: the literal 1e-10 is REAL(4) and is
// promoted to double (diabatization/intor.f90:140, std/intor.f90:78,223).
const double SCREEN_THRESH = static_cast<double>(1e-10f);
// Value skips of intor_df2c_mo (std/intor.f90:247 real(4), :269 real(8)).
const double DF2C_SKIP1 = static_cast<double>(1e-10f);
const double DF2C_SKIP2 = 1e-10;

int g_boys_mode = 0;
int g_skip_metric = 0;
// Triplet estimate of contract_coulomb_densities_2d: 0 = schwarz_estimate (the
// reference's active line, diabatization/intor.f90:138), 1 = qvl_estimate (its
// commented-out alternative at :137, common/screening.f90:267-299).
int g_screening = 0;
// Optional diagonal shift of (P|Q) before the factorization (0 = the reference).
double g_metric_shift = 0.0;
OracleStats g_stats{};

// ---------------------------------------------------------------------------
// BLAS / LAPACK hooks (Fortran ABI), as called by common/linalg.f90:60-82,
// diabatization/intor.f90:198, std/intor.f90:116,137,290.
typedef void (*dpotrf_t)(const char*, const int*, double*, const int*, int*);
typedef void (*dtrtri_t)(const char*, const char*, const int*, double*, const int*, int*);
typedef void (*dtrmm_t)(const char*, const char*, const char*, const char*, const int*,
                        const int*, const double*, const double*, const int*, double*,
                        const int*);
typedef void (*dgemm_t)(const char*, const char*, const int*, const int*, const int*,
                        const double*, const double*, const int*, const double*, const int*,
                        const double*, double*, const int*);
dpotrf_t p_dpotrf = nullptr;
dtrtri_t p_dtrtri = nullptr;
dtrmm_t p_dtrmm = nullptr;
dgemm_t p_dgemm = nullptr;

double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// ---------------------------------------------------------------------------
// Boys function F_n(x) = int_0^1 t^(2n) exp(-x t^2) dt.

// Exact mode: series F_n(x) = e^-x sum_k (2x)^k / ((2n+1)(2n+3)...(2n+2k+1)) for the
// highest order and downward recursion for x < 30; erf-based F_0 and upward
// recursion above. Evaluated in long double.
void boys_exact_ld(int nmax, long double x, long double* F) {
  if (x < 1e-30L) {
    for (int n = 0; n <= nmax; ++n) F[n] = 1.0L / (2 * n + 1);
    return;
  }
  const long double ex = expl(-x);
  if (x < 30.0L) {
    long double term = 1.0L / (2 * nmax + 1);
    long double sum = term;
    for (int k = 1; k < 2000; ++k) {
      term *= 2.0L * x / (2 * nmax + 2 * k + 1);
      sum += term;
      if (term < 1e-22L * sum) break;
    }
    F[nmax] = ex * sum;
    for (int n = nmax - 1; n >= 0; --n) F[n] = (2.0L * x * F[n + 1] + ex) / (2 * n + 1);
  } else {
    F[0] = 0.5L * sqrtl(PI / x) * erfl(sqrtl(x));
    for (int n = 0; n < nmax; ++n) F[n + 1] = ((2 * n + 1) * F[n] - ex) / (2.0L * x);
  }
}

void boys_exact(int nmax, double x, double* F) {
  long double Fl[BOYS_NMAX + 1];
  boys_exact_ld(nmax, x, Fl);
  for (int n = 0; n <= nmax; ++n) F[n] = static_cast<double>(Fl[n]);
}

// Reference-compatible mode (common/integrals/boys.f90:22-97): table on
// x_i = i * 0.01 (i = 0 .. 2710, boys.f90:22-30), 5-point Neville
// interpolation through points i0 .. i0+4 with i0 = int(100 x) (:53-85), and
// for x >= 27 the asymptotic formula (2n-1)!! / 2^(n+1) * sqrt(pi / x^(2n+1))
// (:44-49, switch at :88-97). The table is regenerated here (exact mode) instead of
// being copied; the reference stores n <= 14 only, this table extends to
// BOYS_NMAX so that high-L Schwarz integrals stay defined.
constexpr int REF_NPTS = 2711;
std::vector<double> g_ref_table;  // [n * REF_NPTS + i]
std::once_flag g_ref_once;

void build_ref_table() {
  g_ref_table.assign(static_cast<size_t>(BOYS_NMAX + 1) * REF_NPTS, 0.0);
  long double F[BOYS_NMAX + 1];
  for (int i = 0; i < REF_NPTS; ++i) {
    const double xi = i * 0.01;
    boys_exact_ld(BOYS_NMAX, xi, F);
    for (int n = 0; n <= BOYS_NMAX; ++n) g_ref_table[n * REF_NPTS + i] = static_cast<double>(F[n]);
  }
}

double double_factorial(int n) {
  double r = 1.0;
  for (int k = n; k > 1; k -= 2) r *= k;
  return r;
}

void boys_reference(int nmax, double x, double* F) {
  std::call_once(g_ref_once, build_ref_table);
  if (x >= 27.0) {
    for (int n = 0; n <= nmax; ++n) {
      const double df = double_factorial(std::max(0, 2 * n - 1));
      F[n] = df / std::pow(2.0, n + 1) * std::sqrt(PI / std::pow(x, 2 * n + 1));
    }
    return;
  }
  const int i0 = static_cast<int>(x * 100);
  double xs[5];
  for (int k = 0; k < 5; ++k) xs[k] = (i0 + k) * 0.01;
  for (int n = 0; n <= nmax; ++n) {
    double p[5];
    for (int k = 0; k < 5; ++k) p[k] = g_ref_table[n * REF_NPTS + i0 + k];
    for (int k = 1; k < 5; ++k)
      for (int j = 0; j + k < 5; ++j)
        p[j] = ((x - xs[j + k]) * p[j] + (xs[j] - x) * p[j + 1]) / (xs[j] - xs[j + k]);
    F[n] = p[0];
  }
}

inline void boys(int nmax, double x, double* F) {
  if (g_boys_mode == 1)
    boys_reference(nmax, x, F);
  else
    boys_exact(nmax, x, F);
}

// ---------------------------------------------------------------------------
// Cartesian component bookkeeping. Components of total degree l are ordered
// x^l, x^(l-1) y, x^(l-1) z, x^(l-2) y^2, ... (i descending, then j
// descending); all degrees 0..L are stored back to back.
constexpr int NCUM_MAX = (2 * MAXL + 1) * (2 * MAXL + 2) * (2 * MAXL + 3) / 6;

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }
inline int ncum(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }
inline int cidx(int i, int j, int k) {
  const int l = i + j + k, li = l - i;
  return l * (l + 1) * (l + 2) / 6 + li * (li + 1) / 2 + (li - j);
}

struct CartTables {
  int xyz[NCUM_MAX][3];
  int minus[NCUM_MAX][3];  // index of e - 1_d, -1 if e_d == 0
  int plus[NCUM_MAX][3];   // index of e + 1_d (if within NCUM_MAX), else -1
  int deg[NCUM_MAX];
  // real solid harmonics, normalized: sph[l][m + l][cart index within degree l]
  std::vector<double> sph[MAXL + 1];
  CartTables() {
    for (int l = 0; l <= 2 * MAXL; ++l)
      for (int i = l; i >= 0; --i)
        for (int j = l - i; j >= 0; --j) {
          const int k = l - i - j, g = cidx(i, j, k);
          xyz[g][0] = i;
          xyz[g][1] = j;
          xyz[g][2] = k;
          deg[g] = l;
        }
    for (int g = 0; g < NCUM_MAX; ++g)
      for (int d = 0; d < 3; ++d) {
        int e[3] = {xyz[g][0], xyz[g][1], xyz[g][2]};
        minus[g][d] = -1;
        plus[g][d] = -1;
        if (e[d] > 0) {
          e[d] -= 1;
          minus[g][d] = cidx(e[0], e[1], e[2]);
          e[d] += 1;
        }
        e[d] += 1;
        if (deg[g] + 1 <= 2 * MAXL) plus[g][d] = cidx(e[0], e[1], e[2]);
      }
    for (int l = 0; l <= MAXL; ++l) build_sph(l);
  }
  static double fact(int n) {
    double r = 1.0;
    for (int k = 2; k <= n; ++k) r *= k;
    return r;
  }
  static double binom(int n, int k) {
    if (k < 0 || k > n) return 0.0;
    return fact(n) / (fact(k) * fact(n - k));
  }
  // Real solid harmonics S_lm (Helgaker, Jorgensen, Olsen, "Molecular
  // Electronic-Structure Theory", eqs. 6.4.47-6.4.50), m = -l..l, then
  // normalized so that S_lm * exp(-a r^2) with the reference's contraction
  // normalization is a unit-norm function.
  void build_sph(int l) {
    const int nc = ncart(l);
    std::vector<double>& T = sph[l];
    T.assign(static_cast<size_t>(2 * l + 1) * nc, 0.0);
    for (int m = -l; m <= l; ++m) {
      const int am = std::abs(m);
      const double Nlm = 1.0 / (std::pow(2.0, am) * fact(l)) *
                         std::sqrt(2.0 * fact(l + am) * fact(l - am) / (m == 0 ? 2.0 : 1.0));
      const int vm2 = m < 0 ? 1 : 0;
      const int v2max = 2 * static_cast<int>(std::floor(am / 2.0 - vm2 / 2.0)) + vm2;
      for (int t = 0; t <= (l - am) / 2; ++t)
        for (int u = 0; u <= t; ++u)
          for (int v2 = vm2; v2 <= v2max; v2 += 2) {
            const int sgn = ((t + (v2 - vm2) / 2) % 2) ? -1 : 1;
            const double C = sgn * std::pow(0.25, t) * binom(l, t) * binom(l - t, am + t) *
                             binom(t, u) * binom(am, v2);
            const int px = 2 * t + am - 2 * u - v2, py = 2 * u + v2, pz = l - 2 * t - am;
            const int g = cidx(px, py, pz) - l * (l + 1) * (l + 2) / 6;
            T[(m + l) * nc + g] += Nlm * C;
          }
      // normalization: sum_cc' T_c T_c' (i+i'-1)!! (j+j'-1)!! (k+k'-1)!! = 1
      double s = 0.0;
      const int off = l * (l + 1) * (l + 2) / 6;
      for (int c1 = 0; c1 < nc; ++c1)
        for (int c2 = 0; c2 < nc; ++c2) {
          const int* e1 = xyz[off + c1];
          const int* e2 = xyz[off + c2];
          double f = T[(m + l) * nc + c1] * T[(m + l) * nc + c2];
          for (int d = 0; d < 3; ++d) {
            const int n = e1[d] + e2[d];
            if (n % 2) {
              f = 0.0;
              break;
            }
            f *= double_factorial(n - 1);
          }
          s += f;
        }
      for (int c = 0; c < nc; ++c) T[(m + l) * nc + c] /= std::sqrt(s);
    }
  }
};

const CartTables& tables() {
  static CartTables t;
  return t;
}

// ---------------------------------------------------------------------------
// Basis unpacking (common/shells.f90:97-187) and contraction normalization
// (common/normalization.f90:10-38).

struct OShell {
  int L = 0;
  int nprim = 0;
  double A[3] = {0, 0, 0};
  std::vector<double> exps, coefs;
  int sph_off = 0;
};

struct OBasis {
  std::vector<OShell> shells;
  int nsph = 0;
  int lmax = -1;
};

void norm_cgto_coeffs(std::vector<double>& c, const std::vector<double>& e, int L) {
  double N = 0.0;
  const double lp = L + 1.5;
  for (size_t i = 0; i < e.size(); ++i)
    for (size_t j = 0; j < e.size(); ++j)
      N += c[i] * c[j] / std::pow(e[i] + e[j], lp) * std::pow(std::sqrt(e[i] * e[j]), lp);
  for (size_t i = 0; i < e.size(); ++i)
    c[i] *= std::sqrt(std::pow(e[i], lp) / (std::pow(PI, 1.5) / std::pow(2.0, L) * N));
}

OBasis make_basis(int nshells, const int* centers, const int* spec, const double* data) {
  OBasis b;
  b.shells.resize(nshells);
  int off = 0;
  for (int i = 0; i < nshells; ++i) {
    OShell& s = b.shells[i];
    const int cptr = centers[i + 2 * nshells] - 1;  // bas_centers(i, 3), 1-based
    for (int d = 0; d < 3; ++d) s.A[d] = data[cptr + d];
    s.L = spec[i + 1 * nshells];
    s.nprim = spec[i + 2 * nshells];
    const int ptr = spec[i + 4 * nshells] - 1;
    s.coefs.assign(data + ptr, data + ptr + s.nprim);
    s.exps.assign(data + ptr + s.nprim, data + ptr + 2 * s.nprim);
    norm_cgto_coeffs(s.coefs, s.exps, s.L);
    s.sph_off = off;
    off += 2 * s.L + 1;
    b.lmax = std::max(b.lmax, s.L);
  }
  b.nsph = off;
  return b;
}

// A "null" shell: unit s function with exponent 0 at the partner's center.
OShell null_shell(const OShell& partner) {
  OShell s;
  s.L = -1;
  s.nprim = 1;
  std::copy(partner.A, partner.A + 3, s.A);
  s.exps = {0.0};
  s.coefs = {1.0};
  return s;
}

// ---------------------------------------------------------------------------
// Obara-Saika VRR + Head-Gordon-Pople HRR for contracted (ab|cd).

struct PrimPair {
  double p, P[3], PA[3], K;
};

void make_pairs(const OShell& a, const OShell& b, std::vector<PrimPair>& out) {
  out.clear();
  double AB2 = 0.0;
  for (int d = 0; d < 3; ++d) AB2 += (a.A[d] - b.A[d]) * (a.A[d] - b.A[d]);
  for (int i = 0; i < a.nprim; ++i)
    for (int j = 0; j < b.nprim; ++j) {
      PrimPair pp;
      const double ai = a.exps[i], bj = b.exps[j];
      pp.p = ai + bj;
      for (int d = 0; d < 3; ++d) {
        pp.P[d] = (ai * a.A[d] + bj * b.A[d]) / pp.p;
        pp.PA[d] = pp.P[d] - a.A[d];
      }
      pp.K = a.coefs[i] * b.coefs[j] * std::exp(-ai * bj / pp.p * AB2);
      out.push_back(pp);
    }
}

struct Workspace {
  std::vector<double> V, acc, h1, h2, t, t2, ketc, cart, s1, s2, s3;
  std::vector<PrimPair> bra, ket;
};

// acc[e][f] (all |e| <= Le, |f| <= Lf) = sum over primitive quartets of [e0|f0]^(0).
void vrr_contracted(const std::vector<PrimPair>& bra, const std::vector<PrimPair>& ket,
                    const double* A, const double* C, int Le, int Lf, Workspace& ws) {
  const CartTables& T = tables();
  const int ne = ncum(Le), nf = ncum(Lf), M = Le + Lf;
  ws.acc.assign(static_cast<size_t>(ne) * nf, 0.0);
  ws.V.resize(static_cast<size_t>(M + 1) * ne * nf);
  double* V = ws.V.data();
  auto at = [&](int m, int e, int f) -> double& {
    return V[(static_cast<size_t>(m) * ne + e) * nf + f];
  };
  double F[BOYS_NMAX + 1];
  for (const PrimPair& bp : bra)
    for (const PrimPair& kp : ket) {
      const double p = bp.p, q = kp.p, pq = p + q, rho = p * q / pq;
      double W[3], WP[3], WQ[3], QC[3], PQ2 = 0.0;
      for (int d = 0; d < 3; ++d) {
        W[d] = (p * bp.P[d] + q * kp.P[d]) / pq;
        WP[d] = W[d] - bp.P[d];
        WQ[d] = W[d] - kp.P[d];
        QC[d] = kp.P[d] - C[d];
        PQ2 += (bp.P[d] - kp.P[d]) * (bp.P[d] - kp.P[d]);
      }
      (void)A;
      boys(M, rho * PQ2, F);
      const double pref = 2.0 * std::pow(PI, 2.5) / (p * q * std::sqrt(pq)) * bp.K * kp.K;
      for (int m = 0; m <= M; ++m) at(m, 0, 0) = pref * F[m];
      // bra build, f = 0
      for (int e = 1; e < ne; ++e) {
        const int le = T.deg[e];
        int d = 0;
        while (T.xyz[e][d] == 0) ++d;
        const int e1 = T.minus[e][d];
        const int e2 = T.minus[e1][d];
        const double c2 = (T.xyz[e1][d]) / (2.0 * p);
        for (int m = 0; m <= M - le; ++m) {
          double v = bp.PA[d] * at(m, e1, 0) + WP[d] * at(m + 1, e1, 0);
          if (e2 >= 0) v += c2 * (at(m, e2, 0) - rho / p * at(m + 1, e2, 0));
          at(m, e, 0) = v;
        }
      }
      // ket build
      for (int f = 1; f < nf; ++f) {
        const int lf = T.deg[f];
        int d = 0;
        while (T.xyz[f][d] == 0) ++d;
        const int f1 = T.minus[f][d];
        const int f2 = T.minus[f1][d];
        const double c2 = T.xyz[f1][d] / (2.0 * q);
        for (int e = 0; e < ne; ++e) {
          const int em = T.minus[e][d];
          const double c3 = T.xyz[e][d] / (2.0 * pq);
          for (int m = 0; m <= Lf - lf; ++m) {
            double v = QC[d] * at(m, e, f1) + WQ[d] * at(m + 1, e, f1);
            if (f2 >= 0) v += c2 * (at(m, e, f2) - rho / q * at(m + 1, e, f2));
            if (em >= 0) v += c3 * at(m + 1, em, f1);
            at(m, e, f) = v;
          }
        }
      }
      for (int e = 0; e < ne; ++e)
        for (int f = 0; f < nf; ++f) ws.acc[static_cast<size_t>(e) * nf + f] += at(0, e, f);
    }
}

// HRR on the leading index: in[e][K] (e over all |e| <= la+lb) ->
// out[a][b][K] for |a| = la, |b| = lb (local Cartesian indices).
void hrr(const double* in, int la, int lb, const double* AB, int K, std::vector<double>& out,
         Workspace& ws) {
  const CartTables& T = tables();
  const int Le = la + lb;
  const int offa = la * (la + 1) * (la + 2) / 6;
  if (lb == 0) {
    const int na = ncart(la);
    out.assign(static_cast<size_t>(na) * K, 0.0);
    for (int a = 0; a < na; ++a)
      std::memcpy(&out[static_cast<size_t>(a) * K], in + static_cast<size_t>(offa + a) * K,
                  sizeof(double) * K);
    return;
  }
  // level j: H_j[a_global over |a| in [la, Le - j]][b_local of degree j][K]
  std::vector<double>& prev = ws.h1;
  std::vector<double>& cur = ws.h2;
  const int ne = ncum(Le);
  prev.assign(static_cast<size_t>(ne) * K, 0.0);
  std::memcpy(prev.data(), in, sizeof(double) * ne * K);
  int nb_prev = 1;
  for (int j = 1; j <= lb; ++j) {
    const int nbj = ncart(j);
    const int amax = Le - j;
    const int na_all = ncum(amax);
    cur.assign(static_cast<size_t>(na_all) * nbj * K, 0.0);
    const int offb = j * (j + 1) * (j + 2) / 6;
    const int offbp = (j - 1) * j * (j + 1) / 6;
    for (int b = 0; b < nbj; ++b) {
      const int bg = offb + b;
      int d = 0;
      while (T.xyz[bg][d] == 0) ++d;
      const int bpg = T.minus[bg][d] - offbp;
      for (int a = offa; a < na_all; ++a) {
        const int ap = T.plus[a][d];
        double* dst = &cur[(static_cast<size_t>(a) * nbj + b) * K];
        const double* s1 = &prev[(static_cast<size_t>(ap) * nb_prev + bpg) * K];
        const double* s2 = &prev[(static_cast<size_t>(a) * nb_prev + bpg) * K];
        for (int k = 0; k < K; ++k) dst[k] = s1[k] + AB[d] * s2[k];
      }
    }
    std::swap(prev, cur);
    nb_prev = nbj;
  }
  const int na = ncart(la), nb = ncart(lb);
  out.assign(static_cast<size_t>(na) * nb * K, 0.0);
  for (int a = 0; a < na; ++a)
    std::memcpy(&out[static_cast<size_t>(a) * nb * K],
                &prev[(static_cast<size_t>(offa + a) * nb) * K], sizeof(double) * nb * K);
}

// Contracted spherical (ab|cd) into out[(ma,mb,mc,md)], md fastest.
// Shells with L < 0 are null (s, exponent 0, coefficient 1).
void eri_sph(const OShell& a, const OShell& b, const OShell& c, const OShell& d, double* out,
             Workspace& ws) {
  const CartTables& T = tables();
  const int la = std::max(a.L, 0), lb = std::max(b.L, 0), lc = std::max(c.L, 0),
            ld = std::max(d.L, 0);
  make_pairs(a, b, ws.bra);
  make_pairs(c, d, ws.ket);
  const int Le = la + lb, Lf = lc + ld;
  vrr_contracted(ws.bra, ws.ket, a.A, c.A, Le, Lf, ws);
  // ket HRR first: transpose acc[e][f] -> t[f][e] and run hrr over f
  const int ne = ncum(Le), nf = ncum(Lf);
  std::vector<double>& t = ws.t;
  t.resize(static_cast<size_t>(nf) * ne);
  for (int e = 0; e < ne; ++e)
    for (int f = 0; f < nf; ++f) t[static_cast<size_t>(f) * ne + e] = ws.acc[static_cast<size_t>(e) * nf + f];
  double CD[3], AB[3];
  for (int k = 0; k < 3; ++k) {
    CD[k] = c.A[k] - d.A[k];
    AB[k] = a.A[k] - b.A[k];
  }
  std::vector<double>& ketc = ws.ketc;  // [c][d][e]
  hrr(t.data(), lc, ld, CD, ne, ketc, ws);
  const int ncc = ncart(lc), ndc = ncart(ld), nac = ncart(la), nbc = ncart(lb);
  // transpose to [e][cd]
  const int ncd = ncc * ndc;
  std::vector<double>& t2 = ws.t2;
  t2.resize(static_cast<size_t>(ne) * ncd);
  for (int cd = 0; cd < ncd; ++cd)
    for (int e = 0; e < ne; ++e) t2[static_cast<size_t>(e) * ncd + cd] = ketc[static_cast<size_t>(cd) * ne + e];
  std::vector<double>& cart = ws.cart;  // [a][b][c][d]
  hrr(t2.data(), la, lb, AB, ncd, cart, ws);
  // spherical transform, one index at a time
  const std::vector<double>& Ta = T.sph[la];
  const std::vector<double>& Tb = T.sph[lb];
  const std::vector<double>& Tc = T.sph[lc];
  const std::vector<double>& Td = T.sph[ld];
  const int nsa = 2 * la + 1, nsb = 2 * lb + 1, nsc = 2 * lc + 1, nsd = 2 * ld + 1;
  // d
  std::vector<double>& s1 = ws.s1;
  s1.assign(static_cast<size_t>(nac) * nbc * ncc * nsd, 0.0);
  for (size_t x = 0; x < static_cast<size_t>(nac) * nbc * ncc; ++x)
    for (int m = 0; m < nsd; ++m) {
      double v = 0.0;
      for (int k = 0; k < ndc; ++k) v += Td[m * ndc + k] * cart[x * ndc + k];
      s1[x * nsd + m] = v;
    }
  // c
  std::vector<double>& s2 = ws.s2;
  s2.assign(static_cast<size_t>(nac) * nbc * nsc * nsd, 0.0);
  for (size_t x = 0; x < static_cast<size_t>(nac) * nbc; ++x)
    for (int m = 0; m < nsc; ++m)
      for (int r = 0; r < nsd; ++r) {
        double v = 0.0;
        for (int k = 0; k < ncc; ++k) v += Tc[m * ncc + k] * s1[(x * ncc + k) * nsd + r];
        s2[(x * nsc + m) * nsd + r] = v;
      }
  // b
  const int rest = nsc * nsd;
  std::vector<double>& s3 = ws.s3;
  s3.assign(static_cast<size_t>(nac) * nsb * rest, 0.0);
  for (int x = 0; x < nac; ++x)
    for (int m = 0; m < nsb; ++m)
      for (int r = 0; r < rest; ++r) {
        double v = 0.0;
        for (int k = 0; k < nbc; ++k)
          v += Tb[m * nbc + k] * s2[(static_cast<size_t>(x) * nbc + k) * rest + r];
        s3[(static_cast<size_t>(x) * nsb + m) * rest + r] = v;
      }
  // a
  const int rest2 = nsb * rest;
  for (int m = 0; m < nsa; ++m)
    for (int r = 0; r < rest2; ++r) {
      double v = 0.0;
      for (int k = 0; k < nac; ++k) v += Ta[m * nac + k] * s3[static_cast<size_t>(k) * rest2 + r];
      out[static_cast<size_t>(m) * rest2 + r] = v;
    }
}

// ---------------------------------------------------------------------------
// Drivers.

// intor_schwarz_aux (common/integrals/intor.f90:97-129): sqrt(||(c|c)||_F).
std::vector<double> schwarz_aux(const OBasis& B) {
  const int n = static_cast<int>(B.shells.size());
  std::vector<double> out(n);
#pragma omp parallel
  {
    Workspace ws;
    std::vector<double> blk;
#pragma omp for schedule(dynamic)
    for (int c = 0; c < n; ++c) {
      const OShell& s = B.shells[c];
      const int sz = (2 * s.L + 1) * (2 * s.L + 1);
      blk.assign(sz, 0.0);
      OShell nul = null_shell(s);
      eri_sph(s, nul, s, nul, blk.data(), ws);
      double n2 = 0.0;
      for (double v : blk) n2 += v * v;
      out[c] = std::sqrt(std::sqrt(n2));
    }
  }
  return out;
}

// intor_schwarz_bra (common/integrals/intor.f90:131-160): sqrt(||(ab|ab)||_F)
// at packed index a(a-1)/2 + b (1-based), b <= a.
// Fingerprint of a basis (every shell's L, center, exponents and
// coefficients), the key of the bra Schwarz cache.
std::vector<double> basis_key(const OBasis& B) {
  std::vector<double> k;
  for (const OShell& s : B.shells) {
    k.push_back(s.L);
    k.push_back(s.nprim);
    k.insert(k.end(), s.A, s.A + 3);
    k.insert(k.end(), s.exps.begin(), s.exps.end());
    k.insert(k.end(), s.coefs.begin(), s.coefs.end());
  }
  return k;
}

// With g_reuse_screening, the bra Schwarz vector of the last orbital basis is
// kept and reused while the basis stays the same (a timing aid: the CPU
// baseline times the three-center work of a sample of auxiliary shells, and
// the O(npairs) screening pass, once per tensor, would dominate a small
// sample). Off by default.
int g_reuse_screening = 0;
std::mutex g_sbra_mu;
std::vector<double> g_sbra_key, g_sbra_val;

std::vector<double> schwarz_bra_compute(const OBasis& B);

std::vector<double> schwarz_bra(const OBasis& B) {
  if (!g_reuse_screening) return schwarz_bra_compute(B);
  std::vector<double> key = basis_key(B);
  {
    std::lock_guard<std::mutex> lk(g_sbra_mu);
    if (key == g_sbra_key) return g_sbra_val;
  }
  std::vector<double> v = schwarz_bra_compute(B);
  std::lock_guard<std::mutex> lk(g_sbra_mu);
  g_sbra_key = std::move(key);
  g_sbra_val = v;
  return v;
}

std::vector<double> schwarz_bra_compute(const OBasis& B) {
  const int n = static_cast<int>(B.shells.size());
  std::vector<double> out(static_cast<size_t>(n) * (n + 1) / 2);
#pragma omp parallel
  {
    Workspace ws;
    std::vector<double> blk;
#pragma omp for schedule(dynamic)
    for (int a = 0; a < n; ++a)
      for (int b = 0; b <= a; ++b) {
        const OShell& sa = B.shells[a];
        const OShell& sb = B.shells[b];
        const int nab = (2 * sa.L + 1) * (2 * sb.L + 1);
        blk.assign(static_cast<size_t>(nab) * nab, 0.0);
        eri_sph(sa, sb, sa, sb, blk.data(), ws);
        double n2 = 0.0;
        for (double v : blk) n2 += v * v;
        out[static_cast<size_t>(a) * (a + 1) / 2 + b] = std::sqrt(std::sqrt(n2));
      }
  }
  return out;
}

// int2c2e_sph / intor2d_sph_symmetric (common/integrals/intor.f90:40-95):
// full symmetric (P|Q), column-major naux x naux.
std::vector<double> metric_2c2e(const OBasis& B) {
  const int n = static_cast<int>(B.shells.size());
  const int N = B.nsph;
  std::vector<double> M(static_cast<size_t>(N) * N, 0.0);
#pragma omp parallel
  {
    Workspace ws;
    std::vector<double> blk;
#pragma omp for schedule(dynamic)
    for (int a = 0; a < n; ++a)
      for (int b = a; b < n; ++b) {
        const OShell& sa = B.shells[a];
        const OShell& sb = B.shells[b];
        const int na = 2 * sa.L + 1, nb = 2 * sb.L + 1;
        blk.assign(static_cast<size_t>(na) * nb, 0.0);
        eri_sph(sa, null_shell(sa), sb, null_shell(sb), blk.data(), ws);
        for (int i = 0; i < na; ++i)
          for (int j = 0; j < nb; ++j) {
            const size_t r = sa.sph_off + i, c = sb.sph_off + j;
            M[r + c * N] = blk[static_cast<size_t>(i) * nb + j];
            M[c + r * N] = blk[static_cast<size_t>(i) * nb + j];
          }
      }
  }
  return M;
}

// inv_chol (common/linalg.f90:60-82): dpotrf("L") then dtrtri("L","N"). The
// lower triangle then holds L^-1. LAPACK's info is ignored, as in the
// reference.
void inv_chol(std::vector<double>& A, int n) {
  if (g_metric_shift != 0.0)
    for (int j = 0; j < n; ++j) A[j + static_cast<size_t>(j) * n] += g_metric_shift;
  if (p_dpotrf && p_dtrtri) {
    int info = 0;
    const char lo = 'L', nu = 'N';
    p_dpotrf(&lo, &n, A.data(), &n, &info);
    p_dtrtri(&lo, &nu, &n, A.data(), &n, &info);
    return;
  }
  double* a = A.data();
  for (int j = 0; j < n; ++j) {
    const double d = std::sqrt(a[j + static_cast<size_t>(j) * n]);
    a[j + static_cast<size_t>(j) * n] = d;
    for (int i = j + 1; i < n; ++i) a[i + static_cast<size_t>(j) * n] /= d;
#pragma omp parallel for schedule(static)
    for (int k = j + 1; k < n; ++k) {
      const double akj = a[k + static_cast<size_t>(j) * n];
      double* colk = a + static_cast<size_t>(k) * n;
      const double* colj = a + static_cast<size_t>(j) * n;
      for (int i = k; i < n; ++i) colk[i] -= colj[i] * akj;
    }
  }
  // dtrti2, lower, non-unit
  for (int j = n - 1; j >= 0; --j) {
    a[j + static_cast<size_t>(j) * n] = 1.0 / a[j + static_cast<size_t>(j) * n];
    const double ajj = -a[j + static_cast<size_t>(j) * n];
    if (j < n - 1) {
      double* x = a + static_cast<size_t>(j) * n;
      for (int jj = n - 1; jj > j; --jj) {
        const double temp = x[jj];
        const double* col = a + static_cast<size_t>(jj) * n;
        for (int i = n - 1; i > jj; --i) x[i] += temp * col[i];
        x[jj] = temp * col[jj];
      }
      for (int i = j + 1; i < n; ++i) x[i] *= ajj;
    }
  }
}

// dtrmm("L","L","N","N", n, m, 1, Linv, n, B, n): B := Linv * B.
void trmm_left_lower(const std::vector<double>& L, int n, double* Bm, int m) {
  if (p_dtrmm) {
    const char s = 'L', u = 'L', t = 'N', dg = 'N';
    const double one = 1.0;
    p_dtrmm(&s, &u, &t, &dg, &n, &m, &one, L.data(), &n, Bm, &n);
    return;
  }
#pragma omp parallel for schedule(static)
  for (int c = 0; c < m; ++c) {
    double* x = Bm + static_cast<size_t>(c) * n;
    for (int k = n - 1; k >= 0; --k) {
      const double temp = x[k];
      const double* col = L.data() + static_cast<size_t>(k) * n;
      for (int i = n - 1; i > k; --i) x[i] += temp * col[i];
      x[k] = temp * col[k];
    }
  }
}

// dtrmm("R","L","T","N", m, n, 1, Linv, n, B, m): B := B * Linv^T.
void trmm_right_lower_trans(const std::vector<double>& L, int n, double* Bm, int m) {
  if (p_dtrmm) {
    const char s = 'R', u = 'L', t = 'T', dg = 'N';
    const double one = 1.0;
    p_dtrmm(&s, &u, &t, &dg, &m, &n, &one, L.data(), &n, Bm, &m);
    return;
  }
#pragma omp parallel
  {
    std::vector<double> r(n);
#pragma omp for schedule(static)
    for (int i = 0; i < m; ++i) {
      for (int k = 0; k < n; ++k) r[k] = Bm[i + static_cast<size_t>(m) * k];
      for (int j = n - 1; j >= 0; --j) {
        double s = 0.0;
        for (int k = 0; k <= j; ++k) s += L[j + static_cast<size_t>(n) * k] * r[k];
        r[j] = s;
      }
      for (int k = 0; k < n; ++k) Bm[i + static_cast<size_t>(m) * k] = r[k];
    }
  }
}

// QVL screener data (t_df_screener%init, common/screening.f90:101-163) and
// qvl_estimate (:267-299). thresh_ws = 1d-4 at every call site
// (diabatization/intor.f90:84); the auxiliary extents use prec = 1d-8 and the
// default min_extent 0.01 (:168-196).
struct QvlScreener {
  std::vector<double> cx, cy, cz, ext_bra, den_bra;  // per bra pair a >= b, index a(a+1)/2 + b
  std::vector<double> ext_aux, beta_aux;             // per auxiliary shell
};

double auxiliary_extent(const std::vector<double>& exps, double prec, double min_extent) {
  double ext = 0.0;
  const double prec_term = -std::log(prec);
  for (double e : exps) {
    const double arg = (prec_term + 0.5 * std::log(e)) / e;
    ext = std::max(ext, arg < 0.0 ? min_extent : std::sqrt(arg));
  }
  return ext;
}

QvlScreener qvl_screener(const OBasis& B, const OBasis& X) {
  QvlScreener q;
  const double erfi = oracle_erfinv(1.0 - 1e-4);
  const int nsh = static_cast<int>(B.shells.size());
  std::vector<double> effexp(nsh);
  for (int i = 0; i < nsh; ++i)
    effexp[i] = *std::min_element(B.shells[i].exps.begin(), B.shells[i].exps.end());
  const size_t np = static_cast<size_t>(nsh) * (nsh + 1) / 2;
  q.cx.resize(np);
  q.cy.resize(np);
  q.cz.resize(np);
  q.ext_bra.resize(np);
  q.den_bra.resize(np);
  for (int a = 0; a < nsh; ++a)
    for (int b = 0; b <= a; ++b) {
      const OShell& sa = B.shells[a];
      const OShell& sb = B.shells[b];
      const size_t k = static_cast<size_t>(a) * (a + 1) / 2 + b;
      double R[3];
      oracle_contracted_center(static_cast<int>(sa.exps.size()), sa.exps.data(), sa.coefs.data(), sa.A,
                               static_cast<int>(sb.exps.size()), sb.exps.data(), sb.coefs.data(), sb.A, R);
      // contracted_extent (:198-232)
      double ext = 0.0;
      for (double ax : sa.exps)
        for (double bx : sb.exps) {
          const double px = ax + bx;
          double d2 = 0.0;
          for (int d = 0; d < 3; ++d) {
            const double P = (ax * sa.A[d] + bx * sb.A[d]) / px;
            d2 += (R[d] - P) * (R[d] - P);
          }
          ext = std::max(ext, std::sqrt(2.0 / px) * erfi + std::sqrt(d2));
        }
      q.cx[k] = R[0];
      q.cy[k] = R[1];
      q.cz[k] = R[2];
      q.ext_bra[k] = ext;
      q.den_bra[k] = std::pow(effexp[a] + effexp[b], 0.25);
    }
  for (const OShell& c : X.shells) {
    q.ext_aux.push_back(auxiliary_extent(c.exps, 1e-8, 0.01));
    const double eff = *std::min_element(c.exps.begin(), c.exps.end());
    q.beta_aux.push_back(std::pow(eff, -(2.0 * c.L + 3.0) / 4.0) * std::sqrt(double_factorial(2 * c.L - 1)));
  }
  return q;
}

double qvl_estimate(const QvlScreener& q, const OBasis& X, const std::vector<double>& sbra,
                    const std::vector<double>& saux, int a, int b, int c) {
  const size_t k = static_cast<size_t>(a) * (a + 1) / 2 + b;
  const OShell& sc = X.shells[c];
  const double dx = q.cx[k] - sc.A[0], dy = q.cy[k] - sc.A[1], dz = q.cz[k] - sc.A[2];
  const double R = std::sqrt(dx * dx + dy * dy + dz * dz);
  if (R <= q.ext_bra[k] + q.ext_aux[c]) return sbra[k] * saux[c];
  double RL = R;
  for (int l = 0; l < sc.L; ++l) RL *= R;
  return sbra[k] * PI * std::sqrt(2.0) * q.beta_aux[c] / (q.den_bra[k] * RL);
}

// contract_coulomb_densities_2d (diabatization/intor.f90:28-200).
void df_contract_2d(const OBasis& B, const OBasis& X, int ndens, int nbf, const double* D,
                    double* df) {
  const double t0 = now();
  const int naux = X.nsph;
  const int nsh = static_cast<int>(B.shells.size());
  const int nsx = static_cast<int>(X.shells.size());
  // screener (common/screening.f90:101-163)
  const std::vector<double> sbra = schwarz_bra(B);
  const std::vector<double> saux = schwarz_aux(X);
  const QvlScreener qvl = g_screening ? qvl_screener(B, X) : QvlScreener{};
  const double t1 = now();
  std::vector<double> metric = metric_2c2e(X);
  const double t2 = now();
  inv_chol(metric, naux);
  const double t3 = now();
  std::fill(df, df + static_cast<size_t>(naux) * ndens, 0.0);
  long long skipped = 0, nints = 0;
#pragma omp parallel reduction(+ : skipped, nints)
  {
    Workspace ws;
    std::vector<double> blk;
#pragma omp for schedule(dynamic)
    for (int c = 0; c < nsx; ++c) {
      const OShell& sc = X.shells[c];
      const OShell nul = null_shell(sc);
      const int nc = 2 * sc.L + 1;
      for (int a = 0; a < nsh; ++a) {
        const OShell& sa = B.shells[a];
        const int na = 2 * sa.L + 1;
        for (int b = 0; b <= a; ++b) {
          const OShell& sb = B.shells[b];
          const int nb = 2 * sb.L + 1;
          const double est = g_screening ? qvl_estimate(qvl, X, sbra, saux, a, b, c)
                                         : sbra[static_cast<size_t>(a) * (a + 1) / 2 + b] * saux[c];
          if (est < SCREEN_THRESH) {
            ++skipped;
            continue;
          }
          blk.assign(static_cast<size_t>(na) * nb * nc, 0.0);
          eri_sph(sa, sb, sc, nul, blk.data(), ws);
          nints += static_cast<long long>(na) * nb * nc;
          for (int d = 0; d < ndens; ++d) {
            int idx = 0;
            for (int i = 0; i < na; ++i)
              for (int j = 0; j < nb; ++j)
                for (int k = 0; k < nc; ++k, ++idx) {
                  const size_t gi = sa.sph_off + i, gj = sb.sph_off + j;
                  double* out = &df[(sc.sph_off + k) + static_cast<size_t>(naux) * d];
                  *out += blk[idx] * D[d + static_cast<size_t>(ndens) * (gi + nbf * gj)];
                  if (a != b) *out += blk[idx] * D[d + static_cast<size_t>(ndens) * (gj + nbf * gi)];
                }
          }
        }
      }
    }
  }
  const double t4 = now();
  if (!g_skip_metric) trmm_left_lower(metric, naux, df, ndens);
  const double t5 = now();
  g_stats.ntriplets = static_cast<long long>(nsh) * (nsh + 1) / 2 * nsx;
  g_stats.nskipped = skipped;
  g_stats.nints = nints;
  g_stats.t_screener = t1 - t0;
  g_stats.t_metric = t2 - t1;
  g_stats.t_chol = t3 - t2;
  g_stats.t_3c = t4 - t3;
  g_stats.t_trmm = t5 - t4;
  g_stats.t_total = t5 - t0;
}

// Coulomb-tensor assembly (diabatization/intor.f90:241-269).
void coulomb_4d(const double* df, int naux, int nstates, double* R) {
  int d1 = 0;
  const size_t ns = nstates;
  auto at = [&](int i, int j, int k, int l) -> double& {
    return R[i + ns * (j + ns * (k + ns * l))];
  };
  for (int i = 0; i < nstates; ++i)
    for (int j = 0; j <= i; ++j) {
      int d2 = 0;
      for (int k = 0; k <= i; ++k) {
        const int lmax = (k == i) ? j : k;
        for (int l = 0; l <= lmax; ++l) {
          double val = 0.0;
          for (int m = 0; m < naux; ++m)
            val += df[m + static_cast<size_t>(naux) * d1] * df[m + static_cast<size_t>(naux) * d2];
          at(i, j, k, l) = val;
          at(j, i, k, l) = val;
          at(i, j, l, k) = val;
          at(j, i, l, k) = val;
          at(k, l, i, j) = val;
          at(k, l, j, i) = val;
          at(l, k, i, j) = val;
          at(l, k, j, i) = val;
          ++d2;
        }
      }
      ++d1;
    }
}

// intor_df1c (std/intor.f90:15-118): (mu mu|P) then * L^-T.
void df1c(const OBasis& B, const OBasis& X, double* T) {
  const int nbf = B.nsph, naux = X.nsph;
  std::vector<double> metric = metric_2c2e(X);
  inv_chol(metric, naux);
  const std::vector<double> sbra = schwarz_bra(B);
  const std::vector<double> saux = schwarz_aux(X);
  std::fill(T, T + static_cast<size_t>(nbf) * naux, 0.0);
  const int nsh = static_cast<int>(B.shells.size()), nsx = static_cast<int>(X.shells.size());
#pragma omp parallel
  {
    Workspace ws;
    std::vector<double> blk;
#pragma omp for schedule(dynamic)
    for (int a = 0; a < nsh; ++a) {
      const OShell& sa = B.shells[a];
      const int na = 2 * sa.L + 1;
      for (int c = 0; c < nsx; ++c) {
        const OShell& sc = X.shells[c];
        const int nc = 2 * sc.L + 1;
        if (sbra[static_cast<size_t>(a) * (a + 1) / 2 + a] * saux[c] < SCREEN_THRESH) continue;
        blk.assign(static_cast<size_t>(na) * na * nc, 0.0);
        eri_sph(sa, sa, sc, null_shell(sc), blk.data(), ws);
        for (int i = 0; i < na; ++i)
          for (int k = 0; k < nc; ++k)
            T[(sa.sph_off + i) + static_cast<size_t>(nbf) * (sc.sph_off + k)] =
                blk[(static_cast<size_t>(i) * na + i) * nc + k];
      }
    }
  }
  if (!g_skip_metric) trmm_right_lower_trans(metric, naux, T, nbf);
}

// intor_df2c_mo (std/intor.f90:141-292).
void df2c_mo(const OBasis& B, const OBasis& X, int nmos, const double* C, double* out) {
  const int nbf = B.nsph, naux = X.nsph;
  const int npack = nmos * (nmos + 1) / 2;
  std::vector<double> metric = metric_2c2e(X);
  inv_chol(metric, naux);
  const std::vector<double> sbra = schwarz_bra(B);
  const std::vector<double> saux = schwarz_aux(X);
  std::fill(out, out + static_cast<size_t>(npack) * naux, 0.0);
  const int nsh = static_cast<int>(B.shells.size()), nsx = static_cast<int>(X.shells.size());
  // The reference loop is serial; aux shells own disjoint output columns, so
  // the c loop is parallelized without changing any summation order.
#pragma omp parallel
  {
    Workspace ws;
    std::vector<double> blk, tmp;
#pragma omp for schedule(dynamic)
    for (int c = 0; c < nsx; ++c) {
      const OShell& sc = X.shells[c];
      const int nc = 2 * sc.L + 1;
      for (int a = 0; a < nsh; ++a) {
        const OShell& sa = B.shells[a];
        const int na = 2 * sa.L + 1;
        for (int b = 0; b < nsh; ++b) {
          const OShell& sb = B.shells[b];
          const int nb = 2 * sb.L + 1;
          const int lo = std::min(a, b), hi = std::max(a, b);
          if (sbra[static_cast<size_t>(hi) * (hi + 1) / 2 + lo] * saux[c] < SCREEN_THRESH) continue;
          blk.assign(static_cast<size_t>(na) * nb * nc, 0.0);
          eri_sph(sa, sb, sc, null_shell(sc), blk.data(), ws);
          tmp.assign(static_cast<size_t>(nmos) * nb * nc, 0.0);  // df_tmp((mo-1)*nb + j1, k1)
          int idx = 0;
          for (int i1 = 0; i1 < na; ++i1) {
            const int i = sa.sph_off + i1;
            for (int j1 = 0; j1 < nb; ++j1)
              for (int k1 = 0; k1 < nc; ++k1, ++idx) {
                const double v = blk[idx];
                if (std::fabs(v) <= DF2C_SKIP1) continue;
                for (int mo = 0; mo < nmos; ++mo)
                  tmp[(static_cast<size_t>(mo) * nb + j1) + static_cast<size_t>(nmos) * nb * k1] +=
                      C[i + static_cast<size_t>(nbf) * mo] * v;
              }
          }
          for (int mo1 = 0; mo1 < nmos; ++mo1)
            for (int j1 = 0; j1 < nb; ++j1) {
              const int j = sb.sph_off + j1;
              for (int k1 = 0; k1 < nc; ++k1) {
                const int k = sc.sph_off + k1;
                const double v =
                    tmp[(static_cast<size_t>(mo1) * nb + j1) + static_cast<size_t>(nmos) * nb * k1];
                if (std::fabs(v) <= DF2C_SKIP2) continue;
                for (int mo2 = 0; mo2 <= mo1; ++mo2) {
                  const size_t pk = static_cast<size_t>(mo1) * (mo1 + 1) / 2 + mo2;
                  out[pk + static_cast<size_t>(npack) * k] += C[j + static_cast<size_t>(nbf) * mo2] * v;
                }
              }
            }
        }
      }
    }
  }
  if (!g_skip_metric) trmm_right_lower_trans(metric, naux, out, npack);
}

// erfinv: rational approximations of Blair, Edwards and Johnson (1976),
// tables 17, 37 and 57, as used by common/erfinv.f90:88-127.
const double P17[7] = {0.160304955844066229311e2, -0.90784959262960326650e2,
                       0.18644914861620987391e3,  -0.16900142734642382420e3,
                       0.6545466284794487048e2,   -0.864213011587247794e1,
                       0.176058782139590e0};
const double Q17[7] = {0.147806470715138316110e2, -0.91374167024260313936e2,
                       0.21015790486205317714e3,  -0.22210254121855132366e3,
                       0.10760453916055123830e3,  -0.206010730328265443e2,
                       0.1000000000000000e1};
const double P37[8] = {-0.152389263440726128e-1, 0.3444556924136125216e0,
                       -0.29344398672542478687e1, 0.11763505705217627302e2,
                       -0.22655292823101104193e2, 0.19121334396580330163e2,
                       -0.5478927619598318769e1,  0.237516689024448000e0};
const double Q37[8] = {-0.108465169602059954e-1, 0.2610628885843078511e0,
                       -0.24068318104393757995e1, 0.10695129973387014469e2,
                       -0.23716715521596581025e2, 0.24640158943917284883e2,
                       -0.10014376349783070835e2, 0.1000000000000000000e1};
const double P57[9] = {0.3100808562552958465e-4,  0.40974876030119399241e-2,
                       0.1214902662897276161664e0, 0.11091676946390282026357e1,
                       0.32283798556639239484387e1, 0.2881691815651598826211e1,
                       0.2047972087262996049729e1, 0.854592208197214832806e0,
                       0.3551095884622383139e-2};
const double Q57[9] = {0.3100809298564522487e-4,  0.40975286786639145041e-2,
                       0.1215907800748757143068e0, 0.11186271676316964210428e1,
                       0.34323639843052901805054e1, 0.4140284677116202150554e1,
                       0.4119797271272204121285e1, 0.2162961962641434560920e1,
                       0.10000000000000000000000e1};

double rational(double x, double base0, const double* P, const double* Q, int n) {
  double num = 0.0, den = 0.0, base = 1.0;
  for (int i = 0; i < n; ++i) {
    num += P[i] * base;
    den += Q[i] * base;
    base *= base0;
  }
  return x * num / den;
}

// ---------------------------------------------------------------------------
// Grid densities (grid/grid.f90) and GDMA primitive densities
// (gdma/prim_dens.f90). Cartesian functions in pysisyphus order (x^L, x^(L-1) y,
// x^(L-1) z, ..., z^L), each scaled by 1/sqrt((2i-1)!! (2j-1)!! (2k-1)!!) --
// the NORM2 / NORM3 / NORM4 / NORM22 constants of grid.f90:9-13.

constexpr double GRID_CUTOFF = -36.0;  // grid.f90:9, prim_dens.f90:13

double cart_norm(int i, int j, int k) {
  auto df = [](int n) {  // (2n - 1)!!
    double r = 1.0;
    for (int m = 2 * n - 1; m > 1; m -= 2) r *= m;
    return r;
  };
  return 1.0 / std::sqrt(df(i) * df(j) * df(k));
}

// Powers (i, j, k) of Cartesian component c of degree L in pysisyphus order.
void cart_powers(int L, int c, int* i, int* j, int* k) {
  int idx = 0;
  for (int a = L; a >= 0; --a)
    for (int b = L - a; b >= 0; --b) {
      if (idx == c) {
        *i = a;
        *j = b;
        *k = L - a - b;
        return;
      }
      ++idx;
    }
}

double ipow(double x, int n) {
  double r = 1.0;
  for (int m = 0; m < n; ++m) r *= x;
  return r;
}

// cart_gto3d_rel (grid.f90:17-108): the Cartesian functions of one shell at
// offset RA from its center; exp arguments below -36 are skipped.
void cart_gto3d(const OShell& s, const double* RA, double* out) {
  const int nc = (s.L + 1) * (s.L + 2) / 2;
  for (int c = 0; c < nc; ++c) out[c] = 0.0;
  const double dist = RA[0] * RA[0] + RA[1] * RA[1] + RA[2] * RA[2];
  for (int p = 0; p < s.nprim; ++p) {
    const double arg = -s.exps[p] * dist;
    if (arg < GRID_CUTOFF) continue;
    const double e = s.coefs[p] * std::exp(arg);
    for (int c = 0; c < nc; ++c) {
      int i = 0, j = 0, k = 0;
      cart_powers(s.L, c, &i, &j, &k);
      out[c] += cart_norm(i, j, k) * ipow(RA[0], i) * ipow(RA[1], j) * ipow(RA[2], k) * e;
    }
  }
}

// eval_densities (grid.f90:110-286): blocks of blk_size points; per block the
// Cartesian functions, their mean |values| over the block, then every pair
// nu <= mu whose estimate factor * D(j, mu, nu) * mean(nu) * mean(mu) reaches
// thresh adds factor * D(j, mu, nu) chi(:, mu) chi(:, nu).
void eval_densities(const OBasis& B, int npoints, const double* grid3d, int ndens, int nbfs,
                    const double* D, double* rho, int blk_size, double thresh) {
  std::vector<int> cart_off(B.shells.size() + 1, 0);
  for (size_t a = 0; a < B.shells.size(); ++a)
    cart_off[a + 1] = cart_off[a] + (B.shells[a].L + 1) * (B.shells[a].L + 2) / 2;
  const int ncart = cart_off.back();
  std::fill(rho, rho + static_cast<size_t>(ndens) * npoints, 0.0);
  if (blk_size <= 0 || ncart != nbfs) return;
  const int nblks = (npoints + blk_size - 1) / blk_size;
#pragma omp parallel
  {
    std::vector<double> chis(static_cast<size_t>(blk_size) * ncart), mean(ncart);
    std::vector<double> scratch(static_cast<size_t>(ndens) * blk_size * ncart);
    std::vector<char> contributed(static_cast<size_t>(ndens) * ncart);
#pragma omp for schedule(dynamic)
    for (int blk = 0; blk < nblks; ++blk) {
      const int start = blk * blk_size;
      const int n = std::min(blk_size, npoints - start);
      for (int i = 0; i < n; ++i) {
        const double* R = grid3d + 3 * static_cast<size_t>(start + i);
        for (size_t a = 0; a < B.shells.size(); ++a) {
          const OShell& sh = B.shells[a];
          const double RA[3] = {R[0] - sh.A[0], R[1] - sh.A[1], R[2] - sh.A[2]};
          double v[15];
          cart_gto3d(sh, RA, v);
          for (int c = 0; c < cart_off[a + 1] - cart_off[a]; ++c)
            chis[i + static_cast<size_t>(blk_size) * (cart_off[a] + c)] = v[c];
        }
      }
      for (int nu = 0; nu < ncart; ++nu) {
        double m = 0.0;
        for (int i = 0; i < n; ++i) m += std::fabs(chis[i + static_cast<size_t>(blk_size) * nu]);
        mean[nu] = m / n;
      }
      std::fill(scratch.begin(), scratch.end(), 0.0);
      std::fill(contributed.begin(), contributed.end(), 0);
      for (int nu = 0; nu < ncart; ++nu)
        for (int mu = nu; mu < ncart; ++mu) {
          const double f = nu == mu ? 1.0 : 2.0;
          for (int j = 0; j < ndens; ++j) {
            const double dnm = D[j + static_cast<size_t>(ndens) * (mu + static_cast<size_t>(nbfs) * nu)];
            const double contrib = f * dnm * mean[nu] * mean[mu];
            if (std::fabs(contrib) >= thresh) {
              double* sc = &scratch[static_cast<size_t>(j) + static_cast<size_t>(ndens) * blk_size * nu];
              const double* cm = &chis[static_cast<size_t>(blk_size) * mu];
              for (int i = 0; i < n; ++i) sc[static_cast<size_t>(ndens) * i] += f * dnm * cm[i];
              contributed[j + static_cast<size_t>(ndens) * nu] = 1;
            }
          }
        }
      for (int nu = 0; nu < ncart; ++nu)
        for (int j = 0; j < ndens; ++j) {
          if (!contributed[j + static_cast<size_t>(ndens) * nu]) continue;
          for (int i = 0; i < n; ++i)
            rho[j + static_cast<size_t>(ndens) * (start + i)] +=
                scratch[j + static_cast<size_t>(ndens) * (i + static_cast<size_t>(blk_size) * nu)] *
                chis[i + static_cast<size_t>(blk_size) * nu];
        }
    }
  }
}

// f_eval_prim_density (gdma/prim_dens.f90:100-259). ls_inds(2, nprims) = (L,
// 0-based Cartesian start index); primdata(5, nprims) = (coefficient,
// exponent, x, y, z); P(nbfs, nbfs) column-major. Pairs ai <= bi with
// ax + bx < switch; a pair is skipped when -mu * (sum_d (A_d - B_d))^2 <= -36
// -- the reference squares the sum of the differences there
// (prim_dens.f90:212), not the sum of their squares; its prefactor K uses the
// squared distance. Cartesian prefactors as prefacts (:17-92) for L <= 3; for
// L = 4 the 15 components of grid.f90's order (prefacts fills 14 of them and
// leaves the 15th unset).
void eval_prim_density(int nprims, int npoints, int nbfs, const int* ls_inds, const double* primdata,
                       const double* coords3d, const double* P, double sw, double* rho) {
  std::fill(rho, rho + npoints, 0.0);
#pragma omp parallel
  {
    std::vector<double> loc(npoints, 0.0);
    double pa[15], pb[15];
#pragma omp for schedule(dynamic)
    for (int ai = 0; ai < nprims; ++ai) {
      const double da = primdata[5 * ai], ax = primdata[5 * ai + 1];
      const double* A = primdata + 5 * ai + 2;
      const int La = ls_inds[2 * ai], ia = ls_inds[2 * ai + 1];
      const int na = (La + 1) * (La + 2) / 2;
      for (int bi = ai; bi < nprims; ++bi) {
        const double db = primdata[5 * bi], bx = primdata[5 * bi + 1];
        if (ax + bx >= sw) continue;
        const double* Bc = primdata + 5 * bi + 2;
        const int Lb = ls_inds[2 * bi], ib = ls_inds[2 * bi + 1];
        const int nb = (Lb + 1) * (Lb + 2) / 2;
        const double px = ax + bx, mux = ax * bx / px;
        const double dsum = (A[0] - Bc[0]) + (A[1] - Bc[1]) + (A[2] - Bc[2]);
        if (-mux * dsum * dsum <= GRID_CUTOFF) continue;
        const double AB2 = (A[0] - Bc[0]) * (A[0] - Bc[0]) + (A[1] - Bc[1]) * (A[1] - Bc[1]) +
                           (A[2] - Bc[2]) * (A[2] - Bc[2]);
        const double K = da * db * (ai == bi ? 1.0 : 2.0) * std::exp(-mux * AB2);
        const double Pc[3] = {(ax * A[0] + bx * Bc[0]) / px, (ax * A[1] + bx * Bc[1]) / px,
                              (ax * A[2] + bx * Bc[2]) / px};
        for (int i = 0; i < npoints; ++i) {
          const double* R = coords3d + 3 * static_cast<size_t>(i);
          const double r2 = (R[0] - Pc[0]) * (R[0] - Pc[0]) + (R[1] - Pc[1]) * (R[1] - Pc[1]) +
                            (R[2] - Pc[2]) * (R[2] - Pc[2]);
          if (-px * r2 <= GRID_CUTOFF) continue;
          const double Pexp = std::exp(-px * r2);
          for (int c = 0; c < na; ++c) {
            int x = 0, y = 0, z = 0;
            cart_powers(La, c, &x, &y, &z);
            pa[c] = cart_norm(x, y, z) * ipow(R[0] - A[0], x) * ipow(R[1] - A[1], y) * ipow(R[2] - A[2], z);
          }
          for (int c = 0; c < nb; ++c) {
            int x = 0, y = 0, z = 0;
            cart_powers(Lb, c, &x, &y, &z);
            pb[c] = cart_norm(x, y, z) * ipow(R[0] - Bc[0], x) * ipow(R[1] - Bc[1], y) * ipow(R[2] - Bc[2], z);
          }
          double acc = 0.0;
          for (int nu = 0; nu < na; ++nu)
            for (int mu = 0; mu < nb; ++mu)
              acc += K * Pexp * P[(ia + nu) + static_cast<size_t>(nbfs) * (ib + mu)] * pa[nu] * pb[mu];
          loc[i] += acc;
        }
      }
    }
#pragma omp critical
    for (int i = 0; i < npoints; ++i) rho[i] += loc[i];
  }
}

// benchmark_int3c2e (intor/benchmark.f90:15-132): for every shell pair a >= b
// that is not concentric (|A - B| > 1e-6) and whose bra Schwarz value exceeds
// 1e-10, and every auxiliary shell c, the record (schwarz_estimate,
// qvl_estimate, ||(ab|c)||_2 over the block, |contracted center - C|) in the
// reference's loop order; *nskipped counts records with qvl_estimate < 1e-10
// (REAL(4) literal, promoted). Returns the number of records; writes at most
// cap records.
long long int3c2e_estimates(const OBasis& B, const OBasis& X, long long cap, double* rec, long long* nskipped) {
  const int nsh = static_cast<int>(B.shells.size()), nsx = static_cast<int>(X.shells.size());
  const std::vector<double> sbra = schwarz_bra(B);
  const std::vector<double> saux = schwarz_aux(X);
  const QvlScreener q = qvl_screener(B, X);
  std::vector<std::pair<int, int>> pairs;
  for (int a = 0; a < nsh; ++a)
    for (int b = 0; b <= a; ++b) {
      const OShell& sa = B.shells[a];
      const OShell& sb = B.shells[b];
      double d2 = 0.0;
      for (int d = 0; d < 3; ++d) d2 += (sa.A[d] - sb.A[d]) * (sa.A[d] - sb.A[d]);
      const bool concentric = std::sqrt(d2) <= 1e-6;
      const bool small = sbra[static_cast<size_t>(a) * (a + 1) / 2 + b] <= 1e-10;
      if (!concentric && !small) pairs.push_back({a, b});
    }
  const long long n = static_cast<long long>(pairs.size()) * nsx;
  long long skipped = 0;
#pragma omp parallel reduction(+ : skipped)
  {
    Workspace ws;
    std::vector<double> blk;
#pragma omp for schedule(dynamic)
    for (long long r = 0; r < n; ++r) {
      const int a = pairs[r / nsx].first, b = pairs[r / nsx].second, c = static_cast<int>(r % nsx);
      const size_t k = static_cast<size_t>(a) * (a + 1) / 2 + b;
      const double sch = sbra[k] * saux[c];
      const double qvl = qvl_estimate(q, X, sbra, saux, a, b, c);
      if (qvl < SCREEN_THRESH) ++skipped;
      if (r >= cap) continue;
      const OShell& sa = B.shells[a];
      const OShell& sb = B.shells[b];
      const OShell& sc = X.shells[c];
      blk.assign(static_cast<size_t>(2 * sa.L + 1) * (2 * sb.L + 1) * (2 * sc.L + 1), 0.0);
      eri_sph(sa, sb, sc, null_shell(sc), blk.data(), ws);
      double ss = 0.0;
      for (double v : blk) ss += v * v;
      const double dx = q.cx[k] - sc.A[0], dy = q.cy[k] - sc.A[1], dz = q.cz[k] - sc.A[2];
      rec[4 * r + 0] = sch;
      rec[4 * r + 1] = qvl;
      rec[4 * r + 2] = std::sqrt(ss);
      rec[4 * r + 3] = std::sqrt(dx * dx + dy * dy + dz * dz);
    }
  }
  *nskipped = skipped;
  return n;
}

}  // namespace

// ---------------------------------------------------------------------------
// C-ABI

extern "C" {

void oracle_set_boys_mode(int mode) { g_boys_mode = mode; }
int oracle_get_boys_mode(void) { return g_boys_mode; }
void oracle_set_skip_metric(int skip) { g_skip_metric = skip ? 1 : 0; }
void oracle_set_metric_shift(double shift) { g_metric_shift = shift; }
void oracle_set_screening(int mode) { g_screening = mode ? 1 : 0; }
void oracle_set_reuse_screening(int reuse) { g_reuse_screening = reuse ? 1 : 0; }
void oracle_set_threads(int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
}
int oracle_get_threads(void) { return omp_get_max_threads(); }
void oracle_register_lapack(void* dpotrf, void* dtrtri, void* dtrmm, void* dgemm) {
  p_dpotrf = reinterpret_cast<dpotrf_t>(dpotrf);
  p_dtrtri = reinterpret_cast<dtrtri_t>(dtrtri);
  p_dtrmm = reinterpret_cast<dtrmm_t>(dtrmm);
  p_dgemm = reinterpret_cast<dgemm_t>(dgemm);
}

void oracle_boys(int nmax, double x, double* out) { boys(nmax, x, out); }

double oracle_erfinv(double x) {
  const double ax = std::fabs(x);
  if (ax <= 0.75) return rational(x, x * x - 0.5625, P17, Q17, 7);
  if (ax <= 0.9375) return rational(x, x * x - 0.87890625, P37, Q37, 8);
  const double base = 1.0 / std::sqrt(-std::log(1.0 - ax));
  return rational(std::copysign(1.0, x) / base, base, P57, Q57, 9);
}

// contracted_center (common/screening.f90:235-265).
void oracle_contracted_center(int na, const double* axs, const double* das, const double* A,
                              int nb, const double* bxs, const double* dbs, const double* B,
                              double* R) {
  double denom = 0.0;
  R[0] = R[1] = R[2] = 0.0;
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) {
      const double px = axs[i] + bxs[j];
      const double w = std::fabs(das[i] * dbs[j]);
      for (int d = 0; d < 3; ++d) R[d] += w * (axs[i] * A[d] + bxs[j] * B[d]) / px;
      denom += w;
    }
  for (int d = 0; d < 3; ++d) R[d] /= denom;
}

int oracle_eri_block(int La, int na, const double* ea, const double* ca, const double* A,
                     int Lb, int nb, const double* eb, const double* cb, const double* B,
                     int Lc, int nc, const double* ec, const double* cc, const double* C,
                     int Ld, int nd, const double* ed, const double* cd, const double* D,
                     double* out) {
  auto mk = [](int L, int n, const double* e, const double* c, const double* X) {
    OShell s;
    s.L = L;
    std::copy(X, X + 3, s.A);
    if (L < 0) {
      s.nprim = 1;
      s.exps = {0.0};
      s.coefs = {1.0};
      return s;
    }
    s.nprim = n;
    s.exps.assign(e, e + n);
    s.coefs.assign(c, c + n);
    norm_cgto_coeffs(s.coefs, s.exps, L);
    return s;
  };
  if (La > MAXL || Lb > MAXL || Lc > MAXL || Ld > MAXL) return 1;
  Workspace ws;
  eri_sph(mk(La, na, ea, ca, A), mk(Lb, nb, eb, cb, B), mk(Lc, nc, ec, cc, C),
          mk(Ld, nd, ed, cd, D), out, ws);
  return 0;
}

void oracle_init(void) { (void)tables(); }

void oracle_int_schwarz_aux(int nshells, int, const int* bc, const int* bs, const double* bd,
                            double* integrals) {
  const OBasis B = make_basis(nshells, bc, bs, bd);
  const std::vector<double> v = schwarz_aux(B);
  std::copy(v.begin(), v.end(), integrals);
}

void oracle_int_schwarz_bra(int nshells, int, const int* bc, const int* bs, const double* bd,
                            double* integrals) {
  const OBasis B = make_basis(nshells, bc, bs, bd);
  const std::vector<double> v = schwarz_bra(B);
  std::copy(v.begin(), v.end(), integrals);
}

void oracle_int2c2e_metric(int nshells, int, const int* bc, const int* bs, const double* bd,
                           int, double* metric) {
  const OBasis B = make_basis(nshells, bc, bs, bd);
  const std::vector<double> v = metric_2c2e(B);
  std::copy(v.begin(), v.end(), metric);
}

void oracle_contract_coulomb_densities_2d(int nshells, int, const int* bc, const int* bs,
                                          const double* bd, int nshells_aux, int,
                                          const int* bca, const int* bsa, const double* bda,
                                          int ndens, int nbfs, const double* densities, int,
                                          double* df_tensor) {
  const OBasis B = make_basis(nshells, bc, bs, bd);
  const OBasis X = make_basis(nshells_aux, bca, bsa, bda);
  df_contract_2d(B, X, ndens, nbfs, densities, df_tensor);
}

void oracle_contract_coulomb_densities_4d(int nshells, int, const int* bc, const int* bs,
                                          const double* bd, int nshells_aux, int,
                                          const int* bca, const int* bsa, const double* bda,
                                          int ndens, int nbfs, const double* densities,
                                          int nstates, double* coulomb_tensor) {
  const OBasis B = make_basis(nshells, bc, bs, bd);
  const OBasis X = make_basis(nshells_aux, bca, bsa, bda);
  std::vector<double> df(static_cast<size_t>(X.nsph) * ndens);
  df_contract_2d(B, X, ndens, nbfs, densities, df.data());
  coulomb_4d(df.data(), X.nsph, nstates, coulomb_tensor);
}

void oracle_intor_eri2c(int nshells, int, const int* bc, const int* bs, const double* bd,
                        int nshells_aux, int, const int* bca, const int* bsa, const double* bda,
                        int nbfs, double* eri2c) {
  const OBasis B = make_basis(nshells, bc, bs, bd);
  const OBasis X = make_basis(nshells_aux, bca, bsa, bda);
  const int naux = X.nsph;
  std::vector<double> T(static_cast<size_t>(nbfs) * naux);
  df1c(B, X, T.data());
  // dgemm("N","T", nbfs, nbfs, naux, 1, T, nbfs, T, nbfs, 0, eri2c, nbfs) (std/intor.f90:137)
  if (p_dgemm) {
    const char n = 'N', t = 'T';
    const double one = 1.0, zero = 0.0;
    p_dgemm(&n, &t, &nbfs, &nbfs, &naux, &one, T.data(), &nbfs, T.data(), &nbfs, &zero, eri2c,
            &nbfs);
    return;
  }
#pragma omp parallel for schedule(dynamic)
  for (int j = 0; j < nbfs; ++j)
    for (int i = 0; i < nbfs; ++i) {
      double v = 0.0;
      for (int k = 0; k < naux; ++k)
        v += T[i + static_cast<size_t>(nbfs) * k] * T[j + static_cast<size_t>(nbfs) * k];
      eri2c[i + static_cast<size_t>(nbfs) * j] = v;
    }
}

void oracle_intor_df1c(int nshells, int, const int* bc, const int* bs, const double* bd,
                       int nshells_aux, int, const int* bca, const int* bsa, const double* bda,
                       int, int, double* out) {
  const OBasis B = make_basis(nshells, bc, bs, bd);
  const OBasis X = make_basis(nshells_aux, bca, bsa, bda);
  df1c(B, X, out);
}

void oracle_intor_df2c_mo(int nshells, int, const int* bc, const int* bs, const double* bd,
                          int nshells_aux, int, const int* bca, const int* bsa, const double* bda,
                          int, int nmos, const double* mo_tensor, int, double* out) {
  const OBasis B = make_basis(nshells, bc, bs, bd);
  const OBasis X = make_basis(nshells_aux, bca, bsa, bda);
  df2c_mo(B, X, nmos, mo_tensor, out);
}

void oracle_last_stats(OracleStats* out) { *out = g_stats; }

long long oracle_int3c2e_estimates(int nshells, int, const int* bc, const int* bs, const double* bd,
                                   int nshells_aux, int, const int* bca, const int* bsa, const double* bda,
                                   long long cap, double* records, long long* nskipped) {
  const OBasis B = make_basis(nshells, bc, bs, bd);
  const OBasis X = make_basis(nshells_aux, bca, bsa, bda);
  return int3c2e_estimates(B, X, cap, records, nskipped);
}

void oracle_eval_densities(int nshells, int, const int* bc, const int* bs, const double* bd, int npoints,
                           const double* grid3d, int ndens, int nbfs, const double* densities,
                           double* grid_densities, int blk_size, double thresh) {
  const OBasis B = make_basis(nshells, bc, bs, bd);
  eval_densities(B, npoints, grid3d, ndens, nbfs, densities, grid_densities, blk_size, thresh);
}

void oracle_eval_prim_density(int nprims, int npoints, int nbfs, const int* ls_inds, const double* primdata,
                              const double* coords3d, const double* P, double sw, double* rho) {
  eval_prim_density(nprims, npoints, nbfs, ls_inds, primdata, coords3d, P, sw, rho);
}

// Extended-precision factor and solve (x87 long double: 64-bit significand,
// unit roundoff 5.4e-20, against 1.1e-16 in double). Not part of the
// reference: a checker for FP64 factorizations of ill-conditioned metrics.
// M is n x n column-major (lower triangle read), B is n x nrhs column-major.
// L = chol(M) and Y = L^-1 B are formed in long double; Y (and, when L_out is
// given, L, rounded, upper triangle zero) are returned in double.
// Returns 0, or the 1-based column of the first non-positive pivot.
int oracle_chol_solve_ld(int n, const double* M, int nrhs, const double* B, double* Y,
                         double* L_out) {
  typedef long double ld;
  std::vector<ld> L(static_cast<size_t>(n) * n, 0.0L);  // row-major: L[i * n + k]
  for (int i = 0; i < n; ++i)
    for (int k = 0; k <= i; ++k) L[static_cast<size_t>(i) * n + k] = M[i + static_cast<size_t>(k) * n];
  int info = 0;
  for (int j = 0; j < n && info == 0; ++j) {
    ld* Lj = L.data() + static_cast<size_t>(j) * n;
    ld d = Lj[j];
    for (int k = 0; k < j; ++k) d -= Lj[k] * Lj[k];
    if (!(d > 0.0L)) {
      info = j + 1;
      break;
    }
    d = std::sqrt(d);
    Lj[j] = d;
#pragma omp parallel for schedule(static)
    for (int i = j + 1; i < n; ++i) {
      ld* Li = L.data() + static_cast<size_t>(i) * n;
      ld s = Li[j];
      for (int k = 0; k < j; ++k) s -= Li[k] * Lj[k];
      Li[j] = s / d;
    }
  }
  if (info) return info;
#pragma omp parallel
  {
    std::vector<ld> y(n);
#pragma omp for schedule(static)
    for (int r = 0; r < nrhs; ++r) {
      for (int i = 0; i < n; ++i) {
        const ld* Li = L.data() + static_cast<size_t>(i) * n;
        ld s = B[i + static_cast<size_t>(n) * r];
        for (int k = 0; k < i; ++k) s -= Li[k] * y[k];
        y[i] = s / Li[i];
      }
      for (int i = 0; i < n; ++i) Y[i + static_cast<size_t>(n) * r] = static_cast<double>(y[i]);
    }
  }
  if (L_out)
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i)
        L_out[i + static_cast<size_t>(n) * j] =
            i >= j ? static_cast<double>(L[static_cast<size_t>(i) * n + j]) : 0.0;
  return 0;
}

// ||L L^T - M||_F / ||M||_F in long double, for L the lower triangle of the
// column-major n x n array Lc (its upper triangle is ignored): the backward
// error of a Cholesky factor.
double oracle_chol_backward_error_ld(int n, const double* M, const double* Lc) {
  typedef long double ld;
  std::vector<ld> L(static_cast<size_t>(n) * n, 0.0L);  // row-major lower
  for (int i = 0; i < n; ++i)
    for (int k = 0; k <= i; ++k) L[static_cast<size_t>(i) * n + k] = Lc[i + static_cast<size_t>(k) * n];
  ld num = 0.0L, den = 0.0L;
#pragma omp parallel for schedule(dynamic) reduction(+ : num, den)
  for (int i = 0; i < n; ++i) {
    const ld* Li = L.data() + static_cast<size_t>(i) * n;
    for (int j = 0; j <= i; ++j) {
      const ld* Lj = L.data() + static_cast<size_t>(j) * n;
      ld s = 0.0L;
      for (int k = 0; k <= j; ++k) s += Li[k] * Lj[k];
      const ld m = M[i + static_cast<size_t>(j) * n];
      const ld w = i == j ? 1.0L : 2.0L;  // symmetric: count the mirrored entry
      num += w * (s - m) * (s - m);
      den += w * m * m;
    }
  }
  return static_cast<double>(std::sqrt(num / den));
}


}  // extern "C"
