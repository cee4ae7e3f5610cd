// Host orchestration and C-ABI of libpa_b200.so.
//
// The density-fitting path (diabatization/intor.f90:28-270) runs entirely on
// the current CUDA device:
//   Schwarz vectors (k_schwarz_bra / k_schwarz_aux)  -> screening
//   class-wise sort of bra units and auxiliary shells by Schwarz value (CUB)
//   density folding of the bra units (k_bra_prep)
//   metric (P|Q) (k_metric) -> Cholesky (k_linalg)
//   screened 3c2e contraction (k_df3c<LAB,LC>) -> ordered reduction
//   B = L^-1 df (blocked forward substitution) [-> Coulomb tensor]
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <limits>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <fstream>
#include <list>
#include <memory>
#include <mutex>
#include <optional>
#include <sstream>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "boys.cuh"
#include "k_df3c.cuh"
#include "k_integrals.cuh"
#include "k_linalg.cuh"
#include "k_std.cuh"
#include "pa_b200.h"
#include "pa_internal.h"

namespace pa {

namespace {

thread_local std::string tl_err;

// NVTX range over the host-side enqueue of one phase (header-only NVTX v3:
// no cost without a tool attached; Nsight Systems shows the ranges on the CPU
// timeline, Nsight Compute can filter launches by them with --nvtx).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

int fail(int code, const std::string& msg) {
  tl_err = msg;
  return code;
}

std::mutex g_opt_mu;
Options g_opts;
pa_stats g_stats{};

// Applies "L_ab L_c variant" lines of a tile table (# starts a comment) to
// g_opts; returns the number of entries applied, -1 if the file cannot be read,
// -2 on a malformed or out-of-range entry (nothing applied then).
int apply_tile_table(const char* path) {
  std::ifstream in(path);
  if (!in) return -1;
  std::vector<int> ent;
  std::string line;
  while (std::getline(in, line)) {
    const size_t h = line.find('#');
    if (h != std::string::npos) line.resize(h);
    std::istringstream ls(line);
    int lab, lc, v;
    if (!(ls >> lab)) continue;
    std::string rest;
    if (!(ls >> lc >> v) || (ls >> rest)) return -2;
    if (lab < 0 || lab > 2 * PA_LMAX || lc < 0 || lc > PA_LAUXMAX || v < 0 || v >= kDf3cVariants) return -2;
    ent.insert(ent.end(), {lab, lc, v});
  }
  std::lock_guard<std::mutex> lk(g_opt_mu);
  for (size_t i = 0; i < ent.size(); i += 3)
    g_opts.tile_variant[ent[i]][ent[i + 1]] = static_cast<signed char>(ent[i + 2]);
  return static_cast<int>(ent.size() / 3);
}

// The tile table read once per process: $PA_B200_TILE_TABLE when set (empty:
// none), else df3c_tiles.txt beside this library when present.
std::string default_tile_table() {
  if (const char* env = std::getenv("PA_B200_TILE_TABLE")) return env;
  Dl_info info{};
  if (!dladdr(reinterpret_cast<void*>(&apply_tile_table), &info) || !info.dli_fname) return "";
  std::string lib = info.dli_fname;
  const size_t slash = lib.rfind('/');
  return (slash == std::string::npos ? std::string() : lib.substr(0, slash + 1)) + "df3c_tiles.txt";
}

static_assert(kDf3cVariants == PA_TILE_VARIANTS, "tile variants of the header and the kernels agree");
std::once_flag g_tile_once;

Options options() {
  std::call_once(g_tile_once, [] {
    const std::string path = default_tile_table();
    if (!path.empty()) apply_tile_table(path.c_str());
  });
  std::lock_guard<std::mutex> lk(g_opt_mu);
  return g_opts;
}

#define PA_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(PA_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));   \
  } while (0)

}  // namespace

// Records the calling thread's error message for pa_last_error (used by the
// C-ABI entry points in other translation units).
int set_error(int code, const std::string& msg) { return fail(code, msg); }

// ---------------------------------------------------------------------------
// Basis unpacking: common/shells.f90:97-187 and common/normalization.f90:10-38.
int unpack_basis(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                 const double* bas_data, int lmax_allowed, HostBasis* out, std::string* err) {
  if (nshells < 0 || ndata < 0) {
    *err = "negative basis sizes";
    return PA_ERR_ARG;
  }
  if (nshells > 0 && (!bas_centers || !bas_spec || !bas_data)) {
    *err = "null basis array";
    return PA_ERR_ARG;
  }
  HostBasis b;
  b.shells.resize(nshells);
  int sph = 0;
  for (int i = 0; i < nshells; ++i) {
    HostShell& s = b.shells[i];
    const long long cptr = bas_centers[i + 2LL * nshells];
    const int L = bas_spec[i + 1LL * nshells];
    const int nprim = bas_spec[i + 2LL * nshells];
    const long long ptr = bas_spec[i + 4LL * nshells];
    if (L < 0) {
      *err = "shell " + std::to_string(i) + ": L must be >= 0";
      return PA_ERR_ARG;
    }
    if (L > lmax_allowed) {
      *err = "shell " + std::to_string(i) + ": L = " + std::to_string(L) +
             " exceeds the compiled maximum " + std::to_string(lmax_allowed);
      return PA_ERR_LMAX;
    }
    if (nprim < 1) {
      *err = "shell " + std::to_string(i) + ": needs at least one primitive";
      return PA_ERR_ARG;
    }
    if (cptr < 1 || cptr + 2 > ndata || ptr < 1 || ptr + 2LL * nprim - 1 > ndata) {
      *err = "shell " + std::to_string(i) + ": pointer outside bas_data (truncated basis?)";
      return PA_ERR_ARG;
    }
    for (int d = 0; d < 3; ++d) s.A[d] = bas_data[cptr - 1 + d];
    s.L = L;
    s.nprim = nprim;
    s.prim_off = static_cast<int>(b.exps.size());
    s.sph_off = sph;
    sph += 2 * L + 1;
    std::vector<double> c(bas_data + ptr - 1, bas_data + ptr - 1 + nprim);
    std::vector<double> e(bas_data + ptr - 1 + nprim, bas_data + ptr - 1 + 2 * nprim);
    bool finite = std::isfinite(s.A[0]) && std::isfinite(s.A[1]) && std::isfinite(s.A[2]);
    for (int k = 0; k < nprim; ++k) finite = finite && std::isfinite(c[k]) && std::isfinite(e[k]) && e[k] > 0.0;
    if (!finite) {
      *err = "shell " + std::to_string(i) + ": non-finite center, coefficient or non-positive exponent";
      return PA_ERR_ARG;
    }
    double N = 0.0;
    const double lp = L + 1.5;
    for (int p = 0; p < nprim; ++p)
      for (int q = 0; q < nprim; ++q)
        N += c[p] * c[q] / std::pow(e[p] + e[q], lp) * std::pow(std::sqrt(e[p] * e[q]), lp);
    for (int p = 0; p < nprim; ++p)
      c[p] *= std::sqrt(std::pow(e[p], lp) / (std::pow(kPi, 1.5) / std::pow(2.0, L) * N));
    b.exps.insert(b.exps.end(), e.begin(), e.end());
    b.coefs.insert(b.coefs.end(), c.begin(), c.end());
    b.lmax = std::max(b.lmax, L);
  }
  b.nsph = sph;
  *out = std::move(b);
  return PA_OK;
}

void build_pair_lists(const HostBasis& b, PairLists* out) {
  PairLists p;
  const int n = static_cast<int>(b.shells.size());
  p.npairs = n * (n + 1) / 2;
  p.lab_max = std::max(0, 2 * b.lmax);
  p.pair_ab.reserve(p.npairs);
  p.pair_unit0.reserve(p.npairs);
  for (int a = 0; a < n; ++a)
    for (int c = 0; c <= a; ++c) {
      const HostShell& sa = b.shells[a];
      const HostShell& sc = b.shells[c];
      const int pair = static_cast<int>(p.pair_ab.size());
      p.pair_ab.push_back(make_int2(a, c));
      p.pair_unit0.push_back(static_cast<int>(p.unit_pair.size()));
      const long long blk = static_cast<long long>(2 * sa.L + 1) * (2 * sc.L + 1) * ncum(sa.L + sc.L);
      for (int i = 0; i < sa.nprim; ++i)
        for (int j = 0; j < sc.nprim; ++j) {
          p.unit_pair.push_back(pair);
          p.unit_prims.push_back(make_int2(sa.prim_off + i, sc.prim_off + j));
          p.unit_esph.push_back(p.esph_total);
          p.esph_total += blk;
        }
    }
  p.nunits = static_cast<int>(p.unit_pair.size());
  p.class_off.assign(p.lab_max + 2, 0);
  std::vector<int> lab(p.nunits);
  for (int u = 0; u < p.nunits; ++u) {
    const int2 ab = p.pair_ab[p.unit_pair[u]];
    lab[u] = b.shells[ab.x].L + b.shells[ab.y].L;
    p.class_off[lab[u] + 1]++;
  }
  for (int c = 0; c <= p.lab_max; ++c) p.class_off[c + 1] += p.class_off[c];
  p.class_unit.assign(p.nunits, 0);
  std::vector<int> fill(p.class_off.begin(), p.class_off.end() - 1);
  for (int u = 0; u < p.nunits; ++u) p.class_unit[fill[lab[u]]++] = u;
  p.pair_class_off.assign(p.lab_max + 2, 0);
  for (int q = 0; q < p.npairs; ++q) {
    const int2 ab = p.pair_ab[q];
    p.pair_class_off[b.shells[ab.x].L + b.shells[ab.y].L + 1]++;
  }
  for (int c = 0; c <= p.lab_max; ++c) p.pair_class_off[c + 1] += p.pair_class_off[c];
  p.class_pair.assign(p.npairs, 0);
  std::vector<int> pfill(p.pair_class_off.begin(), p.pair_class_off.end() - 1);
  for (int q = 0; q < p.npairs; ++q) {
    const int2 ab = p.pair_ab[q];
    p.class_pair[pfill[b.shells[ab.x].L + b.shells[ab.y].L]++] = q;
  }
  *out = std::move(p);
}

void build_aux_lists(const HostBasis& b, AuxLists* out) {
  AuxLists x;
  x.lc_max = std::max(0, b.lmax);
  x.class_off.assign(x.lc_max + 2, 0);
  for (const HostShell& s : b.shells) x.class_off[s.L + 1]++;
  for (int c = 0; c <= x.lc_max; ++c) x.class_off[c + 1] += x.class_off[c];
  x.class_shell.assign(b.shells.size(), 0);
  std::vector<int> fill(x.class_off.begin(), x.class_off.end() - 1);
  for (int i = 0; i < static_cast<int>(b.shells.size()); ++i)
    x.class_shell[fill[b.shells[i].L]++] = i;
  *out = std::move(x);
}

// erf^-1(y) for 0 <= y < 1 by Newton's method on erf(x) - y
// (d/dx erf = 2/sqrt(pi) exp(-x^2)), started from x = 1 and clipped to
// stay positive; converges to full double precision in a few steps.
double erfinv_newton(double y) {
  double x = 1.0;
  for (int it = 0; it < 100; ++it) {
    const double f = std::erf(x) - y;
    const double step = f / (2.0 / std::sqrt(kPi) * std::exp(-x * x));
    double xn = x - step;
    if (xn <= 0.0) xn = 0.5 * x;
    if (std::fabs(xn - x) <= 1e-16 * std::fabs(xn)) return xn;
    x = xn;
  }
  return x;
}

void build_qvl_pairs(const HostBasis& b, const PairLists& P, std::vector<double4>* cen_ext,
                     std::vector<double>* den, double* den_min) {
  // thresh_ws = 1d-4 at every call site (diabatization/intor.f90:84,
  // std/intor.f90:60,201); contracted_extent uses erf^-1(1 - thresh_ws)
  const double erfi = erfinv_newton(1.0 - 1e-4);
  const int n = static_cast<int>(b.shells.size());
  std::vector<double> effexp(n);
  for (int i = 0; i < n; ++i) {
    const HostShell& s = b.shells[i];
    effexp[i] = *std::min_element(b.exps.begin() + s.prim_off, b.exps.begin() + s.prim_off + s.nprim);
  }
  cen_ext->resize(P.pair_ab.size());
  den->resize(P.pair_ab.size());
  double dmin = std::numeric_limits<double>::infinity();
  for (size_t q = 0; q < P.pair_ab.size(); ++q) {
    const HostShell& sa = b.shells[P.pair_ab[q].x];
    const HostShell& sb = b.shells[P.pair_ab[q].y];
    // contracted_center (common/screening.f90:235-265): |d_a d_b|-weighted
    // mean of the primitive product centers
    double R[3] = {0.0, 0.0, 0.0}, wsum = 0.0;
    for (int i = 0; i < sa.nprim; ++i)
      for (int j = 0; j < sb.nprim; ++j) {
        const double ax = b.exps[sa.prim_off + i], bx = b.exps[sb.prim_off + j];
        const double w = std::fabs(b.coefs[sa.prim_off + i] * b.coefs[sb.prim_off + j]);
        const double px = ax + bx;
        for (int d = 0; d < 3; ++d) R[d] += w * (ax * sa.A[d] + bx * sb.A[d]) / px;
        wsum += w;
      }
    for (int d = 0; d < 3; ++d) R[d] /= wsum;
    // contracted_extent (:198-232): max over primitive pairs of
    // sqrt(2 / p) erf^-1(1 - thresh_ws) + |R - P|
    double ext = 0.0;
    for (int i = 0; i < sa.nprim; ++i)
      for (int j = 0; j < sb.nprim; ++j) {
        const double ax = b.exps[sa.prim_off + i], bx = b.exps[sb.prim_off + j];
        const double px = ax + bx;
        double d2 = 0.0;
        for (int d = 0; d < 3; ++d) {
          const double Pd = (ax * sa.A[d] + bx * sb.A[d]) / px;
          d2 += (R[d] - Pd) * (R[d] - Pd);
        }
        ext = std::max(ext, std::sqrt(2.0 / px) * erfi + std::sqrt(d2));
      }
    (*cen_ext)[q] = make_double4(R[0], R[1], R[2], ext);
    const double dn = std::pow(effexp[P.pair_ab[q].x] + effexp[P.pair_ab[q].y], 0.25);
    (*den)[q] = dn;
    dmin = std::min(dmin, dn);
  }
  *den_min = P.pair_ab.empty() ? 1.0 : dmin;
}

void build_qvl_aux(const HostBasis& b, std::vector<double2>* ext_beta) {
  ext_beta->resize(b.shells.size());
  const double prec_term = -std::log(1e-8);  // auxiliary_extent(exps, 1d-8), min_extent 0.01
  for (size_t i = 0; i < b.shells.size(); ++i) {
    const HostShell& s = b.shells[i];
    double ext = 0.0, emin = std::numeric_limits<double>::infinity();
    for (int k = 0; k < s.nprim; ++k) {
      const double e = b.exps[s.prim_off + k];
      const double arg = (prec_term + 0.5 * std::log(e)) / e;
      ext = std::max(ext, arg < 0.0 ? 0.01 : std::sqrt(arg));
      emin = std::min(emin, e);
    }
    double dfact = 1.0;  // (2L - 1)!!
    for (int k = 2 * s.L - 1; k > 1; k -= 2) dfact *= k;
    (*ext_beta)[i] = make_double2(ext, std::pow(emin, -(2.0 * s.L + 3.0) / 4.0) * std::sqrt(dfact));
  }
}

cudaError_t Arena::reserve(size_t bytes) {
  if (bytes <= cap) return cudaSuccess;
  if (base) {
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return e;
    cudaFree(base);
    base = nullptr;
    cap = 0;
  }
  const size_t want = bytes + bytes / 4 + (64 << 20);
  cudaError_t e = cudaMalloc(&base, want);
  if (e != cudaSuccess) {
    base = nullptr;
    return e;
  }
  cap = want;
  return cudaSuccess;
}

}  // namespace pa

// ---------------------------------------------------------------------------
// Opaque basis handle.
struct pa_basis_s {
  int device = 0;
  long long serial = 0;  // unique per handle in the process
  pa::HostBasis host;
  pa::PairLists pairs;
  pa::AuxLists aux;
  char* dmem = nullptr;
  pa::DevBasis dev;
  // Shell-pair lists: built on the first use as an orbital basis (an
  // auxiliary basis never needs them).
  std::mutex pair_mu;
  bool pairs_ready = false;
  char* dpair = nullptr;
  int2* d_pair_ab = nullptr;
  int* d_pair_unit0 = nullptr;
  int* d_unit_pair = nullptr;
  int2* d_unit_prims = nullptr;
  long long* d_unit_esph = nullptr;
  int* d_class_unit = nullptr;   // units grouped by Lab
  int* d_class_off = nullptr;    // [lab_max + 2]
  int* d_class_pair = nullptr;   // pairs grouped by Lab
  int* d_aux_shell = nullptr;    // aux shells grouped by L
  int* d_aux_off = nullptr;      // [lc_max + 2]
  // QVL screener data: per shell (as an auxiliary basis) and per shell pair
  // (as an orbital basis, built with the pair lists)
  std::vector<double2> aux_qvl;  // (extent, beta)
  double2* d_aux_qvl = nullptr;
  // (the pair data only once QVL screening is used with this basis)
  bool qvl_ready = false;
  std::vector<double4> pair_qvl;  // (contracted center, extent)
  std::vector<double> pair_den;   // (zeta_a + zeta_b)^(1/4)
  double qvl_den_min = 1.0;
  char* dqvl = nullptr;
  double4* d_pair_qvl = nullptr;
  double* d_pair_den = nullptr;
};

namespace pa {
namespace {

struct Ctx {
  std::mutex mu;
  Arena arena;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEvent_t ph[5] = {};  // phase boundaries on the main stream: screen | bra | 3c | solve
  cudaStream_t stream2 = nullptr;     // metric + Cholesky + inverse, overlapped with the 3c work
  cudaStream_t sscr = nullptr;        // screening of the single-molecule path (highest priority)
  cudaEvent_t ev_scr0 = nullptr, ev_scr1 = nullptr;
  cudaEvent_t fork = nullptr, m0 = nullptr, m1 = nullptr;
  cudaEvent_t ev_bra[2 * PA_LMAX + 1] = {};  // density folding of each L_ab class done
  // streams of the three-center class launches: the tail of one class overlaps
  // the start of the next
  static constexpr int kNs3c = 4;
  cudaStream_t s3c[kNs3c] = {};
  cudaEvent_t j3c[kNs3c] = {};
  int* h_info = nullptr;  // pinned
  // Stream-ordered pool of the host-buffer entry points (densities, df, R).
  // Freed blocks stay mapped in this private pool, so repeated calls of the
  // same size do not map device memory again; the device's default pool and
  // other allocators in the process are untouched.
  cudaMemPool_t pool = nullptr;
  // host-buffer path: the density upload runs on its own stream and only the
  // density folding waits for it (screening and metric do not need it)
  cudaStream_t scopy = nullptr;
  cudaEvent_t ev_alloc = nullptr, ev_copied = nullptr;
  // batched form: metric chains of different molecules on their own streams
  cudaStream_t smet[kNs3c] = {};
  cudaStream_t sscrw[kNs3c] = {};  // batched form: screening + folding (highest priority)
  // batched form: folding of each L_ab class done by screening worker i (for
  // the last molecule it folds, hence for all of its molecules)
  cudaEvent_t ev_bra_w[kNs3c][2 * PA_LMAX + 1] = {};
  cudaEvent_t jmet[kNs3c] = {};
  cudaEvent_t jscr[kNs3c] = {};  // batched form: screening worker i done
  // lookahead streams of the Cholesky factorization: la2 for the chains on
  // stream2 and for pa_cholesky_solve, la_met[i] for the chain on smet[i]
  CholLookahead la2;
  CholLookahead la_met[kNs3c];
  struct BatchPlan* plan = nullptr;  // the last batch, kept for replay
  // class timing (Options::class_timing): an event pair per class run
  std::vector<cudaEvent_t> ct_ev;
};

// Per-class device times of the last single-molecule run in class-timing mode.
struct ClassTime {
  int lab, lc;
  double ms;
};
std::mutex g_ct_mu;
std::vector<ClassTime> g_class_times;

std::mutex g_ctx_mu;
std::vector<Ctx*> g_ctx;

int current_ctx(Ctx** out, DeviceTables* dt) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(PA_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  std::string err;
  const int st = get_device_tables(dt, &err);
  if (st != PA_OK) return fail(st, err);
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (static_cast<int>(g_ctx.size()) <= dev) g_ctx.resize(dev + 1, nullptr);
  if (!g_ctx[dev]) {
    Ctx* c = new Ctx();
    PA_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    PA_CUDA(cudaEventCreate(&c->ev0));
    PA_CUDA(cudaEventCreate(&c->ev1));
    for (auto& e : c->ph) PA_CUDA(cudaEventCreate(&e));
    // The metric + Cholesky chain is a long sequence of small dependent
    // launches; at the highest priority each of its blocks takes the next SM
    // that a 3c block frees instead of queueing behind the whole 3c grid.
    int prio_lo = 0, prio_hi = 0;
    PA_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    // The screening is on the critical path and the metric chain has slack:
    // screening at the highest priority, the metric chain one level below
    // (still above the three-center kernels at the default level).
    const int prio_met = prio_hi < prio_lo ? prio_hi + 1 : prio_hi;
    PA_CUDA(cudaStreamCreateWithPriority(&c->sscr, cudaStreamNonBlocking, prio_hi));
    PA_CUDA(cudaEventCreateWithFlags(&c->ev_scr0, cudaEventDisableTiming));
    PA_CUDA(cudaEventCreateWithFlags(&c->ev_scr1, cudaEventDisableTiming));
    PA_CUDA(cudaStreamCreateWithPriority(&c->stream2, cudaStreamNonBlocking, prio_met));
    PA_CUDA(cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming));
    for (auto& e : c->ev_bra) PA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto& row : c->ev_bra_w)
      for (auto& e : row) PA_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    PA_CUDA(cudaStreamCreateWithFlags(&c->scopy, cudaStreamNonBlocking));
    PA_CUDA(cudaEventCreateWithFlags(&c->ev_alloc, cudaEventDisableTiming));
    PA_CUDA(cudaEventCreateWithFlags(&c->ev_copied, cudaEventDisableTiming));
    for (int i = 0; i < Ctx::kNs3c; ++i) {
      PA_CUDA(cudaStreamCreateWithFlags(&c->s3c[i], cudaStreamNonBlocking));
      PA_CUDA(cudaEventCreateWithFlags(&c->j3c[i], cudaEventDisableTiming));
      // batched form: screening and folding at the highest priority, the
      // metric chains one level below, the class kernels at the default (as
      // in the single-molecule path)
      PA_CUDA(cudaStreamCreateWithPriority(&c->smet[i], cudaStreamNonBlocking, prio_met));
      PA_CUDA(cudaStreamCreateWithPriority(&c->sscrw[i], cudaStreamNonBlocking, prio_hi));
      PA_CUDA(cudaEventCreateWithFlags(&c->jmet[i], cudaEventDisableTiming));
      PA_CUDA(cudaEventCreateWithFlags(&c->jscr[i], cudaEventDisableTiming));
    }
    for (int i = 0; i <= Ctx::kNs3c; ++i) {
      CholLookahead& la = i < Ctx::kNs3c ? c->la_met[i] : c->la2;
      PA_CUDA(cudaStreamCreateWithPriority(&la.aux, cudaStreamNonBlocking, prio_met));
      PA_CUDA(cudaEventCreateWithFlags(&la.ev_panel, cudaEventDisableTiming));
      PA_CUDA(cudaEventCreateWithFlags(&la.ev_rest, cudaEventDisableTiming));
    }
    PA_CUDA(cudaEventCreate(&c->m0));
    PA_CUDA(cudaEventCreate(&c->m1));
    PA_CUDA(cudaMallocHost(&c->h_info, sizeof(int) * 4));
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    PA_CUDA(cudaMemPoolCreate(&c->pool, &props));
    unsigned long long keep = ~0ull;
    PA_CUDA(cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    g_ctx[dev] = c;
  }
  *out = g_ctx[dev];
  return PA_OK;
}

// Arena carving that can also just count bytes.
struct Carver {
  char* base = nullptr;
  size_t used = 0;
  template <class T>
  T* take(size_t count) {
    const size_t bytes = ((count * sizeof(T)) + 255) & ~size_t(255);
    T* p = base ? reinterpret_cast<T*>(base + used) : nullptr;
    used += bytes;
    return p;
  }
};

__global__ void k_gather_unit_keys(int n, const int* __restrict__ class_unit,
                                   const int* __restrict__ unit_pair, const double* __restrict__ Qab,
                                   double* keys, int* vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  keys[i] = Qab[unit_pair[class_unit[i]]];
  vals[i] = i;  // input position; class_sort_desc maps it back to the unit
}

// Sort keys of the auxiliary shells: Q_c, or with QVL screening (qvl != null)
// the bound max(Q_c, pi sqrt(2) beta_c / (den_min ext_c^(L_c + 1))) of
// qvl_estimate / Q_ab: beyond the distance ext_ab + ext_c > ext_c the QVL
// estimate is below Q_ab times the second term, inside it equals Q_ab Q_c. With
// these keys the staircase of sorted units and shells stays a valid bound.
__global__ void k_gather_aux_keys(int n, const int* __restrict__ shells, const double* __restrict__ Qc,
                                  const int4* __restrict__ shell_info, const double2* __restrict__ qvl,
                                  double den_min, double* keys, int* vals) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = shells[i];
  double key = Qc[s];
  if (qvl) {
    const double2 eb = qvl[s];
    double rl = eb.x;
    for (int l = 0; l < shell_info[s].x; ++l) rl *= eb.x;
    key = fmax(key, kPi * sqrt(2.0) * eb.y / (den_min * rl));
  }
  keys[i] = key;
  vals[i] = i;  // input position; class_sort_desc maps it back to the shell
}

// Per auxiliary slot: (Q_c, extent, beta, 0) of the sorted shell (QVL screening).
__global__ void k_aux_slot_qvl(int n, const int* __restrict__ sorted_aux, const double* __restrict__ Qc,
                               const double2* __restrict__ qvl, double4* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = sorted_aux[i];
  out[i] = make_double4(Qc[s], qvl[s].x, qvl[s].y, 0.0);
}

__global__ void k_boys_eval(DeviceTables dt, int mode, int nmax, int n, const double* T, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n * (nmax + 1)) return;
  const int k = i / (nmax + 1), m = i - k * (nmax + 1);
  out[i] = boys_n(dt, mode, m, T[k]);
}

// Class of each entry of a globally sorted list, found from its input
// position (inputs are ordered by class, class c at [off[c], off[c+1])).
__global__ void k_class_of_sorted(int n, const int* __restrict__ pos, const int* __restrict__ off,
                                  int nseg, unsigned char* cls, int* idx) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int i = pos[j];
  int c = 0;
  while (c + 1 < nseg && i >= off[c + 1]) ++c;
  cls[j] = static_cast<unsigned char>(c);
  idx[j] = j;
}

__global__ void k_class_sort_finish(int n, const int* __restrict__ order, const double* __restrict__ keys,
                                    const int* __restrict__ pos, const int* __restrict__ ids,
                                    double* keys_out, int* ids_out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const int j = order[k];
  keys_out[k] = keys[j];
  ids_out[k] = ids[pos[j]];
}

// Buffers of one density-fitting run.
struct DfBuffers {
  double *Qab, *Qc, *qmax, *esph, *ukeys, *slot_Q, *akeys, *aux_Q, *G, *M, *partial, *lawork,
      *df_raw;
  double4 *unit_pP, *slot_pP;
  // QVL screening: per unit slot (contracted center, extent of its pair) and
  // (zeta_a + zeta_b)^(1/4); per auxiliary slot (Q_c, extent, beta, 0)
  double4 *slot_qvl, *aux_slot_qvl;
  double* slot_den;
  int *uvals, *sorted_unit, *avals, *sorted_aux, *info;
  int* counters = nullptr;  // one work counter per class run
  // class_sort_desc scratch (max(nunits, naux shells) entries each)
  double* sort_k;
  int *sort_p, *sort_j, *sort_j2;
  unsigned char *sort_c, *sort_c2;
  void* cub_tmp;
  size_t cub_bytes;
  std::vector<long long> g_off;      // per Lab class
  int dw = 8;                        // density chunk width of G (multiple of 8, <= 40)
  bool split = false;                // mixed form: the weak triplets run on their own kernels
  struct ClassRun {
    int lab, lc, ny;
    double* partial;
    int variant;  // tile-shape variant of the class kernel
    bool weak;    // weak-triplet kernel (mixed form)
  };
  std::vector<ClassRun> runs;
};

size_t cub_temp_bytes(const pa_basis_s* orb, const pa_basis_s* aux) {
  size_t need = 0;
  for (const int n : {orb->pairs.nunits, static_cast<int>(aux->host.shells.size())}) {
    size_t b1 = 0, b2 = 0, b3 = 0;
    cub::DeviceRadixSort::SortPairsDescending(nullptr, b1, (const double*)nullptr, (double*)nullptr,
                                              (const int*)nullptr, (int*)nullptr, n, 0, 64);
    cub::DeviceRadixSort::SortPairs(nullptr, b2, (const unsigned char*)nullptr, (unsigned char*)nullptr,
                                    (const int*)nullptr, (int*)nullptr, n, 0, 8);
    cub::DeviceReduce::Max(nullptr, b3, (const double*)nullptr, (double*)nullptr, n);
    need = std::max(need, std::max(b1, std::max(b2, b3)));
  }
  return need;
}

// Stable descending sort of keys[0, n) inside each class segment
// [off[c], off[c+1]), c < nseg, of a class-ordered input: one global stable
// sort by key (position as value), then a stable sort by class. Within a class
// this is key-descending with ties in input order, the order of a segmented
// radix sort, but every pass runs on all SMs (a segmented sort gives each
// segment one block, and there are only a handful of classes). Writes the
// sorted keys and ids[position] of the entries.
static_assert(2 * PA_LMAX + 1 <= 256, "class ids of the sort are unsigned char");
int class_sort_desc(DfBuffers& b, const double* keys, const int* positions, const int* ids,
                    const int* d_off, int nseg, int n, double* keys_out, int* ids_out, cudaStream_t s) {
  if (n <= 0) return 0;
  size_t bytes = b.cub_bytes;
  PA_CUDA(cub::DeviceRadixSort::SortPairsDescending(b.cub_tmp, bytes, keys, b.sort_k, positions, b.sort_p,
                                                    n, 0, 64, s));
  const int grid = (n + 255) / 256;
  k_class_of_sorted<<<grid, 256, 0, s>>>(n, b.sort_p, d_off, nseg, b.sort_c, b.sort_j);
  int bits = 1;
  while ((1 << bits) < nseg) ++bits;
  bytes = b.cub_bytes;
  PA_CUDA(cub::DeviceRadixSort::SortPairs(b.cub_tmp, bytes, b.sort_c, b.sort_c2, b.sort_j, b.sort_j2, n, 0,
                                          bits, s));
  k_class_sort_finish<<<grid, 256, 0, s>>>(n, b.sort_j2, b.sort_k, b.sort_p, ids, keys_out, ids_out);
  return 4;  // two kernels of this file + two CUB sort calls
}

// Lays out all buffers of a run (counting when c.base == nullptr).
void layout_df(Carver& c, const pa_basis_s* orb, const pa_basis_s* aux, int nd, DfBuffers* b,
               const Options& o) {
  int items_per_sm = o.items_per_sm;
  const PairLists& P = orb->pairs;
  const int nx = static_cast<int>(aux->host.shells.size());
  const long long naux = aux->host.nsph;
  b->Qab = c.take<double>(P.npairs);
  b->Qc = c.take<double>(nx);
  b->qmax = c.take<double>(1);
  b->unit_pP = c.take<double4>(P.nunits);
  b->esph = c.take<double>(P.esph_total);
  b->ukeys = c.take<double>(P.nunits);
  b->uvals = c.take<int>(P.nunits);
  b->slot_Q = c.take<double>(P.nunits);
  b->sorted_unit = c.take<int>(P.nunits);
  b->slot_pP = c.take<double4>(P.nunits);
  b->slot_qvl = c.take<double4>(P.nunits);
  b->slot_den = c.take<double>(P.nunits);
  b->aux_slot_qvl = c.take<double4>(nx);
  b->akeys = c.take<double>(nx);
  b->avals = c.take<int>(nx);
  b->aux_Q = c.take<double>(nx);
  b->sorted_aux = c.take<int>(nx);
  b->info = c.take<int>(4);
  b->dw = std::min(40, std::max(8, (nd + 7) / 8 * 8));
  const int nz = nd > 0 ? (nd + b->dw - 1) / b->dw : 0;
  b->g_off.assign(P.lab_max + 2, 0);
  for (int lab = 0; lab <= P.lab_max; ++lab) {
    const long long nu = P.class_off[lab + 1] - P.class_off[lab];
    b->g_off[lab + 1] = b->g_off[lab] + nu * ncum(lab) * nz * b->dw;
  }
  b->G = c.take<double>(b->g_off[P.lab_max + 1]);
  b->split = o.precision == PA_PRECISION_MIXED && o.mixed_kernels != 0 && o.fp32_thresh > o.screen_thresh;

  b->M = c.take<double>(naux * naux);
  b->lawork = c.take<double>(linalg_workspace_doubles(static_cast<int>(naux)));
  b->df_raw = c.take<double>(static_cast<size_t>(naux) * nd);
  const int nsort = std::max(P.nunits, nx);
  b->sort_k = c.take<double>(nsort);
  b->sort_p = c.take<int>(nsort);
  b->sort_j = c.take<int>(nsort);
  b->sort_j2 = c.take<int>(nsort);
  b->sort_c = c.take<unsigned char>(nsort);
  b->sort_c2 = c.take<unsigned char>(nsort);
  b->cub_bytes = cub_temp_bytes(orb, aux);
  b->cub_tmp = c.take<char>(b->cub_bytes);
  // partial slabs; the work-item granularity grows with the system size (on
  // B200, with every item a chunk of its tile's surviving units: 2 items per
  // SM and class at 40 atoms, 8 at 200 atoms were best)
  if (items_per_sm <= 0) {
    const double T = static_cast<double>(P.npairs) * aux->host.shells.size();
    items_per_sm = static_cast<int>(std::lround(2.0 * std::pow(std::max(T, 1.0) / 1.85e7, 0.55)));
    items_per_sm = std::min(8, std::max(2, items_per_sm));
  }
  b->runs.clear();
  size_t part_total = 0;
  const AuxLists& X = aux->aux;
  // class runs grouped by L_c, highest first (light L_c = 0 classes last, so
  // the cheapest reduction closes the phase), L_ab ascending within a group
  for (int lc = X.lc_max; lc >= 0 && nd > 0; --lc) {
    const int nxc = X.class_off[lc + 1] - X.class_off[lc];
    if (nxc == 0) continue;
    for (int lab = 0; lab <= P.lab_max; ++lab) {
      const int nu = P.class_off[lab + 1] - P.class_off[lab];
      if (nu == 0) continue;
      const int variant = o.tile_variant[lab][lc];
      // the FP64 run, then (mixed form) the weak-triplet run of the class
      for (int weak = 0; weak <= (b->split ? 1 : 0); ++weak) {
        Df3cClassInfo ci;
        if (weak)
          df3c_class_info_w(lab, lc, &ci);
        else
          df3c_class_info(lab, lc, variant, &ci);
        const int bx = (nxc + ci.tc - 1) / ci.tc;
        const int bz = nz;
        const int target = items_per_sm * 148;  // work items per class (persistent blocks pull them)
        int ny = std::max(1, (target + bx * bz - 1) / (bx * bz));
        const int max_ny = (nu + ci.ub - 1) / ci.ub;
        ny = std::min(ny, max_ny);
        int upc = (nu + ny - 1) / ny;
        upc = ((upc + ci.ub - 1) / ci.ub) * ci.ub;
        ny = (nu + upc - 1) / upc;
        DfBuffers::ClassRun r{lab, lc, ny, nullptr, variant, weak != 0};
        b->runs.push_back(r);
        part_total += static_cast<size_t>(ny) * nxc * (2 * lc + 1) * nd;
      }
    }
  }
  double* part = c.take<double>(part_total);
  b->counters = c.take<int>(std::max<size_t>(b->runs.size(), 1));
  size_t off = 0;
  for (auto& r : b->runs) {
    const int nxc = X.class_off[r.lc + 1] - X.class_off[r.lc];
    r.partial = part ? part + off : nullptr;
    off += static_cast<size_t>(r.ny) * nxc * (2 * r.lc + 1) * nd;
  }
}

UnitArrays unit_arrays(const pa_basis_s* orb, const DfBuffers& b) {
  UnitArrays U;
  U.unit_pair = orb->d_unit_pair;
  U.unit_prims = orb->d_unit_prims;
  U.unit_esph = orb->d_unit_esph;
  U.unit_pP = b.unit_pP;
  U.esph = b.esph;
  return U;
}

// Schwarz vectors of both bases and the sorted class lists.
int run_screening(const pa_basis_s* orb, const pa_basis_s* aux, const DeviceTables& dt,
                  const Options& o, DfBuffers& b, cudaStream_t s, int* launches) {
  const PairLists& P = orb->pairs;
  const int nx = static_cast<int>(aux->host.shells.size());
  UnitArrays U = unit_arrays(orb, b);
  *launches += launch_unit_setup(orb->dev, orb->d_pair_ab, orb->d_class_unit, P, U, dt, s);
  *launches += launch_schwarz_bra(orb->dev, orb->d_pair_ab, orb->d_pair_unit0, orb->d_class_pair, P, U, dt,
                                  o.boys_mode, b.Qab, s);
  *launches += launch_schwarz_aux(aux->dev, dt, o.boys_mode, b.Qc, s);
  const bool qvl = o.screening == PA_SCREEN_QVL;
  if (nx > 0) {
    k_gather_aux_keys<<<(nx + 255) / 256, 256, 0, s>>>(nx, aux->d_aux_shell, b.Qc, aux->dev.shell,
                                                       qvl ? aux->d_aux_qvl : nullptr, orb->qvl_den_min,
                                                       b.akeys, b.avals);
    ++*launches;
    size_t bytes = b.cub_bytes;
    PA_CUDA(cub::DeviceReduce::Max(b.cub_tmp, bytes, b.akeys, b.qmax, nx, s));  // largest key
    ++*launches;
  }
  if (P.nunits > 0) {
    k_gather_unit_keys<<<(P.nunits + 255) / 256, 256, 0, s>>>(P.nunits, orb->d_class_unit,
                                                              orb->d_unit_pair, b.Qab, b.ukeys, b.uvals);
    ++*launches;
    *launches += class_sort_desc(b, b.ukeys, b.uvals, orb->d_class_unit, orb->d_class_off, P.lab_max + 1,
                                 P.nunits, b.slot_Q, b.sorted_unit, s);
  }
  if (nx > 0) {
    *launches += class_sort_desc(b, b.akeys, b.avals, aux->d_aux_shell, aux->d_aux_off, aux->aux.lc_max + 1,
                                 nx, b.aux_Q, b.sorted_aux, s);
    if (qvl) {
      k_aux_slot_qvl<<<(nx + 255) / 256, 256, 0, s>>>(nx, b.sorted_aux, b.Qc, aux->d_aux_qvl, b.aux_slot_qvl);
      ++*launches;
    }
  }
  return PA_OK;
}

// ---------------------------------------------------------------------------
// Stages of one density-fitting run, shared by the single-molecule path
// (run_df) and the batched path (pa_df_4d_batch).

// (P|Q) [+ shift], its Cholesky factor and the inverted diagonal blocks.
void stage_metric(const pa_basis_s* aux, DfBuffers& b, const DeviceTables& dt, const Options& o,
                  cudaStream_t s2, const CholLookahead* la, int* launches) {
  const int naux = aux->host.nsph;
  *launches += launch_metric(aux->dev, dt, o.boys_mode, b.M, s2);
  *launches += add_diagonal(b.M, naux, o.metric_shift, s2);
  *launches += cholesky_lower(b.M, naux, b.info, b.lawork, s2, la);
}

// Density folding of the sorted bra units, per L_ab class.
// With ev_lab, ev_lab[lab] is recorded on s once class lab is folded (also for
// empty classes), so that three-center launches can wait for their class alone.
void stage_bra_prep(const pa_basis_s* orb, const pa_basis_s* aux, int nd, const double* d_dens,
                    long long sd, long long si, long long sj, DfBuffers& b, const Options& o,
                    cudaStream_t s, int* launches, cudaEvent_t* ev_lab = nullptr) {
  const PairLists& P = orb->pairs;
  UnitArrays U = unit_arrays(orb, b);
  for (int lab = 0; lab <= P.lab_max; ++lab) {
    BraPrepArgs a;
    a.slot0 = P.class_off[lab];
    a.slot_end = P.class_off[lab + 1];
    if (a.slot_end <= a.slot0 || nd == 0 || aux->host.shells.empty()) {
      if (ev_lab) cudaEventRecord(ev_lab[lab], s);
      continue;
    }
    a.slot_Q = b.slot_Q;
    a.qmax_aux = b.qmax;
    a.thresh = o.screen_thresh;
    a.sorted_unit = b.sorted_unit;
    a.nd = nd;
    a.dens = d_dens;
    a.sd = sd;
    a.si = si;
    a.sj = sj;
    a.slot_pP = b.slot_pP;
    a.G = b.G;
    a.g_base = b.g_off[lab];
    a.dw = b.dw;
    a.n_class = a.slot_end - a.slot0;
    if (o.screening == PA_SCREEN_QVL) {
      a.pair_qvl = orb->d_pair_qvl;
      a.pair_den = orb->d_pair_den;
      a.slot_qvl = b.slot_qvl;
      a.slot_den = b.slot_den;
    }
    *launches += launch_bra_prep(orb->dev, orb->d_pair_ab, U, a, lab, s);
    if (ev_lab) cudaEventRecord(ev_lab[lab], s);
  }
}

// Kernel arguments of one (L_ab, L_c) class run.
Df3cArgs class_args(const pa_basis_s* orb, const pa_basis_s* aux, int nd, const DfBuffers& b,
                    const DeviceTables& dt, const Options& o, const DfBuffers::ClassRun& r) {
  const PairLists& P = orb->pairs;
  const AuxLists& X = aux->aux;
  Df3cArgs a;
  a.X = aux->dev;
  a.dt = dt;
  a.boys_mode = o.boys_mode;
  a.thresh = o.screen_thresh;
  a.thr32 = o.precision == PA_PRECISION_MIXED ? o.fp32_thresh : 0.0;
  if (b.split && !r.weak) {
    // the FP64 kernel takes the strong triplets only (Q_ab Q_c >= thr32)
    a.thresh = std::max(o.screen_thresh, o.fp32_thresh);
    a.thr32 = 0.0;
  }
  if (r.weak) a.err = b.info + 2;
  a.unit_slot0 = P.class_off[r.lab];
  a.n_units = P.class_off[r.lab + 1] - P.class_off[r.lab];
  a.unit_Q = b.slot_Q;
  a.slot_pP = b.slot_pP;
  a.G = b.G + b.g_off[r.lab];
  a.dw = b.dw;
  a.aux_slot0 = X.class_off[r.lc];
  a.n_aux = X.class_off[r.lc + 1] - X.class_off[r.lc];
  a.sorted_aux = b.sorted_aux;
  a.aux_Q = b.aux_Q;
  a.nd = nd;
  a.partial = r.partial;
  if (o.screening == PA_SCREEN_QVL) {
    a.qvl = 1;
    a.slot_qvl = b.slot_qvl;
    a.slot_den = b.slot_den;
    a.aux_qvl = b.aux_slot_qvl;
  }
  return a;
}

// Ordered sum of the partial slabs of auxiliary class lc into df_raw (the
// classes in L_ab order, as they appear in b.runs).
void stage_reduce_lc(const pa_basis_s* aux, int nd, DfBuffers& b, int lc, cudaStream_t s, int* launches) {
  const AuxLists& X = aux->aux;
  if (lc < 0 || lc > X.lc_max) return;  // no auxiliary shells of this L
  {
    Df3cReduceArgs ra;
    ra.X = aux->dev;
    ra.aux_slot0 = X.class_off[lc];
    ra.n_aux = X.class_off[lc + 1] - X.class_off[lc];
    if (ra.n_aux == 0 || nd <= 0) return;
    ra.nc = 2 * lc + 1;
    ra.nd = nd;
    ra.naux = aux->host.nsph;
    ra.sorted_aux = b.sorted_aux;
    ra.nclasses = 0;
    for (const auto& r : b.runs)
      if (r.lc == lc) {
        if (ra.nclasses >= kMaxRunsPerLc) break;  // unreachable: layout_df makes at most two runs per (L_ab, L_c)
        ra.part[ra.nclasses] = r.partial;
        ra.ny[ra.nclasses] = r.ny;
        ++ra.nclasses;
      }
    ra.df = b.df_raw;
    *launches += launch_df3c_reduce(ra, s);
  }
}

// All auxiliary classes, after every class run is done.
void stage_reduce(const pa_basis_s* aux, int nd, DfBuffers& b, cudaStream_t s, int* launches) {
  for (int lc = 0; lc <= aux->aux.lc_max; ++lc) stage_reduce_lc(aux, nd, b, lc, s, launches);
}

// d_df = L^-1 df_raw (or df_raw itself when the metric is skipped).
int stage_solve(const pa_basis_s* aux, int nd, DfBuffers& b, const Options& o, double* d_df,
                cudaStream_t s, int* launches) {
  const int naux = aux->host.nsph;
  if (nd <= 0) return PA_OK;
  if (o.skip_metric)
    PA_CUDA(cudaMemcpyAsync(d_df, b.df_raw, sizeof(double) * naux * nd, cudaMemcpyDeviceToDevice, s));
  else
    *launches += trsm_lower_left(b.M, naux, b.lawork, b.df_raw, naux, nd, d_df, naux, s);
  return PA_OK;
}

// df[naux, nd] (column-major) = L^-1 sum (ab|P) Dsym, into d_df.
int run_df(const pa_basis_s* orb, const pa_basis_s* aux, int nd, const double* d_dens,
           long long sd, long long si, long long sj, double* d_df, DfBuffers& b,
           const DeviceTables& dt, const Options& o, cudaStream_t s, int* launches,
           Ctx* ctx, int* launches_3c, cudaEvent_t dens_ready) {
  cudaEvent_t* ph = ctx->ph;
  // metric (P|Q), its Cholesky factor and L^-1 on the second stream: independent
  // of everything until the final L^-1 df
  // (the critical-path screening is enqueued first: the metric chain's ~100
  // launches would otherwise delay its start by their host-side launch time)
  cudaStream_t s2 = ctx->stream2;
  PA_CUDA(cudaEventRecord(ctx->fork, s));
  PA_CUDA(cudaEventRecord(ctx->ev_scr0, s));
  PA_CUDA(cudaStreamWaitEvent(ctx->sscr, ctx->ev_scr0, 0));
  int st = PA_OK;
  {
    NvtxRange r("pa: screening");
    st = run_screening(orb, aux, dt, o, b, ctx->sscr, launches);
  }
  if (st != PA_OK) return st;
  PA_CUDA(cudaStreamWaitEvent(s2, ctx->fork, 0));
  PA_CUDA(cudaEventRecord(ctx->m0, s2));
  {
    NvtxRange r("pa: metric and Cholesky");
    stage_metric(aux, b, dt, o, s2, &ctx->la2, launches);
  }
  PA_CUDA(cudaEventRecord(ctx->m1, s2));
  PA_CUDA(cudaEventRecord(ctx->ev_scr1, ctx->sscr));
  PA_CUDA(cudaStreamWaitEvent(s, ctx->ev_scr1, 0));
  PA_CUDA(cudaEventRecord(ph[0], s));
  if (dens_ready) PA_CUDA(cudaStreamWaitEvent(s, dens_ready, 0));
  // the class streams start after the screening; each class launch then waits
  // only for the folding of its own L_ab class
  const bool run3c = nd > 0 && !b.runs.empty();
  if (run3c) {
    PA_CUDA(cudaMemsetAsync(b.counters, 0, sizeof(int) * b.runs.size(), s));
    PA_CUDA(cudaMemsetAsync(b.info + 2, 0, sizeof(int), s));
    PA_CUDA(cudaEventRecord(ctx->fork, s));
    for (int i = 0; i < Ctx::kNs3c; ++i) PA_CUDA(cudaStreamWaitEvent(ctx->s3c[i], ctx->fork, 0));
  }
  {
    NvtxRange r("pa: density folding");
    stage_bra_prep(orb, aux, nd, d_dens, sd, si, sj, b, o, s, launches, ctx->ev_bra);
  }
  PA_CUDA(cudaEventRecord(ph[1], s));
  // three-center contraction: one persistent launch per class, on four streams
  const int before3c = *launches;
  std::optional<NvtxRange> r3c;
  r3c.emplace("pa: three-center classes");
  if (run3c) {
    // the runs come grouped by L_c: once a group is enqueued, the main stream
    // waits for the class streams and reduces that group while the next
    // groups run
    const int nr = static_cast<int>(b.runs.size());
    if (o.class_timing)
      while (static_cast<int>(ctx->ct_ev.size()) < 2 * nr) {
        cudaEvent_t e;
        PA_CUDA(cudaEventCreate(&e));
        ctx->ct_ev.push_back(e);
      }
    for (int ri = 0; ri < nr; ++ri) {
      const auto& r = b.runs[ri];
      Df3cArgs a = class_args(orb, aux, nd, b, dt, o, r);
      a.counter = b.counters + ri;
      // class timing: every class on the first class stream, one after another
      cudaStream_t cs = ctx->s3c[o.class_timing ? 0 : ri % Ctx::kNs3c];
      PA_CUDA(cudaStreamWaitEvent(cs, ctx->ev_bra[r.lab], 0));
      if (o.class_timing) PA_CUDA(cudaEventRecord(ctx->ct_ev[2 * ri], cs));
      *launches += r.weak ? launch_df3c_class_w(r.lab, r.lc, a, r.ny, cs)
                          : launch_df3c_class(r.lab, r.lc, r.variant, a, r.ny, cs);
      if (o.class_timing) PA_CUDA(cudaEventRecord(ctx->ct_ev[2 * ri + 1], cs));
      if (ri + 1 == nr || b.runs[ri + 1].lc != r.lc) {
        for (int i = 0; i < Ctx::kNs3c; ++i) {
          PA_CUDA(cudaEventRecord(ctx->j3c[i], ctx->s3c[i]));
          PA_CUDA(cudaStreamWaitEvent(s, ctx->j3c[i], 0));
        }
        stage_reduce_lc(aux, nd, b, r.lc, s, launches);
      }
    }
  }
  *launches_3c = *launches - before3c;
  r3c.reset();
  PA_CUDA(cudaEventRecord(ph[2], s));
  PA_CUDA(cudaStreamWaitEvent(s, ctx->m1, 0));  // join the metric stream
  NvtxRange rs("pa: solve");
  return stage_solve(aux, nd, b, o, d_df, s, launches);
}

int finish(Ctx* c, const DfBuffers& b, cudaStream_t s, int launches, float* ms) {
  PA_CUDA(cudaGetLastError());
  PA_CUDA(cudaEventRecord(c->ev1, s));
  PA_CUDA(cudaMemcpyAsync(c->h_info, b.info, sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  PA_CUDA(cudaEventElapsedTime(ms, c->ev0, c->ev1));
  float t[5];
  PA_CUDA(cudaEventElapsedTime(&t[0], c->ev0, c->ph[0]));
  PA_CUDA(cudaEventElapsedTime(&t[1], c->ph[0], c->ph[1]));
  PA_CUDA(cudaEventElapsedTime(&t[2], c->m0, c->m1));  // concurrent with screening..3c
  PA_CUDA(cudaEventElapsedTime(&t[3], c->ph[1], c->ph[2]));
  PA_CUDA(cudaEventElapsedTime(&t[4], c->ph[2], c->ev1));
  g_stats.ms_screen = t[0];
  g_stats.ms_bra = t[1];
  g_stats.ms_metric = t[2];
  g_stats.ms_3c = t[3];
  g_stats.ms_solve = t[4];
  g_stats.kernel_launches = launches;
  g_stats.ms_total = *ms;
  if (options().class_timing && !b.runs.empty() && c->ct_ev.size() >= 2 * b.runs.size()) {
    std::vector<ClassTime> ct;
    for (size_t ri = 0; ri < b.runs.size(); ++ri) {
      float t = 0.f;
      PA_CUDA(cudaEventElapsedTime(&t, c->ct_ev[2 * ri], c->ct_ev[2 * ri + 1]));
      ct.push_back({b.runs[ri].lab, b.runs[ri].lc, static_cast<double>(t)});
    }
    std::lock_guard<std::mutex> lk(g_ct_mu);
    g_class_times = std::move(ct);
  }
  if (b.split && c->h_info[2] != 0)
    return fail(PA_ERR_TIMEOUT, "weak-triplet kernel: a tensor-core completion wait gave up");
  if (*c->h_info != 0)
    return fail(PA_ERR_NOT_SPD, "metric (P|Q) is not positive definite (Cholesky pivot " +
                                    std::to_string(*c->h_info) + ")");
  return PA_OK;
}

// Builds and uploads the shell-pair / primitive-pair lists of an orbital basis
// once; later calls return at once.
int ensure_pairs(pa_basis b) {
  std::lock_guard<std::mutex> lk(b->pair_mu);
  if (b->pairs_ready) return PA_OK;
  if (b->host.lmax > PA_LMAX) return fail(PA_ERR_LMAX, "orbital basis L above the compiled maximum");
  PairLists P;
  build_pair_lists(b->host, &P);
  Carver cnt;
  char* dpair = nullptr;
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) {
      if (cudaMalloc(&dpair, std::max<size_t>(cnt.used, 256)) != cudaSuccess)
        return fail(PA_ERR_CUDA, "cudaMalloc(pair lists) failed");
      cnt = Carver();
      cnt.base = dpair;
    }
    b->d_pair_ab = cnt.take<int2>(P.pair_ab.size());
    b->d_pair_unit0 = cnt.take<int>(P.pair_unit0.size());
    b->d_unit_pair = cnt.take<int>(P.unit_pair.size());
    b->d_unit_prims = cnt.take<int2>(P.unit_prims.size());
    b->d_unit_esph = cnt.take<long long>(P.unit_esph.size());
    b->d_class_unit = cnt.take<int>(P.class_unit.size());
    b->d_class_off = cnt.take<int>(P.class_off.size());
    b->d_class_pair = cnt.take<int>(P.class_pair.size());
  }
  std::vector<char> stage(cnt.used);
  auto put = [&](const void* dst, const void* src, size_t bytes) {
    if (bytes) std::memcpy(stage.data() + (static_cast<const char*>(dst) - dpair), src, bytes);
  };
  put(b->d_pair_ab, P.pair_ab.data(), sizeof(int2) * P.pair_ab.size());
  put(b->d_pair_unit0, P.pair_unit0.data(), sizeof(int) * P.pair_unit0.size());
  put(b->d_unit_pair, P.unit_pair.data(), sizeof(int) * P.unit_pair.size());
  put(b->d_unit_prims, P.unit_prims.data(), sizeof(int2) * P.unit_prims.size());
  put(b->d_unit_esph, P.unit_esph.data(), sizeof(long long) * P.unit_esph.size());
  put(b->d_class_unit, P.class_unit.data(), sizeof(int) * P.class_unit.size());
  put(b->d_class_off, P.class_off.data(), sizeof(int) * P.class_off.size());
  put(b->d_class_pair, P.class_pair.data(), sizeof(int) * P.class_pair.size());
  const cudaError_t e = cudaMemcpy(dpair, stage.data(), cnt.used, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(dpair);
    return fail(PA_ERR_CUDA, std::string("pair-list upload: ") + cudaGetErrorString(e));
  }
  b->pairs = std::move(P);
  b->dpair = dpair;
  b->pairs_ready = true;
  return PA_OK;
}

// QVL pair data of an orbital basis (pair lists built), once, on first use of
// QVL screening with it.
int ensure_qvl(pa_basis b) {
  std::lock_guard<std::mutex> lk(b->pair_mu);
  if (b->qvl_ready) return PA_OK;
  std::vector<double4> pair_qvl;
  std::vector<double> pair_den;
  double den_min = 1.0;
  build_qvl_pairs(b->host, b->pairs, &pair_qvl, &pair_den, &den_min);
  Carver cnt;
  char* d = nullptr;
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1) {
      if (cudaMalloc(&d, std::max<size_t>(cnt.used, 256)) != cudaSuccess)
        return fail(PA_ERR_CUDA, "cudaMalloc(QVL pair data) failed");
      cnt = Carver();
      cnt.base = d;
    }
    b->d_pair_qvl = cnt.take<double4>(pair_qvl.size());
    b->d_pair_den = cnt.take<double>(pair_den.size());
  }
  cudaError_t e = cudaMemcpy(b->d_pair_qvl, pair_qvl.data(), sizeof(double4) * pair_qvl.size(),
                             cudaMemcpyHostToDevice);
  if (e == cudaSuccess)
    e = cudaMemcpy(b->d_pair_den, pair_den.data(), sizeof(double) * pair_den.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    cudaFree(d);
    return fail(PA_ERR_CUDA, std::string("QVL pair data upload: ") + cudaGetErrorString(e));
  }
  b->pair_qvl = std::move(pair_qvl);
  b->pair_den = std::move(pair_den);
  b->qvl_den_min = den_min;
  b->dqvl = d;
  b->qvl_ready = true;
  return PA_OK;
}

int check_pair(pa_basis orb, pa_basis aux) {
  if (!orb || !aux) return fail(PA_ERR_ARG, "null basis handle");
  int dev = 0;
  cudaGetDevice(&dev);
  if (orb->device != dev || aux->device != dev)
    return fail(PA_ERR_ARG, "basis handle belongs to another device");
  const int st = ensure_pairs(orb);
  if (st != PA_OK || options().screening != PA_SCREEN_QVL) return st;
  return ensure_qvl(orb);
}

int df_device(pa_basis orb, pa_basis aux, int ndens, int nbf, const double* d_dens, int layout,
              double* d_df, int nstates, double* d_R, cudaStream_t user_stream,
              cudaEvent_t dens_ready = nullptr) {
  int st = check_pair(orb, aux);
  if (st != PA_OK) return st;
  if (ndens < 0 || nbf != orb->host.nsph)
    return fail(PA_ERR_ARG, "nbf (" + std::to_string(nbf) + ") does not match the orbital basis (" +
                                std::to_string(orb->host.nsph) + ")");
  if (layout != PA_LAYOUT_FORTRAN && layout != PA_LAYOUT_C) return fail(PA_ERR_ARG, "unknown layout");
  if (ndens > 0 && (!d_dens || !d_df)) return fail(PA_ERR_ARG, "null density or output pointer");
  Ctx* c = nullptr;
  DeviceTables dt;
  st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  const Options o = options();
  cudaStream_t s = user_stream;
  DfBuffers b;
  Carver cnt;
  layout_df(cnt, orb, aux, ndens, &b, o);
  if (d_R) cnt.take<double>(static_cast<size_t>(ndens) * ndens);
  PA_CUDA(c->arena.reserve(cnt.used));
  Carver real;
  real.base = c->arena.base;
  layout_df(real, orb, aux, ndens, &b, o);
  double* gram = d_R ? real.take<double>(static_cast<size_t>(ndens) * ndens) : nullptr;
  const long long n = nbf;
  long long sd, si, sj;
  if (layout == PA_LAYOUT_FORTRAN) {
    sd = 1;
    si = ndens;
    sj = static_cast<long long>(ndens) * n;
  } else {
    sd = n * n;
    si = n;
    sj = 1;
  }
  PA_CUDA(cudaEventRecord(c->ev0, s));
  int launches = 0, launches_3c = 0;
  st = run_df(orb, aux, ndens, d_dens, sd, si, sj, d_df, b, dt, o, s, &launches, c, &launches_3c, dens_ready);
  if (st != PA_OK) return st;
  g_stats.launches_3c = launches_3c;
  if (d_R) launches += coulomb_4d(d_df, aux->host.nsph, ndens, nstates, gram, d_R, s);
  float ms = 0.f;
  g_stats.ntriplets = static_cast<long long>(orb->pairs.npairs) * aux->host.shells.size();
  g_stats.nskipped = -1;
  g_stats.nints = -1;
  return finish(c, b, s, launches, &ms);
}

// ---------------------------------------------------------------------------
// Batched form: the Coulomb tensors of many molecules in one sequence --
// every molecule's screening, density folding and metric chain, then one
// persistent launch per shell-triplet class over the work items of all
// molecules, then the reductions, solves and tensors -- recorded once as a
// CUDA graph and replayed while the batch (handles, sizes, pointers and
// options) stays the same.
struct BatchPlan {
  std::vector<long long> sig;
  char* dmem = nullptr;
  std::vector<DfBuffers> bufs;
  std::vector<double*> df, gram;
  int* infos = nullptr;      // device: 4 ints per molecule
  int* h_infos = nullptr;    // pinned copy
  int* counters = nullptr;   // one per class launch
  cudaGraphExec_t exec = nullptr;
  int launches = 0;
  ~BatchPlan() {
    if (exec) cudaGraphExecDestroy(exec);
    if (dmem) cudaFree(dmem);
    if (h_infos) cudaFreeHost(h_infos);
  }
};

struct BatchMol {
  pa_basis orb, aux;
  int nd, ns;
  const double* dens;
  double* R;
  long long sd, si, sj;
};

// Records the whole batch on c->stream (the origin of a capture when graphed).
int record_batch(Ctx* c, BatchPlan& plan, const std::vector<BatchMol>& mols, const DeviceTables& dt,
                 const Options& o, const std::vector<int>& class_lab, const std::vector<int>& class_lc,
                 const std::vector<int>& class_weak, const std::vector<const Df3cArgs*>& class_args_d,
                 const std::vector<const int*>& class_off_d, const std::vector<int>& class_nm,
                 const std::vector<int>& class_items, const std::vector<Df3cArgs>& class_single, int* launches) {
  cudaStream_t s = c->stream;
  const int nmol = static_cast<int>(mols.size());
  constexpr int W = Ctx::kNs3c;
  constexpr int NLAB = 2 * PA_LMAX + 1;
  const int ncls = static_cast<int>(class_lab.size());
  // the class counters are zeroed and the class streams forked first: each
  // class launch then waits only for the folding of its own L_ab on every
  // screening worker, so the three-center work starts while later classes
  // are still folded (as in the single-molecule path)
  if (ncls > 0) PA_CUDA(cudaMemsetAsync(plan.counters, 0, sizeof(int) * ncls, s));
  // status words of every molecule (the weak-triplet kernels' flag among them)
  PA_CUDA(cudaMemsetAsync(plan.infos, 0, sizeof(int) * 4 * std::max(nmol, 1), s));
  PA_CUDA(cudaEventRecord(c->fork, s));
  for (int i = 0; i < W; ++i) {
    PA_CUDA(cudaStreamWaitEvent(c->sscrw[i], c->fork, 0));
    PA_CUDA(cudaStreamWaitEvent(c->smet[i], c->fork, 0));
    PA_CUDA(cudaStreamWaitEvent(c->s3c[i], c->fork, 0));
  }
  // per molecule: screening + folding on a screening worker (enqueued first:
  // the critical path), then the metric chain on a metric stream
  const int nworkers = std::min(nmol, W);
  for (int m = 0; m < nmol; ++m) {
    const BatchMol& M = mols[m];
    DfBuffers& b = plan.bufs[m];
    const int w = m % W;
    const int st = run_screening(M.orb, M.aux, dt, o, b, c->sscrw[w], launches);
    if (st != PA_OK) return st;
    const bool last = m + W >= nmol;  // the worker's last molecule
    stage_bra_prep(M.orb, M.aux, M.nd, M.dens, M.sd, M.si, M.sj, b, o, c->sscrw[w], launches,
                   last ? c->ev_bra_w[w] : nullptr);
    if (last)  // classes above this molecule's L_ab: done with everything before
      for (int lab = M.orb->pairs.lab_max + 1; lab < NLAB; ++lab)
        PA_CUDA(cudaEventRecord(c->ev_bra_w[w][lab], c->sscrw[w]));
  }
  for (int m = 0; m < nmol; ++m)
    stage_metric(mols[m].aux, plan.bufs[m], dt, o, c->smet[m % W], &c->la_met[m % W], launches);
  // the classes come grouped by L_c: once a group is enqueued, the main stream
  // waits for the class streams and reduces that group of every molecule while
  // the next groups run (as the single-molecule path does)
  bool reduced[PA_LAUXMAX + 1] = {};
  bool joined = false;  // the main stream has waited for the screening workers
  for (int k = 0; k < ncls; ++k) {
    for (int w = 0; w < nworkers; ++w)
      PA_CUDA(cudaStreamWaitEvent(c->s3c[k % W], c->ev_bra_w[w][class_lab[k]], 0));
    const int variant = o.tile_variant[class_lab[k]][class_lc[k]];
    if (class_nm[k] == 1) {
      // one molecule has items of this class: the single-molecule kernel, its
      // descriptor a kernel parameter (the batched kernel reads it from
      // shared memory on every use)
      Df3cArgs a1 = class_single[k];
      a1.counter = plan.counters + k;
      *launches += class_weak[k] ? launch_df3c_class_w(class_lab[k], class_lc[k], a1, a1.nby, c->s3c[k % W])
                                 : launch_df3c_class(class_lab[k], class_lc[k], variant, a1, a1.nby, c->s3c[k % W]);
    } else if (class_weak[k]) {
      *launches += launch_df3c_class_batch_w(class_lab[k], class_lc[k], class_args_d[k], class_off_d[k], class_nm[k],
                                             class_items[k], plan.counters + k, c->s3c[k % W]);
    } else {
      *launches += launch_df3c_class_batch(class_lab[k], class_lc[k], variant, class_args_d[k], class_off_d[k],
                                           class_nm[k], class_items[k], plan.counters + k, c->s3c[k % W]);
    }
    if (k + 1 == ncls || class_lc[k + 1] != class_lc[k]) {
      for (int i = 0; i < W; ++i) {
        PA_CUDA(cudaEventRecord(c->j3c[i], c->s3c[i]));
        PA_CUDA(cudaStreamWaitEvent(s, c->j3c[i], 0));
        if (!joined) {  // the reductions read the screening's sorted lists
          PA_CUDA(cudaEventRecord(c->jscr[i], c->sscrw[i]));
          PA_CUDA(cudaStreamWaitEvent(s, c->jscr[i], 0));
        }
      }
      joined = true;
      for (int m = 0; m < nmol; ++m) stage_reduce_lc(mols[m].aux, mols[m].nd, plan.bufs[m], class_lc[k], s, launches);
      reduced[class_lc[k]] = true;
    }
  }
  for (int i = 0; i < W; ++i) {
    PA_CUDA(cudaEventRecord(c->j3c[i], c->s3c[i]));
    PA_CUDA(cudaStreamWaitEvent(s, c->j3c[i], 0));
    if (!joined) {
      PA_CUDA(cudaEventRecord(c->jscr[i], c->sscrw[i]));
      PA_CUDA(cudaStreamWaitEvent(s, c->jscr[i], 0));
    }
  }
  for (int lc = 0; lc <= PA_LAUXMAX; ++lc)  // groups without class launches (zero rows)
    if (!reduced[lc])
      for (int m = 0; m < nmol; ++m) stage_reduce_lc(mols[m].aux, mols[m].nd, plan.bufs[m], lc, s, launches);
  // per molecule: (after its metric chain) solve and tensor
  PA_CUDA(cudaEventRecord(c->fork, s));
  for (int i = 0; i < W; ++i) {
    PA_CUDA(cudaStreamWaitEvent(c->s3c[i], c->fork, 0));
    PA_CUDA(cudaEventRecord(c->jmet[i], c->smet[i]));
    PA_CUDA(cudaStreamWaitEvent(c->s3c[i], c->jmet[i], 0));
  }
  for (int m = 0; m < nmol; ++m) {
    const BatchMol& M = mols[m];
    DfBuffers& b = plan.bufs[m];
    cudaStream_t w = c->s3c[m % W];
    const int st = stage_solve(M.aux, M.nd, b, o, plan.df[m], w, launches);
    if (st != PA_OK) return st;
    *launches += coulomb_4d(plan.df[m], M.aux->host.nsph, M.nd, M.ns, plan.gram[m], M.R, w);
  }
  for (int i = 0; i < W; ++i) {
    PA_CUDA(cudaEventRecord(c->j3c[i], c->s3c[i]));
    PA_CUDA(cudaStreamWaitEvent(s, c->j3c[i], 0));
  }
  return PA_OK;
}

int batch_4d(int nmol, const pa_basis* orbs, const pa_basis* auxs, const int* ndens,
             const double* const* d_dens, int layout, const int* nstates, double* const* d_R,
             int use_graph, cudaStream_t user_stream) {
  NvtxRange range("pa: batched Coulomb tensors");
  if (nmol < 0 || (nmol > 0 && (!orbs || !auxs || !ndens || !d_dens || !nstates || !d_R)))
    return fail(PA_ERR_ARG, "invalid batch arguments");
  if (layout != PA_LAYOUT_FORTRAN && layout != PA_LAYOUT_C) return fail(PA_ERR_ARG, "unknown layout");
  std::vector<BatchMol> mols(nmol);
  for (int m = 0; m < nmol; ++m) {
    int st = check_pair(orbs[m], auxs[m]);
    if (st != PA_OK) return st;
    const int nd = ndens[m], ns = nstates[m];
    if (ns <= 0 || ns * (ns + 1) / 2 != nd) return fail(PA_ERR_ARG, "molecule " + std::to_string(m) + ": ndens must equal nstates (nstates + 1) / 2");
    if (!d_dens[m] || !d_R[m]) return fail(PA_ERR_ARG, "molecule " + std::to_string(m) + ": null pointer");
    const long long n = orbs[m]->host.nsph;
    BatchMol& M = mols[m];
    M.orb = orbs[m];
    M.aux = auxs[m];
    M.nd = nd;
    M.ns = ns;
    M.dens = d_dens[m];
    M.R = d_R[m];
    if (layout == PA_LAYOUT_FORTRAN) {
      M.sd = 1;
      M.si = nd;
      M.sj = static_cast<long long>(nd) * n;
    } else {
      M.sd = n * n;
      M.si = n;
      M.sj = 1;
    }
  }
  Ctx* c = nullptr;
  DeviceTables dt;
  int st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  const Options o = options();
  // signature of the batch: options, then per molecule handles, sizes, pointers
  std::vector<long long> sig{nmol, layout, use_graph ? 1 : 0, o.boys_mode, o.skip_metric, o.precision,
                             o.mixed_kernels, o.items_per_sm, o.screening};
  for (const auto& row : o.tile_variant)
    for (signed char v : row) sig.push_back(v);
  for (double v : {o.screen_thresh, o.fp32_thresh, o.metric_shift}) {
    long long bits;
    std::memcpy(&bits, &v, sizeof bits);
    sig.push_back(bits);
  }
  for (const BatchMol& M : mols) {
    sig.push_back(M.orb->serial);
    sig.push_back(M.aux->serial);
    sig.push_back(M.nd);
    sig.push_back(reinterpret_cast<long long>(M.dens));
    sig.push_back(reinterpret_cast<long long>(M.R));
  }
  // the user's stream is ordered before the batch, the batch before the return
  PA_CUDA(cudaStreamSynchronize(user_stream));
  BatchPlan* plan = c->plan;
  const bool reuse = use_graph && plan && plan->sig == sig && plan->exec;
  int launches = 0;
  if (!reuse) {
    if (plan) {
      PA_CUDA(cudaStreamSynchronize(c->stream));
      delete plan;
      c->plan = nullptr;
    }
    plan = new BatchPlan();
    plan->sig = sig;
    plan->bufs.resize(nmol);
    plan->df.resize(nmol);
    plan->gram.resize(nmol);
    // classes present in the batch, and for each the molecules' runs
    std::vector<int> class_lab, class_lc, class_weak, class_nm, class_items;
    // classes grouped by auxiliary L, highest first (as the single-molecule
    // path orders its class launches); in the mixed form every class has an
    // FP64 run and a weak-triplet run
    const bool split = o.precision == PA_PRECISION_MIXED && o.mixed_kernels != 0 && o.fp32_thresh > o.screen_thresh;
    for (int lc = PA_LAUXMAX; lc >= 0; --lc)
      for (int lab = 0; lab <= 2 * PA_LMAX; ++lab)
        for (int weak = 0; weak <= (split ? 1 : 0); ++weak) {
          class_lab.push_back(lab);
          class_lc.push_back(lc);
          class_weak.push_back(weak);
        }
    // count, allocate, carve
    std::vector<size_t> off(nmol + 1, 0);
    for (int pass = 0; pass < 2; ++pass) {
      Carver cv;
      if (pass == 1) cv.base = plan->dmem;
      for (int m = 0; m < nmol; ++m) {
        const BatchMol& M = mols[m];
        layout_df(cv, M.orb, M.aux, M.nd, &plan->bufs[m], o);
        plan->df[m] = cv.take<double>(static_cast<size_t>(M.aux->host.nsph) * M.nd);
        plan->gram[m] = cv.take<double>(static_cast<size_t>(M.nd) * M.nd);
      }
      plan->infos = cv.take<int>(4 * std::max(nmol, 1));
      plan->counters = cv.take<int>(class_lab.size());
      if (pass == 0) {
        off[0] = cv.used;
        // room for the class descriptors: at most one per (class, molecule)
        cv.take<Df3cArgs>(class_lab.size() * std::max(nmol, 1));
        cv.take<int>(class_lab.size() * (std::max(nmol, 1) + 1));
        if (cudaMalloc(&plan->dmem, std::max<size_t>(cv.used, 256)) != cudaSuccess) {
          delete plan;
          return fail(PA_ERR_CUDA, "cudaMalloc(batch plan) failed");
        }
      }
    }
    for (int m = 0; m < nmol; ++m) plan->bufs[m].info = plan->infos + 4 * m;
    Df3cArgs* d_args = reinterpret_cast<Df3cArgs*>(plan->dmem + off[0]);
    int* d_off = reinterpret_cast<int*>(d_args + class_lab.size() * std::max(nmol, 1));
    // class descriptors (host), molecules by decreasing work within a class
    std::vector<Df3cArgs> h_args(class_lab.size() * std::max(nmol, 1));
    std::vector<int> h_off(class_lab.size() * (std::max(nmol, 1) + 1), 0);
    std::vector<const Df3cArgs*> args_d;
    std::vector<const int*> off_d;
    std::vector<int> keep_lab, keep_lc, keep_weak;
    std::vector<Df3cArgs> class_single;  // the first (heaviest) molecule's descriptor of each class
    for (size_t k = 0; k < class_lab.size(); ++k) {
      std::vector<std::pair<long long, Df3cArgs>> items;
      for (int m = 0; m < nmol; ++m) {
        const BatchMol& M = mols[m];
        const DfBuffers& b = plan->bufs[m];
        for (const auto& r : b.runs) {
          if (r.lab != class_lab[k] || r.lc != class_lc[k] || r.weak != (class_weak[k] != 0)) continue;
          Df3cArgs a = class_args(M.orb, M.aux, M.nd, b, dt, o, r);
          if (r.weak)
            df3c_fill_items_w(r.lab, r.lc, &a, r.ny);
          else
            df3c_fill_items(r.lab, r.lc, r.variant, &a, r.ny);
          const long long work = static_cast<long long>(a.n_units) * a.n_aux * a.nd;
          if (a.n_items > 0) items.push_back({work, a});
        }
      }
      if (items.empty()) continue;
      std::stable_sort(items.begin(), items.end(),
                       [](const auto& x, const auto& y) { return x.first > y.first; });
      const size_t slot = keep_lab.size();
      Df3cArgs* ha = h_args.data() + slot * std::max(nmol, 1);
      int* ho = h_off.data() + slot * (std::max(nmol, 1) + 1);
      ho[0] = 0;
      for (size_t i = 0; i < items.size(); ++i) {
        ha[i] = items[i].second;
        ho[i + 1] = ho[i] + items[i].second.n_items;
      }
      keep_lab.push_back(class_lab[k]);
      keep_lc.push_back(class_lc[k]);
      keep_weak.push_back(class_weak[k]);
      class_nm.push_back(static_cast<int>(items.size()));
      class_single.push_back(items[0].second);
      class_items.push_back(ho[items.size()]);
      args_d.push_back(d_args + slot * std::max(nmol, 1));
      off_d.push_back(d_off + slot * (std::max(nmol, 1) + 1));
    }
    PA_CUDA(cudaMemcpy(d_args, h_args.data(), sizeof(Df3cArgs) * h_args.size(), cudaMemcpyHostToDevice));
    PA_CUDA(cudaMemcpy(d_off, h_off.data(), sizeof(int) * h_off.size(), cudaMemcpyHostToDevice));
    PA_CUDA(cudaMallocHost(&plan->h_infos, sizeof(int) * 4 * std::max(nmol, 1)));
    c->plan = plan;
    if (use_graph) {
      cudaGraph_t graph = nullptr;
      PA_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
      st = record_batch(c, *plan, mols, dt, o, keep_lab, keep_lc, keep_weak, args_d, off_d, class_nm,
                        class_items, class_single, &launches);
      const cudaError_t ec = cudaStreamEndCapture(c->stream, &graph);
      if (st != PA_OK || ec != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        c->plan = nullptr;
        delete plan;
        if (st != PA_OK) return st;
        return fail(PA_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
      }
      // node priorities from the capturing streams (screening and metric
      // chains ahead of the persistent class kernels)
      const cudaError_t ei = cudaGraphInstantiateWithFlags(&plan->exec, graph, cudaGraphInstantiateFlagUseNodePriority);
      cudaGraphDestroy(graph);
      if (ei != cudaSuccess) {
        c->plan = nullptr;
        delete plan;
        return fail(PA_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ei));
      }
      plan->launches = launches;
    } else {
      PA_CUDA(cudaEventRecord(c->ev0, c->stream));
      st = record_batch(c, *plan, mols, dt, o, keep_lab, keep_lc, keep_weak, args_d, off_d, class_nm,
                        class_items, class_single, &launches);
      plan->launches = launches;
      if (st != PA_OK) {
        cudaStreamSynchronize(c->stream);
        c->plan = nullptr;
        delete plan;
        return st;
      }
    }
  }
  if (use_graph) {
    PA_CUDA(cudaEventRecord(c->ev0, c->stream));
    PA_CUDA(cudaGraphLaunch(plan->exec, c->stream));
  }
  PA_CUDA(cudaGetLastError());
  PA_CUDA(cudaEventRecord(c->ev1, c->stream));
  PA_CUDA(cudaMemcpyAsync(plan->h_infos, plan->infos, sizeof(int) * 4 * std::max(nmol, 1),
                          cudaMemcpyDeviceToHost, c->stream));
  PA_CUDA(cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  g_stats = pa_stats{};
  g_stats.ms_total = ms;
  g_stats.kernel_launches = plan->launches;
  g_stats.ntriplets = g_stats.nskipped = g_stats.nints = -1;
  if (!use_graph) {
    // an ungraphed plan is not kept for replay
    c->plan = nullptr;
    const int nm = nmol;
    std::vector<int> infos(plan->h_infos, plan->h_infos + 4 * std::max(nm, 1));
    delete plan;
    for (int m = 0; m < nm; ++m)
      if (infos[4 * m + 2] != 0)
        return fail(PA_ERR_TIMEOUT, "molecule " + std::to_string(m) + ": weak-triplet kernel: a tensor-core completion wait gave up");
    for (int m = 0; m < nm; ++m)
      if (infos[4 * m] != 0)
        return fail(PA_ERR_NOT_SPD, "molecule " + std::to_string(m) + ": metric (P|Q) is not positive definite (Cholesky pivot " +
                                        std::to_string(infos[4 * m]) + ")");
    return PA_OK;
  }
  for (int m = 0; m < nmol; ++m) {
    if (plan->h_infos[4 * m + 2] != 0)
      return fail(PA_ERR_TIMEOUT, "molecule " + std::to_string(m) + ": weak-triplet kernel: a tensor-core completion wait gave up");
    if (plan->h_infos[4 * m] != 0)
      return fail(PA_ERR_NOT_SPD, "molecule " + std::to_string(m) + ": metric (P|Q) is not positive definite (Cholesky pivot " +
                                      std::to_string(plan->h_infos[4 * m]) + ")");
  }
  return PA_OK;
}

int nstates_of(int ndens) {
  const int ns = static_cast<int>(std::lround((std::sqrt(8.0 * ndens + 1.0) - 1.0) / 2.0));
  return ns * (ns + 1) / 2 == ndens ? ns : -1;
}

// Host-buffer path: copies in, runs on the library stream, copies out.
int df_host(pa_basis orb, pa_basis aux, int ndens, int nbf, const double* dens, int layout,
            double* out, int nstates) {
  int st = check_pair(orb, aux);
  if (st != PA_OK) return st;
  Ctx* c = nullptr;
  DeviceTables dt;
  st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  const size_t nd_bytes = sizeof(double) * static_cast<size_t>(ndens) * nbf * nbf;
  const size_t df_count = static_cast<size_t>(aux->host.nsph) * ndens;
  const size_t out_count = nstates > 0 ? static_cast<size_t>(nstates) * nstates * nstates * nstates : df_count;
  double *d_dens = nullptr, *d_df = nullptr, *d_R = nullptr;
  PA_CUDA(cudaMallocFromPoolAsync(&d_dens, std::max<size_t>(nd_bytes, 8), c->pool, c->stream));
  PA_CUDA(cudaMallocFromPoolAsync(&d_df, sizeof(double) * std::max<size_t>(df_count, 1), c->pool, c->stream));
  if (nstates > 0) PA_CUDA(cudaMallocFromPoolAsync(&d_R, sizeof(double) * out_count, c->pool, c->stream));
  cudaEvent_t ready = nullptr;
  if (nd_bytes) {
    PA_CUDA(cudaEventRecord(c->ev_alloc, c->stream));
    PA_CUDA(cudaStreamWaitEvent(c->scopy, c->ev_alloc, 0));
    PA_CUDA(cudaMemcpyAsync(d_dens, dens, nd_bytes, cudaMemcpyHostToDevice, c->scopy));
    PA_CUDA(cudaEventRecord(c->ev_copied, c->scopy));
    ready = c->ev_copied;
  }
  st = df_device(orb, aux, ndens, nbf, d_dens, layout, d_df, nstates, d_R, c->stream, ready);
  if (st != PA_OK && ready) cudaStreamWaitEvent(c->stream, ready, 0);  // the copy ends before the free
  if (st == PA_OK) {
    cudaMemcpyAsync(out, nstates > 0 ? d_R : d_df, sizeof(double) * out_count, cudaMemcpyDeviceToHost,
                    c->stream);
  }
  cudaFreeAsync(d_dens, c->stream);
  cudaFreeAsync(d_df, c->stream);
  if (d_R) cudaFreeAsync(d_R, c->stream);
  const cudaError_t e = cudaStreamSynchronize(c->stream);
  if (st != PA_OK) return st;
  if (e != cudaSuccess) return fail(PA_ERR_CUDA, std::string("download: ") + cudaGetErrorString(e));
  return PA_OK;
}

// ---------------------------------------------------------------------------
// sTDDFT tensors (std/intor.f90). kind: 0 = df1c (nbf x naux), 1 = eri2c
// (nbf x nbf), 2 = df2c_mo (nmos(nmos+1)/2 x naux); all column-major.
enum StdKind { kStdDf1c = 0, kStdEri2c = 1, kStdDf2cMo = 2 };

// Doubles of W per batch of the df2c_mo half transformation (1 GiB).
constexpr size_t kStdWBudget = size_t(1) << 27;

int std_device(pa_basis orb, pa_basis aux, int kind, int nmos, const double* d_mo, double* d_out,
               cudaStream_t s) {
  NvtxRange range(kind == kStdDf1c ? "pa: std df1c" : (kind == kStdEri2c ? "pa: std eri2c" : "pa: std df2c_mo"));
  int st = check_pair(orb, aux);
  if (st != PA_OK) return st;
  if (kind == kStdDf2cMo && (nmos < 0 || (nmos > 0 && !d_mo))) return fail(PA_ERR_ARG, "invalid MO tensor");
  if (!d_out) return fail(PA_ERR_ARG, "null output pointer");
  if (orb->host.shells.size() > 65535) return fail(PA_ERR_ARG, "more than 65535 orbital shells");
  Ctx* c = nullptr;
  DeviceTables dt;
  st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  const Options o = options();
  const PairLists& P = orb->pairs;
  const int nbf = orb->host.nsph, naux = aux->host.nsph;
  const int nx = static_cast<int>(aux->host.shells.size());
  const long long npack = static_cast<long long>(nmos) * (nmos + 1) / 2;
  const long long ncols = kind == kStdDf2cMo ? npack : nbf;
  // auxiliary shell batches of the df2c_mo half transformation
  std::vector<int> batch{0};
  size_t wmax = 0, resmax = 0;
  if (kind == kStdDf2cMo && nmos > 0) {
    const size_t per_fn = static_cast<size_t>(nmos) * nbf;
    size_t fns = 0;
    for (int i = 0; i < nx; ++i) {
      const size_t f = 2 * aux->host.shells[i].L + 1;
      if (fns > 0 && (fns + f) * per_fn > kStdWBudget) {
        batch.push_back(i);
        fns = 0;
      }
      fns += f;
      wmax = std::max(wmax, fns * per_fn);
      resmax = std::max(resmax, fns * static_cast<size_t>(nmos) * nmos);
    }
  }
  batch.push_back(nx);
  Carver cnt;
  // one layout, carved twice (count, then real)
  struct Bufs {
    double *Qab, *Qc, *esph, *M, *lawork, *raw, *y, *W, *res;
    double4* pP;
    int* info;
  } b{};
  for (int pass = 0; pass < 2; ++pass) {
    Carver cv;
    if (pass == 1) {
      PA_CUDA(c->arena.reserve(cnt.used));
      cv.base = c->arena.base;
    }
    b.Qab = cv.take<double>(P.npairs);
    b.Qc = cv.take<double>(nx);
    b.pP = cv.take<double4>(P.nunits);
    b.esph = cv.take<double>(P.esph_total);
    b.M = cv.take<double>(static_cast<size_t>(naux) * naux);
    b.lawork = cv.take<double>(linalg_workspace_doubles(naux));
    b.info = cv.take<int>(4);
    b.raw = cv.take<double>(static_cast<size_t>(naux) * ncols);
    b.y = cv.take<double>(static_cast<size_t>(naux) * ncols);
    b.W = cv.take<double>(wmax);
    b.res = cv.take<double>(resmax);
    if (pass == 0) cnt = cv;
  }
  PA_CUDA(cudaEventRecord(c->ev0, s));
  int launches = 0;
  // metric + Cholesky on the second stream
  cudaStream_t s2 = c->stream2;
  PA_CUDA(cudaEventRecord(c->fork, s));
  PA_CUDA(cudaStreamWaitEvent(s2, c->fork, 0));
  PA_CUDA(cudaEventRecord(c->m0, s2));
  launches += launch_metric(aux->dev, dt, o.boys_mode, b.M, s2);
  launches += add_diagonal(b.M, naux, o.metric_shift, s2);
  launches += cholesky_lower(b.M, naux, b.info, b.lawork, s2, &c->la2);
  PA_CUDA(cudaEventRecord(c->m1, s2));
  // Schwarz vectors (screener%init, common/screening.f90:101-163)
  UnitArrays U;
  U.unit_pair = orb->d_unit_pair;
  U.unit_prims = orb->d_unit_prims;
  U.unit_esph = orb->d_unit_esph;
  U.unit_pP = b.pP;
  U.esph = b.esph;
  launches += launch_unit_setup(orb->dev, orb->d_pair_ab, orb->d_class_unit, P, U, dt, s);
  launches += launch_schwarz_bra(orb->dev, orb->d_pair_ab, orb->d_pair_unit0, orb->d_class_pair, P, U, dt,
                                 o.boys_mode, b.Qab, s);
  launches += launch_schwarz_aux(aux->dev, dt, o.boys_mode, b.Qc, s);
  PA_CUDA(cudaEventRecord(c->ph[0], s));
  StdArgs a;
  a.B = orb->dev;
  a.X = aux->dev;
  a.dt = dt;
  a.boys_mode = o.boys_mode;
  a.thresh = o.screen_thresh;
  a.pair_ab = orb->d_pair_ab;
  a.pair_unit0 = orb->d_pair_unit0;
  a.unit_pP = b.pP;
  a.esph = b.esph;
  a.unit_esph = orb->d_unit_esph;
  a.Qab = b.Qab;
  a.Qc = b.Qc;
  const size_t raw_bytes = sizeof(double) * static_cast<size_t>(naux) * ncols;
  if (kind != kStdDf2cMo) {
    // screened (a, a, c) entries stay zero (the reference's output starts zeroed)
    if (raw_bytes) PA_CUDA(cudaMemsetAsync(b.raw, 0, raw_bytes, s));
    launches += launch_std_df1c(a, b.raw, s);
  } else if (nmos > 0) {
    for (size_t bi = 0; bi + 1 < batch.size(); ++bi) {
      const int c0 = batch[bi], c1 = batch[bi + 1];
      if (c1 <= c0) continue;
      const int k0 = aux->host.shells[c0].sph_off;
      const int k1 = c1 < nx ? aux->host.shells[c1].sph_off : naux;
      const int nk = k1 - k0;
      launches += launch_std_df2c_half(a, c0, c1, k0, nmos, d_mo, b.W, s);
      // Res[(kk, p), q] = sum_nu W[(kk, p)][nu] C[nu, q] (std/intor.f90:263-279)
      launches += gemm(true, false, nk * nmos, nmos, nbf, 1.0, b.W, nbf, d_mo, nbf, 0.0, b.res,
                       static_cast<long long>(nk) * nmos, false, s);
      launches += launch_std_pack(b.res, nk, nmos, k0, naux, b.raw, s);
    }
  }
  PA_CUDA(cudaEventRecord(c->ph[1], s));
  PA_CUDA(cudaStreamWaitEvent(s, c->m1, 0));
  const double* y = b.raw;
  if (!o.skip_metric && ncols > 0 && naux > 0) {
    // T L^-T = (L^-1 T^T)^T (std/intor.f90:116,290: dtrmm("R","L","T","N"))
    launches += trsm_lower_left(b.M, naux, b.lawork, b.raw, naux, static_cast<int>(ncols), b.y, naux, s);
    y = b.y;
  }
  if (kind == kStdEri2c) {
    // (mu mu|nu nu) = T T^T (std/intor.f90:137)
    launches += gemm(true, false, nbf, nbf, naux, 1.0, y, naux, y, naux, 0.0, d_out, nbf, false, s);
    if (naux == 0 && nbf > 0)
      PA_CUDA(cudaMemsetAsync(d_out, 0, sizeof(double) * static_cast<size_t>(nbf) * nbf, s));
  } else {
    launches += launch_transpose(y, static_cast<int>(ncols), naux, d_out, s);
  }
  PA_CUDA(cudaGetLastError());
  PA_CUDA(cudaEventRecord(c->ev1, s));
  PA_CUDA(cudaMemcpyAsync(c->h_info, b.info, sizeof(int), cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  float t[4] = {0, 0, 0, 0};
  PA_CUDA(cudaEventElapsedTime(&t[0], c->ev0, c->ev1));
  PA_CUDA(cudaEventElapsedTime(&t[1], c->ev0, c->ph[0]));
  PA_CUDA(cudaEventElapsedTime(&t[2], c->ph[0], c->ph[1]));
  PA_CUDA(cudaEventElapsedTime(&t[3], c->m0, c->m1));
  g_stats = pa_stats{};
  g_stats.ms_total = t[0];
  g_stats.ms_screen = t[1];
  g_stats.ms_3c = t[2];
  g_stats.ms_metric = t[3];
  g_stats.ms_solve = t[0] - t[1] - t[2];
  g_stats.kernel_launches = launches;
  g_stats.launches_3c = 0;
  g_stats.ntriplets = -1;
  g_stats.nskipped = -1;
  g_stats.nints = -1;
  if (*c->h_info != 0)
    return fail(PA_ERR_NOT_SPD, "metric (P|Q) is not positive definite (Cholesky pivot " +
                                    std::to_string(*c->h_info) + ")");
  return PA_OK;
}

// Host-buffer std call: uploads the MO tensor, runs, downloads.
int std_host(pa_basis orb, pa_basis aux, int kind, int nmos, const double* mo, double* out,
             size_t out_count) {
  int st = check_pair(orb, aux);
  if (st != PA_OK) return st;
  Ctx* c = nullptr;
  DeviceTables dt;
  st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  const size_t mo_bytes = sizeof(double) * static_cast<size_t>(orb->host.nsph) * std::max(nmos, 0);
  double *d_mo = nullptr, *d_out = nullptr;
  PA_CUDA(cudaMallocFromPoolAsync(&d_mo, std::max<size_t>(mo_bytes, 8), c->pool, c->stream));
  PA_CUDA(cudaMallocFromPoolAsync(&d_out, sizeof(double) * std::max<size_t>(out_count, 1), c->pool, c->stream));
  if (mo_bytes) PA_CUDA(cudaMemcpyAsync(d_mo, mo, mo_bytes, cudaMemcpyHostToDevice, c->stream));
  st = std_device(orb, aux, kind, nmos, d_mo, d_out, c->stream);
  if (st == PA_OK && out_count)
    cudaMemcpyAsync(out, d_out, sizeof(double) * out_count, cudaMemcpyDeviceToHost, c->stream);
  cudaFreeAsync(d_mo, c->stream);
  cudaFreeAsync(d_out, c->stream);
  const cudaError_t e = cudaStreamSynchronize(c->stream);
  if (st != PA_OK) return st;
  if (e != cudaSuccess) return fail(PA_ERR_CUDA, std::string("download: ") + cudaGetErrorString(e));
  return PA_OK;
}

// Bases of the f_* entry points. Their callers pass the same basis arrays call
// after call, so the unpacked basis with its device copy and shell-pair lists
// is kept for later calls with byte-identical arrays (same device and angular
// momentum limit): at most kBasisCacheSize per process, least recently used
// first out. A call holds a reference for its duration, so an eviction by
// another thread never frees a basis in use. pa_basis_cache_clear() empties
// the cache.
constexpr size_t kBasisCacheSize = 8;
struct BasisEntry {
  int device = 0, lmax = 0, nshells = 0, ndata = 0;
  std::vector<int> centers, spec;
  std::vector<double> data;
  std::shared_ptr<pa_basis_s> basis;
};
struct BasisCache {
  std::mutex mu;
  std::list<BasisEntry> entries;  // most recently used first
};
// never destroyed: no device frees run during process teardown
BasisCache& basis_cache() {
  static BasisCache* c = new BasisCache();
  return *c;
}

struct BasisGuard {
  pa_basis b = nullptr;
  std::shared_ptr<pa_basis_s> keep;
};

int acquire_basis(int nshells, int ndata, const int* centers, const int* spec, const double* data, int lmax,
                  BasisGuard* g) {
  const bool valid = nshells >= 0 && ndata >= 0 && (nshells == 0 || (centers && spec)) && (ndata == 0 || data);
  int dev = 0;
  cudaGetDevice(&dev);
  BasisCache& cache = basis_cache();
  if (valid) {
    std::lock_guard<std::mutex> lk(cache.mu);
    for (auto it = cache.entries.begin(); it != cache.entries.end(); ++it) {
      if (it->device != dev || it->lmax != lmax || it->nshells != nshells || it->ndata != ndata) continue;
      if (nshells > 0 && (std::memcmp(it->centers.data(), centers, sizeof(int) * 3 * nshells) != 0 ||
                          std::memcmp(it->spec.data(), spec, sizeof(int) * 5 * nshells) != 0))
        continue;
      if (ndata > 0 && std::memcmp(it->data.data(), data, sizeof(double) * ndata) != 0) continue;
      cache.entries.splice(cache.entries.begin(), cache.entries, it);
      g->keep = cache.entries.front().basis;
      g->b = g->keep.get();
      return PA_OK;
    }
  }
  pa_basis b = nullptr;
  const int st = pa_basis_create(nshells, ndata, centers, spec, data, lmax, &b);
  if (st != PA_OK) return st;
  g->keep = std::shared_ptr<pa_basis_s>(b, [](pa_basis p) { pa_basis_destroy(p); });
  g->b = b;
  BasisEntry e;
  e.device = dev;
  e.lmax = lmax;
  e.nshells = nshells;
  e.ndata = ndata;
  e.centers.assign(centers, centers + 3 * static_cast<size_t>(nshells));
  e.spec.assign(spec, spec + 5 * static_cast<size_t>(nshells));
  if (ndata > 0) e.data.assign(data, data + ndata);
  e.basis = g->keep;
  std::lock_guard<std::mutex> lk(cache.mu);
  cache.entries.push_front(std::move(e));
  while (cache.entries.size() > kBasisCacheSize) cache.entries.pop_back();
  return PA_OK;
}

}  // namespace
}  // namespace pa

// ---------------------------------------------------------------------------
// C-ABI
using namespace pa;

extern "C" {

const char* pa_last_error(void) { return tl_err.c_str(); }

int pa_set_boys_mode(int mode) {
  if (mode != PA_BOYS_EXACT && mode != PA_BOYS_REFERENCE) return fail(PA_ERR_ARG, "unknown Boys mode");
  std::lock_guard<std::mutex> lk(g_opt_mu);
  g_opts.boys_mode = mode;
  return PA_OK;
}

int pa_get_boys_mode(void) {
  std::lock_guard<std::mutex> lk(g_opt_mu);
  return g_opts.boys_mode;
}

int pa_set_screen_threshold(double thresh) {
  if (!(thresh >= 0.0)) return fail(PA_ERR_ARG, "threshold must be >= 0");
  std::lock_guard<std::mutex> lk(g_opt_mu);
  g_opts.screen_thresh = thresh;
  return PA_OK;
}

int pa_set_precision(int mode, double fp32_thresh) {
  if (mode != PA_PRECISION_FP64 && mode != PA_PRECISION_MIXED) return fail(PA_ERR_ARG, "unknown precision mode");
  if (!(fp32_thresh >= 0.0) || !std::isfinite(fp32_thresh)) return fail(PA_ERR_ARG, "FP32 threshold must be finite and >= 0");
  std::lock_guard<std::mutex> lk(g_opt_mu);
  g_opts.precision = mode;
  g_opts.fp32_thresh = fp32_thresh;
  return PA_OK;
}

int pa_get_precision(void) {
  std::lock_guard<std::mutex> lk(g_opt_mu);
  return g_opts.precision;
}

int pa_basis_cache_clear(void) {
  pa::BasisCache& cache = pa::basis_cache();
  std::lock_guard<std::mutex> lk(cache.mu);
  cache.entries.clear();
  return PA_OK;
}

int pa_get_device(int* device) {
  if (!device) return fail(PA_ERR_ARG, "null output pointer");
  const cudaError_t e = cudaGetDevice(device);
  if (e != cudaSuccess) return fail(PA_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  return PA_OK;
}

int pa_set_class_grid(int mode) {
  if (mode != 0 && mode != 1) return fail(PA_ERR_ARG, "class grid: 0 (persistent blocks) or 1 (one block per work item)");
  pa::set_df3c_block_per_item(mode);
  return PA_OK;
}

int pa_set_mixed_kernels(int mode) {
  if (mode != 0 && mode != 1) return fail(PA_ERR_ARG, "mixed-form kernels: 0 (FP32 recurrences in the FP64 kernels) or 1 (weak-triplet kernels)");
  std::lock_guard<std::mutex> lk(g_opt_mu);
  g_opts.mixed_kernels = mode;
  return PA_OK;
}

int pa_get_mixed_kernels(void) {
  std::lock_guard<std::mutex> lk(g_opt_mu);
  return g_opts.mixed_kernels;
}

int pa_set_screening(int mode) {
  if (mode != PA_SCREEN_SCHWARZ && mode != PA_SCREEN_QVL) return fail(PA_ERR_ARG, "unknown screening mode");
  std::lock_guard<std::mutex> lk(g_opt_mu);
  g_opts.screening = mode;
  return PA_OK;
}

int pa_get_screening(void) {
  std::lock_guard<std::mutex> lk(g_opt_mu);
  return g_opts.screening;
}

int pa_set_items_per_sm(int items) {
  if (items < 0 || items > 1024) return fail(PA_ERR_ARG, "items per SM must be in [0, 1024] (0 = by size)");
  std::lock_guard<std::mutex> lk(g_opt_mu);
  g_opts.items_per_sm = items;
  return PA_OK;
}

int pa_set_class_timing(int on) {
  std::lock_guard<std::mutex> lk(g_opt_mu);
  g_opts.class_timing = on ? 1 : 0;
  return PA_OK;
}

int pa_get_class_times(int cap, int* lab, int* lc, double* ms) {
  std::lock_guard<std::mutex> lk(g_ct_mu);
  const int n = static_cast<int>(g_class_times.size());
  for (int i = 0; i < std::min(n, cap); ++i) {
    if (lab) lab[i] = g_class_times[i].lab;
    if (lc) lc[i] = g_class_times[i].lc;
    if (ms) ms[i] = g_class_times[i].ms;
  }
  return n;
}

int pa_set_tile_variant(int lab, int lc, int variant) {
  if (lab < 0 || lab > 2 * PA_LMAX || lc < 0 || lc > PA_LAUXMAX)
    return fail(PA_ERR_ARG, "tile variant: class (L_ab, L_c) out of range");
  if (variant < 0 || variant >= kDf3cVariants) return fail(PA_ERR_ARG, "tile variant out of range");
  options();  // the default table is applied first, so it cannot override this call later
  std::lock_guard<std::mutex> lk(g_opt_mu);
  g_opts.tile_variant[lab][lc] = static_cast<signed char>(variant);
  return PA_OK;
}

int pa_get_tile_variant(int lab, int lc, int* variant) {
  if (lab < 0 || lab > 2 * PA_LMAX || lc < 0 || lc > PA_LAUXMAX || !variant)
    return fail(PA_ERR_ARG, "tile variant: class (L_ab, L_c) out of range");
  *variant = options().tile_variant[lab][lc];
  return PA_OK;
}

int pa_tile_shape(int lab, int lc, int variant, int* out) {
  if (lab < 0 || lab > 2 * PA_LMAX || lc < 0 || lc > PA_LAUXMAX || variant < 0 || variant >= kDf3cVariants ||
      !out)
    return fail(PA_ERR_ARG, "tile shape: class or variant out of range");
  Df3cClassInfo ci;
  df3c_class_info(lab, lc, variant, &ci);
  out[0] = ci.tc;
  out[1] = ci.ub;
  out[2] = ci.lanes;
  out[3] = ci.blocks_per_sm;
  out[4] = static_cast<int>(ci.smem);
  return PA_OK;
}

int pa_load_tile_table(const char* path, int* napplied) {
  options();  // the default table first (a later explicit table wins)
  const std::string p = path ? std::string(path) : default_tile_table();
  const int n = p.empty() ? 0 : apply_tile_table(p.c_str());
  if (n == -1 && path) return fail(PA_ERR_ARG, "tile table: cannot read " + p);
  if (n == -2) return fail(PA_ERR_ARG, "tile table: malformed or out-of-range entry in " + p);
  if (napplied) *napplied = std::max(n, 0);
  return PA_OK;
}

int pa_set_metric_shift(double shift) {
  if (!(shift >= 0.0) || !std::isfinite(shift)) return fail(PA_ERR_ARG, "metric shift must be finite and >= 0");
  std::lock_guard<std::mutex> lk(g_opt_mu);
  g_opts.metric_shift = shift;
  return PA_OK;
}

int pa_set_skip_metric(int skip) {
  std::lock_guard<std::mutex> lk(g_opt_mu);
  g_opts.skip_metric = skip ? 1 : 0;
  return PA_OK;
}

int pa_get_stats(pa_stats* out) {
  if (!out) return fail(PA_ERR_ARG, "null stats pointer");
  *out = g_stats;
  return PA_OK;
}

int f_init(void) {
  Ctx* c = nullptr;
  DeviceTables dt;
  return current_ctx(&c, &dt);
}

int pa_basis_create(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                    const double* bas_data, int lmax_allowed, pa_basis* out) {
  if (!out) return fail(PA_ERR_ARG, "null output handle");
  *out = nullptr;
  if (lmax_allowed < 0 || lmax_allowed > std::max(PA_LMAX, PA_LAUXMAX))
    lmax_allowed = std::max(PA_LMAX, PA_LAUXMAX);
  Ctx* c = nullptr;
  DeviceTables dt;
  int st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  pa_basis b = new pa_basis_s();
  {
    static std::atomic<long long> next_serial{1};
    b->serial = next_serial++;
  }
  cudaGetDevice(&b->device);
  std::string err;
  st = unpack_basis(nshells, ndata, bas_centers, bas_spec, bas_data, lmax_allowed, &b->host, &err);
  if (st != PA_OK) {
    delete b;
    return fail(st, err);
  }
  build_aux_lists(b->host, &b->aux);
  build_qvl_aux(b->host, &b->aux_qvl);
  const HostBasis& h = b->host;
  const int ns = static_cast<int>(h.shells.size());
  Carver cnt;
  for (int pass = 0; pass < 2; ++pass) {
    Carver& cv = cnt;
    if (pass == 1) {
      if (cudaMalloc(&b->dmem, std::max<size_t>(cnt.used, 256)) != cudaSuccess) {
        delete b;
        return fail(PA_ERR_CUDA, "cudaMalloc(basis) failed");
      }
      cv = Carver();
      cv.base = b->dmem;
    }
    b->dev.shell = cv.take<int4>(ns);
    b->dev.center = cv.take<double4>(ns);
    b->dev.prim = cv.take<double2>(h.exps.size());
    b->d_aux_shell = cv.take<int>(b->aux.class_shell.size());
    b->d_aux_off = cv.take<int>(b->aux.class_off.size());
    b->d_aux_qvl = cv.take<double2>(b->aux_qvl.size());
  }
  std::vector<int4> shell(ns);
  std::vector<double4> center(ns);
  for (int i = 0; i < ns; ++i) {
    const HostShell& s = h.shells[i];
    shell[i] = make_int4(s.L, s.nprim, s.prim_off, s.sph_off);
    center[i] = make_double4(s.A[0], s.A[1], s.A[2], 0.0);
  }
  std::vector<double2> prim(h.exps.size());
  for (size_t k = 0; k < prim.size(); ++k) prim[k] = make_double2(h.exps[k], h.coefs[k]);
  // one host image of the carved block, one copy
  std::vector<char> stage(cnt.used);
  auto put = [&](const void* dst, const void* src, size_t bytes) {
    if (bytes) std::memcpy(stage.data() + (static_cast<const char*>(dst) - b->dmem), src, bytes);
  };
  put(b->dev.shell, shell.data(), sizeof(int4) * ns);
  put(b->dev.center, center.data(), sizeof(double4) * ns);
  put(b->dev.prim, prim.data(), sizeof(double2) * prim.size());
  put(b->d_aux_shell, b->aux.class_shell.data(), sizeof(int) * b->aux.class_shell.size());
  put(b->d_aux_off, b->aux.class_off.data(), sizeof(int) * b->aux.class_off.size());
  put(b->d_aux_qvl, b->aux_qvl.data(), sizeof(double2) * b->aux_qvl.size());
  const cudaError_t e = cnt.used ? cudaMemcpy(b->dmem, stage.data(), cnt.used, cudaMemcpyHostToDevice) : cudaSuccess;
  if (e != cudaSuccess) {
    cudaFree(b->dmem);
    delete b;
    return fail(PA_ERR_CUDA, std::string("basis upload: ") + cudaGetErrorString(e));
  }
  b->dev.nshells = ns;
  b->dev.nprims = static_cast<int>(h.exps.size());
  b->dev.nsph = h.nsph;
  b->dev.lmax = h.lmax;
  *out = b;
  return PA_OK;
}

int pa_basis_destroy(pa_basis basis) {
  if (!basis) return PA_OK;
  if (basis->dmem) cudaFree(basis->dmem);
  if (basis->dpair) cudaFree(basis->dpair);
  if (basis->dqvl) cudaFree(basis->dqvl);
  delete basis;
  return PA_OK;
}

int pa_basis_info(pa_basis basis, int* nshells, int* nsph, int* lmax) {
  if (!basis) return fail(PA_ERR_ARG, "null basis handle");
  if (nshells) *nshells = static_cast<int>(basis->host.shells.size());
  if (nsph) *nsph = basis->host.nsph;
  if (lmax) *lmax = basis->host.lmax;
  return PA_OK;
}

int pa_df_2d(pa_basis orbital, pa_basis aux, int ndens, int nbf, const double* d_densities,
             int layout, double* d_df, void* stream) {
  if (orbital && orbital->host.lmax > PA_LMAX)
    return fail(PA_ERR_LMAX, "orbital basis L above the compiled maximum");
  return df_device(orbital, aux, ndens, nbf, d_densities, layout, d_df, 0, nullptr,
                   static_cast<cudaStream_t>(stream));
}

int pa_df_4d(pa_basis orbital, pa_basis aux, int ndens, int nbf, const double* d_densities,
             int layout, int nstates, double* d_coulomb, void* stream) {
  if (nstates < 0 || nstates * (nstates + 1) / 2 != ndens)
    return fail(PA_ERR_ARG, "ndens must equal nstates (nstates + 1) / 2");
  if (!d_coulomb) return fail(PA_ERR_ARG, "null output pointer");
  Ctx* c = nullptr;
  DeviceTables dt;
  int st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  double* d_df = nullptr;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  PA_CUDA(cudaMallocFromPoolAsync(&d_df, sizeof(double) * std::max<size_t>(1, static_cast<size_t>(aux ? aux->host.nsph : 0) * ndens), c->pool, s));
  st = df_device(orbital, aux, ndens, nbf, d_densities, layout, d_df, nstates, d_coulomb, s);
  cudaFreeAsync(d_df, s);
  return st;
}

int pa_contract_coulomb_densities_2d(pa_basis orbital, pa_basis aux, int ndens, int nbf,
                                     const double* densities, int layout, double* df_tensor) {
  return df_host(orbital, aux, ndens, nbf, densities, layout, df_tensor, 0);
}

int pa_contract_coulomb_densities_4d(pa_basis orbital, pa_basis aux, int ndens, int nbf,
                                     const double* densities, int layout, int nstates,
                                     double* coulomb_tensor) {
  if (nstates <= 0 || nstates * (nstates + 1) / 2 != ndens)
    return fail(PA_ERR_ARG, "ndens must equal nstates (nstates + 1) / 2");
  return df_host(orbital, aux, ndens, nbf, densities, layout, coulomb_tensor, nstates);
}

int f_contract_coulomb_densities_2d(int nshells, int ndata, const int* bas_centers,
                                    const int* bas_spec, const double* bas_data, int nshells_aux,
                                    int ndata_aux, const int* bas_centers_aux,
                                    const int* bas_spec_aux, const double* bas_data_aux,
                                    int ndens, int nbfs, const double* densities, int naux,
                                    double* df_tensor) {
  BasisGuard orb, aux;
  int st = acquire_basis(nshells, ndata, bas_centers, bas_spec, bas_data, PA_LMAX, &orb);
  if (st != PA_OK) return st;
  st = acquire_basis(nshells_aux, ndata_aux, bas_centers_aux, bas_spec_aux, bas_data_aux,
                       PA_LAUXMAX, &aux);
  if (st != PA_OK) return st;
  if (naux != aux.b->host.nsph)
    return fail(PA_ERR_ARG, "naux (" + std::to_string(naux) + ") does not match the auxiliary basis (" +
                                std::to_string(aux.b->host.nsph) + ")");
  return df_host(orb.b, aux.b, ndens, nbfs, densities, PA_LAYOUT_FORTRAN, df_tensor, 0);
}

int f_contract_coulomb_densities_4d(int nshells, int ndata, const int* bas_centers,
                                    const int* bas_spec, const double* bas_data, int nshells_aux,
                                    int ndata_aux, const int* bas_centers_aux,
                                    const int* bas_spec_aux, const double* bas_data_aux,
                                    int ndens, int nbfs, const double* densities, int nstates,
                                    double* coulomb_tensor) {
  if (nstates <= 0 || nstates * (nstates + 1) / 2 != ndens)
    return fail(PA_ERR_ARG, "ndens must equal nstates (nstates + 1) / 2");
  BasisGuard orb, aux;
  int st = acquire_basis(nshells, ndata, bas_centers, bas_spec, bas_data, PA_LMAX, &orb);
  if (st != PA_OK) return st;
  st = acquire_basis(nshells_aux, ndata_aux, bas_centers_aux, bas_spec_aux, bas_data_aux,
                       PA_LAUXMAX, &aux);
  if (st != PA_OK) return st;
  return df_host(orb.b, aux.b, ndens, nbfs, densities, PA_LAYOUT_FORTRAN, coulomb_tensor, nstates);
}

// Schwarz vectors through the screening stage of the pipeline.
static int schwarz_impl(pa_basis orb, pa_basis aux, double* q_bra, double* q_aux) {
  Ctx* c = nullptr;
  DeviceTables dt;
  int st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  const Options o = options();
  cudaStream_t s = c->stream;
  int launches = 0;
  if (orb) {
    const int pst = ensure_pairs(orb);
    if (pst != PA_OK) return pst;
    const PairLists& P = orb->pairs;
    Carver cnt;
    double* Qab = cnt.take<double>(P.npairs);
    double4* pP = cnt.take<double4>(P.nunits);
    double* esph = cnt.take<double>(P.esph_total);
    PA_CUDA(c->arena.reserve(cnt.used));
    Carver r;
    r.base = c->arena.base;
    Qab = r.take<double>(P.npairs);
    pP = r.take<double4>(P.nunits);
    esph = r.take<double>(P.esph_total);
    UnitArrays U;
    U.unit_pair = orb->d_unit_pair;
    U.unit_prims = orb->d_unit_prims;
    U.unit_esph = orb->d_unit_esph;
    U.unit_pP = pP;
    U.esph = esph;
    launches += launch_unit_setup(orb->dev, orb->d_pair_ab, orb->d_class_unit, P, U, dt, s);
    launches += launch_schwarz_bra(orb->dev, orb->d_pair_ab, orb->d_pair_unit0, orb->d_class_pair, P, U, dt,
                                   o.boys_mode, Qab, s);
    if (P.npairs) PA_CUDA(cudaMemcpyAsync(q_bra, Qab, sizeof(double) * P.npairs, cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaStreamSynchronize(s));
  }
  if (aux) {
    const int nx = static_cast<int>(aux->host.shells.size());
    PA_CUDA(c->arena.reserve(sizeof(double) * nx + 256));
    double* Qc = reinterpret_cast<double*>(c->arena.base);
    launches += launch_schwarz_aux(aux->dev, dt, o.boys_mode, Qc, s);
    if (nx) PA_CUDA(cudaMemcpyAsync(q_aux, Qc, sizeof(double) * nx, cudaMemcpyDeviceToHost, s));
    PA_CUDA(cudaStreamSynchronize(s));
  }
  PA_CUDA(cudaGetLastError());
  g_stats.kernel_launches = launches;
  return PA_OK;
}

int f_int_schwarz_aux(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                      const double* bas_data, double* integrals) {
  BasisGuard b;
  int st = acquire_basis(nshells, ndata, bas_centers, bas_spec, bas_data, PA_LAUXMAX, &b);
  if (st != PA_OK) return st;
  if (nshells > 0 && !integrals) return fail(PA_ERR_ARG, "null output pointer");
  return schwarz_impl(nullptr, b.b, nullptr, integrals);
}

int f_int_schwarz_bra(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                      const double* bas_data, double* integrals) {
  BasisGuard b;
  int st = acquire_basis(nshells, ndata, bas_centers, bas_spec, bas_data, PA_LMAX, &b);
  if (st != PA_OK) return st;
  if (nshells > 0 && !integrals) return fail(PA_ERR_ARG, "null output pointer");
  return schwarz_impl(b.b, nullptr, integrals, nullptr);
}

int pa_count_triplets(pa_basis orbital, pa_basis aux, long long* ntriplets, long long* ncomputed,
                      long long* nints) {
  int st = check_pair(orbital, aux);
  if (st != PA_OK) return st;
  std::vector<double> qb(orbital->pairs.npairs), qc(aux->host.shells.size());
  st = schwarz_impl(orbital, aux, qb.data(), qc.data());
  if (st != PA_OK) return st;
  const Options o = options();
  const double thr = o.screen_thresh;
  if (o.screening == PA_SCREEN_QVL) {
    // every (pair, shell) with the estimate of the kernels (qvl_estimate)
    long long ncomp = 0, ni = 0;
    const HostBasis& X = aux->host;
    for (int p = 0; p < orbital->pairs.npairs; ++p) {
      const int2 ab = orbital->pairs.pair_ab[p];
      const long long nab = static_cast<long long>(2 * orbital->host.shells[ab.x].L + 1) *
                            (2 * orbital->host.shells[ab.y].L + 1);
      const double4 pq = orbital->pair_qvl[p];
      for (size_t c = 0; c < X.shells.size(); ++c) {
        const HostShell& sc = X.shells[c];
        const double dx = pq.x - sc.A[0], dy = pq.y - sc.A[1], dz = pq.z - sc.A[2];
        const double R = std::sqrt(dx * dx + dy * dy + dz * dz);
        double est;
        if (R <= pq.w + aux->aux_qvl[c].x) {
          est = qb[p] * qc[c];
        } else {
          double RL = R;
          for (int l = 0; l < sc.L; ++l) RL *= R;
          est = qb[p] * kPi * 1.4142135623730951 * aux->aux_qvl[c].y / (orbital->pair_den[p] * RL);
        }
        if (est >= thr) {
          ++ncomp;
          ni += nab * (2 * sc.L + 1);
        }
      }
    }
    const long long all = static_cast<long long>(orbital->pairs.npairs) * qc.size();
    if (ntriplets) *ntriplets = all;
    if (ncomputed) *ncomputed = ncomp;
    if (nints) *nints = ni;
    g_stats.ntriplets = all;
    g_stats.nskipped = all - ncomp;
    g_stats.nints = ni;
    return PA_OK;
  }
  std::vector<std::pair<double, int>> sc;
  for (size_t i = 0; i < qc.size(); ++i) sc.push_back({qc[i], 2 * aux->host.shells[i].L + 1});
  std::sort(sc.begin(), sc.end(), [](const auto& x, const auto& y) { return x.first > y.first; });
  std::vector<long long> pre(sc.size() + 1, 0);
  for (size_t i = 0; i < sc.size(); ++i) pre[i + 1] = pre[i] + sc[i].second;
  long long ncomp = 0, ni = 0;
  for (int p = 0; p < orbital->pairs.npairs; ++p) {
    const double q = qb[p];
    size_t lo = 0, hi = sc.size();  // count of leading entries with q * qc >= thr
    while (lo < hi) {
      const size_t mid = (lo + hi) / 2;
      if (q * sc[mid].first >= thr)
        lo = mid + 1;
      else
        hi = mid;
    }
    const int2 ab = orbital->pairs.pair_ab[p];
    const long long nab = static_cast<long long>(2 * orbital->host.shells[ab.x].L + 1) *
                          (2 * orbital->host.shells[ab.y].L + 1);
    ncomp += static_cast<long long>(lo);
    ni += nab * pre[lo];
  }
  if (ntriplets) *ntriplets = static_cast<long long>(orbital->pairs.npairs) * qc.size();
  if (ncomputed) *ncomputed = ncomp;
  if (nints) *nints = ni;
  g_stats.ntriplets = static_cast<long long>(orbital->pairs.npairs) * qc.size();
  g_stats.nskipped = g_stats.ntriplets - ncomp;
  g_stats.nints = ni;
  return PA_OK;
}

// The estimator study of intor/benchmark.f90:15-132 (benchmark_int3c2e):
// records (schwarz_estimate, qvl_estimate, ||(ab|c)||_2, |contracted center -
// C|) for every shell pair a >= b that is not concentric (|A - B| > 1e-6) and
// whose Schwarz value exceeds 1e-10, and every auxiliary shell c, in the
// reference's loop order. The block norms come from explicit (ab|c) blocks on
// the device (k_std_block_norm); the estimates are the screener's formulas
// on the host. With records == nullptr only the counts are returned.
int pa_int3c2e_estimates(pa_basis orbital, pa_basis aux, long long cap, double* records, long long* nrecords,
                         long long* nskipped) {
  int st = check_pair(orbital, aux);
  if (st != PA_OK) return st;
  if (orbital->host.shells.size() > 65535 && records)
    return fail(PA_ERR_ARG, "more than 65535 orbital shells");
  st = ensure_qvl(orbital);
  if (st != PA_OK) return st;
  const PairLists& P = orbital->pairs;
  const HostBasis& B = orbital->host;
  const HostBasis& X = aux->host;
  const int nx = static_cast<int>(X.shells.size());
  std::vector<double> qb(P.npairs), qc(nx);
  st = schwarz_impl(orbital, aux, qb.data(), qc.data());
  if (st != PA_OK) return st;
  std::vector<int> keep;
  for (int p = 0; p < P.npairs; ++p) {
    const int2 ab = P.pair_ab[p];
    const double* A = B.shells[ab.x].A;
    const double* Bc = B.shells[ab.y].A;
    const double d = std::sqrt((A[0] - Bc[0]) * (A[0] - Bc[0]) + (A[1] - Bc[1]) * (A[1] - Bc[1]) +
                               (A[2] - Bc[2]) * (A[2] - Bc[2]));
    if (d <= 1e-6 || qb[p] <= 1e-10) continue;  // benchmark.f90:88-93
    keep.push_back(p);
  }
  const long long n = static_cast<long long>(keep.size()) * nx;
  const double thr = static_cast<double>(1e-10f);  // benchmark.f90:100, REAL(4) literal
  long long skipped = 0;
  std::vector<double> est;
  if (records) {
    if (cap < n) return fail(PA_ERR_ARG, "records buffer holds " + std::to_string(cap) + " of " + std::to_string(n));
    est.resize(static_cast<size_t>(3) * n);
  }
  for (size_t k = 0; k < keep.size(); ++k) {
    const int p = keep[k];
    const double4 pq = orbital->pair_qvl[p];
    for (int c = 0; c < nx; ++c) {
      const HostShell& sc = X.shells[c];
      const double dx = pq.x - sc.A[0], dy = pq.y - sc.A[1], dz = pq.z - sc.A[2];
      const double R = std::sqrt(dx * dx + dy * dy + dz * dz);
      const double sch = qb[p] * qc[c];
      double qvl = sch;  // qvl_estimate (common/screening.f90:267-299)
      if (R > pq.w + aux->aux_qvl[c].x) {
        double RL = R;
        for (int l = 0; l < sc.L; ++l) RL *= R;
        qvl = qb[p] * kPi * 1.4142135623730951 * aux->aux_qvl[c].y / (orbital->pair_den[p] * RL);
      }
      if (qvl < thr) ++skipped;
      if (records) {
        const size_t r = k * nx + c;
        est[3 * r] = sch;
        est[3 * r + 1] = qvl;
        est[3 * r + 2] = R;
      }
    }
  }
  if (nrecords) *nrecords = n;
  if (nskipped) *nskipped = skipped;
  if (!records || n == 0) return PA_OK;
  // block norms on the device
  Ctx* c = nullptr;
  DeviceTables dt;
  st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  const Options o = options();
  cudaStream_t s = c->stream;
  Carver cnt;
  double *Qab = nullptr, *esph = nullptr, *norms = nullptr;
  double4* pP = nullptr;
  int* d_keep = nullptr;
  for (int pass = 0; pass < 2; ++pass) {
    Carver cv;
    if (pass == 1) {
      PA_CUDA(c->arena.reserve(cnt.used));
      cv.base = c->arena.base;
    }
    Qab = cv.take<double>(P.npairs);
    pP = cv.take<double4>(P.nunits);
    esph = cv.take<double>(P.esph_total);
    d_keep = cv.take<int>(keep.size());
    norms = cv.take<double>(n);
    if (pass == 0) cnt = cv;
  }
  UnitArrays U;
  U.unit_pair = orbital->d_unit_pair;
  U.unit_prims = orbital->d_unit_prims;
  U.unit_esph = orbital->d_unit_esph;
  U.unit_pP = pP;
  U.esph = esph;
  int launches = launch_unit_setup(orbital->dev, orbital->d_pair_ab, orbital->d_class_unit, P, U, dt, s);
  PA_CUDA(cudaMemcpyAsync(d_keep, keep.data(), sizeof(int) * keep.size(), cudaMemcpyHostToDevice, s));
  StdArgs a;
  a.B = orbital->dev;
  a.X = aux->dev;
  a.dt = dt;
  a.boys_mode = o.boys_mode;
  a.thresh = o.screen_thresh;
  a.pair_ab = orbital->d_pair_ab;
  a.pair_unit0 = orbital->d_pair_unit0;
  a.unit_pP = pP;
  a.esph = esph;
  a.unit_esph = orbital->d_unit_esph;
  a.Qab = Qab;
  launches += launch_std_block_norms(a, d_keep, static_cast<int>(keep.size()), norms, s);
  PA_CUDA(cudaGetLastError());
  std::vector<double> h_norms(n);
  PA_CUDA(cudaMemcpyAsync(h_norms.data(), norms, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  PA_CUDA(cudaStreamSynchronize(s));
  for (long long r = 0; r < n; ++r) {
    records[4 * r] = est[3 * r];
    records[4 * r + 1] = est[3 * r + 1];
    records[4 * r + 2] = h_norms[r];
    records[4 * r + 3] = est[3 * r + 2];
  }
  g_stats = pa_stats{};
  g_stats.kernel_launches = launches;
  return PA_OK;
}

// f_benchmark_int3c2e (intor/benchmark_wrapper.f90:13-37): prints the basis
// sizes, the time of the study and the number of triplets the QVL estimate
// skips, and writes the records to int_estimates.bin in the working
// directory (a stream of 4 doubles per record, benchmark.f90:117).
int f_benchmark_int3c2e(int nshells, int ndata, const int* bas_centers, const int* bas_spec, const double* bas_data,
                        int nshells_aux, int ndata_aux, const int* bas_centers_aux, const int* bas_spec_aux,
                        const double* bas_data_aux) {
  BasisGuard orb, aux;
  int st = acquire_basis(nshells, ndata, bas_centers, bas_spec, bas_data, PA_LMAX, &orb);
  if (st != PA_OK) return st;
  st = acquire_basis(nshells_aux, ndata_aux, bas_centers_aux, bas_spec_aux, bas_data_aux, PA_LAUXMAX, &aux);
  if (st != PA_OK) return st;
  std::printf("Main basis:%6d shells, %6d basis functions\n", nshells, orb.b->host.nsph);
  std::printf("Aux. basis:%6d shells, %6d basis functions\n", nshells_aux, aux.b->host.nsph);
  const auto t0 = std::chrono::steady_clock::now();
  long long n = 0, skipped = 0;
  st = pa_int3c2e_estimates(orb.b, aux.b, 0, nullptr, &n, &skipped);
  if (st != PA_OK) return st;
  std::vector<double> rec(static_cast<size_t>(4) * std::max(n, 1LL));
  st = pa_int3c2e_estimates(orb.b, aux.b, n, rec.data(), &n, &skipped);
  if (st != PA_OK) return st;
  const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  std::printf("Estimates and block norms took %8.4f s.\n", dt);
  const long long ntrip = static_cast<long long>(nshells) * (nshells + 1) / 2 * nshells_aux;
  std::printf("Skipped %12lld of %12lld integral triplets (%8.2f%%)\n", skipped, ntrip,
              ntrip ? 100.0 * static_cast<double>(skipped) / static_cast<double>(ntrip) : 0.0);
  std::fflush(stdout);
  FILE* f = std::fopen("int_estimates.bin", "wb");
  if (!f) return fail(PA_ERR_ARG, "cannot open int_estimates.bin for writing");
  const size_t w = std::fwrite(rec.data(), sizeof(double), static_cast<size_t>(4) * n, f);
  std::fclose(f);
  if (w != static_cast<size_t>(4) * n) return fail(PA_ERR_ARG, "short write to int_estimates.bin");
  return PA_OK;
}

int pa_boys_eval(int mode, int nmax, int n, const double* T, double* out) {
  if (nmax < 0 || nmax > PA_BOYS_NMAX || n < 0 || (n > 0 && (!T || !out)))
    return fail(PA_ERR_ARG, "invalid Boys evaluation request");
  if (mode != PA_BOYS_EXACT && mode != PA_BOYS_REFERENCE) return fail(PA_ERR_ARG, "unknown Boys mode");
  for (int i = 0; i < n; ++i)
    if (!(T[i] >= 0.0) || !std::isfinite(T[i])) return fail(PA_ERR_ARG, "Boys argument must be finite and >= 0");
  Ctx* c = nullptr;
  DeviceTables dt;
  int st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  const size_t nout = static_cast<size_t>(n) * (nmax + 1);
  PA_CUDA(c->arena.reserve(sizeof(double) * (n + nout) + 512));
  double* dT = reinterpret_cast<double*>(c->arena.base);
  double* dO = dT + ((n + 31) / 32) * 32;
  if (n == 0) return PA_OK;
  PA_CUDA(cudaMemcpyAsync(dT, T, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  k_boys_eval<<<static_cast<int>((nout + 255) / 256), 256, 0, c->stream>>>(dt, mode, nmax, n, dT, dO);
  PA_CUDA(cudaGetLastError());
  PA_CUDA(cudaMemcpyAsync(out, dO, sizeof(double) * nout, cudaMemcpyDeviceToHost, c->stream));
  PA_CUDA(cudaStreamSynchronize(c->stream));
  return PA_OK;
}

int pa_metric(pa_basis aux, double* metric) {
  if (!aux || !metric) return fail(PA_ERR_ARG, "null argument");
  Ctx* c = nullptr;
  DeviceTables dt;
  int st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  const size_t n = aux->host.nsph;
  PA_CUDA(c->arena.reserve(sizeof(double) * n * n + 256));
  double* M = reinterpret_cast<double*>(c->arena.base);
  PA_CUDA(cudaEventRecord(c->ev0, c->stream));
  const int launches = launch_metric(aux->dev, dt, options().boys_mode, M, c->stream);
  PA_CUDA(cudaGetLastError());
  PA_CUDA(cudaEventRecord(c->ev1, c->stream));
  PA_CUDA(cudaMemcpyAsync(metric, M, sizeof(double) * n * n, cudaMemcpyDeviceToHost, c->stream));
  PA_CUDA(cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  g_stats = pa_stats{};
  g_stats.ms_metric = g_stats.ms_total = ms;
  g_stats.kernel_launches = launches;
  return PA_OK;
}

// The metric half of the path on device buffers: (P|Q) of the auxiliary basis
// (+ the metric shift), its Cholesky factor, d_df = L^-1 d_raw and, with
// nstates > 0, the Coulomb tensor. The same stages as the end of run_df
// (stage_metric, stage_solve, coulomb_4d), for a raw contraction assembled
// from auxiliary-shell shards computed elsewhere (other ranks).
int pa_df_solve(pa_basis aux, int ndens, const double* d_raw, double* d_df, int nstates, double* d_coulomb,
                void* stream) {
  if (!aux) return fail(PA_ERR_ARG, "null basis handle");
  if (ndens < 0 || (ndens > 0 && (!d_raw || !d_df))) return fail(PA_ERR_ARG, "null raw or df pointer");
  if (nstates < 0 || (nstates > 0 && (nstates * (nstates + 1) / 2 != ndens || !d_coulomb)))
    return fail(PA_ERR_ARG, "nstates must be 0, or satisfy ndens = nstates (nstates + 1) / 2 with an output");
  int dev = 0;
  cudaGetDevice(&dev);
  if (aux->device != dev) return fail(PA_ERR_ARG, "basis handle belongs to another device");
  Ctx* c = nullptr;
  DeviceTables dt;
  int st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  const Options o = options();
  const int naux = aux->host.nsph;
  const size_t nn = static_cast<size_t>(naux) * naux;
  Carver cnt;
  for (int pass = 0; pass < 2; ++pass) {
    Carver cv;
    if (pass == 1) {
      PA_CUDA(c->arena.reserve(cnt.used));
      cv.base = c->arena.base;
    }
    DfBuffers b;
    b.M = cv.take<double>(nn);
    b.lawork = cv.take<double>(linalg_workspace_doubles(naux));
    b.info = cv.take<int>(4);
    double* gram = cv.take<double>(static_cast<size_t>(ndens) * ndens);
    double* raw_copy = cv.take<double>(static_cast<size_t>(naux) * ndens);  // the solve overwrites its input
    if (pass == 0) {
      cnt = cv;
      continue;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    PA_CUDA(cudaEventRecord(c->ev0, s));
    int launches = 0;
    stage_metric(aux, b, dt, o, s, nullptr, &launches);
    if (ndens > 0) {
      PA_CUDA(cudaMemcpyAsync(raw_copy, d_raw, sizeof(double) * naux * ndens, cudaMemcpyDeviceToDevice, s));
      b.df_raw = raw_copy;
      st = stage_solve(aux, ndens, b, o, d_df, s, &launches);
      if (st != PA_OK) return st;
      if (nstates > 0) launches += coulomb_4d(d_df, naux, ndens, nstates, gram, d_coulomb, s);
    }
    PA_CUDA(cudaEventRecord(c->ph[0], s));
    PA_CUDA(cudaEventRecord(c->ph[1], s));
    PA_CUDA(cudaEventRecord(c->m0, s));
    PA_CUDA(cudaEventRecord(c->m1, s));
    PA_CUDA(cudaEventRecord(c->ph[2], s));
    float ms = 0.f;
    g_stats = pa_stats{};
    return finish(c, b, s, launches, &ms);
  }
  return PA_OK;
}

int pa_cholesky_solve(int n, double* A, int nrhs, double* B) {
  if (n < 0 || nrhs < 0 || (n > 0 && !A) || (n > 0 && nrhs > 0 && !B))
    return fail(PA_ERR_ARG, "invalid Cholesky arguments");
  Ctx* c = nullptr;
  DeviceTables dt;
  int st = current_ctx(&c, &dt);
  if (st != PA_OK) return st;
  std::lock_guard<std::mutex> lk(c->mu);
  const size_t nn = static_cast<size_t>(n) * n, nb = static_cast<size_t>(n) * nrhs;
  PA_CUDA(c->arena.reserve(sizeof(double) * (nn + 2 * nb + linalg_workspace_doubles(n)) + 4096));
  Carver cv;
  cv.base = c->arena.base;
  double* dA = cv.take<double>(nn);
  double* dB = cv.take<double>(nb);
  int* info = cv.take<int>(1);
  if (n == 0) return PA_OK;
  PA_CUDA(cudaMemcpyAsync(dA, A, sizeof(double) * nn, cudaMemcpyHostToDevice, c->stream));
  if (nb) PA_CUDA(cudaMemcpyAsync(dB, B, sizeof(double) * nb, cudaMemcpyHostToDevice, c->stream));
  double* work = cv.take<double>(linalg_workspace_doubles(n));
  double* dC = cv.take<double>(nb);
  PA_CUDA(cudaEventRecord(c->ev0, c->stream));
  int launches = cholesky_lower(dA, n, info, work, c->stream, &c->la2);
  if (nb) launches += trsm_lower_left(dA, n, work, dB, n, nrhs, dC, n, c->stream);
  PA_CUDA(cudaGetLastError());
  PA_CUDA(cudaEventRecord(c->ev1, c->stream));
  PA_CUDA(cudaMemcpyAsync(A, dA, sizeof(double) * nn, cudaMemcpyDeviceToHost, c->stream));
  if (nb) PA_CUDA(cudaMemcpyAsync(B, dC, sizeof(double) * nb, cudaMemcpyDeviceToHost, c->stream));
  PA_CUDA(cudaMemcpyAsync(c->h_info, info, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  PA_CUDA(cudaStreamSynchronize(c->stream));
  float ms = 0.f;
  PA_CUDA(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  g_stats = pa_stats{};
  g_stats.ms_solve = g_stats.ms_total = ms;
  g_stats.kernel_launches = launches;
  if (*c->h_info != 0)
    return fail(PA_ERR_NOT_SPD, "matrix is not positive definite (Cholesky pivot " +
                                    std::to_string(*c->h_info) + ")");
  return PA_OK;
}

}  // extern "C"

extern "C" {

int pa_std_df1c(pa_basis orbital, pa_basis aux, double* d_out, void* stream) {
  return std_device(orbital, aux, kStdDf1c, 0, nullptr, d_out, static_cast<cudaStream_t>(stream));
}

int pa_std_eri2c(pa_basis orbital, pa_basis aux, double* d_out, void* stream) {
  return std_device(orbital, aux, kStdEri2c, 0, nullptr, d_out, static_cast<cudaStream_t>(stream));
}

int pa_std_df2c_mo(pa_basis orbital, pa_basis aux, int nmos, const double* d_mo, double* d_out,
                   void* stream) {
  return std_device(orbital, aux, kStdDf2cMo, nmos, d_mo, d_out, static_cast<cudaStream_t>(stream));
}

int f_intor_eri2c(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                  const double* bas_data, int nshells_aux, int ndata_aux,
                  const int* bas_centers_aux, const int* bas_spec_aux,
                  const double* bas_data_aux, int nbfs, double* eri2c_tensor) {
  BasisGuard orb, aux;
  int st = acquire_basis(nshells, ndata, bas_centers, bas_spec, bas_data, PA_LMAX, &orb);
  if (st != PA_OK) return st;
  st = acquire_basis(nshells_aux, ndata_aux, bas_centers_aux, bas_spec_aux, bas_data_aux,
                       PA_LAUXMAX, &aux);
  if (st != PA_OK) return st;
  if (nbfs != orb.b->host.nsph)
    return fail(PA_ERR_ARG, "nbfs does not match the orbital basis");
  if (nbfs > 0 && !eri2c_tensor) return fail(PA_ERR_ARG, "null output pointer");
  return std_host(orb.b, aux.b, kStdEri2c, 0, nullptr, eri2c_tensor,
                  static_cast<size_t>(nbfs) * nbfs);
}

int f_intor_df1c(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                 const double* bas_data, int nshells_aux, int ndata_aux,
                 const int* bas_centers_aux, const int* bas_spec_aux, const double* bas_data_aux,
                 int nbfs, int nbfs_aux, double* df1c_tensor) {
  BasisGuard orb, aux;
  int st = acquire_basis(nshells, ndata, bas_centers, bas_spec, bas_data, PA_LMAX, &orb);
  if (st != PA_OK) return st;
  st = acquire_basis(nshells_aux, ndata_aux, bas_centers_aux, bas_spec_aux, bas_data_aux,
                       PA_LAUXMAX, &aux);
  if (st != PA_OK) return st;
  if (nbfs != orb.b->host.nsph || nbfs_aux != aux.b->host.nsph)
    return fail(PA_ERR_ARG, "nbfs / nbfs_aux do not match the bases");
  if (static_cast<long long>(nbfs) * nbfs_aux > 0 && !df1c_tensor) return fail(PA_ERR_ARG, "null output pointer");
  return std_host(orb.b, aux.b, kStdDf1c, 0, nullptr, df1c_tensor,
                  static_cast<size_t>(nbfs) * nbfs_aux);
}

int f_intor_df2c_mo(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                    const double* bas_data, int nshells_aux, int ndata_aux,
                    const int* bas_centers_aux, const int* bas_spec_aux,
                    const double* bas_data_aux, int nbfs, int nmos, const double* mo_tensor,
                    int nbfs_aux, double* df2c_mo_tensor) {
  BasisGuard orb, aux;
  int st = acquire_basis(nshells, ndata, bas_centers, bas_spec, bas_data, PA_LMAX, &orb);
  if (st != PA_OK) return st;
  st = acquire_basis(nshells_aux, ndata_aux, bas_centers_aux, bas_spec_aux, bas_data_aux,
                       PA_LAUXMAX, &aux);
  if (st != PA_OK) return st;
  if (nbfs != orb.b->host.nsph || nbfs_aux != aux.b->host.nsph)
    return fail(PA_ERR_ARG, "nbfs / nbfs_aux do not match the bases");
  if (nmos < 0 || (nmos > 0 && (!mo_tensor || !df2c_mo_tensor)))
    return fail(PA_ERR_ARG, "invalid MO tensor or output");
  const size_t npack = static_cast<size_t>(nmos) * (nmos + 1) / 2;
  return std_host(orb.b, aux.b, kStdDf2cMo, nmos, mo_tensor, df2c_mo_tensor, npack * nbfs_aux);
}

}  // extern "C"

extern "C" int pa_df_4d_batch(int nmol, const pa_basis* orbital, const pa_basis* aux, const int* ndens,
                              const double* const* d_densities, int layout, const int* nstates,
                              double* const* d_coulomb, int use_graph, void* stream) {
  return pa::batch_4d(nmol, orbital, aux, ndens, d_densities, layout, nstates, d_coulomb, use_graph,
                      static_cast<cudaStream_t>(stream));
}

