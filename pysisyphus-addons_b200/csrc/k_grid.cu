// Densities on grid points and the GDMA primitive density.
//
// f_eval_densities (grid/grid_wrapper.f90:12-38, driver grid/grid.f90:110-286):
//   rho_j(r) = sum_(nu <= mu) f D_j(mu, nu) chi_mu(r) chi_nu(r), f = 1 on the
//   diagonal and 2 off it, over Cartesian basis functions chi in pysisyphus
//   order, with the reference's per-block screening: the points are cut into
//   consecutive blocks of blk_size, and a pair (nu, mu) contributes to a block
//   only when |f D_j(mu, nu) mean_nu mean_mu| >= thresh, mean = the mean |chi|
//   over the block's points.
// f_eval_prim_density (gdma/prim_dens.f90:100-259): the density of the
//   primitive pairs whose total exponent is below `switch`, on grid points.
//
// Device layout of f_eval_densities. One CTA (128 threads) takes one block of
// points at a time (persistent over the blocks):
//   1. chi of every Cartesian function at the block's points into the CTA's
//      slice of a global scratch array ([function][point], row stride bp);
//   2. the block means, each a sequential sum over the points in order (the
//      reference's order, so the screening decisions are the reference's);
//   3. the functions that can pass the test (mean_x dmax_x max_mean >= thresh,
//      dmax_x = the largest |f D| of x's pairs) compacted into an ordered list;
//   4. per density, 32 x 32 tiles of the pair matrix W[mu][nu] = f D(mu, nu)
//      (masked by the test, mu >= nu) staged in shared memory -- tiles with no
//      surviving pair are skipped -- and every thread (one grid point)
//      accumulates T[nu] = sum_mu W[mu][nu] chi_mu in registers, then
//      rho += sum_nu chi_nu T[nu].
// Bound: FP64 FMA over the surviving pairs (the pair matrix is read from L2).
//
// f_eval_prim_density: the surviving primitive pairs (the reference's two
// tests, on the host, in its ai <= bi order) go to the device; one thread per
// grid point sums over all pairs, staged 64 at a time in shared memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "pa_internal.h"  // before pa_b200.h: its status macros would rename the enum
#include "pa_b200.h"

namespace pa {
int set_error(int code, const std::string& msg);

namespace {

constexpr double kExpCutoff = -36.0;  // grid.f90:9, prim_dens.f90:13
constexpr int kGridThreads = 128;
constexpr int kTile = 32;
constexpr int kGridLmax = 4;  // cart_gto3d_rel / prefacts cover s..g

// 1 / sqrt((2i-1)!! (2j-1)!! (2k-1)!!) of every Cartesian component of
// degree <= 4 (cidx order): the NORM2 / NORM3 / NORM4 / NORM22 factors of
// grid.f90:9-13 and prim_dens.f90:7-10.
__constant__ double c_cart_norm[ncum(kGridLmax)];
__constant__ unsigned char c_cart_pow[ncum(kGridLmax)][3];

struct GridArgs {
  int nshells, ncart, npoints, ndens, nbfs, blk, bp, nblks;
  const int4* shell;      // (L, nprim, prim_off, cart_off)
  const double4* center;  // (x, y, z, 0)
  const double2* prim;    // (exponent, normalized coefficient)
  const double* grid;     // [npoints][3]
  const double* D;        // D[j + ndens (mu + nbfs nu)] (reference layout)
  const double* dmax;     // [ncart]
  double thresh;
  double* chi;            // [slot][ncart][bp]
  double* mean;           // [slot][ncart]
  int* act;               // [slot][ncart]
  double* rho;            // rho[j + ndens i]
};

__device__ __forceinline__ double ipow(double x, int n) {
  double r = 1.0;
  for (int m = 0; m < n; ++m) r *= x;
  return r;
}

__global__ void __launch_bounds__(kGridThreads) k_grid_density(GridArgs a) {
  __shared__ double W[kTile][kTile + 1];
  __shared__ int s_cnt[kGridThreads / 32];
  __shared__ double s_red[kGridThreads / 32];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double* chi = a.chi + static_cast<long long>(blockIdx.x) * a.ncart * a.bp;
  double* mean = a.mean + static_cast<long long>(blockIdx.x) * a.ncart;
  int* act = a.act + static_cast<long long>(blockIdx.x) * a.ncart;
  for (int blk = blockIdx.x; blk < a.nblks; blk += gridDim.x) {
    const int start = blk * a.blk;
    const int n = min(a.blk, a.npoints - start);
    // 1. chi of every shell at every point of the block
    for (long long item = tid; item < static_cast<long long>(a.nshells) * n; item += kGridThreads) {
      const int sh = static_cast<int>(item / n), i = static_cast<int>(item - static_cast<long long>(sh) * n);
      const int4 s = a.shell[sh];
      const double4 C = a.center[sh];
      const double* R = a.grid + 3LL * (start + i);
      const double x = R[0] - C.x, y = R[1] - C.y, z = R[2] - C.z;
      const double dist = x * x + y * y + z * z;
      double e = 0.0;
      for (int p = 0; p < s.y; ++p) {
        const double2 pr = a.prim[s.z + p];
        const double arg = -pr.x * dist;
        if (arg < kExpCutoff) continue;
        e += pr.y * exp(arg);
      }
      const int c0 = ncum(s.x - 1), nc = ncart(s.x);
      for (int c = 0; c < nc; ++c) {
        const unsigned char* pw = c_cart_pow[c0 + c];
        chi[static_cast<long long>(s.w + c) * a.bp + i] =
            c_cart_norm[c0 + c] * ipow(x, pw[0]) * ipow(y, pw[1]) * ipow(z, pw[2]) * e;
      }
    }
    __syncthreads();
    // 2. block means, summed over the points in order
    double mmax = 0.0;
    for (int nu = tid; nu < a.ncart; nu += kGridThreads) {
      const double* row = chi + static_cast<long long>(nu) * a.bp;
      double m = 0.0;
      for (int i = 0; i < n; ++i) m += fabs(row[i]);
      m /= n;
      mean[nu] = m;
      mmax = fmax(mmax, m);
    }
    for (int o = 16; o > 0; o >>= 1) mmax = fmax(mmax, __shfl_xor_sync(0xffffffffu, mmax, o));
    if (lane == 0) s_red[warp] = mmax;
    __syncthreads();
    mmax = s_red[0];
    for (int w = 1; w < kGridThreads / 32; ++w) mmax = fmax(mmax, s_red[w]);
    // 3. ordered list of the functions that can pass the test (a superset:
    //    the bound is relaxed by 1e-12 for rounding)
    int na = 0;
    for (int base = 0; base < a.ncart; base += kGridThreads) {
      const int nu = base + tid;
      const bool keep = nu < a.ncart && mean[nu] * a.dmax[nu] * mmax >= a.thresh * (1.0 - 1e-12);
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (lane == 0) s_cnt[warp] = __popc(bal);
      __syncthreads();
      int off = na;
      for (int w = 0; w < warp; ++w) off += s_cnt[w];
      if (keep) act[off + __popc(bal & ((1u << lane) - 1u))] = nu;
      int tot = 0;
      for (int w = 0; w < kGridThreads / 32; ++w) tot += s_cnt[w];
      na += tot;
      __syncthreads();
    }
    // 4. masked pair products, per density and per group of points
    for (int j = 0; j < a.ndens; ++j) {
      for (int p0 = 0; p0 < n; p0 += kGridThreads) {
        const int i = p0 + tid;
        const bool pt = i < n;
        double rho = 0.0;
        for (int t0 = 0; t0 < na; t0 += kTile) {
          double T[kTile];
#pragma unroll
          for (int k = 0; k < kTile; ++k) T[k] = 0.0;
          for (int s0 = t0; s0 < na; s0 += kTile) {
            bool any = false;
            for (int e = tid; e < kTile * kTile; e += kGridThreads) {
              const int m = e / kTile, k = e % kTile;
              double w = 0.0;
              if (t0 + k < na && s0 + m < na) {
                const int nu = act[t0 + k], mu = act[s0 + m];
                if (mu >= nu) {
                  const double f = nu == mu ? 1.0 : 2.0;
                  const double d = a.D[j + static_cast<long long>(a.ndens) * (mu + static_cast<long long>(a.nbfs) * nu)];
                  const double contrib = f * d * mean[nu] * mean[mu];
                  if (fabs(contrib) >= a.thresh) w = f * d;
                }
              }
              W[m][k] = w;
              any = any || w != 0.0;
            }
            if (!__syncthreads_or(any)) continue;
            if (pt) {
              for (int m = 0; m < kTile && s0 + m < na; ++m) {
                const double x = chi[static_cast<long long>(act[s0 + m]) * a.bp + i];
#pragma unroll
                for (int k = 0; k < kTile; ++k) T[k] = fma(W[m][k], x, T[k]);
              }
            }
            __syncthreads();
          }
          if (pt) {
#pragma unroll
            for (int k = 0; k < kTile; ++k)
              if (t0 + k < na) rho = fma(chi[static_cast<long long>(act[t0 + k]) * a.bp + i], T[k], rho);
          }
        }
        if (pt) a.rho[j + static_cast<long long>(a.ndens) * (start + i)] = rho;
      }
    }
    __syncthreads();  // the slice is rewritten by the next block
  }
}

// GDMA primitive pairs (host-filtered, in the reference's ai <= bi order).
struct PrimPairG {
  double K, px, P[3], A[3], B[3];
  int La, Lb, ia, ib;
};

__device__ __forceinline__ void cart_prefactors(int L, double x, double y, double z, double* out) {
  const int c0 = ncum(L - 1), nc = ncart(L);
  for (int c = 0; c < nc; ++c) {
    const unsigned char* pw = c_cart_pow[c0 + c];
    out[c] = c_cart_norm[c0 + c] * ipow(x, pw[0]) * ipow(y, pw[1]) * ipow(z, pw[2]);
  }
}

constexpr int kPairChunk = 64;

__global__ void __launch_bounds__(128) k_prim_density(const PrimPairG* __restrict__ pairs, int npairs,
                                                      const double* __restrict__ coords, int npoints,
                                                      const double* __restrict__ P, int nbfs,
                                                      double* __restrict__ rho) {
  __shared__ PrimPairG sp[kPairChunk];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool pt = i < npoints;
  double R[3] = {0.0, 0.0, 0.0};
  if (pt)
    for (int d = 0; d < 3; ++d) R[d] = coords[3LL * i + d];
  double acc = 0.0;
  double pa[ncart(kGridLmax)], pb[ncart(kGridLmax)];
  for (int c0 = 0; c0 < npairs; c0 += kPairChunk) {
    const int nc = min(kPairChunk, npairs - c0);
    __syncthreads();
    for (int k = threadIdx.x; k < nc; k += blockDim.x) sp[k] = pairs[c0 + k];
    __syncthreads();
    if (!pt) continue;
    for (int k = 0; k < nc; ++k) {
      const PrimPairG& q = sp[k];
      const double dx = R[0] - q.P[0], dy = R[1] - q.P[1], dz = R[2] - q.P[2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (-q.px * r2 <= kExpCutoff) continue;
      const double pexp = exp(-q.px * r2);
      cart_prefactors(q.La, R[0] - q.A[0], R[1] - q.A[1], R[2] - q.A[2], pa);
      cart_prefactors(q.Lb, R[0] - q.B[0], R[1] - q.B[1], R[2] - q.B[2], pb);
      const int na = ncart(q.La), nb = ncart(q.Lb);
      double s = 0.0;
      for (int nu = 0; nu < na; ++nu) {
        double t = 0.0;
        for (int mu = 0; mu < nb; ++mu)
          t = fma(__ldg(P + (q.ia + nu) + static_cast<long long>(nbfs) * (q.ib + mu)), pb[mu], t);
        s = fma(pa[nu], t, s);
      }
      acc = fma(q.K * pexp, s, acc);
    }
  }
  if (pt) rho[i] = acc;
}

std::once_flag g_tables_once[64];
cudaError_t g_tables_err[64];

cudaError_t upload_cart_tables() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::call_once(g_tables_once[dev], [dev]() {
    double norm[ncum(kGridLmax)];
    unsigned char pw[ncum(kGridLmax)][3];
    auto df = [](int k) {  // (2k - 1)!!
      double r = 1.0;
      for (int m = 2 * k - 1; m > 1; m -= 2) r *= m;
      return r;
    };
    int idx = 0;
    for (int L = 0; L <= kGridLmax; ++L)
      for (int x = L; x >= 0; --x)
        for (int y = L - x; y >= 0; --y, ++idx) {
          const int z = L - x - y;
          norm[idx] = 1.0 / std::sqrt(df(x) * df(y) * df(z));
          pw[idx][0] = static_cast<unsigned char>(x);
          pw[idx][1] = static_cast<unsigned char>(y);
          pw[idx][2] = static_cast<unsigned char>(z);
        }
    g_tables_err[dev] = cudaMemcpyToSymbol(c_cart_norm, norm, sizeof(norm));
    if (g_tables_err[dev] == cudaSuccess) g_tables_err[dev] = cudaMemcpyToSymbol(c_cart_pow, pw, sizeof(pw));
  });
  return g_tables_err[dev];
}

// Device buffers of one call, released when the call returns.
struct DevBuf {
  std::vector<void*> ptrs;
  cudaStream_t s = nullptr;
  ~DevBuf() {
    for (void* p : ptrs) cudaFreeAsync(p, s);
    if (s) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
  }
  template <class T>
  cudaError_t get(T** p, size_t n) {
    *p = nullptr;
    const cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(p), std::max<size_t>(n, 1) * sizeof(T), s);
    if (e == cudaSuccess) ptrs.push_back(*p);
    return e;
  }
};

#define PA_GRID_CUDA(x)                                                                                  \
  do {                                                                                                   \
    const cudaError_t e_ = (x);                                                                          \
    if (e_ != cudaSuccess) return set_error(PA_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
  } while (0)

}  // namespace
}  // namespace pa

using namespace pa;

extern "C" {

int f_eval_densities(int nshells, int ndata, const int* bas_centers, const int* bas_spec, const double* bas_data,
                     int npoints, const double* grid3d, int ndens, int nbfs, const double* densities,
                     double* grid_densities, int blk_size, double thresh) {
  HostBasis b;
  std::string err;
  int st = unpack_basis(nshells, ndata, bas_centers, bas_spec, bas_data, kGridLmax, &b, &err);
  if (st != PA_OK) return set_error(st, "f_eval_densities: " + err);
  int ncart_tot = 0;
  for (const HostShell& s : b.shells) ncart_tot += ncart(s.L);
  if (npoints < 0 || ndens < 0 || nbfs != ncart_tot)
    return set_error(PA_ERR_ARG, "f_eval_densities: nbfs (" + std::to_string(nbfs) +
                                     ") must equal the Cartesian size of the basis (" + std::to_string(ncart_tot) + ")");
  if (blk_size < 1 || blk_size > 4096) return set_error(PA_ERR_ARG, "f_eval_densities: blk_size must be in [1, 4096]");
  if (!(thresh >= 0.0) || !std::isfinite(thresh)) return set_error(PA_ERR_ARG, "f_eval_densities: thresh must be >= 0");
  if ((npoints > 0 && (!grid3d || !grid_densities)) || (ndens > 0 && nbfs > 0 && !densities))
    return set_error(PA_ERR_ARG, "f_eval_densities: null array");
  if (npoints == 0 || ndens == 0) return PA_OK;
  if (nbfs == 0) {
    std::fill(grid_densities, grid_densities + static_cast<size_t>(ndens) * npoints, 0.0);
    return PA_OK;
  }
  PA_GRID_CUDA(upload_cart_tables());
  // per function: the largest |f D_j(mu, nu)| over its pairs and the densities
  std::vector<double> dmax(nbfs, 0.0);
  for (int nu = 0; nu < nbfs; ++nu)
    for (int mu = nu; mu < nbfs; ++mu) {
      const double f = nu == mu ? 1.0 : 2.0;
      double m = 0.0;
      for (int j = 0; j < ndens; ++j)
        m = std::max(m, std::fabs(f * densities[j + static_cast<size_t>(ndens) * (mu + static_cast<size_t>(nbfs) * nu)]));
      dmax[nu] = std::max(dmax[nu], m);
      dmax[mu] = std::max(dmax[mu], m);
    }
  std::vector<int4> shell(b.shells.size());
  std::vector<double4> center(b.shells.size());
  std::vector<double2> prim(b.exps.size());
  int off = 0;
  for (size_t k = 0; k < b.shells.size(); ++k) {
    const HostShell& s = b.shells[k];
    shell[k] = make_int4(s.L, s.nprim, s.prim_off, off);
    center[k] = make_double4(s.A[0], s.A[1], s.A[2], 0.0);
    off += ncart(s.L);
  }
  for (size_t p = 0; p < b.exps.size(); ++p) prim[p] = make_double2(b.exps[p], b.coefs[p]);
  DevBuf buf;
  PA_GRID_CUDA(cudaStreamCreateWithFlags(&buf.s, cudaStreamNonBlocking));
  GridArgs a;
  a.nshells = static_cast<int>(b.shells.size());
  a.ncart = nbfs;
  a.npoints = npoints;
  a.ndens = ndens;
  a.nbfs = nbfs;
  a.blk = blk_size;
  a.bp = (blk_size + 1) / 2 * 2;
  a.nblks = (npoints + blk_size - 1) / blk_size;
  a.thresh = thresh;
  int dev = 0, sms = 148;
  PA_GRID_CUDA(cudaGetDevice(&dev));
  PA_GRID_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // slots of the chi scratch: at most 4 per SM, at most ~1 GiB in total
  const size_t slot_bytes = sizeof(double) * (static_cast<size_t>(nbfs) * a.bp + nbfs) + sizeof(int) * nbfs;
  int slots = std::min(a.nblks, 4 * sms);
  slots = std::max(1, std::min<int>(slots, static_cast<int>((size_t(1) << 30) / slot_bytes)));
  int4* d_shell;
  double4* d_center;
  double2* d_prim;
  double *d_grid, *d_D, *d_dmax, *d_chi, *d_mean, *d_rho;
  int* d_act;
  const size_t nD = static_cast<size_t>(ndens) * nbfs * nbfs;
  PA_GRID_CUDA(buf.get(&d_shell, shell.size()));
  PA_GRID_CUDA(buf.get(&d_center, center.size()));
  PA_GRID_CUDA(buf.get(&d_prim, prim.size()));
  PA_GRID_CUDA(buf.get(&d_grid, 3 * static_cast<size_t>(npoints)));
  PA_GRID_CUDA(buf.get(&d_D, nD));
  PA_GRID_CUDA(buf.get(&d_dmax, nbfs));
  PA_GRID_CUDA(buf.get(&d_chi, static_cast<size_t>(slots) * nbfs * a.bp));
  PA_GRID_CUDA(buf.get(&d_mean, static_cast<size_t>(slots) * nbfs));
  PA_GRID_CUDA(buf.get(&d_act, static_cast<size_t>(slots) * nbfs));
  PA_GRID_CUDA(buf.get(&d_rho, static_cast<size_t>(ndens) * npoints));
  PA_GRID_CUDA(cudaMemcpyAsync(d_shell, shell.data(), sizeof(int4) * shell.size(), cudaMemcpyHostToDevice, buf.s));
  PA_GRID_CUDA(cudaMemcpyAsync(d_center, center.data(), sizeof(double4) * center.size(), cudaMemcpyHostToDevice, buf.s));
  if (!prim.empty())
    PA_GRID_CUDA(cudaMemcpyAsync(d_prim, prim.data(), sizeof(double2) * prim.size(), cudaMemcpyHostToDevice, buf.s));
  PA_GRID_CUDA(cudaMemcpyAsync(d_grid, grid3d, sizeof(double) * 3 * npoints, cudaMemcpyHostToDevice, buf.s));
  PA_GRID_CUDA(cudaMemcpyAsync(d_D, densities, sizeof(double) * nD, cudaMemcpyHostToDevice, buf.s));
  PA_GRID_CUDA(cudaMemcpyAsync(d_dmax, dmax.data(), sizeof(double) * nbfs, cudaMemcpyHostToDevice, buf.s));
  a.shell = d_shell;
  a.center = d_center;
  a.prim = d_prim;
  a.grid = d_grid;
  a.D = d_D;
  a.dmax = d_dmax;
  a.chi = d_chi;
  a.mean = d_mean;
  a.act = d_act;
  a.rho = d_rho;
  k_grid_density<<<slots, kGridThreads, 0, buf.s>>>(a);
  PA_GRID_CUDA(cudaGetLastError());
  PA_GRID_CUDA(cudaMemcpyAsync(grid_densities, d_rho, sizeof(double) * ndens * static_cast<size_t>(npoints),
                               cudaMemcpyDeviceToHost, buf.s));
  PA_GRID_CUDA(cudaStreamSynchronize(buf.s));
  return PA_OK;
}

int f_eval_prim_density(int nprims, int npoints, int nbfs, const int* ls_inds, const double* primdata,
                        const double* coords3d, const double* P, double sw, double* rho) {
  if (nprims < 0 || npoints < 0 || nbfs < 0) return set_error(PA_ERR_ARG, "f_eval_prim_density: negative size");
  if ((nprims > 0 && (!ls_inds || !primdata)) || (npoints > 0 && (!coords3d || !rho)) || (nbfs > 0 && !P))
    return set_error(PA_ERR_ARG, "f_eval_prim_density: null array");
  for (int ai = 0; ai < nprims; ++ai) {
    const int La = ls_inds[2 * ai], ia = ls_inds[2 * ai + 1];
    if (La < 0 || La > kGridLmax)
      return set_error(PA_ERR_LMAX, "f_eval_prim_density: primitive " + std::to_string(ai) + " has L = " +
                                        std::to_string(La) + " (s..g supported)");
    if (ia < 0 || ia + ncart(La) > nbfs)
      return set_error(PA_ERR_ARG, "f_eval_prim_density: primitive " + std::to_string(ai) +
                                       ": Cartesian index outside the density matrix");
  }
  if (npoints == 0) return PA_OK;
  std::vector<PrimPairG> pairs;
  for (int ai = 0; ai < nprims; ++ai) {
    const double da = primdata[5 * ai], ax = primdata[5 * ai + 1];
    const double* A = primdata + 5 * ai + 2;
    for (int bi = ai; bi < nprims; ++bi) {
      const double db = primdata[5 * bi], bx = primdata[5 * bi + 1];
      if (ax + bx >= sw) continue;
      const double* B = primdata + 5 * bi + 2;
      const double px = ax + bx, mux = ax * bx / px;
      // prim_dens.f90:212 squares the sum of the differences (kept as is)
      const double dsum = (A[0] - B[0]) + (A[1] - B[1]) + (A[2] - B[2]);
      if (-mux * dsum * dsum <= kExpCutoff) continue;
      const double AB2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
      PrimPairG q;
      q.K = da * db * (ai == bi ? 1.0 : 2.0) * std::exp(-mux * AB2);
      q.px = px;
      for (int d = 0; d < 3; ++d) {
        q.P[d] = (ax * A[d] + bx * B[d]) / px;
        q.A[d] = A[d];
        q.B[d] = B[d];
      }
      q.La = ls_inds[2 * ai];
      q.ia = ls_inds[2 * ai + 1];
      q.Lb = ls_inds[2 * bi];
      q.ib = ls_inds[2 * bi + 1];
      pairs.push_back(q);
    }
  }
  PA_GRID_CUDA(upload_cart_tables());
  DevBuf buf;
  PA_GRID_CUDA(cudaStreamCreateWithFlags(&buf.s, cudaStreamNonBlocking));
  PrimPairG* d_pairs;
  double *d_coords, *d_P, *d_rho;
  PA_GRID_CUDA(buf.get(&d_pairs, pairs.size()));
  PA_GRID_CUDA(buf.get(&d_coords, 3 * static_cast<size_t>(npoints)));
  PA_GRID_CUDA(buf.get(&d_P, static_cast<size_t>(nbfs) * nbfs));
  PA_GRID_CUDA(buf.get(&d_rho, npoints));
  if (!pairs.empty())
    PA_GRID_CUDA(cudaMemcpyAsync(d_pairs, pairs.data(), sizeof(PrimPairG) * pairs.size(), cudaMemcpyHostToDevice, buf.s));
  PA_GRID_CUDA(cudaMemcpyAsync(d_coords, coords3d, sizeof(double) * 3 * npoints, cudaMemcpyHostToDevice, buf.s));
  if (nbfs > 0)
    PA_GRID_CUDA(cudaMemcpyAsync(d_P, P, sizeof(double) * nbfs * static_cast<size_t>(nbfs), cudaMemcpyHostToDevice, buf.s));
  k_prim_density<<<(npoints + 127) / 128, 128, 0, buf.s>>>(d_pairs, static_cast<int>(pairs.size()), d_coords,
                                                           npoints, d_P, nbfs, d_rho);
  PA_GRID_CUDA(cudaGetLastError());
  PA_GRID_CUDA(cudaMemcpyAsync(rho, d_rho, sizeof(double) * npoints, cudaMemcpyDeviceToHost, buf.s));
  PA_GRID_CUDA(cudaStreamSynchronize(buf.s));
  return PA_OK;
}

}  // extern "C"
