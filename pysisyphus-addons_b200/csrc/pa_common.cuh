// Shared definitions of the B200 density-fitting library (libpa_b200.so).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

// Compiled angular-momentum limits. The reference builds its integral
// kernels for lmax = 4 (orbital) and lauxmax = 5 (auxiliary) by default
// (meson.options:1-4); shells above these limits are rejected with
// PA_ERR_LMAX instead of the reference's build-time absence of a kernel.
#define PA_LMAX 4
#define PA_LAUXMAX 5
// Highest Boys order: (gg|gg) Schwarz integrals need 4 * PA_LMAX.
#define PA_BOYS_NMAX 16
// Largest total Hermite degree handled by a single R build: 4 * PA_LMAX.
#define PA_LTOT_MAX 16

namespace pa {

constexpr double kPi = 3.141592653589793238462643383279502884;
// 2 pi^(5/2)
constexpr double kTwoPi52 = 34.98683665524972497;

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }
// number of Cartesian (or Hermite) components of total degree <= l
__host__ __device__ constexpr int ncum(int l) { return (l + 1) * (l + 2) * (l + 3) / 6; }
__host__ __device__ constexpr int nsph(int l) { return 2 * l + 1; }
// Index of component (i, j, k) among all components of degree <= i+j+k.
// Within a degree: x^l, x^(l-1) y, x^(l-1) z, x^(l-2) y^2, ... (i descending,
// then j descending).
__host__ __device__ constexpr int cidx(int i, int j, int k) {
  return (i + j + k) * (i + j + k + 1) * (i + j + k + 2) / 6 +
         (j + k) * (j + k + 1) / 2 + k;
}

constexpr int kNCumMax = ncum(PA_LTOT_MAX);  // 969

// Decoded Cartesian / Hermite index tables (global memory, read through L1).
struct IndexTables {
  uint8_t xyz[kNCumMax][4];    // (i, j, k, degree)
  int16_t minus[kNCumMax][3];  // index of e - 1_d, or -1
};

// Device-resident constant data built once per device.
struct DeviceTables {
  const IndexTables* idx;
  // Boys tables
  const double* boys_taylor;  // [npts][nord] F_n(i*h), exact mode
  const double* boys_ref;     // [nord_ref][2711] F_n(i*0.01), reference mode
  // Real solid harmonics, sparse rows: for each l, m: entries (cart index, coef)
  const int* sph_start;       // [(PA_LAUXMAX+1)^2 + 1] row starts into sph_col/sph_val
  const int16_t* sph_col;     // local Cartesian index within degree l
  const double* sph_val;
  // sum_idx[i * kNSum + j] = index of the multi-index sum (i) + (j) for
  // components i, j of degree <= 2 * PA_LMAX
  const int16_t* sum_idx;
  // Hermite recursion descriptor of every component idx > 0 (kNCumMax
  // entries): s1 | s2 << 10 | d << 20 | c << 22, where d is the first
  // direction with a nonzero exponent e_d, s1 = idx - 1_d, s2 = idx - 2_d and
  // c = e_d - 1, so R(idx) = X_d R'(s1) + c R'(s2).
  const int* rdesc;
};

__device__ __forceinline__ int rdesc_s1(int dsc) { return dsc & 1023; }
__device__ __forceinline__ int rdesc_s2(int dsc) { return (dsc >> 10) & 1023; }
__device__ __forceinline__ int rdesc_d(int dsc) { return (dsc >> 20) & 3; }
__device__ __forceinline__ int rdesc_c(int dsc) { return dsc >> 22; }

constexpr int kNSum = ncum(2 * PA_LMAX);  // 165

enum : int {
  PA_OK = 0,
  PA_ERR_ARG = 1,
  PA_ERR_LMAX = 2,
  PA_ERR_NOT_SPD = 3,
  PA_ERR_CUDA = 4,
  PA_ERR_TIMEOUT = 5,
  PA_ERR_NO_DEVICE = 6,
  PA_ERR_SCRATCH = 7,
};

}  // namespace pa
