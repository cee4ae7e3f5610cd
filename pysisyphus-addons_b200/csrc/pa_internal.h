// Host-side structures and kernel launchers of libpa_b200.so (internal).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "pa_common.cuh"

namespace pa {

// ---------------------------------------------------------------------------
// Basis on the host, unpacked like common/shells.f90:97-187 and normalized like
// common/normalization.f90:10-38.
struct HostShell {
  int L = 0, nprim = 0, prim_off = 0, sph_off = 0;
  double A[3] = {0, 0, 0};
};

struct HostBasis {
  std::vector<HostShell> shells;
  std::vector<double> exps, coefs;  // coefs renormalized
  int nsph = 0;
  int lmax = -1;
};

// Returns PA_OK or an error code (message in *err).
int unpack_basis(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                 const double* bas_data, int lmax_allowed, HostBasis* out, std::string* err);

// ---------------------------------------------------------------------------
// Device copy of a basis (structure of arrays).
struct DevBasis {
  int nshells = 0, nprims = 0, nsph = 0, lmax = -1;
  int4* shell = nullptr;      // (L, nprim, prim_off, sph_off)
  double4* center = nullptr;  // (x, y, z, 0)
  double2* prim = nullptr;    // (exponent, normalized coefficient)
};

// Orbital shell pairs a >= b and their primitive pairs ("bra units"), grouped
// by Lab = la + lb. Built on the host from the basis alone.
struct PairLists {
  int npairs = 0;
  int nunits = 0;
  int lab_max = 0;
  std::vector<int2> pair_ab;          // pair -> (a, b)
  std::vector<int> pair_unit0;        // pair -> first unit (units of a pair are contiguous)
  std::vector<int> unit_pair;         // unit -> pair
  std::vector<int2> unit_prims;       // unit -> (prim index in a, prim index in b), global
  std::vector<long long> unit_esph;   // unit -> offset of its E_sph block (doubles)
  long long esph_total = 0;
  // units sorted by class: class_units[c] = list of units with Lab = c (host order)
  std::vector<int> class_off;         // [lab_max + 2] offsets into class_unit
  std::vector<int> class_unit;        // units grouped by class
  // shell pairs grouped by class Lab (host order within a class)
  std::vector<int> pair_class_off;    // [lab_max + 2] offsets into class_pair
  std::vector<int> class_pair;
};

struct AuxLists {
  int lc_max = 0;
  std::vector<int> class_off;   // [lc_max + 2]
  std::vector<int> class_shell; // aux shells grouped by L
};

void build_pair_lists(const HostBasis& b, PairLists* out);
void build_aux_lists(const HostBasis& b, AuxLists* out);

// QVL screener data of t_df_screener%init (common/screening.f90:101-163):
// per shell pair (order of PairLists::pair_ab) the contracted center and
// extent (x, y, z, extent) and (zeta_a,min + zeta_b,min)^(1/4); the smallest of
// the latter in *den_min.
void build_qvl_pairs(const HostBasis& b, const PairLists& P, std::vector<double4>* cen_ext,
                     std::vector<double>* den, double* den_min);
// Per auxiliary shell: (extent, beta) of auxiliary_extent(exps, 1d-8) and
// beta = zeta_min^(-(2L+3)/4) sqrt((2L-1)!!).
void build_qvl_aux(const HostBasis& b, std::vector<double2>* ext_beta);

// ---------------------------------------------------------------------------
// Options and statistics.
struct Options {
  int boys_mode = 1;          // 1 = reference-compatible (default), 0 = exact
  double screen_thresh = static_cast<double>(1e-10f);
  int verbose = 0;
  int skip_metric = 0;
  double metric_shift = 0.0;  // added to the diagonal of (P|Q) before the Cholesky
  int precision = 0;          // 0 = FP64 throughout, 1 = mixed (FP32 recurrences for weak triplets)
  double fp32_thresh = 1e-6;  // Schwarz bound below which the mixed form uses FP32
  // mixed form: 0 = FP32 recurrences inside the FP64 class kernels (default),
  // 1 = the weak triplets on their own kernels (FP32 X, split-BF16
  // tensor-core product)
  int mixed_kernels = 0;
  int items_per_sm = 0;       // work items per SM and class of the three-center kernel (0 = by size)
  int screening = 0;          // triplet estimate: 0 = Schwarz (reference), 1 = QVL
  int class_timing = 0;       // 1: class launches serialized on one stream, each timed with events
  // tile-shape variant of each three-center class [L_ab][L_c] (0 = default)
  signed char tile_variant[2 * PA_LMAX + 1][PA_LAUXMAX + 1] = {};
};

struct Stats {
  long long ntriplets = 0, nskipped = 0, nints = 0;
  long long n3c_flops_model = 0;
  double ms_screen = 0, ms_metric = 0, ms_chol = 0, ms_bra = 0, ms_3c = 0, ms_trsm = 0,
         ms_total = 0;
  int kernel_launches = 0;
};

// ---------------------------------------------------------------------------
// Device tables (built once per device).
int get_device_tables(DeviceTables* out, std::string* err);

// ---------------------------------------------------------------------------
// Stream-ordered scratch arena (grow-only, one per device).
struct Arena {
  char* base = nullptr;
  size_t cap = 0, used = 0;
  cudaError_t reserve(size_t bytes);
  void reset() { used = 0; }
  template <class T>
  T* take(size_t count) {
    const size_t bytes = ((count * sizeof(T)) + 255) & ~size_t(255);
    T* p = reinterpret_cast<T*>(base + used);
    used += bytes;
    return p;
  }
};

// ---------------------------------------------------------------------------
// Kernel launchers (return the number of kernel launches issued).
struct UnitArrays {
  // per unit (host order)
  const int* unit_pair;
  const int2* unit_prims;
  const long long* unit_esph;
  double4* unit_pP;   // (p, Px, Py, Pz)
  double* esph;       // E_sph blocks
};

// Unit data of all bra units: classes L_ab <= 2 one warp per unit, the others
// one block per unit (class_unit: device copy of P.class_unit).
int launch_unit_setup(const DevBasis& B, const int2* pair_ab, const int* class_unit, const PairLists& P,
                      UnitArrays U, const DeviceTables& dt, cudaStream_t s);
// Schwarz values of all pairs: pairs with Lab <= 4 one warp each, the others
// one block each (class_pair: device copy of P.class_pair).
int launch_schwarz_bra(const DevBasis& B, const int2* pair_ab, const int* pair_unit0,
                       const int* class_pair, const PairLists& P, UnitArrays U, const DeviceTables& dt,
                       int boys_mode, double* Qab, cudaStream_t s);
int launch_schwarz_aux(const DevBasis& X, const DeviceTables& dt, int boys_mode, double* Qc,
                       cudaStream_t s);
int launch_metric(const DevBasis& X, const DeviceTables& dt, int boys_mode, double* M,
                  cudaStream_t s);

}  // namespace pa
