// Launch interface of the three-center contraction (k_df3c.cu, the class
// kernels in k_df3c_impl.cuh instantiated by k_df3c_l<LAB>.cu).
#pragma once

#include "pa_internal.h"

namespace pa {

// Arguments of one class (LAB, LC) launch. Pointers already point at the
// class's first slot where noted.
struct Df3cArgs {
  DevBasis X;                        // auxiliary basis
  DeviceTables dt;
  int boys_mode = 1;
  double thresh = 0.0;
  // triplets with Q_ab * Q_c below thr32 build X with FP32 recurrences
  // (precision form); 0 keeps every triplet in FP64
  double thr32 = 0.0;
  // bra units of class LAB, sorted by Schwarz value (descending)
  int unit_slot0 = 0, n_units = 0;   // global slot offset, count
  const double* unit_Q = nullptr;    // [slot]
  const double4* slot_pP = nullptr;  // [slot] (p, P)
  const double* G = nullptr;         // class base: [z][s][tuv][dw]
  int dw = 8;                        // density chunk width (multiple of 8, <= 40)
  // auxiliary shells of class LC, sorted by Schwarz value (descending)
  int aux_slot0 = 0, n_aux = 0;
  const int* sorted_aux = nullptr;   // [slot] -> shell
  const double* aux_Q = nullptr;     // [slot]
  int nd = 0;
  double* partial = nullptr;         // [chunk][n_aux * NC][nd]
  // QVL screening (qvl = 1): aux_Q then holds the sort keys (bounds of the
  // estimate / Q_ab); per unit slot (contracted center, extent) and
  // (zeta_a + zeta_b)^(1/4); per auxiliary slot (Q_c, extent, beta, 0)
  int qvl = 0;
  const double4* slot_qvl = nullptr;
  const double* slot_den = nullptr;
  const double4* aux_qvl = nullptr;
  // persistent scheduling (filled in by launch_df3c_class): work items are
  // (aux tile, bra chunk, density chunk), pulled from *counter (zeroed before
  // the launch)
  int* counter = nullptr;
  int n_items = 0, nbx = 0, nby = 0, nbz = 0;
  // weak-triplet kernels (precision form): a device flag set to 1 when a
  // tensor-core completion wait gave up
  int* err = nullptr;
};

// Class runs of one auxiliary L: an FP64 run per L_ab, and in the mixed form a
// weak-triplet run beside each.
constexpr int kMaxRunsPerLc = 2 * (2 * PA_LMAX + 1);

struct Df3cReduceArgs {
  DevBasis X;
  int aux_slot0 = 0, n_aux = 0, nc = 1, nd = 0, naux = 0;
  const int* sorted_aux = nullptr;
  int nclasses = 0;
  const double* part[kMaxRunsPerLc] = {};
  int ny[kMaxRunsPerLc] = {};
  double* df = nullptr;              // [naux][nd] column-major (naux rows)
};

struct Df3cClassInfo {
  int tc = 0, ub = 0, ndc = 0;
  int lanes = 0;          // lanes per triplet in the X build (TPT or team size)
  int blocks_per_sm = 0;  // occupancy the shape is sized for
  size_t smem = 0;
};

// Tile-shape variants per class (k_df3c_impl.cuh, Cfg); Options::tile_variant
// selects one per class.
constexpr int kDf3cVariants = 3;

void df3c_class_info(int lab, int lc, int variant, Df3cClassInfo* ci);
int launch_df3c_class(int lab, int lc, int variant, const Df3cArgs& a, int ny, cudaStream_t s);
// Fills a->nbx, nby, nbz and n_items of one class run (host side).
void df3c_fill_items(int lab, int lc, int variant, Df3cArgs* a, int ny);
// One persistent launch of class (lab, lc) over the runs of nm molecules:
// d_args[m] (device) with items [d_item_off[m], d_item_off[m + 1]).
int launch_df3c_class_batch(int lab, int lc, int variant, const Df3cArgs* d_args, const int* d_item_off,
                            int nm, int total_items, int* counter, cudaStream_t s);
int launch_df3c_reduce(const Df3cReduceArgs& r, cudaStream_t s);
// The same four entry points for the weak-triplet kernels (k_df3c_w.cuh).
void df3c_class_info_w(int lab, int lc, Df3cClassInfo* ci);
int launch_df3c_class_w(int lab, int lc, const Df3cArgs& a, int ny, cudaStream_t s);
void df3c_fill_items_w(int lab, int lc, Df3cArgs* a, int ny);
int launch_df3c_class_batch_w(int lab, int lc, const Df3cArgs* d_args, const int* d_item_off, int nm,
                              int total_items, int* counter, cudaStream_t s);
// Row normalization of the solid harmonics (constant memory of every class
// translation unit).
cudaError_t upload_sph_rownorm(const double* rownorm, cudaStream_t s);

// Grid of a class launch of n_items work items when `resident` blocks fit the
// device: persistent (min(n_items, resident) blocks that pull items until none
// is left), or one block per item (set_df3c_block_per_item(1)), whose blocks
// retire item by item so that higher-priority streams (the metric chain) get
// SM slots while the class runs.
int df3c_grid(int n_items, int resident);
void set_df3c_block_per_item(int on);

// Dispatch row of one LAB (defined by k_df3c_l<LAB>.cu).
struct Df3cRow {
  using LaunchFn = int (*)(const Df3cArgs&, int, cudaStream_t);
  using InfoFn = void (*)(Df3cClassInfo*);
  using FillFn = void (*)(Df3cArgs*, int);
  using BatchFn = int (*)(const Df3cArgs*, const int*, int, int, int*, cudaStream_t);
  LaunchFn launch[kDf3cVariants][PA_LAUXMAX + 1] = {};
  InfoFn info[kDf3cVariants][PA_LAUXMAX + 1] = {};
  FillFn fill[kDf3cVariants][PA_LAUXMAX + 1] = {};
  BatchFn batch[kDf3cVariants][PA_LAUXMAX + 1] = {};
  // weak-triplet kernels of the precision form (one shape per class)
  LaunchFn launch_w[PA_LAUXMAX + 1] = {};
  InfoFn info_w[PA_LAUXMAX + 1] = {};
  FillFn fill_w[PA_LAUXMAX + 1] = {};
  BatchFn batch_w[PA_LAUXMAX + 1] = {};
  cudaError_t (*upload_rownorm)(const double*, cudaStream_t) = nullptr;
};
void df3c_row_0(Df3cRow*);
void df3c_row_1(Df3cRow*);
void df3c_row_2(Df3cRow*);
void df3c_row_3(Df3cRow*);
void df3c_row_4(Df3cRow*);
void df3c_row_5(Df3cRow*);
void df3c_row_6(Df3cRow*);
void df3c_row_7(Df3cRow*);
void df3c_row_8(Df3cRow*);

}  // namespace pa
