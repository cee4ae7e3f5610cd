// Host side of the screened three-center contraction: the run-time dispatch
// over (LAB, LC, tile-shape variant) to the class kernels (k_df3c_impl.cuh,
// one translation unit per LAB), the per-class variant table, and the ordered
// reduction of the per-chunk partial slabs.
#include "k_df3c.cuh"

#include <algorithm>
#include <atomic>
#include <mutex>

namespace pa {

namespace {

// df_raw[sph_off(P) + m][d] (column-major, naux rows) = sum over LAB classes and
// bra chunks of the partial slabs of class LC. A block takes 32 consecutive
// outputs (one per lane, coalesced reads of every slab); its eight warps sum
// eight consecutive ranges of the slab sequence (classes in L_ab order, chunks
// in order), and warp 0 adds the eight partial sums in order: a fixed order,
// so the results are deterministic, with dependent chains an eighth as long.
__global__ void __launch_bounds__(256) k_df3c_reduce(Df3cReduceArgs r) {
  __shared__ double part[8][32];
  const long long total = static_cast<long long>(r.n_aux) * r.nc * r.nd;
  const long long slab = static_cast<long long>(r.n_aux) * r.nc * r.nd;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int nslabs = 0;
  for (int c = 0; c < r.nclasses; ++c)
    if (r.part[c]) nslabs += r.ny[c];
  const int j0 = static_cast<int>(static_cast<long long>(nslabs) * w / 8);
  const int j1 = static_cast<int>(static_cast<long long>(nslabs) * (w + 1) / 8);
  for (long long base = blockIdx.x * 32LL; base < total; base += gridDim.x * 32LL) {
    const long long idx = base + lane;
    double s = 0.0;
    if (idx < total) {
      int j = 0;
      for (int c = 0; c < r.nclasses && j < j1; ++c) {
        const double* p = r.part[c];
        if (!p) continue;
        const int ny = r.ny[c];
        // chunks y of this class with j0 <= j + y < j1
        const int y0 = max(0, j0 - j), y1 = min(ny, j1 - j);
        for (int y = y0; y < y1; ++y) s += p[y * slab + idx];
        j += ny;
      }
    }
    part[w][lane] = s;
    __syncthreads();
    if (w == 0 && idx < total) {
      double t = part[0][lane];
#pragma unroll
      for (int k = 1; k < 8; ++k) t += part[k][lane];
      const long long fn = idx / r.nd;
      const int d = static_cast<int>(idx - fn * r.nd);
      const int pos = static_cast<int>(fn / r.nc), m = static_cast<int>(fn - pos * r.nc);
      const int sh = r.sorted_aux[r.aux_slot0 + pos];
      const long long row = r.X.shell[sh].w + m;
      r.df[row + static_cast<long long>(r.naux) * d] = t;
    }
    __syncthreads();
  }
}

constexpr int kNLab = 2 * PA_LMAX + 1;

const Df3cRow* rows() {
  static Df3cRow table[kNLab];
  static std::once_flag once;
  std::call_once(once, [] {
    df3c_row_0(&table[0]);
    df3c_row_1(&table[1]);
    df3c_row_2(&table[2]);
    df3c_row_3(&table[3]);
    df3c_row_4(&table[4]);
    df3c_row_5(&table[5]);
    df3c_row_6(&table[6]);
    df3c_row_7(&table[7]);
    df3c_row_8(&table[8]);
  });
  return table;
}

int checked(int v) { return (v >= 0 && v < kDf3cVariants) ? v : 0; }

std::atomic<int> g_block_per_item{0};

}  // namespace

int df3c_grid(int n_items, int resident) {
  return g_block_per_item.load(std::memory_order_relaxed) ? n_items : std::min(n_items, resident);
}

void set_df3c_block_per_item(int on) { g_block_per_item.store(on ? 1 : 0, std::memory_order_relaxed); }

void df3c_class_info(int lab, int lc, int variant, Df3cClassInfo* ci) {
  rows()[lab].info[checked(variant)][lc](ci);
}

int launch_df3c_class(int lab, int lc, int variant, const Df3cArgs& a, int ny, cudaStream_t s) {
  return rows()[lab].launch[checked(variant)][lc](a, ny, s);
}

void df3c_fill_items(int lab, int lc, int variant, Df3cArgs* a, int ny) {
  rows()[lab].fill[checked(variant)][lc](a, ny);
}

int launch_df3c_class_batch(int lab, int lc, int variant, const Df3cArgs* d_args, const int* d_item_off,
                            int nm, int total_items, int* counter, cudaStream_t s) {
  return rows()[lab].batch[checked(variant)][lc](d_args, d_item_off, nm, total_items, counter, s);
}

int launch_df3c_reduce(const Df3cReduceArgs& r, cudaStream_t s) {
  const long long total = static_cast<long long>(r.n_aux) * r.nc * r.nd;
  if (total == 0) return 0;
  const int blocks = static_cast<int>(std::min<long long>((total + 31) / 32, 148 * 8));
  k_df3c_reduce<<<blocks, 256, 0, s>>>(r);
  return 1;
}

void df3c_class_info_w(int lab, int lc, Df3cClassInfo* ci) { rows()[lab].info_w[lc](ci); }

int launch_df3c_class_w(int lab, int lc, const Df3cArgs& a, int ny, cudaStream_t s) {
  return rows()[lab].launch_w[lc](a, ny, s);
}

void df3c_fill_items_w(int lab, int lc, Df3cArgs* a, int ny) { rows()[lab].fill_w[lc](a, ny); }

int launch_df3c_class_batch_w(int lab, int lc, const Df3cArgs* d_args, const int* d_item_off, int nm,
                              int total_items, int* counter, cudaStream_t s) {
  return rows()[lab].batch_w[lc](d_args, d_item_off, nm, total_items, counter, s);
}

cudaError_t upload_sph_rownorm(const double* rownorm, cudaStream_t s) {
  for (int lab = 0; lab < kNLab; ++lab) {
    const cudaError_t e = rows()[lab].upload_rownorm(rownorm, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace pa
