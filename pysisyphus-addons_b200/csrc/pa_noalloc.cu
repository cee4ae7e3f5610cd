// Allocation-free Cholesky solve: pa_cholesky_solve_noalloc.
//
// Same arithmetic as pa_cholesky_solve (blocked Cholesky, inverted 64 x 64
// diagonal blocks, blocked forward substitution; k_linalg.cu), but on device
// buffers the caller owns and with every scratch byte taken from one
// file-scope device array instead of cudaMalloc / a memory pool. It exists
// for callers that cannot allocate device memory themselves at call time:
// applications whose GPU memory is handed out entirely by another allocator
// (a framework's caching allocator that reserved the device up front), and
// code that must not call cudaMalloc / cudaFree because those calls can
// synchronize the whole device and stall unrelated work in flight.
//
// Scratch layout inside g_noalloc_scratch (doubles):
//   [0, nblk * 4096)                  inverses of L's 64 x 64 diagonal blocks
//   [nblk * 4096, + n * nrhs)         working copy of B (the substitution
//                                     overwrites its right-hand side)
//   last 32 doubles of the used part  pivot status word (int), cleared by
//                                     every call before the factorization
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "k_linalg.cuh"
#include "pa_b200.h"

namespace pa {
// Thread-local error message of the C-ABI (pa_api.cu).
int set_error(int code, const std::string& msg);
}  // namespace pa

namespace {

constexpr size_t kScratchDoubles = PA_NOALLOC_SCRATCH_DOUBLES;

// Every GPU that loads this library holds this array until the process exits.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

// Device address of g_noalloc_scratch in the current context. The host-side
// name is only a stand-in for the symbol; the address belongs to a context
// (it changes after cudaDeviceReset, and differs on a non-primary context of
// the same device), so it is looked up on every call -- a host-side table
// lookup once the module is loaded on the device.
int scratch_address(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return pa::set_error(PA_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
  *out = static_cast<double*>(p);
  return PA_OK;
}

bool overlaps(const void* a, size_t abytes, const void* b, size_t bbytes) {
  const auto x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
  return abytes && bbytes && x < y + bbytes && y < x + abytes;
}

}  // namespace

extern "C" int pa_cholesky_solve_noalloc(int n, double* d_A, int nrhs, const double* d_B, double* d_X,
                                         void* stream) {
  if (n < 0 || nrhs < 0 || (n > 0 && !d_A) || (n > 0 && nrhs > 0 && (!d_B || !d_X)))
    return pa::set_error(PA_ERR_ARG, "invalid Cholesky arguments");
  const size_t nblk = (static_cast<size_t>(n) + 63) / 64;
  const size_t dinv = nblk * 64 * 64;
  const size_t need = dinv + static_cast<size_t>(n) * nrhs + 32;
  if (need > kScratchDoubles)
    return pa::set_error(PA_ERR_SCRATCH,
                         "pa_cholesky_solve_noalloc: n = " + std::to_string(n) + ", nrhs = " +
                             std::to_string(nrhs) + " needs " + std::to_string(need) +
                             " scratch doubles; the fixed maximum is " + std::to_string(kScratchDoubles) +
                             " (64 * ceil(n / 64) * 64 + n * nrhs + 32 <= " +
                             std::to_string(kScratchDoubles) + ")");
  const size_t nb = static_cast<size_t>(n) * nrhs;
  // X is written while L is still being read: it must not overlap A (X == B is fine,
  // B is copied to the scratch array before anything is written)
  if (nb && overlaps(d_X, sizeof(double) * nb, d_A, sizeof(double) * n * static_cast<size_t>(n)))
    return pa::set_error(PA_ERR_ARG, "pa_cholesky_solve_noalloc: d_X overlaps d_A");
  // an error left by earlier, unrelated work is reported as such and not cleared
  cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess)
    return pa::set_error(PA_ERR_CUDA, std::string("a CUDA error from earlier work is pending: ") +
                                          cudaGetErrorString(e));
  double* scratch = nullptr;
  int st = scratch_address(&scratch);
  if (st != PA_OK) return st;
  if (n == 0) return PA_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* work = scratch;
  double* Bw = scratch + dinv;
  int* info = reinterpret_cast<int*>(scratch + dinv + static_cast<size_t>(n) * nrhs);
  if (nb) {
    e = cudaMemcpyAsync(Bw, d_B, sizeof(double) * nb, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess)
      return pa::set_error(PA_ERR_CUDA, std::string("copy of B: ") + cudaGetErrorString(e));
  }
  pa::cholesky_lower(d_A, n, info, work, s);  // clears *info first
  if (nb) pa::trsm_lower_left(d_A, n, work, Bw, n, nrhs, d_X, n, s);
  int h_info = 0;
  e = cudaGetLastError();  // nothing was pending on entry: this is this call's own launch error
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return pa::set_error(PA_ERR_CUDA, std::string("Cholesky solve: ") + cudaGetErrorString(e));
  if (h_info != 0)
    return pa::set_error(PA_ERR_NOT_SPD, "matrix is not positive definite (Cholesky pivot " +
                                             std::to_string(h_info) + ")");
  return PA_OK;
}
