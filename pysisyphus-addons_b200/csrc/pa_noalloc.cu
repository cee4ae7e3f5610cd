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

#include <mutex>
#include <string>

#include "k_linalg.cuh"
#include "pa_b200.h"

namespace pa {
// Thread-local error message of the C-ABI (pa_api.cu).
int set_error(int code, const std::string& msg);
}  // namespace pa

namespace {

constexpr size_t kScratchDoubles = PA_NOALLOC_SCRATCH_DOUBLES;
constexpr int kMaxDevices = 64;

// Every GPU that loads this library holds this array until the process exits.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device, looked up once
// per device (the host-side name is only a stand-in for the symbol).
int scratch_address(double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return pa::set_error(PA_ERR_NO_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return pa::set_error(PA_ERR_ARG, "device index out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return pa::set_error(PA_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") +
                                            cudaGetErrorString(e));
    g_scratch_addr[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_addr[dev];
  return PA_OK;
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
  double* scratch = nullptr;
  int st = scratch_address(&scratch);
  if (st != PA_OK) return st;
  if (n == 0) return PA_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  double* work = scratch;
  double* Bw = scratch + dinv;
  int* info = reinterpret_cast<int*>(scratch + dinv + static_cast<size_t>(n) * nrhs);
  const size_t nb = static_cast<size_t>(n) * nrhs;
  if (nb) {
    const cudaError_t e = cudaMemcpyAsync(Bw, d_B, sizeof(double) * nb, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess)
      return pa::set_error(PA_ERR_CUDA, std::string("copy of B: ") + cudaGetErrorString(e));
  }
  pa::cholesky_lower(d_A, n, info, work, s);  // clears *info first
  if (nb) pa::trsm_lower_left(d_A, n, work, Bw, n, nrhs, d_X, n, s);
  int h_info = 0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&h_info, info, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return pa::set_error(PA_ERR_CUDA, std::string("Cholesky solve: ") + cudaGetErrorString(e));
  if (h_info != 0)
    return pa::set_error(PA_ERR_NOT_SPD, "matrix is not positive definite (Cholesky pivot " +
                                             std::to_string(h_info) + ")");
  return PA_OK;
}
