// pa_split_product_check: the split-BF16 tensor-core product of the precision
// form (umma.cuh) on caller matrices, one block. It runs the same shared-memory
// layout, descriptors, tensor-memory accumulator and drain as the weak-triplet
// three-center kernels, so a test can compare them with an FP64 product on
// plain inputs (including operands with fewer real rows than the MMA shape).
#include <cuda_runtime.h>

#include <string>

#include "pa_b200.h"
#include "umma.cuh"

namespace pa {
int set_error(int code, const std::string& msg);
}  // namespace pa

namespace {

constexpr int kThreads = 256;
constexpr int kN = 48;       // MMA N (accumulator columns); B has at most 48 real rows
// padding after each operand: its virtual rows (M = 128, N = 48) read at most
// 2048 (A) and 768 (B) bytes past the last k column; 8 KB keeps every read of
// the block inside its own buffers even for descriptor offsets read the other
// way round
constexpr int kPadA = 8192;
constexpr int kPadB = 8192;

// C[m][n] = sum_k A[m][k] B[n][k] (row-major inputs, m <= 128, n <= 48, k <= 128).
__global__ void __launch_bounds__(kThreads) k_split_product_check(int m, int n, int k, const double* __restrict__ A,
                                                                  const double* __restrict__ B, double* __restrict__ C,
                                                                  int* __restrict__ status) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint32_t s_tmem;
  __shared__ __align__(8) uint64_t s_bar;
  const int ar = (m + 7) / 8 * 8, br = (n + 7) / 8 * 8, K = (k + 15) / 16 * 16;
  const uint32_t a_slice = static_cast<uint32_t>(K * ar * 2), b_slice = static_cast<uint32_t>(K * br * 2);
  unsigned char* a0 = smem;
  unsigned char* b0 = smem + 3 * a_slice + kPadA;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < ar * K; i += kThreads) {
    const int r = i / K, c = i - r * K;
    const double v = (r < m && c < k) ? A[static_cast<long long>(r) * k + c] : 0.0;
    __nv_bfloat16 s[3];
    pa::umma::split3(v, s[0], s[1], s[2]);
    const uint32_t off = pa::umma::kmajor_off(r, c, ar);
    for (int j = 0; j < 3; ++j) *reinterpret_cast<__nv_bfloat16*>(a0 + j * a_slice + off) = s[j];
  }
  for (int i = tid; i < br * K; i += kThreads) {
    const int r = i / K, c = i - r * K;
    const double v = (r < n && c < k) ? B[static_cast<long long>(r) * k + c] : 0.0;
    __nv_bfloat16 s[3];
    pa::umma::split3(v, s[0], s[1], s[2]);
    const uint32_t off = pa::umma::kmajor_off(r, c, br);
    for (int j = 0; j < 3; ++j) *reinterpret_cast<__nv_bfloat16*>(b0 + j * b_slice + off) = s[j];
  }
  // the paddings (virtual rows) hold finite values
  for (int i = tid; i < kPadA / 4; i += kThreads) reinterpret_cast<float*>(a0 + 3 * a_slice)[i] = 0.f;
  for (int i = tid; i < kPadB / 4; i += kThreads) reinterpret_cast<float*>(b0 + 3 * b_slice)[i] = 0.f;
  if (tid == 0) pa::umma::mbar_init(&s_bar, 1);
  if (warp == 0) pa::umma::tmem_alloc(&s_tmem, 64);
  pa::umma::fence_async_smem();
  pa::umma::fence_before();
  __syncthreads();
  pa::umma::fence_after();
  const uint32_t tmem = s_tmem;
  if (tid == 0) {
    pa::umma::issue_split_product(tmem, pa::umma::smem_addr(a0), a_slice, ar, pa::umma::smem_addr(b0), b_slice,
                                  br, K, pa::umma::idesc_bf16(128, kN));
    pa::umma::commit(pa::umma::smem_addr(&s_bar));
  }
  const bool ok = pa::umma::mbar_wait(&s_bar, 0);
  if (__syncthreads_and(ok)) {
    pa::umma::fence_after();
    const int q = warp & 3, h = warp >> 2;
    float v[24];
    for (int j = 0; j < 3; ++j) pa::umma::tmem_ld8(tmem + (static_cast<uint32_t>(32 * q) << 16) + 24 * h + 8 * j, v + 8 * j);
    pa::umma::tmem_wait_ld();
    const int row = 32 * q + (tid & 31);
    if (row < m)
      for (int j = 0; j < 24; ++j) {
        const int col = 24 * h + j;
        if (col < n) C[static_cast<long long>(row) * n + col] = static_cast<double>(v[j]);
      }
  } else if (tid == 0) {
    *status = 1;
  }
  pa::umma::fence_before();
  __syncthreads();
  if (warp == 0) {
    pa::umma::fence_after();
    pa::umma::tmem_free(tmem, 64);
  }
}

}  // namespace

extern "C" int pa_split_product_check(int m, int n, int k, const double* A, const double* B, double* C) {
  if (m < 1 || m > 128 || n < 1 || n > kN || k < 1 || k > 128 || !A || !B || !C)
    return pa::set_error(PA_ERR_ARG, "pa_split_product_check: need 1 <= m <= 128, 1 <= n <= 48, 1 <= k <= 128");
  const int ar = (m + 7) / 8 * 8, br = (n + 7) / 8 * 8, K = (k + 15) / 16 * 16;
  const size_t smem = 3 * static_cast<size_t>(K) * (ar + br) * 2 + kPadA + kPadB;
  double *dA = nullptr, *dB = nullptr, *dC = nullptr;
  int* dst = nullptr;
  auto cleanup = [&] {
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dC);
    cudaFree(dst);
  };
  cudaError_t e = cudaMalloc(&dA, sizeof(double) * m * k);
  if (e == cudaSuccess) e = cudaMalloc(&dB, sizeof(double) * n * k);
  if (e == cudaSuccess) e = cudaMalloc(&dC, sizeof(double) * m * n);
  if (e == cudaSuccess) e = cudaMalloc(&dst, sizeof(int));
  if (e == cudaSuccess) e = cudaMemcpy(dA, A, sizeof(double) * m * k, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dB, B, sizeof(double) * n * k, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(dst, 0, sizeof(int));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_split_product_check, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
  if (e != cudaSuccess) {
    cleanup();
    return pa::set_error(PA_ERR_CUDA, std::string("pa_split_product_check: ") + cudaGetErrorString(e));
  }
  k_split_product_check<<<1, kThreads, smem>>>(m, n, k, dA, dB, dC, dst);
  int st = 0;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(C, dC, sizeof(double) * m * n, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(&st, dst, sizeof(int), cudaMemcpyDeviceToHost);
  cleanup();
  if (e != cudaSuccess) return pa::set_error(PA_ERR_CUDA, std::string("pa_split_product_check: ") + cudaGetErrorString(e));
  if (st != 0) return pa::set_error(PA_ERR_TIMEOUT, "pa_split_product_check: tensor-core completion wait timed out");
  return PA_OK;
}
