// Warm-start network of the solver (no counterpart in the reference): an MLP
// with BF16 weights and activations and FP32 accumulation whose forward and
// backward contractions run on the tcgen05 GEMM of aero_mlp_gemm.cuh.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <vector>

#include "../../include/aerocfd_gpu.h"
#include "aero_mlp_gemm.cuh"

namespace aero {
int set_last_error(int code, const char* msg);  // aero_runtime.cu

namespace mlp {
namespace {

#define MCK(call)                                                                      \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      char b_[200];                                                                    \
      std::snprintf(b_, sizeof b_, "%s: %s", #call, cudaGetErrorString(e_));           \
      return set_last_error(e_ == cudaErrorMemoryAllocation ? AERO_ERR_NOMEM : AERO_ERR_CUDA, b_); \
    }                                                                                  \
  } while (0)

// Fixed-order sum of the split-K partial tiles: out[i] = sum_s part[s][i].
__global__ void k_splitk_reduce(const float* __restrict__ part, int splits, long n, float* __restrict__ out) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = 0.f;
  for (int x = 0; x < splits; ++x) s += part[(long)x * n + i];
  out[i] = s;
}

}  // namespace

// C = A * B^T on the device; splits > 1 reduces the partial tiles into C with
// `scratch` (splits * M * N floats).
int gemm(const uint16_t* A, const uint16_t* B, float* C, int M, int N, int K, int splits, float* scratch,
         unsigned* status, cudaStream_t st) {
  if (M % kBM || N % kBN || K % kBK || splits < 1)
    return set_last_error(AERO_ERR_ARG, "tensor-core GEMM needs M, N multiples of 128 and K a multiple of 64");
  int ktiles = K / kBK;
  if (splits > ktiles) splits = ktiles;
  int klen = ((ktiles + splits - 1) / splits) * kBK;
  splits = (K + klen - 1) / klen;
  dim3 grid(N / kBN, M / kBM, splits);
  k_gemm_bf16<<<grid, 128, 0, st>>>(A, B, splits > 1 ? scratch : C, M, N, K, klen, status);
  MCK(cudaGetLastError());
  if (splits > 1) {
    long n = (long)M * N;
    k_splitk_reduce<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(scratch, splits, n, C);
    MCK(cudaGetLastError());
  }
  return AERO_OK;
}

}  // namespace mlp
}  // namespace aero

using namespace aero;

extern "C" int aero_mlp_gemm(const uint16_t* a, const uint16_t* b, float* c, int M, int N, int K, int splits) {
  if (M <= 0 || N <= 0 || K <= 0 || M % 128 || N % 128 || K % 64 || splits < 1)
    return set_last_error(AERO_ERR_ARG, "aero_mlp_gemm: M, N multiples of 128, K a multiple of 64, splits >= 1");
  uint16_t *dA = nullptr, *dB = nullptr;
  float *dC = nullptr, *dS = nullptr;
  unsigned* dst = nullptr;
  int rc = AERO_OK;
  auto cleanup = [&] {
    cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(dS); cudaFree(dst);
  };
  size_t na = (size_t)M * K, nb = (size_t)N * K, nc = (size_t)M * N;
  if (cudaMalloc(&dA, na * 2) || cudaMalloc(&dB, nb * 2) || cudaMalloc(&dC, nc * 4) ||
      cudaMalloc(&dS, nc * 4 * (size_t)splits) || cudaMalloc(&dst, 4)) {
    cleanup();
    return set_last_error(AERO_ERR_NOMEM, "aero_mlp_gemm: device allocation failed");
  }
  cudaMemcpy(dA, a, na * 2, cudaMemcpyHostToDevice);
  cudaMemcpy(dB, b, nb * 2, cudaMemcpyHostToDevice);
  cudaMemset(dst, 0, 4);
  rc = mlp::gemm(dA, dB, dC, M, N, K, splits, dS, dst, 0);
  unsigned st = 0;
  if (!rc) {
    cudaError_t e = cudaMemcpy(c, dC, nc * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&st, dst, 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = set_last_error(AERO_ERR_CUDA, cudaGetErrorString(e));
    else if (st) rc = set_last_error(AERO_ERR_DEVICE, "aero_mlp_gemm: a tensor-core wait timed out");
  }
  cleanup();
  return rc;
}
