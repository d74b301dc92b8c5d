// aero_math_eval: the device's crm::pow / crm::exp (aero_crmath.h) on host
// arrays, so that tests can compare the device's bits with the host build of
// the same functions.
#include <cuda_runtime.h>

#include "../../include/aerocfd_gpu.h"
#include "aero_device.cuh"

namespace aero {

int set_last_error(int code, const char* msg);  // aero_runtime.cu

namespace {
__global__ void k_math_eval(int fn, const double* __restrict__ x, const double* __restrict__ y, double* __restrict__ out,
                            long n) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  out[t] = fn == 1 ? crm::exp(x[t]) : crm::pow(x[t], y[t]);
}
}  // namespace
}  // namespace aero

extern "C" int aero_math_eval(int fn, const double* x, const double* y, double* out, long long n) {
  using aero::set_last_error;
  if (n < 0 || !x || !out || (fn == 0 && !y) || (fn != 0 && fn != 1))
    return set_last_error(AERO_ERR_ARG, "aero_math_eval: fn must be 0 (pow) or 1 (exp), arrays non-null, n >= 0");
  if (n == 0) return AERO_OK;
  double* d = nullptr;
  const size_t bytes = (size_t)n * sizeof(double);
  cudaError_t e = cudaMalloc(&d, 3 * bytes);
  if (e != cudaSuccess) return set_last_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && fn == 0) e = cudaMemcpy(d + n, y, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    aero::k_math_eval<<<(unsigned)((n + 255) / 256), 256>>>(fn, d, d + n, d + 2 * n, (long)n);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, d + 2 * n, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return set_last_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  return AERO_OK;
}
