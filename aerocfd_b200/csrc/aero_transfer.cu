// Layout conversion between the reference's host arrays a(nc, is:ie, js:je, ks:ke)
// (column-major, component fastest) and the device's component planes.
#include "aero_device.cuh"
#include "aero_kernels.h"

namespace aero {

__global__ void k_aos_to_soa(const double* __restrict__ src, double* __restrict__ dst, long n,
                             int nc, long plane) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  for (int c = 0; c < nc; ++c) dst[(long)c * plane + t] = src[t * nc + c];
}

__global__ void k_soa_to_aos(const double* __restrict__ src, double* __restrict__ dst, long n,
                             int nc, long plane) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  for (int c = 0; c < nc; ++c) dst[t * nc + c] = src[(long)c * plane + t];
}

__global__ void k_fill_plane(double* __restrict__ p, long n, double val) {
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) p[t] = val;
}

}  // namespace aero
