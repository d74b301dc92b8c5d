// aero_residual_device_noalloc: the residual norms of sub_output_residual.f90:8-67
// over arrays the caller already holds on the device, computed without any
// allocation.
//
// The per-CTA partial sums that aero_residual keeps in a buffer allocated at
// set-up live here in one file-scope device array of fixed size.  Its address
// is looked up (cudaGetSymbolAddress, with the device current) on the first
// call made on a device and kept together with the CUDA context it belongs
// to; a later call in the same context reuses it, and a call that finds
// another context current (the primary context was reset and re-created,
// which reloads the module at another address) looks it up again.  A lookup
// that fails is not kept: the next call tries again.
//
// Scratch contents: slot p holds the six partial sums of CTA p of the current
// call.  Every slot the final reduction reads is written by the partial kernel
// of the same call first, so nothing has to start at zero and no clearing is
// done.  The one array is shared by every call on a device: two calls whose
// kernels overlap (different streams, or host threads racing) overwrite each
// other's partial sums.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/aerocfd_gpu.h"
#include "aero_device.cuh"
#include "aero_kernels.h"

namespace aero {

int set_last_error(int code, const char* msg);  // aero_runtime.cu

namespace {

constexpr int kThreads = 256;  // nodes per partial, as aero_residual
constexpr int kMaxDevices = 64;

// One block of the call: its index boxes and device arrays in the reference
// layout, rhs(5, is:ie, js:je, ks:ke) and dt / inv_j / sa_rhs (is:ie, ...).
struct ResidBlock {
  const double* rhs;
  const double* dt;
  const double* inv_j;
  const double* sa_rhs;  // nullptr: turbulence norm is 0
  Box b, b1;
};
struct ResidBlocks {
  ResidBlock blk[AERO_NOALLOC_MAX_BLOCKS];
};

static __device__ __align__(256) double s_part[AERO_NOALLOC_MAX_PARTS * 6];

// Partial sums of block blockIdx.y over its updated nodes, kThreads nodes per
// CTA, reduced in the same order as k_residual_partial so that the result is
// the one aero_residual gives for the same data.
__global__ void k_residual_partial_ref(ResidBlocks rb, double* __restrict__ part) {
  const ResidBlock& R = rb.blk[blockIdx.y];
  const Box& b1 = R.b1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  if (t < b1.size()) {
    int i = b1.is + (int)(t % b1.nx());
    long r = t / b1.nx();
    int j = b1.js + (int)(r % b1.ny());
    int k = b1.ks + (int)(r / b1.ny());
    long n = (long)(i - R.b.is) + (long)R.b.nx() * ((long)(j - R.b.js) + (long)R.b.ny() * (long)(k - R.b.ks));
    double dt = R.dt[n], ij = R.inv_j[n];
#pragma unroll
    for (int c = 0; c < 5; ++c) v[c] = p2(R.rhs[5 * n + c] * dt / ij);
    if (R.sa_rhs) v[5] = p2(R.sa_rhs[n] * dt);
  }
  __shared__ double sm[6][32];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double x = v[c];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sm[c][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    int nw = blockDim.x >> 5;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      double x = threadIdx.x < nw ? sm[c][threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (threadIdx.x == 0) part[6 * ((long)blockIdx.y * gridDim.x + blockIdx.x) + c] = x;
    }
  }
}

// The scratch address of one device, valid in the context whose unique ID
// (cuCtxGetId: never reused within a process, unlike a context handle, which
// a re-created primary context may get again) is `ctx_id`.
struct DeviceScratch {
  unsigned long long ctx_id = 0;
  double* part = nullptr;
};
DeviceScratch s_dev[kMaxDevices];
std::mutex s_dev_mu;

// cuCtxGetCurrent and cuCtxGetId through the runtime's driver entry point
// table (the library does not link libcuda itself); CUresult is an int-sized
// enum, 0 = success.
typedef int (*CtxGetCurrentFn)(void**);
typedef int (*CtxGetIdFn)(void*, unsigned long long*);
void* driver_fn(const char* name) {
  void* p = nullptr;
  cudaDriverEntryPointQueryResult q;
  if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
    return nullptr;
  return p;
}

// Unique ID of the current context (0 when none is current or on failure).
unsigned long long current_ctx_id() {
  static CtxGetCurrentFn get = (CtxGetCurrentFn)driver_fn("cuCtxGetCurrent");
  static CtxGetIdFn get_id = (CtxGetIdFn)driver_fn("cuCtxGetId");
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (!get || !get_id || get(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
  return id;
}

// Device address of s_part for device `dev` in the current context.
cudaError_t scratch_address(int dev, double** part) {
  std::lock_guard<std::mutex> lock(s_dev_mu);
  DeviceScratch& S = s_dev[dev];
  unsigned long long id = current_ctx_id();
  if (id && S.part && S.ctx_id == id) {
    *part = S.part;
    return cudaSuccess;
  }
  // on a first call no context may be current yet: cudaGetSymbolAddress makes
  // the device's primary context current, and the ID is read after it
  double* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress((void**)&p, s_part);
  if (e != cudaSuccess) return e;  // not kept: the next call tries again
  if (!(id = current_ctx_id())) return cudaErrorDeviceUninitialized;
  S.ctx_id = id;
  S.part = p;
  *part = p;
  return cudaSuccess;
}

bool valid_box(const int* x) { return x[0] <= x[1] && x[2] <= x[3] && x[4] <= x[5]; }
bool inside(const int* in, const int* out) {
  return in[0] >= out[0] && in[1] <= out[1] && in[2] >= out[2] && in[3] <= out[3] && in[4] >= out[4] &&
         in[5] <= out[5];
}

}  // namespace
}  // namespace aero

using namespace aero;

extern "C" int aero_residual_device_noalloc(int nblocks, const double* const* rhs, const double* const* dt,
                                            const double* const* inv_j, const double* const* sa_rhs,
                                            const int* boxes, double totalnodes, double* out7, void* stream) {
  char msg[200];
  if (nblocks < 1 || nblocks > AERO_NOALLOC_MAX_BLOCKS) {
    snprintf(msg, sizeof msg, "aero_residual_device_noalloc: %d blocks, the limit is 1..%d", nblocks,
             AERO_NOALLOC_MAX_BLOCKS);
    return set_last_error(AERO_ERR_ARG, msg);
  }
  if (!rhs || !dt || !inv_j || !boxes || !out7 || !(totalnodes > 0.0))
    return set_last_error(AERO_ERR_ARG, "aero_residual_device_noalloc: null array or totalnodes <= 0");
  ResidBlocks rb{};
  long max_n1 = 0;
  for (int m = 0; m < nblocks; ++m) {
    const int* bx = boxes + 12 * m;
    if (!valid_box(bx) || !valid_box(bx + 6) || !inside(bx + 6, bx) || !rhs[m] || !dt[m] || !inv_j[m]) {
      snprintf(msg, sizeof msg, "aero_residual_device_noalloc: block %d has a bad box or a null array", m + 1);
      return set_last_error(AERO_ERR_ARG, msg);
    }
    ResidBlock& R = rb.blk[m];
    R.rhs = rhs[m];
    R.dt = dt[m];
    R.inv_j = inv_j[m];
    R.sa_rhs = sa_rhs ? sa_rhs[m] : nullptr;
    R.b = Box{bx[0], bx[1], bx[2], bx[3], bx[4], bx[5]};
    R.b1 = Box{bx[6], bx[7], bx[8], bx[9], bx[10], bx[11]};
    max_n1 = R.b1.size() > max_n1 ? R.b1.size() : max_n1;
  }
  long ctas = (max_n1 + kThreads - 1) / kThreads;
  if (ctas * nblocks > AERO_NOALLOC_MAX_PARTS) {
    snprintf(msg, sizeof msg,
             "aero_residual_device_noalloc: %d blocks x %ld partial sums (largest block %ld updated nodes) "
             "exceed the %d-slot scratch",
             nblocks, ctas, max_n1, AERO_NOALLOC_MAX_PARTS);
    return set_last_error(AERO_ERR_ARG, msg);
  }

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return set_last_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return set_last_error(AERO_ERR_ARG, "aero_residual_device_noalloc: device ordinal out of range");
  double* part = nullptr;
  if ((e = scratch_address(dev, &part)) != cudaSuccess)
    return set_last_error(AERO_ERR_CUDA, cudaGetErrorString(e));

  cudaStream_t st = (cudaStream_t)stream;
  k_residual_partial_ref<<<dim3((unsigned)ctas, nblocks), kThreads, 0, st>>>(rb, part);
  if ((e = cudaGetLastError()) != cudaSuccess) return set_last_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  k_residual_final<<<1, 256, 0, st>>>(part, ctas * nblocks, totalnodes, out7, nullptr);
  if ((e = cudaGetLastError()) != cudaSuccess) return set_last_error(AERO_ERR_CUDA, cudaGetErrorString(e));
  return AERO_OK;
}
