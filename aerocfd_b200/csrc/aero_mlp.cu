// Warm-start network of the solver (no counterpart in the reference): an MLP
// with BF16 weights and activations and FP32 accumulation whose forward and
// backward contractions run on the tcgen05 GEMM of aero_mlp_gemm.cuh.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
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

__device__ __forceinline__ uint16_t to_bf16(float f) {  // round to nearest even
  uint32_t u = __float_as_uint(f);
  if ((u & 0x7F800000u) == 0x7F800000u) return (uint16_t)(u >> 16);  // inf / nan
  u += 0x7FFFu + ((u >> 16) & 1u);
  return (uint16_t)(u >> 16);
}
__device__ __forceinline__ float sigmoid(float z) { return 1.0f / (1.0f + expf(-z)); }

// rows x cols FP32 (row stride ld_in) -> BF16 rows x ld_out, zero-padded
// to ld_out columns and `rows_pad` rows.
__global__ void k_pack_bf16(const float* __restrict__ in, int rows, int cols, int ld_in, uint16_t* __restrict__ out,
                            int rows_pad, int ld_out) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)rows_pad * ld_out) return;
  int r = (int)(i / ld_out), c = (int)(i % ld_out);
  out[i] = (r < rows && c < cols) ? to_bf16(in[(long)r * ld_in + c]) : (uint16_t)0;
}

// z += b per column; h = bf16(silu(z)).
__global__ void k_bias_silu(float* __restrict__ z, const float* __restrict__ b, uint16_t* __restrict__ h, int rows,
                            int cols) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)rows * cols) return;
  float v = z[i] + b[i % cols];
  z[i] = v;
  h[i] = to_bf16(v * sigmoid(v));
}

// Output layer: y = c + b; masked difference to the target; dy for the
// backward GEMMs (BF16) and for the bias gradient (FP32); per-CTA loss sums.
__global__ void k_out_loss(const float* __restrict__ c, const float* __restrict__ b, const float* __restrict__ t,
                           int n_real, int n_out, int rows, int cols, float inv_count, float* __restrict__ y,
                           uint16_t* __restrict__ dy, float* __restrict__ dyf, float* __restrict__ loss_part) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (i < (long)rows * cols) {
    int r = (int)(i / cols), j = (int)(i % cols);
    float v = c[i] + b[j];
    y[i] = v;
    float d = (r < n_real && j < n_out && t) ? v - t[(long)r * n_out + j] : 0.f;
    l = d * d;
    float g = 2.f * d * inv_count;
    dy[i] = to_bf16(g);
    dyf[i] = g;
  }
  __shared__ float sm[256];
  sm[threadIdx.x] = l;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0 && loss_part) loss_part[blockIdx.x] = sm[0];
}

// dz = dh * silu'(z), BF16 for the GEMMs and FP32 for the bias gradient.
__global__ void k_silu_back(const float* __restrict__ dh, const float* __restrict__ z, uint16_t* __restrict__ dz,
                            float* __restrict__ dzf, long n) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float s = sigmoid(z[i]);
  float g = dh[i] * (s * (1.f + z[i] * (1.f - s)));
  dz[i] = to_bf16(g);
  dzf[i] = g;
}

// out[c][r] = in[r][c] for a rows x cols BF16 matrix (32 x 32 tiles).
__global__ void k_transpose_bf16(const uint16_t* __restrict__ in, int rows, int cols, uint16_t* __restrict__ out) {
  __shared__ uint16_t tile[32][33];
  int c = blockIdx.x * 32 + threadIdx.x, r0 = blockIdx.y * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    int r = r0 + y;
    if (r < rows && c < cols) tile[y][threadIdx.x] = in[(long)r * cols + c];
  }
  __syncthreads();
  int r = r0 + threadIdx.x, cc0 = blockIdx.x * 32;
  for (int y = threadIdx.y; y < 32; y += blockDim.y) {
    int cc = cc0 + y;
    if (cc < cols && r < rows) out[(long)cc * rows + r] = tile[threadIdx.x][y];
  }
}

// Column sums of a rows x cols FP32 matrix in a fixed order: CTA (x, y) sums
// rows [y*chunk, (y+1)*chunk) of columns 32x..32x+31 into part[y][col].
__global__ void k_colsum_part(const float* __restrict__ in, int rows, int cols, int chunk, float* __restrict__ part) {
  int col = blockIdx.x * 32 + threadIdx.x;
  int r0 = blockIdx.y * chunk, r1 = min(rows, r0 + chunk);
  __shared__ float sm[8][33];
  float s = 0.f;
  if (col < cols)
    for (int r = r0 + threadIdx.y; r < r1; r += blockDim.y) s += in[(long)r * cols + col];
  sm[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && col < cols) {
    float t = 0.f;
    for (int y = 0; y < (int)blockDim.y; ++y) t += sm[y][threadIdx.x];
    part[(long)blockIdx.y * cols + col] = t;
  }
}

// Adam (Kingma & Ba 2015) on FP32 master parameters, with the BF16 copy.
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       uint16_t* __restrict__ wb, long n, float lr, float b1, float b2, float c1, float c2, float eps) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float gi = g[i];
  float mi = b1 * m[i] + (1.f - b1) * gi;
  float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  w[i] = wi;
  if (wb) wb[i] = to_bf16(wi);
}

// Row gather of the training set into a batch (FP32), padded rows zero.
__global__ void k_gather_rows(const float* __restrict__ src, const int* __restrict__ idx, int n_idx, int cols,
                              float* __restrict__ dst, int rows_pad) {
  long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long)rows_pad * cols) return;
  int r = (int)(i / cols), c = (int)(i % cols);
  dst[i] = r < n_idx ? src[(long)idx[r] * cols + c] : 0.f;
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
  static int smem_dev = -1;  // device whose limit was raised (one device per process)
  int dev = 0;
  MCK(cudaGetDevice(&dev));
  if (smem_dev != dev) {
    MCK(cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGemmSmem));
    smem_dev = dev;
  }
  k_gemm_bf16<<<grid, kGemmThreads, kGemmSmem, st>>>(A, B, splits > 1 ? scratch : C, M, N, K, klen, status);
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

extern "C" int aero_mlp_gemm_timed(int M, int N, int K, int reps, double* ms_per_gemm) {
  if (M <= 0 || N <= 0 || K <= 0 || M % 128 || N % 128 || K % 64 || reps < 1 || !ms_per_gemm)
    return set_last_error(AERO_ERR_ARG, "aero_mlp_gemm_timed: M, N multiples of 128, K a multiple of 64, reps >= 1");
  uint16_t *dA = nullptr, *dB = nullptr;
  float* dC = nullptr;
  unsigned* dst = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto cleanup = [&] {
    cudaFree(dA); cudaFree(dB); cudaFree(dC); cudaFree(dst);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  size_t na = (size_t)M * K, nb = (size_t)N * K, nc = (size_t)M * N;
  if (cudaMalloc(&dA, na * 2) || cudaMalloc(&dB, nb * 2) || cudaMalloc(&dC, nc * 4) || cudaMalloc(&dst, 4)) {
    cleanup();
    return set_last_error(AERO_ERR_NOMEM, "aero_mlp_gemm_timed: device allocation failed");
  }
  // operands: every byte 0x3c, i.e. BF16 0x3c3c (about 0.0115) everywhere; the
  // values do not change the time
  cudaMemset(dA, 0x3c, na * 2);
  cudaMemset(dB, 0x3c, nb * 2);
  cudaMemset(dst, 0, 4);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int rc = mlp::gemm(dA, dB, dC, M, N, K, 1, nullptr, dst, 0);  // warm-up
  if (!rc) {
    cudaEventRecord(e0, 0);
    for (int r = 0; r < reps && !rc; ++r) rc = mlp::gemm(dA, dB, dC, M, N, K, 1, nullptr, dst, 0);
    cudaEventRecord(e1, 0);
  }
  unsigned st = 0;
  if (!rc) {
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    if (e == cudaSuccess) e = cudaMemcpy(&st, dst, 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) rc = set_last_error(AERO_ERR_CUDA, cudaGetErrorString(e));
    else if (st) rc = set_last_error(AERO_ERR_DEVICE, "aero_mlp_gemm_timed: a tensor-core wait timed out");
    *ms_per_gemm = ms / reps;
  }
  cleanup();
  return rc;
}

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

// ---------------------------------------------------------------- the network
namespace aero {
namespace mlp {
namespace {

// Layer l maps nin inputs to nout outputs (padded sizes: multiples of 128).
struct Layer {
  int nin = 0, nout = 0;
  float *w = nullptr, *b = nullptr;                        // FP32 master
  float *mw = nullptr, *vw = nullptr, *mb = nullptr, *vb = nullptr;  // Adam moments
  float *gw = nullptr, *gb = nullptr;                      // gradients
  uint16_t *wb = nullptr, *wt = nullptr;                   // BF16 copy and its transpose
};

struct Net {
  bool ok = false;
  int n_in = 0, n_out = 0, width = 0, depth = 0, batch = 0;
  int kin = 128, nout = 128;  // padded input and output widths
  std::vector<Layer> L;       // depth hidden layers, then the output layer
  std::vector<uint16_t*> h;   // h[0] input, h[l] = silu(z[l-1]); BF16 batch x width
  std::vector<float*> z;      // pre-activations, FP32
  float *c_out = nullptr, *y = nullptr, *dyf = nullptr, *dh = nullptr, *dzf = nullptr;
  uint16_t *dy = nullptr, *dz = nullptr, *tA = nullptr, *tB = nullptr;
  float *scratch = nullptr, *cpart = nullptr, *lpart = nullptr, *lhist = nullptr;
  float *xb = nullptr, *tb = nullptr, *xall = nullptr, *tall = nullptr;
  int* idx = nullptr;
  unsigned* status = nullptr;
  long n_all = 0;
  int adam_t = 0;
  std::vector<void*> allocs;
} g_net;

constexpr int kSplitMax = 32;
constexpr int kColChunk = 512;

template <class T>
int alloc(T*& p, size_t n) {
  p = nullptr;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) return set_last_error(AERO_ERR_NOMEM, "warm-start network: device allocation failed");
  g_net.allocs.push_back(p);
  cudaMemset(p, 0, n * sizeof(T));
  return AERO_OK;
}

void release() {
  for (void* p : g_net.allocs) cudaFree(p);
  cudaFree(g_net.xall);
  cudaFree(g_net.tall);
  g_net = Net{};
}

unsigned cdiv(long a, long b) { return (unsigned)((a + b - 1) / b); }

int transpose(const uint16_t* in, int rows, int cols, uint16_t* out) {
  k_transpose_bf16<<<dim3(cols / 32, rows / 32), dim3(32, 8)>>>(in, rows, cols, out);
  MCK(cudaGetLastError());
  return AERO_OK;
}
int colsum(const float* in, int rows, int cols, float* out) {
  int chunks = (rows + kColChunk - 1) / kColChunk;
  k_colsum_part<<<dim3(cdiv(cols, 32), chunks), dim3(32, 8)>>>(in, rows, cols, kColChunk, g_net.cpart);
  MCK(cudaGetLastError());
  k_splitk_reduce<<<cdiv(cols, 256), 256>>>(g_net.cpart, chunks, cols, out);
  MCK(cudaGetLastError());
  return AERO_OK;
}
int refresh_transposes() {
  for (Layer& l : g_net.L) {
    int rc = transpose(l.wb, l.nout, l.nin, l.wt);
    if (rc) return rc;
  }
  return AERO_OK;
}

// Forward pass of the current batch (xb: batch x n_in FP32); with targets tb,
// the loss parts and dy for the backward pass.
int forward(int n_real, bool with_loss) {
  Net& N = g_net;
  const int B = N.batch;
  int rc;
  k_pack_bf16<<<cdiv((long)B * N.kin, 256), 256>>>(N.xb, n_real, N.n_in, N.n_in, N.h[0], B, N.kin);
  MCK(cudaGetLastError());
  for (int l = 0; l < N.depth; ++l) {
    if ((rc = gemm(N.h[l], N.L[l].wb, N.z[l], B, N.width, N.L[l].nin, 1, N.scratch, N.status, 0))) return rc;
    k_bias_silu<<<cdiv((long)B * N.width, 256), 256>>>(N.z[l], N.L[l].b, N.h[l + 1], B, N.width);
    MCK(cudaGetLastError());
  }
  Layer& O = N.L[N.depth];
  if ((rc = gemm(N.h[N.depth], O.wb, N.c_out, B, N.nout, N.width, 1, N.scratch, N.status, 0))) return rc;
  float inv = 1.0f / ((float)n_real * (float)N.n_out);
  k_out_loss<<<cdiv((long)B * N.nout, 256), 256>>>(N.c_out, O.b, with_loss ? N.tb : nullptr, n_real, N.n_out, B,
                                                    N.nout, inv, N.y, N.dy, N.dyf, N.lpart);
  MCK(cudaGetLastError());
  return AERO_OK;
}

// Gradients of the loss of the last forward pass into every layer's gw, gb.
int backward() {
  Net& N = g_net;
  const int B = N.batch;
  int rc;
  int split = std::min(kSplitMax, B / 512);
  Layer& O = N.L[N.depth];
  if ((rc = transpose(N.dy, B, N.nout, N.tA))) return rc;
  if ((rc = transpose(N.h[N.depth], B, N.width, N.tB))) return rc;
  if ((rc = gemm(N.tA, N.tB, O.gw, N.nout, N.width, B, split, N.scratch, N.status, 0))) return rc;
  if ((rc = colsum(N.dyf, B, N.nout, O.gb))) return rc;
  if ((rc = gemm(N.dy, O.wt, N.dh, B, N.width, N.nout, 1, N.scratch, N.status, 0))) return rc;
  for (int l = N.depth - 1; l >= 0; --l) {
    Layer& Ly = N.L[l];
    k_silu_back<<<cdiv((long)B * N.width, 256), 256>>>(N.dh, N.z[l], N.dz, N.dzf, (long)B * N.width);
    MCK(cudaGetLastError());
    if ((rc = transpose(N.dz, B, N.width, N.tA))) return rc;
    if ((rc = transpose(N.h[l], B, Ly.nin, N.tB))) return rc;
    if ((rc = gemm(N.tA, N.tB, Ly.gw, N.width, Ly.nin, B, split, N.scratch, N.status, 0))) return rc;
    if ((rc = colsum(N.dzf, B, N.width, Ly.gb))) return rc;
    if (l > 0 && (rc = gemm(N.dz, Ly.wt, N.dh, B, Ly.nin, N.width, 1, N.scratch, N.status, 0))) return rc;
  }
  return AERO_OK;
}

int adam_step(float lr) {
  Net& N = g_net;
  ++N.adam_t;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  float c1 = 1.f - std::pow(b1, (float)N.adam_t), c2 = 1.f - std::pow(b2, (float)N.adam_t);
  for (Layer& l : N.L) {
    long nw = (long)l.nin * l.nout;
    k_adam<<<cdiv(nw, 256), 256>>>(l.w, l.gw, l.mw, l.vw, l.wb, nw, lr, b1, b2, c1, c2, eps);
    MCK(cudaGetLastError());
    k_adam<<<cdiv(l.nout, 256), 256>>>(l.b, l.gb, l.mb, l.vb, nullptr, l.nout, lr, b1, b2, c1, c2, eps);
    MCK(cudaGetLastError());
  }
  return refresh_transposes();
}

int check_status() {
  unsigned st = 0;
  MCK(cudaMemcpy(&st, g_net.status, 4, cudaMemcpyDeviceToHost));
  if (st) return set_last_error(AERO_ERR_DEVICE, "warm-start network: a tensor-core wait timed out");
  return AERO_OK;
}

// splitmix64 for reproducible initial weights and batch order
uint64_t mix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
double unit(uint64_t& s) { return (mix(s) >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace
}  // namespace mlp
}  // namespace aero

// ------------------------------------------------------------------- C ABI
extern "C" {

int aero_mlp_create(int n_in, int n_out, int width, int depth, int batch, unsigned long long seed) {
  using namespace aero::mlp;
  release();
  if (n_in < 1 || n_in > 128 || n_out < 1 || n_out > 128 || width < 128 || width % 128 || width > 1024 ||
      depth < 1 || depth > 32 || batch < 512 || batch % 512)
    return set_last_error(AERO_ERR_ARG,
                          "aero_mlp_create: n_in, n_out in 1..128, width a multiple of 128 up to 1024, depth 1..32, "
                          "batch a multiple of 512");
  Net& N = g_net;
  N.n_in = n_in; N.n_out = n_out; N.width = width; N.depth = depth; N.batch = batch;
  int rc;
  uint64_t s = seed;
  for (int l = 0; l <= depth; ++l) {
    Layer y;
    y.nin = l == 0 ? N.kin : width;
    y.nout = l == depth ? N.nout : width;
    size_t nw = (size_t)y.nin * y.nout;
    if ((rc = alloc(y.w, nw)) || (rc = alloc(y.b, y.nout)) || (rc = alloc(y.mw, nw)) || (rc = alloc(y.vw, nw)) ||
        (rc = alloc(y.mb, y.nout)) || (rc = alloc(y.vb, y.nout)) || (rc = alloc(y.gw, nw)) ||
        (rc = alloc(y.gb, y.nout)) || (rc = alloc(y.wb, nw)) || (rc = alloc(y.wt, nw)))
      return rc;
    // Glorot-uniform over the real fan-in / fan-out; padded rows/columns stay 0
    int fin = l == 0 ? n_in : width, fout = l == depth ? n_out : width;
    double a = std::sqrt(6.0 / (fin + fout));
    std::vector<float> w(nw, 0.f);
    std::vector<uint16_t> wb(nw, 0);
    for (int r = 0; r < fout; ++r)
      for (int c = 0; c < fin; ++c) {
        float v = (float)((2.0 * unit(s) - 1.0) * a);
        w[(size_t)r * y.nin + c] = v;
      }
    for (size_t i = 0; i < nw; ++i) {  // round to BF16 (nearest even) on the host
      uint32_t u;
      std::memcpy(&u, &w[i], 4);
      u += 0x7FFFu + ((u >> 16) & 1u);
      wb[i] = (uint16_t)(u >> 16);
    }
    MCK(cudaMemcpy(y.w, w.data(), nw * 4, cudaMemcpyHostToDevice));
    MCK(cudaMemcpy(y.wb, wb.data(), nw * 2, cudaMemcpyHostToDevice));
    N.L.push_back(y);
  }
  N.h.resize(depth + 1);
  N.z.resize(depth);
  if ((rc = alloc(N.h[0], (size_t)batch * N.kin))) return rc;
  for (int l = 1; l <= depth; ++l)
    if ((rc = alloc(N.h[l], (size_t)batch * width))) return rc;
  for (int l = 0; l < depth; ++l)
    if ((rc = alloc(N.z[l], (size_t)batch * width))) return rc;
  size_t wmax = (size_t)std::max(width, 128);
  if ((rc = alloc(N.c_out, (size_t)batch * N.nout)) || (rc = alloc(N.y, (size_t)batch * N.nout)) ||
      (rc = alloc(N.dyf, (size_t)batch * N.nout)) || (rc = alloc(N.dy, (size_t)batch * N.nout)) ||
      (rc = alloc(N.dh, (size_t)batch * width)) || (rc = alloc(N.dzf, (size_t)batch * width)) ||
      (rc = alloc(N.dz, (size_t)batch * width)) || (rc = alloc(N.tA, (size_t)batch * wmax)) ||
      (rc = alloc(N.tB, (size_t)batch * wmax)) || (rc = alloc(N.scratch, (size_t)kSplitMax * wmax * wmax)) ||
      (rc = alloc(N.cpart, (size_t)(batch / kColChunk + 1) * wmax)) ||
      (rc = alloc(N.lpart, (size_t)cdiv((long)batch * N.nout, 256))) || (rc = alloc(N.xb, (size_t)batch * n_in)) ||
      (rc = alloc(N.tb, (size_t)batch * n_out)) || (rc = alloc(N.idx, (size_t)batch)) || (rc = alloc(N.status, 1)))
    return rc;
  if ((rc = refresh_transposes())) return rc;
  MCK(cudaDeviceSynchronize());
  N.ok = true;
  return AERO_OK;
}

int aero_mlp_destroy(void) {
  aero::mlp::release();
  return AERO_OK;
}

int aero_mlp_param_count(long long* count) {
  using namespace aero::mlp;
  if (!g_net.ok) return set_last_error(AERO_ERR_STATE, "aero_mlp_create has not been called");
  long long n = 0;
  for (Layer& l : g_net.L) n += (long long)l.nin * l.nout + l.nout;
  *count = n;
  return AERO_OK;
}

int aero_mlp_get_params(float* out) {
  using namespace aero::mlp;
  if (!g_net.ok) return set_last_error(AERO_ERR_STATE, "aero_mlp_create has not been called");
  for (Layer& l : g_net.L) {
    size_t nw = (size_t)l.nin * l.nout;
    MCK(cudaMemcpy(out, l.w, nw * 4, cudaMemcpyDeviceToHost));
    out += nw;
    MCK(cudaMemcpy(out, l.b, (size_t)l.nout * 4, cudaMemcpyDeviceToHost));
    out += l.nout;
  }
  return AERO_OK;
}

int aero_mlp_gradients(const float* x, const float* t, int n, float* loss, float* grad) {
  using namespace aero::mlp;
  Net& N = g_net;
  if (!N.ok) return set_last_error(AERO_ERR_STATE, "aero_mlp_create has not been called");
  if (n < 1 || n > N.batch) return set_last_error(AERO_ERR_ARG, "aero_mlp_gradients: 1 <= n <= batch");
  MCK(cudaMemset(N.xb, 0, (size_t)N.batch * N.n_in * 4));
  MCK(cudaMemcpy(N.xb, x, (size_t)n * N.n_in * 4, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(N.tb, t, (size_t)n * N.n_out * 4, cudaMemcpyHostToDevice));
  int rc;
  if ((rc = forward(n, true)) || (rc = backward())) return rc;
  int np = (int)cdiv((long)N.batch * N.nout, 256);
  std::vector<float> lp(np);
  MCK(cudaMemcpy(lp.data(), N.lpart, np * 4, cudaMemcpyDeviceToHost));
  double sum = 0;
  for (float v : lp) sum += v;
  *loss = (float)(sum / ((double)n * N.n_out));
  for (Layer& l : N.L) {
    size_t nw = (size_t)l.nin * l.nout;
    MCK(cudaMemcpy(grad, l.gw, nw * 4, cudaMemcpyDeviceToHost));
    grad += nw;
    MCK(cudaMemcpy(grad, l.gb, (size_t)l.nout * 4, cudaMemcpyDeviceToHost));
    grad += l.nout;
  }
  return check_status();
}

int aero_mlp_train(const float* x, const float* t, long long n, int steps, float lr, unsigned long long seed,
                   float* loss_hist) {
  using namespace aero::mlp;
  Net& N = g_net;
  if (!N.ok) return set_last_error(AERO_ERR_STATE, "aero_mlp_create has not been called");
  if (n < N.batch || steps < 1) return set_last_error(AERO_ERR_ARG, "aero_mlp_train: n >= batch and steps >= 1");
  int rc = AERO_OK;
  if (N.n_all != n) {
    if (N.xall) { cudaFree(N.xall); cudaFree(N.tall); N.xall = N.tall = nullptr; }
    MCK(cudaMalloc(&N.xall, (size_t)n * N.n_in * 4));
    MCK(cudaMalloc(&N.tall, (size_t)n * N.n_out * 4));
    N.n_all = n;
  }
  MCK(cudaMemcpy(N.xall, x, (size_t)n * N.n_in * 4, cudaMemcpyHostToDevice));
  MCK(cudaMemcpy(N.tall, t, (size_t)n * N.n_out * 4, cudaMemcpyHostToDevice));
  float* dhist = nullptr;
  MCK(cudaMalloc(&dhist, (size_t)steps * 4));
  uint64_t s = seed;
  std::vector<int> perm(n);
  for (long long i = 0; i < n; ++i) perm[i] = (int)i;
  long long pos = n;
  std::vector<int> bidx(N.batch);
  int np = (int)cdiv((long)N.batch * N.nout, 256);
  for (int step = 0; step < steps && !rc; ++step) {
    if (pos + N.batch > n) {  // new epoch: Fisher-Yates shuffle
      for (long long i = n - 1; i > 0; --i) {
        long long j = (long long)(mix(s) % (uint64_t)(i + 1));
        std::swap(perm[i], perm[j]);
      }
      pos = 0;
    }
    std::copy(perm.begin() + pos, perm.begin() + pos + N.batch, bidx.begin());
    pos += N.batch;
    if (cudaMemcpy(N.idx, bidx.data(), (size_t)N.batch * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
      rc = set_last_error(AERO_ERR_CUDA, "aero_mlp_train: copy of the batch indices failed");
      break;
    }
    k_gather_rows<<<cdiv((long)N.batch * N.n_in, 256), 256>>>(N.xall, N.idx, N.batch, N.n_in, N.xb, N.batch);
    k_gather_rows<<<cdiv((long)N.batch * N.n_out, 256), 256>>>(N.tall, N.idx, N.batch, N.n_out, N.tb, N.batch);
    if ((rc = forward(N.batch, true)) || (rc = backward()) || (rc = adam_step(lr))) break;
    k_splitk_reduce<<<1, 32>>>(N.lpart, np, 1, dhist + step);  // sum of squared errors of the step
  }
  if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = set_last_error(AERO_ERR_CUDA, "aero_mlp_train failed");
  if (!rc && loss_hist) {
    if (cudaMemcpy(loss_hist, dhist, (size_t)steps * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
      rc = set_last_error(AERO_ERR_CUDA, "aero_mlp_train: copy of the loss history failed");
    for (int i = 0; i < steps; ++i) loss_hist[i] /= (float)((double)N.batch * N.n_out);
  }
  cudaFree(dhist);
  if (!rc) rc = check_status();
  return rc;
}

int aero_mlp_predict(const float* x, long long n, float* y) {
  using namespace aero::mlp;
  Net& N = g_net;
  if (!N.ok) return set_last_error(AERO_ERR_STATE, "aero_mlp_create has not been called");
  int rc;
  std::vector<float> yb((size_t)N.batch * N.nout);
  for (long long r0 = 0; r0 < n; r0 += N.batch) {
    int m = (int)std::min<long long>(N.batch, n - r0);
    MCK(cudaMemset(N.xb, 0, (size_t)N.batch * N.n_in * 4));
    MCK(cudaMemcpy(N.xb, x + r0 * N.n_in, (size_t)m * N.n_in * 4, cudaMemcpyHostToDevice));
    if ((rc = forward(m, false))) return rc;
    MCK(cudaMemcpy(yb.data(), N.y, yb.size() * 4, cudaMemcpyDeviceToHost));
    for (int r = 0; r < m; ++r)
      for (int c = 0; c < N.n_out; ++c) y[(r0 + r) * N.n_out + c] = yb[(size_t)r * N.nout + c];
  }
  return check_status();
}

}  // extern "C"
