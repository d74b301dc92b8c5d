// BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a) for the
// warm-start network: C[M x N] (FP32) = A[M x K] * B[N x K]^T, A and B
// row-major BF16 (K-major operands), M and N multiples of 128, K a multiple of
// 64.  Split-K: blockIdx.z = s covers K rows [s*klen, (s+1)*klen) and writes
// its partial tile to C + s*M*N (a fixed-order reduction adds the partials).
//
// Per CTA (128 threads): one 128 x 128 FP32 accumulator in tensor memory (128
// columns), A and B tiles of 128 x 64 BF16 staged in shared memory by the
// threads in the canonical no-swizzle K-major layout (8-row x 16-byte core
// matrices; LBO = 128 B between core matrices along K, SBO = 1024 B between
// 8-row groups), two stages so that staging overlaps the MMAs, four kind::f16
// MMAs of K = 16 per tile issued by one thread, completion through
// tcgen05.commit on the stage's mbarrier, and the epilogue reading tensor
// memory with tcgen05.ld (warp w reads lanes 32w..32w+31 = rows).
// Every wait is bounded; the tensor memory is always released.
#pragma once
#include <cstdint>

namespace aero {
namespace mlp {

constexpr int kBM = 128, kBN = 128, kBK = 64;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (tcgen05): start >> 4 in [0,14), LBO >> 4 in
// [16,30), SBO >> 4 in [32,46), version 1 in [46,48), no swizzle.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= 1ull << 46;
  return d;
}
// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 in [17,23), M >> 4 in [24,29).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

constexpr long kGemmSpin = 1L << 22;
// Dynamic shared memory of k_gemm_bf16: two stages of A and B tiles (2 x 2 x
// 16 KB) plus slack to align the first tile to 1024 bytes.
constexpr int kGemmStages = 2;
constexpr size_t kGemmSmem = (size_t)kGemmStages * (kBM + kBN) * kBK * sizeof(uint16_t) + 1024;

__device__ __forceinline__ bool gemm_try_wait(uint32_t bar, unsigned parity) {
  unsigned done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(bar), "r"(parity)
      : "memory");
  return done != 0;
}
__device__ __forceinline__ bool gemm_wait(uint32_t bar, unsigned parity, long budget) {
  for (long spins = 0; spins < budget; ++spins)
    if (gemm_try_wait(bar, parity)) return true;
  return false;
}

// Two-stage pipeline: the threads stage K-tile t into shared-memory stage
// t % 2 while the tensor cores still run the MMAs of tile t - 1 from the other
// stage; before restaging a stage they wait for the commit of the MMAs that
// read it two tiles earlier (tcgen05.commit arrives on that stage's mbarrier
// once every MMA issued before it is done).
__global__ void __launch_bounds__(128) k_gemm_bf16(const uint16_t* __restrict__ A, const uint16_t* __restrict__ B,
                                                  float* __restrict__ C, int M, int N, int K, int klen,
                                                  unsigned* status) {
  extern __shared__ uint8_t gemm_smem[];
  __shared__ __align__(8) unsigned long long bar[kGemmStages];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int kbeg = blockIdx.z * klen, kend = min(K, kbeg + klen);
  float* Cs = C + (long)blockIdx.z * M * N;
  // stage s: A tile at base + s * 32 KB, B tile 16 KB after it
  const uint32_t raw = smem_addr(gemm_smem);
  const uint32_t base_s = (raw + 1023u) & ~1023u;
  uint8_t* base = gemm_smem + (base_s - raw);
  const uint32_t stage_bytes = (kBM + kBN) * kBK * sizeof(uint16_t);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(kBN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    abort_flag = 0;
    for (int s = 0; s < kGemmStages; ++s)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[s])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = idesc_bf16(kBM, kBN);
  // per stage: parity of the next commit to wait for, and whether one is
  // pending (scalars, so nothing goes to local memory)
  unsigned ph0 = 0u, ph1 = 0u;
  bool pend0 = false, pend1 = false;
  int it = 0;
  for (int k0 = kbeg; k0 < kend; k0 += kBK, ++it) {
    const int s = it & 1;
    uint16_t* sA = (uint16_t*)(base + s * stage_bytes);
    uint16_t* sB = sA + kBM * kBK;
    if (s ? pend1 : pend0) {  // the MMAs that read this stage two tiles ago
      if (gemm_wait(smem_addr(&bar[s]), s ? ph1 : ph0, kGemmSpin)) {
        if (s) { ph1 ^= 1u; pend1 = false; } else { ph0 ^= 1u; pend0 = false; }
      } else {
        abort_flag = 1;
      }
      __syncthreads();
      if (abort_flag) break;
    }
    // stage A and B: 128 rows x 8 chunks of 8 BF16 each, 8 chunks per thread
#pragma unroll
    for (int x = 0; x < 8; ++x) {
      int c = tid + 128 * x;
      int r = c >> 3, kc = c & 7;
      int so = (r >> 3) * 512 + kc * 64 + (r & 7) * 8;  // in BF16 elements (1024 B, 128 B, 16 B)
      *(uint4*)(sA + so) = *(const uint4*)(A + (long)(m0 + r) * K + k0 + kc * 8);
      *(uint4*)(sB + so) = *(const uint4*)(B + (long)(n0 + r) * K + k0 + kc * 8);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for (int kk = 0; kk < kBK / 16; ++kk) {
        uint64_t da = umma_desc(smem_addr(sA) + kk * 256, 128, 1024);
        uint64_t db = umma_desc(smem_addr(sB) + kk * 256, 128, 1024);
        uint32_t acc = (k0 > kbeg || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&bar[s]))
                   : "memory");
    }
    if (s) pend1 = true; else pend0 = true;
  }
  // every commit still pending: the last tile's covers all MMAs issued
  if (!abort_flag) {
    if (pend0) {
      if (gemm_wait(smem_addr(&bar[0]), ph0, kGemmSpin)) pend0 = false; else abort_flag = 1;
    }
    if (pend1) {
      if (gemm_wait(smem_addr(&bar[1]), ph1, kGemmSpin)) pend1 = false; else abort_flag = 1;
    }
    __syncthreads();
  }
  if (abort_flag) {
    // MMAs committed on a stage whose wait ran out may still read the staged
    // tiles and write the accumulator: wait once more, with a longer bound,
    // for each pending commit before the accumulator is freed.  If such a
    // wait runs out too, the status bit below is the only guarantee left.
    if (tid == 0) {
      if (pend0) gemm_wait(smem_addr(&bar[0]), ph0, 16 * kGemmSpin);
      if (pend1) gemm_wait(smem_addr(&bar[1]), ph1, 16 * kGemmSpin);
    }
    __syncthreads();
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!abort_flag) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int j = 0; j < kBN; j += 8) {
      uint32_t v[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)j));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      float* out = Cs + (long)row * N + n0 + j;
      *(float4*)out = make_float4(__uint_as_float(v[0]), __uint_as_float(v[1]), __uint_as_float(v[2]),
                                  __uint_as_float(v[3]));
      *(float4*)(out + 4) = make_float4(__uint_as_float(v[4]), __uint_as_float(v[5]), __uint_as_float(v[6]),
                                        __uint_as_float(v[7]));
    }
  } else if (tid == 0 && status) {
    atomicOr(status, 8u);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kBN));
  }
}

}  // namespace mlp
}  // namespace aero
