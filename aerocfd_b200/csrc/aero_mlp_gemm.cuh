// BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a) for the
// warm-start network: C[M x N] (FP32) = A[M x K] * B[N x K]^T, A and B
// row-major BF16 (K-major operands), M and N multiples of 128, K a multiple of
// 64.  Split-K: blockIdx.z = s covers K rows [s*klen, (s+1)*klen) and writes
// its partial tile to C + s*M*N (a fixed-order reduction adds the partials).
//
// Per CTA (128 threads): one 128 x 128 FP32 accumulator in tensor memory (128
// columns), A and B tiles of 128 x 64 BF16 staged in shared memory by the
// threads' asynchronous 16-byte copies (cp.async) in the 128-byte-swizzled
// K-major layout (each tile row one 128-byte line, its 16-byte chunk c stored
// at chunk c ^ (row % 8); SBO = 1024 B between 8-row groups, the K = 16 steps
// 32 bytes apart inside the row), so a warp's copies fill four whole lines
// (no bank conflicts) from four whole rows of global memory, three stages so
// that the copies of the next two K-tiles are in flight while the tensor cores
// work, and two CTAs per SM (97 KB of shared memory and 128 TMEM columns
// each), so one CTA's copies, MMAs or epilogue overlap the other's; four
// kind::f16 MMAs of K = 16 per tile issued by one thread,
// completion through tcgen05.commit on the stage's mbarrier, and the epilogue
// reading tensor memory with tcgen05.ld (warp w reads lanes 32w..32w+31 =
// rows).  Every wait is bounded; the tensor memory is always released.
#pragma once
#include <cstdint>

namespace aero {
namespace mlp {

constexpr int kBM = 128, kBN = 128, kBK = 64;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor (tcgen05) of a tile in the 128-byte-swizzled
// K-major layout (1024-byte aligned 8-row groups): start >> 4 in [0,14), the
// leading offset in [16,30) (not used when the K step stays inside the
// 128-byte row), SBO = 1024 B >> 4 in [32,46), version 1 in [46,48), layout
// type SWIZZLE_128B (2) in [61,64).
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;
  d |= (uint64_t)(1024 >> 4) << 32;
  d |= 1ull << 46;
  d |= 2ull << 61;
  return d;
}
// Instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N >> 3 in [17,23), M >> 4 in [24,29).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

constexpr long kGemmSpin = 1L << 22;
// Dynamic shared memory of k_gemm_bf16: three stages of A and B tiles (3 x 2 x
// 16 KB) plus slack to align the first tile to 1024 bytes; two CTAs of
// kGemmThreads fit on an SM.
constexpr int kGemmStages = 3;
constexpr int kGemmThreads = 128;
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

// Pipeline over the K-tiles t = 0 .. nt-1 of the CTA's K range, stage t % S
// (S = kGemmStages): every thread copies its 16 chunks of tile t with
// cp.async, one commit group per tile, S-1 tiles ahead.  For tile t the
// threads wait for their own copies (cp.async.wait_group), make them visible
// to the tensor cores (fence.proxy.async, then a CTA barrier), and one thread
// issues the tile's MMAs and commits them on the stage's mbarrier; then the
// stage of tile t-1 is refilled with tile t+S-1 once that tile's commit has
// arrived (its MMAs have read the stage).
__global__ void __launch_bounds__(kGemmThreads, 2) k_gemm_bf16(const uint16_t* __restrict__ A, const uint16_t* __restrict__ B,
                                                  float* __restrict__ C, int M, int N, int K, int klen,
                                                  unsigned* status) {
  constexpr int S = kGemmStages;
  extern __shared__ uint8_t gemm_smem[];
  __shared__ __align__(8) unsigned long long bar[S];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kBM, n0 = blockIdx.x * kBN;
  const int kbeg = blockIdx.z * klen, kend = min(K, kbeg + klen);
  const int nt = (kend - kbeg) / kBK;  // K-tiles of this CTA (K and klen are multiples of kBK)
  float* Cs = C + (long)blockIdx.z * M * N;
  // stage s: A tile at base + s * 32 KB, B tile 16 KB after it
  const uint32_t raw = smem_addr(gemm_smem);
  const uint32_t base_s = (raw + 1023u) & ~1023u;
  const uint32_t stage_bytes = (kBM + kBN) * kBK * sizeof(uint16_t);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                 "r"(kBN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    abort_flag = 0;
    for (int x = 0; x < S; ++x)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&bar[x])) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t idesc = idesc_bf16(kBM, kBN);
  // this thread's 16-byte chunks of tile t into stage x: chunk c = tid +
  // kGemmThreads j of the A and of the B tile (1024 chunks each), row c / 8,
  // K-chunk c % 8, stored at row * 128 + ((K-chunk ^ row % 8) * 16)
  auto copy_tile = [&](int t, int x) {
    const int k0 = kbeg + t * kBK;
    const uint32_t sA = base_s + (uint32_t)x * stage_bytes;
    const uint32_t sB = sA + kBM * kBK * sizeof(uint16_t);
#pragma unroll
    for (int j = 0; j < 1024 / kGemmThreads; ++j) {
      const int c = tid + kGemmThreads * j;
      const int r = c >> 3, kc = c & 7;
      const uint32_t so = (uint32_t)(r * 128 + ((kc ^ (r & 7)) << 4));
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sA + so),
                   "l"(A + (long)(m0 + r) * K + k0 + kc * 8)
                   : "memory");
      asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sB + so),
                   "l"(B + (long)(n0 + r) * K + k0 + kc * 8)
                   : "memory");
    }
  };
  for (int t = 0; t < S - 1; ++t) {
    if (t < nt) copy_tile(t, t);
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  int last = -1;  // the last tile whose MMAs were committed
  for (int t = 0; t < nt; ++t) {
    const int x = t % S;
    // tile t's copies are the oldest of the S-1 groups in flight
    asm volatile("cp.async.wait_group %0;" ::"n"(S - 2) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t sA = base_s + (uint32_t)x * stage_bytes;
      const uint32_t sB = sA + kBM * kBK * sizeof(uint16_t);
#pragma unroll
      for (int kk = 0; kk < kBK / 16; ++kk) {
        uint64_t da = umma_desc_sw128(sA + kk * 32);
        uint64_t db = umma_desc_sw128(sB + kk * 32);
        uint32_t acc = (t > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(tmem),
            "l"(da), "l"(db), "r"(idesc), "r"(acc)
            : "memory");
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(&bar[x]))
                   : "memory");
    }
    last = t;
    // refill the stage of tile t-1 with tile t+S-1 once tile t-1's MMAs are
    // done (their commit is the (t-1)/S-th completion of that stage's barrier)
    const int tn = t + S - 1;
    if (tn < nt) {
      const int xp = tn % S;
      if (t >= 1 && !gemm_wait(smem_addr(&bar[xp]), (unsigned)(((t - 1) / S) & 1), kGemmSpin)) abort_flag = 1;
      __syncthreads();
      if (abort_flag) break;
      copy_tile(tn, xp);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  }
  // no copy may still be landing in shared memory when the CTA goes on
  asm volatile("cp.async.wait_all;" ::: "memory");
  // the last commit covers every MMA issued before it
  if (!abort_flag && last >= 0 && !gemm_wait(smem_addr(&bar[last % S]), (unsigned)((last / S) & 1), kGemmSpin))
    abort_flag = 1;
  __syncthreads();
  if (abort_flag) {
    // MMAs committed before a wait ran out may still read the staged tiles
    // and write the accumulator: wait once more, with a longer bound, for the
    // last commit before the accumulator is freed.  If that wait runs out too,
    // the status bit below is the only guarantee left.
    if (tid == 0 && last >= 0) gemm_wait(smem_addr(&bar[last % S]), (unsigned)((last / S) & 1), 16 * kGemmSpin);
    __syncthreads();
  }
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!abort_flag) {
    // warp w reads accumulator lanes 32 (w % 4) .. +31 (its rows) and the
    // (w / 4)-th share of the columns
    const int quarter = warp & 3;
    const int ncol = kBN / (kGemmThreads / 128), col0 = (warp >> 2) * ncol;
    const int row = m0 + quarter * 32 + lane;
#pragma unroll 1
    for (int j = col0; j < col0 + ncol; j += 8) {
      uint32_t v[8];
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                   : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                   : "r"(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)j));
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
