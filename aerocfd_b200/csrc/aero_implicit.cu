// 1st-order implicit LU-SGS update (sub_timeadvancement_1stimplicit.f90 and
// sub_timeadvancement_jac.f90) as an exact-order hyperplane wavefront.
//
// The reference sweeps k, j, i serially.  Node (i,j,k) of the forward sweep
// depends only on (i-1,j,k), (i,j-1,k), (i,j,k-1), so all nodes with the same
// (i-is1)+(j-js1)+(k-ks1) = h can run together once plane h-1 is done; the
// per-node arithmetic is the reference's, so the result is bit-identical to the
// serial loop.  Neighbours outside the updated box hold dq = 0 in the
// reference (dq and dqstar are zero-filled), so their block contributes an
// exact zero and is skipped.
#include <cmath>

#include "aero_device.cuh"
#include "aero_kernels.h"

namespace aero {

// sub_timeadvancement_1stimplicit.f90:72-156: rhs on the updated nodes and the
// spectral radii ra, rb, rc and the diagonal on the updated box grown by one.
__global__ void k_lusgs_prep(const BlockView* __restrict__ blocks, CaseConsts cc) {
  const BlockView& B = blocks[blockIdx.y];
  const Box& b1 = B.b1;
  Box e{b1.is - 1, b1.ie + 1, b1.js - 1, b1.je + 1, b1.ks - 1, b1.ke + 1};
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= e.size()) return;
  int i = e.is + (int)(t % e.nx());
  long r = t / e.nx();
  int j = e.js + (int)(r % e.ny());
  int k = e.ks + (int)(r / e.ny());
  long n = B.at(i, j, k);
  if (b1.contains(i, j, k)) {
#pragma unroll
    for (int c = 1; c <= 5; ++c) B.v(F_RHS, c, n) = B.v(F_RHSI, c, n) + B.v(F_RHSV, c, n);
  }
  double phi = cc.cfl >= 1.0e3 ? 0.0 : 1.0;
  double u = B.v(F_PRI, 2, n), v = B.v(F_PRI, 3, n), w = B.v(F_PRI, 4, n), c = B.v(F_PRI, 7, n);
  double rr[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double x0 = B.v(F_DXIDX, 3 * d + 1, n), y0 = B.v(F_DXIDX, 3 * d + 2, n), z0 = B.v(F_DXIDX, 3 * d + 3, n);
    double temp = p2(x0) + p2(y0) + p2(z0);
    temp = sqrt(temp);
    double cu = x0 * u + y0 * v + z0 * w;
    rr[d] = fabs(cu) + fabs(c * temp);
  }
  B.s(F_RA, n) = rr[0];
  B.s(F_RB, n) = rr[1];
  B.s(F_RC, n) = rr[2];
  B.s(F_DIAG, n) = phi * 1.0 / B.s(F_DT, n) + rr[0] + rr[1] + rr[2];
}

// calc_jm (sub_timeadvancement_jac.f90:17-62) at node n with the metric row
// starting at component cbase; A is row-major, A[r*5+c] = a(r+1,c+1).
__device__ __forceinline__ void calc_jm(const BlockView& B, long n, int cbase, double gamma,
                                        double A[25]) {
  double rho = B.v(F_Q, 1, n), mu0 = B.v(F_Q, 2, n), mv0 = B.v(F_Q, 3, n);
  double mw0 = B.v(F_Q, 4, n), e0 = B.v(F_Q, 5, n);
  double dxidx = B.v(F_DXIDX, cbase, n), dxidy = B.v(F_DXIDX, cbase + 1, n);
  double dxidz = B.v(F_DXIDX, cbase + 2, n);
  double a2 = gamma - 1.0, a3 = gamma - 2.0;
  double uu = (dxidx * mu0 + dxidy * mv0 + dxidz * mw0) / rho;
  double phi = 0.5 * a2 * (p2(mu0) + p2(mv0) + p2(mw0)) / p2(rho);
  double a1 = gamma * e0 / rho - phi;
  A[0] = 0.0; A[1] = dxidx; A[2] = dxidy; A[3] = dxidz; A[4] = 0.0;
  A[5] = phi * dxidx - uu * mu0 / rho;
  A[6] = uu - a3 * dxidx * mu0 / rho;
  A[7] = dxidy * mu0 / rho - a2 * dxidx * mv0 / rho;
  A[8] = dxidz * mu0 / rho - a2 * dxidx * mw0 / rho;
  A[9] = a2 * dxidx;
  A[10] = phi * dxidy - uu * mv0 / rho;
  A[11] = dxidx * mv0 / rho - a2 * dxidy * mu0 / rho;
  A[12] = uu - a3 * dxidy * mv0 / rho;
  A[13] = dxidz * mv0 / rho - a2 * dxidy * mw0 / rho;
  A[14] = a2 * dxidy;
  A[15] = phi * dxidz - uu * mw0 / rho;
  A[16] = dxidx * mw0 / rho - a2 * dxidz * mu0 / rho;
  A[17] = dxidy * mw0 / rho - a2 * dxidz * mv0 / rho;
  A[18] = uu - a3 * dxidz * mw0 / rho;
  A[19] = a2 * dxidz;
  A[20] = (phi - a1) * uu;
  A[21] = a1 * dxidx - a2 * uu * mu0 / rho;
  A[22] = a1 * dxidy - a2 * uu * mv0 / rho;
  A[23] = a1 * dxidz - a2 * uu * mw0 / rho;
  A[24] = gamma * uu;
}

// Position of updated-box offsets (a,b,c) in the hyperplane-major order:
// planes h = a+b+c one after another; inside a plane, c ascending, then b.
__device__ __forceinline__ long plane_pos(const BlockView& B, int a, int b, int c) {
  int nx1 = B.b1.nx(), ny1 = B.b1.ny();
  int h = a + b + c;
  long pos = B.poff[h];
  int cmin = max(0, h - (nx1 - 1) - (ny1 - 1));
  for (int cc = cmin; cc < c; ++cc) {
    int r = h - cc;
    int bmin = max(0, r - (nx1 - 1)), bmax = min(ny1 - 1, r);
    if (bmax >= bmin) pos += bmax - bmin + 1;
  }
  int bmin = max(0, (h - c) - (nx1 - 1));
  return pos + (b - bmin);
}

// Hyperplane-major index of every updated node: its natural (box) index and
// the positions of its six neighbours (-1 outside the updated box).  Fixed
// for a block, so resident blocks fill it once.
__global__ void k_plane_index(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  const Box& b1 = B.b1;
  long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= b1.size()) return;
  int nx1 = b1.nx(), ny1 = b1.ny(), nz1 = b1.nz();
  int a = (int)(u % nx1);
  long r = u / nx1;
  int b = (int)(r % ny1);
  int c = (int)(r / ny1);
  const int off[3] = {a, b, c};
  const int lim[3] = {nx1, ny1, nz1};
  long pos = plane_pos(B, a, b, c);
  B.nat[pos] = B.at(b1.is + a, b1.js + b, b1.ks + c);
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    int lo[3] = {a, b, c}, hi[3] = {a, b, c};
    lo[e] -= 1;
    hi[e] += 1;
    B.nbr[6 * pos + e] = off[e] > 0 ? (int)plane_pos(B, lo[0], lo[1], lo[2]) : -1;
    B.nbr[6 * pos + 3 + e] = off[e] < lim[e] - 1 ? (int)plane_pos(B, hi[0], hi[1], hi[2]) : -1;
  }
}

// The off-diagonal blocks of both sweeps, off the critical path.  For every
// updated node (the provider) and direction d: A = calc_jm at the provider,
// S+ = 0.5*(A + r*I)*inv_j goes to the forward record of the node one step up
// in d, S- = 0.5*(A - r*I)*inv_j to the backward record of the node one step
// down (sub_timeadvancement_1stimplicit.f90:283-301, :459-477, same
// operations).  Each node also stores rhs, diag and inv_j in its record.
__global__ void k_lusgs_mats(const BlockView* __restrict__ blocks, CaseConsts cc) {
  const BlockView& B = blocks[blockIdx.y];
  const Box& b1 = B.b1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long N1 = b1.size();
  if (t >= 3 * N1) return;
  int d = (int)(t % 3);
  long u = t / 3;
  int nx1 = b1.nx(), ny1 = b1.ny(), nz1 = b1.nz();
  int a = (int)(u % nx1);
  long r = u / nx1;
  int b = (int)(r % ny1);
  int c = (int)(r / ny1);
  long n = B.at(b1.is + a, b1.js + b, b1.ks + c);
  int off[3] = {a, b, c};
  const int lim[3] = {nx1, ny1, nz1};
  long pos = plane_pos(B, a, b, c);
  if (d == 0) {
    double* sc = B.sca + 8 * pos;
#pragma unroll
    for (int x = 0; x < 5; ++x) sc[x] = B.v(F_RHS, x + 1, n);
    sc[5] = B.s(F_DIAG, n);
    sc[6] = B.s(F_INVJ, n);
    sc[7] = 0.0;
  }
  bool up = off[d] < lim[d] - 1;    // a forward consumer exists
  bool down = off[d] > 0;           // a backward consumer exists
  if (!up && !down) return;
  double A[25];
  calc_jm(B, n, 3 * d + 1, cc.gamma, A);
  const int radf[3] = {F_RA, F_RB, F_RC};
  double rad = B.s(radf[d], n);
  double invj = B.s(F_INVJ, n);
  if (up) {
    int q[3] = {a, b, c};
    q[d] += 1;
    double* dst = B.rec_f + kRec * plane_pos(B, q[0], q[1], q[2]) + 25 * d;
#pragma unroll
    for (int x = 0; x < 25; ++x) {
      double v = (x % 6 == 0) ? A[x] + rad : A[x];
      dst[x] = 0.5 * v * invj;
    }
  }
  if (down) {
    int q[3] = {a, b, c};
    q[d] -= 1;
    double* dst = B.rec_b + kRec * plane_pos(B, q[0], q[1], q[2]) + 25 * d;
#pragma unroll
    for (int x = 0; x < 25; ++x) {
      double v = (x % 6 == 0) ? A[x] - rad : A[x];
      dst[x] = 0.5 * v * invj;
    }
  }
}

// ---------------------------------------------------------------- sweeps
namespace {

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bulk (non-tensor) copy global -> this CTA's shared memory, completion counted
// on `bar`.  Both addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// Offsets (a,b,c) of node t of hyperplane h, and the index of offsets (b,c)
// of plane h inside that plane (c ascending, then b) - the order of plane_pos.
__device__ __forceinline__ void plane_abc(int h, int t, int nx1, int ny1, int& a, int& b, int& c) {
  c = max(0, h - (nx1 - 1) - (ny1 - 1));
  for (;; ++c) {
    int r = h - c;
    int bmin = max(0, r - (nx1 - 1)), bmax = min(ny1 - 1, r);
    int cnt = bmax - bmin + 1;
    if (t < cnt) {
      b = bmin + t;
      a = r - b;
      return;
    }
    t -= cnt;
  }
}
__device__ __forceinline__ int within(int h, int b, int c, int nx1, int ny1) {
  int w = 0;
  for (int cc = max(0, h - (nx1 - 1) - (ny1 - 1)); cc < c; ++cc) {
    int r = h - cc;
    int bmin = max(0, r - (nx1 - 1)), bmax = min(ny1 - 1, r);
    if (bmax >= bmin) w += bmax - bmin + 1;
  }
  return w + (b - max(0, (h - c) - (nx1 - 1)));
}

__device__ __forceinline__ double row_dot(const double* m, const double* x) {
  double s = m[0] * x[0];
  s = s + m[1] * x[1];
  s = s + m[2] * x[2];
  s = s + m[3] * x[3];
  s = s + m[4] * x[4];
  return s;
}

constexpr long kSpinLimit = 1L << 20;  // bounded mbarrier wait (well under a second)

}  // namespace

// Forward and backward hyperplane sweeps for one block per CTA.  Thread t of a
// plane handles equation row t%5 of node t/5: the row of the three neighbour
// blocks times the neighbours' dq, summed in the reference's order
// (sub_timeadvancement_1stimplicit.f90:346-364, :522-540).  The previous
// plane's results sit in shared memory.
//
// With STAGED, the records of the next NST planes (contiguous in the
// hyperplane-major layout) are brought into shared memory by bulk copies
// issued by one thread and tracked by mbarriers, so a plane's loads are never
// on the critical path.  Without it (planes too large for shared memory) the
// records are read from global memory.  Waits are bounded: on a timeout the
// kernel raises ST_TIMEOUT in `status` and stops.
template <bool STAGED>
__device__ __forceinline__ void lusgs_sweep(const BlockView* __restrict__ blocks, int nst, unsigned* status) {
  const BlockView& B = blocks[blockIdx.x];
  extern __shared__ __align__(16) unsigned char smem[];
  const int P = B.pmax;
  const int H = B.nplanes;
  const int nx1 = B.b1.nx(), ny1 = B.b1.ny();
  const long* poff = B.poff;
  // shared layout: ring (2 planes x 5*P) | stages (nst x P*(kRec + 8 + 8)) | mbarriers
  double* ring = (double*)smem;
  double* stage0 = ring + 10 * P;
  const int sdoubles = P * (kRec + 16);
  unsigned long long* bars = (unsigned long long*)(stage0 + (STAGED ? nst * sdoubles : 0));
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    abort_flag = 0;
    if (STAGED) {
      for (int x = 0; x < nst; ++x) mbar_init(&bars[x], 1);
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
  }
  __syncthreads();
  // Steps gs = 0 .. 2H-1 run the forward planes then the backward planes; step
  // gs uses stage gs % nst, whose mbarrier completes once per use, so the
  // phase to wait for has parity (gs / nst) & 1.
  for (int pass = 0; pass < 2; ++pass) {
    const bool fwd = pass == 0;
    const double* rec_g = fwd ? B.rec_f : B.rec_b;
    auto plane_of = [&](int st) { return fwd ? st : H - 1 - st; };
    auto issue = [&](int st) {  // copies of step st of this pass
      int gs = pass * H + st;
      int h = plane_of(st);
      long base = poff[h];
      unsigned cnt = (unsigned)(poff[h + 1] - base);
      double* stg = stage0 + (gs % nst) * sdoubles;
      unsigned long long* bar = &bars[gs % nst];
      mbar_expect_tx(bar, cnt * (kRec + 8 + (fwd ? 0 : 8)) * 8u);
      bulk_g2s(stg, rec_g + kRec * base, cnt * kRec * 8u, bar);
      bulk_g2s(stg + P * kRec, B.sca + 8 * base, cnt * 64u, bar);
      if (!fwd) bulk_g2s(stg + P * (kRec + 8), B.dqs + 8 * base, cnt * 64u, bar);
    };
    if (STAGED && threadIdx.x == 0) {
      // the generic reads of the stage buffers are ordered before the
      // async-proxy writes into them (the dq* stores of the forward pass are
      // fenced for the async proxy by every thread at the end of that pass)
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      for (int st = 0; st < nst && st < H; ++st) issue(st);
    }
    for (int st = 0; st < H; ++st) {
      int gs = pass * H + st;
      int h = plane_of(st);
      long base = poff[h];
      int cnt = (int)(poff[h + 1] - base);
      int hn = fwd ? h - 1 : h + 1;  // plane holding the neighbours
      double* prev = ring + 5 * P * ((st + 1) & 1);
      double* cur = ring + 5 * P * (st & 1);
      const double* stg = stage0 + (gs % nst) * sdoubles;
      if (STAGED) {
        unsigned parity = (unsigned)((gs / nst) & 1);
        long spins = 0;
        while (!mbar_try_wait(&bars[gs % nst], parity)) {
          if (++spins > kSpinLimit) {
            abort_flag = 1;
            break;
          }
        }
      }
      for (int t = threadIdx.x; t < 5 * cnt && !abort_flag; t += blockDim.x) {
        int node = t / 5, row = t - 5 * node;
        int a, b, c;
        plane_abc(h, node, nx1, ny1, a, b, c);
        const double* rec = STAGED ? stg + kRec * node : rec_g + kRec * (base + node);
        const double* sc = STAGED ? stg + P * kRec + 8 * node : B.sca + 8 * (base + node);
        const int off[3] = {a, b, c};
        const int lim[3] = {nx1, ny1, B.b1.nz()};
        double acc[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          bool has = fwd ? off[d] > 0 : off[d] < lim[d] - 1;
          if (!has) {
            acc[d] = 0.0;
          } else {
            int sgn = fwd ? -1 : 1;
            int nb = d == 1 ? b + sgn : b;
            int nc = d == 2 ? c + sgn : c;
            int w = within(hn, nb, nc, nx1, ny1);
            acc[d] = row_dot(rec + 25 * d + 5 * row, prev + 5 * w);
          }
        }
        double v;
        if (fwd) {
          v = (sc[row] + (acc[0] + acc[1] + acc[2])) / sc[5] / sc[6];
          B.dqs[8 * (base + node) + row] = v;
        } else {
          double ds = STAGED ? stg[P * (kRec + 8) + 8 * node + row] : B.dqs[8 * (base + node) + row];
          v = ds - (acc[0] + acc[1] + acc[2]) / sc[6] / sc[5];
          B.dq[5 * (base + node) + row] = v;
        }
        cur[t] = v;
      }
      __syncthreads();
      if (abort_flag) {
        if (threadIdx.x == 0 && status) atomicOr(status, (unsigned)ST_TIMEOUT);
        return;
      }
      if (STAGED && threadIdx.x == 0 && st + nst < H) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue(st + nst);
      }
    }
    // every thread orders its dq* stores before the backward bulk copies read them
    if (STAGED && fwd) asm volatile("fence.proxy.async.global;" ::: "memory");
    __syncthreads();
  }
}

__global__ void k_lusgs_sweep_staged(const BlockView* __restrict__ blocks, int nst, unsigned* status) {
  lusgs_sweep<true>(blocks, nst, status);
}
__global__ void k_lusgs_sweep_global(const BlockView* __restrict__ blocks, int nst, unsigned* status) {
  lusgs_sweep<false>(blocks, 1, status);
}

// q = q + dq on every updated node (sub_timeadvancement_1stimplicit.f90:568-574).
__global__ void k_lusgs_update(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  long pos = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= B.b1.size()) return;
  long n = B.nat[pos];
#pragma unroll
  for (int x = 1; x <= 5; ++x) B.v(F_Q, x, n) = B.v(F_Q, x, n) + B.dq[5 * pos + x - 1];
}

}  // namespace aero
