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

// sub_timeadvancement_1stimplicit.f90:108-156, first half: the spectral
// radii ra, rb, rc on the updated box grown by one (2-D: in i and j only).  They need only the
// primitives and the metrics, so they (and the off-diagonal blocks made from
// them) can be formed while the fluxes and the time step are computed.
__global__ void k_lusgs_radii(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const Box e = grown_box(B);
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= e.size()) return;
  int i = e.is + (int)(t % e.nx());
  long r = t / e.nx();
  int j = e.js + (int)(r % e.ny());
  int k = e.ks + (int)(r / e.ny());
  long n = B.at(i, j, k);
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
}

// sub_timeadvancement_1stimplicit.f90:72-156, second half: rhs = rhsi + rhsv
// on the updated nodes and diag = phi/dt + ra + rb + rc on the grown box
// (phi = 0 if cfl >= 1000), from the radii k_lusgs_radii stored.
__global__ void k_lusgs_prep(const BlockView* __restrict__ blocks, CaseConsts cc_launch) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
  const Box& b1 = B.b1;
  const Box e = grown_box(B);
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
  if (B.planar())  // 2-D (:157-210): no zeta radius
    B.s(F_DIAG, n) = phi * 1.0 / B.s(F_DT, n) + B.s(F_RA, n) + B.s(F_RB, n);
  else
    B.s(F_DIAG, n) = phi * 1.0 / B.s(F_DT, n) + B.s(F_RA, n) + B.s(F_RB, n) + B.s(F_RC, n);
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
  B.pidx[u] = (int)pos;
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    int lo[3] = {a, b, c}, hi[3] = {a, b, c};
    lo[e] -= 1;
    hi[e] += 1;
    B.nbr[6 * pos + e] = off[e] > 0 ? (int)plane_pos(B, lo[0], lo[1], lo[2]) : -1;
    B.nbr[6 * pos + 3 + e] = off[e] < lim[e] - 1 ? (int)plane_pos(B, hi[0], hi[1], hi[2]) : -1;
  }
}

// Plane-local record layout of the sweeps.  The records of hyperplane h
// (cnt = poff[h+1]-poff[h] nodes) form one contiguous chunk starting at
// kRec*poff[h] (rec_f, rec_b) or 8*poff[h] (sca, dqs); element x of the node
// with plane-local index t sits at x*cnt + t, so the threads of a warp, which
// take consecutive t, read consecutive words.
//   rec_f/rec_b x = 25*d + 5*row + col : block of neighbour direction d
//               x = 75                 : neighbours' plane-local indices, packed
//   sca         x = 0..4 rhs, 5 diag, 6 inv_j, 7 1/diag, 8 1/inv_j (kSca per node)
//   dqs         x = 0..4 dq* (forward result)
__device__ __forceinline__ long rec_at(const BlockView& B, long pos, int h, int stride, int x) {
  long base = B.poff[h];
  long cnt = B.poff[h + 1] - base;
  return stride * base + x * cnt + (pos - base);
}

// Record formats: the 5x5 blocks in FP64 (76 words per node: 75 entries and
// the packed neighbours at 75*cnt) or, in mixed precision, in FP32 (80
// floats per node: 75 entries, the packed neighbours as one 64-bit word at
// float offset 76*cnt, 3 unused), so a plane's chunk stays a multiple of 16
// bytes for the bulk copies.  Products and sums are FP64 either way.
template <typename R>
struct RecFmt;
template <>
struct RecFmt<double> {
  static constexpr int kWords = kRec;
  __device__ static double packed(const double* chunk, int cnt, int t) { return chunk[75 * cnt + t]; }
  __device__ static const double* packed_ptr(const double* chunk, int cnt) { return chunk + 75 * cnt; }
  __device__ static void set_packed(double* chunk, int cnt, long t, double v) { chunk[75 * cnt + t] = v; }
};
template <>
struct RecFmt<float> {
  static constexpr int kWords = 80;
  __device__ static double packed(const float* chunk, int cnt, int t) {
    return reinterpret_cast<const double*>(chunk + 76 * cnt)[t];
  }
  __device__ static const double* packed_ptr(const float* chunk, int cnt) {
    return reinterpret_cast<const double*>(chunk + 76 * cnt);
  }
  __device__ static void set_packed(float* chunk, int cnt, long t, double v) {
    reinterpret_cast<double*>(chunk + 76 * cnt)[t] = v;
  }
};
template <typename R>
__device__ __forceinline__ R* recs(const BlockView& B, bool fwd) {
  return reinterpret_cast<R*>(fwd ? B.rec_f : B.rec_b);
}

// The off-diagonal blocks of both sweeps, off the critical path.  For every
// updated node (the provider) and direction d: A = calc_jm at the provider,
// S+ = 0.5*(A + r*I)*inv_j goes to the forward record of the node one step up
// in d, S- = 0.5*(A - r*I)*inv_j to the backward record of the node one step
// down (sub_timeadvancement_1stimplicit.f90:283-301, :459-477, same
// operations).  They need q, the metrics, inv_j and the radii only, so they
// are formed beside the flux and time-step kernels.  R is the record format.
template <typename R>
__device__ __forceinline__ void lusgs_mats_body(const BlockView* __restrict__ blocks, CaseConsts cc) {
  constexpr int W = RecFmt<R>::kWords;
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const Box& b1 = B.b1;
  // thread t: direction d = t / N1 and provider position p = t % N1 in the
  // hyperplane-major order, so a warp's record stores go to consecutive
  // plane-local slots of one consumer plane
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long N1 = b1.size();
  if (t >= 3 * N1) return;
  int d = (int)(t / N1);
  long p = t - d * N1;
  long n = B.nat[p];
  long r = n / B.nx;
  int i = B.b.is + (int)(n - r * B.nx);
  int j = B.b.js + (int)(r % B.ny);
  int k = B.b.ks + (int)(r / B.ny);
  const int h = (i - b1.is) + (j - b1.js) + (k - b1.ks);
  const int* nb = B.nbr + 6 * p;
  const int up = nb[3 + d];    // forward consumer: the neighbour one step up in d
  const int down = nb[d];      // backward consumer: one step down
  if (up < 0 && down < 0) return;
  // calc_jm's common terms (sub_timeadvancement_jac.f90:17-62); every entry is
  // then formed, and written to both records, one at a time, which keeps few
  // values live
  const int cb = 3 * d + 1;
  const double gamma = cc.gamma;
  const double rho = B.v(F_Q, 1, n), mu0 = B.v(F_Q, 2, n), mv0 = B.v(F_Q, 3, n);
  const double mw0 = B.v(F_Q, 4, n), e0 = B.v(F_Q, 5, n);
  const double dxidx = B.v(F_DXIDX, cb, n), dxidy = B.v(F_DXIDX, cb + 1, n), dxidz = B.v(F_DXIDX, cb + 2, n);
  const double a2 = gamma - 1.0, a3 = gamma - 2.0;
  // every division by rho through its reciprocal (div_rn_lean: the same bits)
  const double rrho = 1.0 / rho;
  auto dv = [&](double x) { return div_rn_lean(x, rho, rrho); };
  const double uu = dv(dxidx * mu0 + dxidy * mv0 + dxidz * mw0);
  const double phi = 0.5 * a2 * (p2(mu0) + p2(mv0) + p2(mw0)) / p2(rho);
  const double a1 = dv(gamma * e0) - phi;
  const double rad = B.s(d == 0 ? F_RA : (d == 1 ? F_RB : F_RC), n);
  const double invj = B.s(F_INVJ, n);
  R* dup = nullptr;
  R* ddn = nullptr;
  long cup = 0, cdn = 0;
  if (up >= 0) {
    long base = B.poff[h + 1];
    cup = B.poff[h + 2] - base;
    dup = recs<R>(B, true) + W * base + 25 * d * cup + (up - base);
  }
  if (down >= 0) {
    long base = B.poff[h - 1];
    cdn = B.poff[h] - base;
    ddn = recs<R>(B, false) + W * base + 25 * d * cdn + (down - base);
  }
#pragma unroll
  for (int x = 0; x < 25; ++x) {
    double a;  // calc_jm's a(x/5+1, x%5+1), the same operations
    switch (x) {
      case 0: a = 0.0; break;
      case 1: a = dxidx; break;
      case 2: a = dxidy; break;
      case 3: a = dxidz; break;
      case 4: a = 0.0; break;
      case 5: a = phi * dxidx - dv(uu * mu0); break;
      case 6: a = uu - dv(a3 * dxidx * mu0); break;
      case 7: a = dv(dxidy * mu0) - dv(a2 * dxidx * mv0); break;
      case 8: a = dv(dxidz * mu0) - dv(a2 * dxidx * mw0); break;
      case 9: a = a2 * dxidx; break;
      case 10: a = phi * dxidy - dv(uu * mv0); break;
      case 11: a = dv(dxidx * mv0) - dv(a2 * dxidy * mu0); break;
      case 12: a = uu - dv(a3 * dxidy * mv0); break;
      case 13: a = dv(dxidz * mv0) - dv(a2 * dxidy * mw0); break;
      case 14: a = a2 * dxidy; break;
      case 15: a = phi * dxidz - dv(uu * mw0); break;
      case 16: a = dv(dxidx * mw0) - dv(a2 * dxidz * mu0); break;
      case 17: a = dv(dxidy * mw0) - dv(a2 * dxidz * mv0); break;
      case 18: a = uu - dv(a3 * dxidz * mw0); break;
      case 19: a = a2 * dxidz; break;
      case 20: a = (phi - a1) * uu; break;
      case 21: a = a1 * dxidx - dv(a2 * uu * mu0); break;
      case 22: a = a1 * dxidy - dv(a2 * uu * mv0); break;
      case 23: a = a1 * dxidz - dv(a2 * uu * mw0); break;
      default: a = gamma * uu; break;
    }
    if (dup) {
      double v = (x % 6 == 0) ? a + rad : a;
      dup[x * cup] = (R)(0.5 * v * invj);
    }
    if (ddn) {
      double v = (x % 6 == 0) ? a - rad : a;
      ddn[x * cdn] = (R)(0.5 * v * invj);
    }
  }
}
__global__ void __launch_bounds__(256, 4) k_lusgs_mats(const BlockView* __restrict__ blocks, CaseConsts cc) {
  lusgs_mats_body<double>(blocks, cc);
}
__global__ void __launch_bounds__(256, 4) k_lusgs_mats_f32(const BlockView* __restrict__ blocks, CaseConsts cc) {
  lusgs_mats_body<float>(blocks, cc);
}

// The per-node part of the sweep records, once rhs and diag are known: rhs,
// diag, inv_j and their reciprocals in the plane-local scalar layout, and the
// packed positions of each node's forward and backward neighbours (with the
// flag that sends its divisions to the IEEE path), one thread per updated
// node in hyperplane-major order.  R is the record format.
template <typename R>
__device__ __forceinline__ void lusgs_sca_body(const BlockView* __restrict__ blocks) {
  constexpr int W = RecFmt<R>::kWords;
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const Box& b1 = B.b1;
  long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= b1.size()) return;
  long n = B.nat[p];
  long r = n / B.nx;
  int i = B.b.is + (int)(n - r * B.nx);
  int j = B.b.js + (int)(r % B.ny);
  int k = B.b.ks + (int)(r / B.ny);
  const int h = (i - b1.is) + (j - b1.js) + (k - b1.ks);
  const int* nb = B.nbr + 6 * p;
  long base = B.poff[h], cnt = B.poff[h + 1] - base, lt = p - base;
  double* sc = B.sca + kSca * base + lt;
#pragma unroll
  for (int x = 0; x < 5; ++x) sc[x * cnt] = B.v(F_RHS, x + 1, n);
  double diag = B.s(F_DIAG, n), invj = B.s(F_INVJ, n);
  sc[5 * cnt] = diag;
  sc[6 * cnt] = invj;
  sc[7 * cnt] = 1.0 / diag;
  sc[8 * cnt] = 1.0 / invj;
  const bool slow = !divisors_ok(diag, invj);
  RecFmt<R>::set_packed(recs<R>(B, true) + W * base, (int)cnt, lt, pack_nbrs(nb, h > 0 ? B.poff[h - 1] : 0, slow));
  RecFmt<R>::set_packed(recs<R>(B, false) + W * base, (int)cnt, lt,
                        pack_nbrs(nb + 3, h + 1 < B.nplanes ? B.poff[h + 1] : 0, slow));
}
__global__ void k_lusgs_sca(const BlockView* __restrict__ blocks) { lusgs_sca_body<double>(blocks); }
__global__ void k_lusgs_sca_f32(const BlockView* __restrict__ blocks) { lusgs_sca_body<float>(blocks); }

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
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
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
// Bulk prefetch of global memory into L2 (no completion to track); both the
// address and the size are multiples of 16 bytes.
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}
// Row t / cnt of item t < 5*cnt of a plane, by comparisons (no division).
__device__ __forceinline__ int row_of(int t, int cnt) {
  return (t >= cnt) + (t >= 2 * cnt) + (t >= 3 * cnt) + (t >= 4 * cnt);
}

template <typename R>
__device__ __forceinline__ double row_dot5(const R* m, int mst, const double* x, int xst) {
  double s = (double)m[0] * x[0];
  s = s + (double)m[mst] * x[xst];
  s = s + (double)m[2 * mst] * x[2 * xst];
  s = s + (double)m[3 * mst] * x[3 * xst];
  s = s + (double)m[4 * mst] * x[4 * xst];
  return s;
}

// Poll budget of the staged sweep's mbarrier waits (well under a second).  It
// takes its budget as an argument (aero_set_poll_budget; this is the default
// and the largest), except for the producer's final wait for its own copies
// in flight, which always has the full budget so that no copy lands after the
// CTA has left.  The cluster sweeps bound their waits by time (wait_bounded).
constexpr long kSpinLimit = 1L << 20;

// Rows r0 .. r0+nr-1 (nr <= 3) of plane-local node `t` of one plane of the
// sweep: each row of the three neighbour blocks times the neighbours' dq,
// summed in the reference's order (sub_timeadvancement_1stimplicit.f90:346-364,
// :522-540); the two divisions are exact (div_rn with the stored
// reciprocals).  rec/sca/dsv point at the plane's chunks (element stride
// cnt); prev holds the previous plane's dq, component c of node w at
// prev[c*pst + w*wst].
template <bool FWD, typename R>
__device__ __forceinline__ void lusgs_rows(const R* rec, const double* sca, const double* dsv, int cnt,
                                           int t, int r0, int nr, const double* prev, long pst, int wst,
                                           double out[3]) {
  double packed = RecFmt<R>::packed(rec, cnt, t);
  double x[3][5];
  bool has[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int w = nbr_local(packed, d);
    has[d] = w >= 0;
#pragma unroll
    for (int c = 0; c < 5; ++c) x[d][c] = has[d] ? prev[c * pst + (long)w * wst] : 0.0;
  }
  const double diag = sca[5 * cnt + t], invj = sca[6 * cnt + t];
  const double rdiag = sca[7 * cnt + t], rinvj = sca[8 * cnt + t];
  const bool bok = !nbr_slow_div(packed);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (k < nr) {
      int row = r0 + k;
      double acc[3];
#pragma unroll
      for (int d = 0; d < 3; ++d)
        acc[d] = has[d] ? row_dot5(rec + (25 * d + 5 * row) * cnt + t, cnt, x[d], 1) : 0.0;
      if (FWD)
        out[k] = div2_rn(sca[row * cnt + t] + (acc[0] + acc[1] + acc[2]), diag, rdiag, invj, rinvj, bok);
      else
        out[k] = dsv[row * cnt + t] - div2_rn(acc[0] + acc[1] + acc[2], invj, rinvj, diag, rdiag, bok);
    }
  }
}

}  // namespace

// Forward and backward hyperplane sweeps of one block per CTA with the plane
// records staged in shared memory.  Warps 0..C/32-1 are consumers: thread
// (row, t) computes equation `row` of node t of every plane; the previous
// plane's dq sits in a two-plane ring in shared memory.  The last warp is the
// producer: it brings the records of the next planes into nst stages with bulk
// copies, each stage guarded by a `full` mbarrier (copies landed) and an
// `empty` mbarrier (every consumer warp done with it).  The backward pass also
// needs dq* of the forward pass, which the consumers publish with a proxy
// fence and the `fwd_done` mbarrier.  Every wait is bounded: a consumer that
// gives up makes all consumers stop at the next plane barrier and raise
// ST_TIMEOUT; the producer then waits (bounded) for its copies in flight.
template <typename R>
__device__ __forceinline__ void lusgs_staged_body(const BlockView* __restrict__ blocks, int nst, unsigned* status,
                                                  long spin_limit, int stall_plane) {
  constexpr int RD = RecFmt<R>::kWords * (int)sizeof(R) / 8;  // record words per node, in doubles
  const BlockView& B = blocks[blockIdx.x];
  if (B.retired()) return;
  extern __shared__ __align__(16) unsigned char smem[];
  const int P = B.pmax;
  const int H = B.nplanes;
  const int C = blockDim.x - 32;  // consumer threads
  // shared layout: plane offsets (H+1, padded to 16 B) | ring (2 planes x 5*P)
  // | nst stages (P*(RD+kSca+8) doubles: records, scalars, dq*) | mbarriers
  long* poff = (long*)smem;
  double* ring = (double*)(poff + ((H + 2) & ~1));
  double* stage0 = ring + 10 * P;
  const int sdoubles = P * (RD + kSca + 8);
  unsigned long long* full = (unsigned long long*)(stage0 + nst * sdoubles);
  unsigned long long* empty = full + nst;
  unsigned long long* fwd_done = empty + nst;
  __shared__ volatile int abort_flag;     // read by the producer
  __shared__ volatile int abort_slot[2];  // consumers: slot k&1 is set before barrier k, read after it
  for (int x = threadIdx.x; x <= H; x += blockDim.x) poff[x] = B.poff[x];
  if (threadIdx.x == 0) {
    abort_flag = 0;
    abort_slot[0] = 0;
    abort_slot[1] = 0;
    for (int x = 0; x < nst; ++x) {
      mbar_init(&full[x], 1);
      mbar_init(&empty[x], C / 32);
    }
    mbar_init(fwd_done, C / 32);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  if (threadIdx.x >= C) {  // ------------------------------------ producer
    if (threadIdx.x != C) return;
    auto stage_of = [&](int gs) { return stage0 + (gs % nst) * sdoubles; };
    auto wait_bar = [&](unsigned long long* bar, unsigned parity) {
      long spins = 0;
      while (!mbar_try_wait(bar, parity)) {
        if (abort_flag || ++spins > spin_limit) return false;
      }
      return true;
    };
    bool ok = true;
    int issued = 0;  // steps whose copies were issued
    // issue the copies of global step gs (forward: gs < H); with_dqs = false
    // leaves the backward dq* copy for later
    auto issue = [&](int gs, bool with_dqs) {
      // fault injection: the copies of this forward plane are never issued,
      // so the consumers' waits for it run out (the producer drains what it
      // did issue and leaves)
      if (gs == stall_plane) return false;
      bool fwd = gs < H;
      int h = fwd ? gs : 2 * H - 1 - gs;
      long base = poff[h];
      unsigned cnt = (unsigned)(poff[h + 1] - base);
      double* stg = stage_of(gs);
      unsigned long long* bar = &full[gs % nst];
      if (gs >= nst && !wait_bar(&empty[gs % nst], (unsigned)((gs / nst - 1) & 1))) return false;
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_expect_tx(bar, cnt * (RD + kSca + (fwd ? 0 : 8)) * 8u);
      bulk_g2s(stg, recs<R>(B, fwd) + RecFmt<R>::kWords * base, cnt * RD * 8u, bar);
      bulk_g2s(stg + P * RD, B.sca + kSca * base, cnt * kSca * 8u, bar);
      if (!fwd && with_dqs) bulk_g2s(stg + P * (RD + kSca), B.dqs + 8 * base, cnt * 64u, bar);
      ++issued;
      return true;
    };
    auto issue_dqs = [&](int gs) {
      int h = 2 * H - 1 - gs;
      long base = poff[h];
      unsigned cnt = (unsigned)(poff[h + 1] - base);
      bulk_g2s(stage_of(gs) + P * (RD + kSca), B.dqs + 8 * base, cnt * 64u, &full[gs % nst]);
    };
    for (int gs = 0; gs < H && ok; ++gs) ok = issue(gs, true);
    int head = nst < H ? nst : H;
    for (int x = 0; x < head && ok; ++x) ok = issue(H + x, false);
    if (ok) ok = wait_bar(fwd_done, 0u);
    if (ok) {
      asm volatile("fence.proxy.async.global;" ::: "memory");
      for (int x = 0; x < head; ++x) issue_dqs(H + x);
    }
    for (int gs = H + head; gs < 2 * H && ok; ++gs) ok = issue(gs, true);
    if (!ok) {
      // drain: wait (bounded) for the copies of the last issued stages
      for (int gs = issued > nst ? issued - nst : 0; gs < issued; ++gs) {
        long spins = 0;
        while (!mbar_try_wait(&full[gs % nst], (unsigned)((gs / nst) & 1)) && ++spins < kSpinLimit) {
        }
      }
    }
    return;
  }

  // ------------------------------------------------------------ consumers
  // Thread t < 5*cnt of a plane computes row t / cnt of node t % cnt (a warp
  // mostly covers consecutive nodes of one row, so its shared-memory reads
  // are consecutive words); warps beyond 5*cnt only take the barrier.  The
  // ring holds the previous plane's dq node-major (5 per node).  The plane's
  // offsets, the wait for its copies, the row mapping, the neighbour
  // positions, rhs or dq*, diagonal and J^-1 are loaded into registers before
  // the barrier that ends the previous plane; the thread's 15 block entries
  // are read from the stage after it (holding them across the barrier costs
  // more registers than it saves).
  const int lane = threadIdx.x & 31;
  double* const g_dqs = B.dqs;
  double* const g_dq = B.dq;
  const double* prev = ring + 5 * P;
  double* cur = ring;
  struct PlaneRegs {
    long base;
    int cnt, row, node;
    bool act, timeout;
    int w[3];
    double rhs, diag, invj, rdiag, rinvj;  // rhs: rhs (forward) or dq* (backward)
    bool bok;                              // divisors in div2_rn's fast range
  };
  auto preload = [&](int gs, int ls, unsigned lph, PlaneRegs& q) {
    const bool fwd = gs < H;
    const int h = fwd ? gs : 2 * H - 1 - gs;
    q.base = poff[h];
    q.cnt = (int)(poff[h + 1] - q.base);
    q.timeout = false;
    long spins = 0;
    while (!mbar_try_wait(&full[ls], lph)) {
      if (++spins > spin_limit) {
        q.timeout = true;
        note_timeout(status, TS_STAGED, (int)blockIdx.x, 0, gs, TW_PLANE);
        break;
      }
    }
    const int t = threadIdx.x;
    q.act = !q.timeout && t < 5 * q.cnt;
    if (!q.act) return;
    const int cnt = q.cnt;
    const int row = row_of(t, cnt);
    const int node = t - row * cnt;
    q.row = row;
    q.node = node;
    const double* stg = stage0 + ls * sdoubles;
    const double* sca = stg + P * RD + node;
    const double packed = RecFmt<R>::packed(reinterpret_cast<const R*>(stg), cnt, node);
#pragma unroll
    for (int d = 0; d < 3; ++d) q.w[d] = nbr_local(packed, d);
    q.rhs = fwd ? sca[row * cnt] : stg[P * (RD + kSca) + row * cnt + node];
    q.diag = sca[5 * cnt];
    q.invj = sca[6 * cnt];
    q.rdiag = sca[7 * cnt];
    q.rinvj = sca[8 * cnt];
    q.bok = !nbr_slow_div(packed);
  };
  PlaneRegs q;
  int ls = 0;  // stage of the current step and its phase parity
  unsigned lph = 0;
  // barrier k (k = 0 before plane 0, k = gs+1 after plane gs) follows the
  // preload of plane k; a thread whose wait gave up sets slot k&1 before it,
  // and every consumer reads that slot after it.  A thread one plane ahead
  // can only write the other slot, so all consumers take the same decision.
  auto give_up = [&](int k) {
    abort_slot[k & 1] = 1;
    abort_flag = 1;
  };
  preload(0, 0, 0u, q);
  if (q.timeout) give_up(0);
  asm volatile("bar.sync 1, %0;" ::"r"(C) : "memory");
  for (int gs = 0; gs < 2 * H; ++gs) {
    if (abort_slot[gs & 1]) {
      if (threadIdx.x == 0) {
        if (status) atomicOr(status, (unsigned)ST_TIMEOUT);
        B.raise(ST_TIMEOUT);
      }
      return;
    }
    const bool fwd = gs < H;
    if (q.act) {
      const R* rec = reinterpret_cast<const R*>(stage0 + ls * sdoubles) + q.node;
      double acc[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        double sd = 0.0;
        if (q.w[d] >= 0) {
          const double* x = prev + 5 * q.w[d];
          const R* mr = rec + (25 * d + 5 * q.row) * q.cnt;
          sd = (double)mr[0] * x[0];
          sd = sd + (double)mr[q.cnt] * x[1];
          sd = sd + (double)mr[2 * q.cnt] * x[2];
          sd = sd + (double)mr[3 * q.cnt] * x[3];
          sd = sd + (double)mr[4 * q.cnt] * x[4];
        }
        acc[d] = sd;
      }
      double v;
      if (fwd) {
        v = div2_rn(q.rhs + (acc[0] + acc[1] + acc[2]), q.diag, q.rdiag, q.invj, q.rinvj, q.bok);
        g_dqs[8 * q.base + q.row * q.cnt + q.node] = v;
      } else {
        v = q.rhs - div2_rn(acc[0] + acc[1] + acc[2], q.invj, q.rinvj, q.diag, q.rdiag, q.bok);
        g_dq[5 * (q.base + q.node) + q.row] = v;
      }
      cur[5 * q.node + q.row] = v;
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[ls]);
    if (gs == H - 1) {
      // every thread orders its dq* stores before the backward bulk copies
      // read them; the producer waits for all consumer warps (before any
      // consumer waits for a backward stage, whose dq* copy needs this)
      asm volatile("fence.proxy.async.global;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(fwd_done);
    }
    if (++ls == nst) {
      ls = 0;
      lph ^= 1u;
    }
    if (gs + 1 < 2 * H) {
      preload(gs + 1, ls, lph, q);
      if (q.timeout) give_up(gs + 1);
    }
    // the barrier orders this plane's ring writes before the next plane's
    // reads, and a timeout flag before every consumer's check
    asm volatile("bar.sync 1, %0;" ::"r"(C) : "memory");
    // the first plane of each pass has no neighbours in the previous one, so
    // the ring needs no reset between passes
    const double* tmp = prev;
    prev = cur;
    cur = (double*)tmp;
  }
}

// 64 registers per thread at most, so that one CTA can hold the 5 rows of
// every node of planes up to 198 nodes (1024 threads).
__global__ void __launch_bounds__(1024, 1)
    k_lusgs_sweep_staged(const BlockView* __restrict__ blocks, int nst, unsigned* status, long spin_limit,
                         int stall_plane) {
  lusgs_staged_body<double>(blocks, nst, status, spin_limit, stall_plane);
}
__global__ void __launch_bounds__(1024, 1)
    k_lusgs_sweep_staged_f32(const BlockView* __restrict__ blocks, int nst, unsigned* status, long spin_limit,
                             int stall_plane) {
  lusgs_staged_body<float>(blocks, nst, status, spin_limit, stall_plane);
}

// The same sweeps with the records read from global memory, for blocks whose
// planes do not fit the shared-memory stages; the previous plane's dq is read
// back from dqs / dq (written before the last __syncthreads).  Thread 0 keeps
// the records of the next kAhead planes on their way into L2 with bulk
// prefetches.
template <typename R>
__device__ __forceinline__ void lusgs_global_body(const BlockView* __restrict__ blocks) {
  constexpr int W = RecFmt<R>::kWords;
  const BlockView& B = blocks[blockIdx.x];
  if (B.retired()) return;
  const int H = B.nplanes;
  const long* poff = B.poff;
  constexpr int kAhead = 3;  // planes prefetched into L2 ahead of the sweep
  // records, scalars (and, backward, dq*) of step st of a pass into L2
  auto prefetch = [&](bool fwd, int st) {
    if (st >= H) return;
    int h = fwd ? st : H - 1 - st;
    long b = poff[h];
    unsigned cnt = (unsigned)(poff[h + 1] - b);
    bulk_prefetch_l2(recs<R>(B, fwd) + W * b, cnt * (unsigned)(W * sizeof(R)));
    bulk_prefetch_l2(B.sca + kSca * b, cnt * kSca * 8u);
    if (!fwd) bulk_prefetch_l2(B.dqs + 8 * b, cnt * 64u);
  };
  for (int pass = 0; pass < 2; ++pass) {
    const bool fwd = pass == 0;
    if (threadIdx.x == 0)
      for (int x = 0; x < kAhead; ++x) prefetch(fwd, x);
    for (int st = 0; st < H; ++st) {
      int h = fwd ? st : H - 1 - st;
      long base = poff[h];
      int cnt = (int)(poff[h + 1] - base);
      if (threadIdx.x == 0) prefetch(fwd, st + kAhead);
      const R* rec = recs<R>(B, fwd) + W * base;
      const double* sca = B.sca + kSca * base;
      const double* dsv = B.dqs + 8 * base;
      // previous plane: forward dq* (plane-local chunk, component stride = its
      // node count), backward dq (node-major, 5 per node)
      const double* prev = sca;
      long pst = 0;
      int wst = 0;
      if (fwd && h > 0) {
        prev = B.dqs + 8 * poff[h - 1];
        pst = poff[h] - poff[h - 1];
        wst = 1;
      } else if (!fwd && h + 1 < H) {
        prev = B.dq + 5 * poff[h + 1];
        pst = 1;
        wst = 5;
      }
      for (int t = threadIdx.x; t < 2 * cnt; t += blockDim.x) {
        int half = t >= cnt;
        int node = t - half * cnt;
        int r0 = half ? 3 : 0, nr = half ? 2 : 3;
        double v[3];
        if (fwd)
          lusgs_rows<true, R>(rec, sca, dsv, cnt, node, r0, nr, prev, pst, wst, v);
        else
          lusgs_rows<false, R>(rec, sca, dsv, cnt, node, r0, nr, prev, pst, wst, v);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          if (k < nr) {
            int row = r0 + k;
            if (fwd)
              B.dqs[8 * base + row * cnt + node] = v[k];
            else
              B.dq[5 * (base + node) + row] = v[k];
          }
        }
      }
      __syncthreads();
    }
  }
}
__global__ void k_lusgs_sweep_global(const BlockView* __restrict__ blocks, int nst, unsigned* status) {
  (void)nst;
  (void)status;
  lusgs_global_body<double>(blocks);
}
__global__ void k_lusgs_sweep_global_f32(const BlockView* __restrict__ blocks, int nst, unsigned* status) {
  (void)nst;
  (void)status;
  lusgs_global_body<float>(blocks);
}

namespace {

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned cluster_size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}

// One row of one node of a plane, as lusgs_rows computes it, with the values
// written during the sweep (previous plane, dq*) loaded from L2: they come
// from other SMs, and a line cached in this SM's L1 before they were written
// would be stale.
template <bool FWD, typename R>
__device__ __forceinline__ double lusgs_row_l2(const R* rec, const double* sca, const double* dsv, int cnt,
                                               int t, int row, const double* prev, long pst, int wst) {
  double packed = RecFmt<R>::packed(rec, cnt, t);
  double acc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int w = nbr_local(packed, d);
    double sd = 0.0;
    if (w >= 0) {
      const double* x = prev + (long)w * wst;
      const R* mr = rec + (25 * d + 5 * row) * cnt + t;
      sd = (double)mr[0] * __ldcg(x);
      sd = sd + (double)mr[cnt] * __ldcg(x + pst);
      sd = sd + (double)mr[2 * cnt] * __ldcg(x + 2 * pst);
      sd = sd + (double)mr[3 * cnt] * __ldcg(x + 3 * pst);
      sd = sd + (double)mr[4 * cnt] * __ldcg(x + 4 * pst);
    }
    acc[d] = sd;
  }
  const double diag = sca[5 * cnt + t], invj = sca[6 * cnt + t];
  const double rdiag = sca[7 * cnt + t], rinvj = sca[8 * cnt + t];
  const bool bok = !nbr_slow_div(packed);
  if (FWD) return div2_rn(sca[row * cnt + t] + (acc[0] + acc[1] + acc[2]), diag, rdiag, invj, rinvj, bok);
  return __ldcg(dsv + row * cnt + t) - div2_rn(acc[0] + acc[1] + acc[2], invj, rinvj, diag, rdiag, bok);
}

}  // namespace

// The records of one row of one node, loaded ahead of the plane barrier (they
// were written before the sweep started).
struct RowRecs {
  double packed, m[15], rhs, diag, invj, rdiag, rinvj;
  int row, node;
};
template <typename R>
__device__ __forceinline__ void load_row_recs(const R* rec, const double* sca, int cnt, int t, RowRecs& r) {
  r.row = row_of(t, cnt);
  r.node = t - r.row * cnt;
  const R* rn = rec + r.node;
  r.packed = RecFmt<R>::packed(rec, cnt, r.node);
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int c = 0; c < 5; ++c) r.m[5 * d + c] = (double)rn[(25 * d + 5 * r.row + c) * cnt];
  const double* sn = sca + r.node;
  r.rhs = sn[r.row * cnt];
  r.diag = sn[5 * cnt];
  r.invj = sn[6 * cnt];
  r.rdiag = sn[7 * cnt];
  r.rinvj = sn[8 * cnt];
  // (the divisor flag in `packed` is read where the row is computed, so that
  // this load of the next plane's row does not wait for its data)
}
// lusgs_rows' arithmetic for one row from preloaded records; the previous
// plane's dq and dq* are loaded from L2 (written by other SMs during the sweep).
template <bool FWD>
__device__ __forceinline__ double row_from_recs(const RowRecs& r, const double* prev, long pst, int wst,
                                                const double* dsv, int cnt) {
  double acc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int w = nbr_local(r.packed, d);
    double sd = 0.0;
    if (w >= 0) {
      const double* x = prev + (long)w * wst;
      sd = r.m[5 * d] * __ldcg(x);
      sd = sd + r.m[5 * d + 1] * __ldcg(x + pst);
      sd = sd + r.m[5 * d + 2] * __ldcg(x + 2 * pst);
      sd = sd + r.m[5 * d + 3] * __ldcg(x + 3 * pst);
      sd = sd + r.m[5 * d + 4] * __ldcg(x + 4 * pst);
    }
    acc[d] = sd;
  }
  const bool bok = !nbr_slow_div(r.packed);  // divisors in div2_rn's fast range
  if (FWD) return div2_rn(r.rhs + (acc[0] + acc[1] + acc[2]), r.diag, r.rdiag, r.invj, r.rinvj, bok);
  return __ldcg(dsv + r.row * cnt + r.node) - div2_rn(acc[0] + acc[1] + acc[2], r.invj, r.rinvj, r.diag, r.rdiag, bok);
}

// The global-memory sweeps of one block spread over a thread-block cluster
// (grid x = blocks x cluster size, cluster dims (CL,1,1)): the CL CTAs of a
// cluster share every plane, one thread per row of a node (t < 5*cnt, row
// t / cnt, consecutive threads on consecutive nodes of one row), and meet at a
// cluster barrier between planes, which orders each plane's dq stores before
// the next plane's loads.  The barrier is split: between its arrive and its
// wait each thread loads the records of its first row of the next plane, so
// only the neighbours' dq loads remain on the path from plane to plane.  All
// CTAs of a cluster are resident together and every thread takes the same 2H
// barriers, so the barrier always completes.  The arithmetic per row is
// lusgs_rows'.
template <typename R>
__device__ __forceinline__ void lusgs_cluster_body(const BlockView* __restrict__ blocks) {
  constexpr int W = RecFmt<R>::kWords;
  const unsigned ncta = cluster_size();
  const BlockView& B = blocks[blockIdx.x / ncta];
  if (B.retired()) return;
  const int H = B.nplanes;
  const long* poff = B.poff;
  const int G = (int)(ncta * blockDim.x);
  const int g = (int)(cluster_rank() * blockDim.x + threadIdx.x);
  // records of this thread's first row of global step gs (forward: gs < H)
  RowRecs pre;
  auto preload = [&](int gs) {
    if (gs >= 2 * H) return;
    const bool fwd = gs < H;
    const int h = fwd ? gs : 2 * H - 1 - gs;
    const long base = poff[h];
    const int cnt = (int)(poff[h + 1] - base);
    if (g < 5 * cnt) load_row_recs(recs<R>(B, fwd) + W * base, B.sca + kSca * base, cnt, g, pre);
  };
  preload(0);
  for (int gs = 0; gs < 2 * H; ++gs) {
    const bool fwd = gs < H;
    const int h = fwd ? gs : 2 * H - 1 - gs;
    const long base = poff[h];
    const int cnt = (int)(poff[h + 1] - base);
    const R* rec = recs<R>(B, fwd) + W * base;
    const double* sca = B.sca + kSca * base;
    const double* dsv = B.dqs + 8 * base;
    const double* prev = sca;
    long pst = 0;
    int wst = 0;
    if (fwd && h > 0) {
      prev = B.dqs + 8 * poff[h - 1];
      pst = poff[h] - poff[h - 1];
      wst = 1;
    } else if (!fwd && h + 1 < H) {
      prev = B.dq + 5 * poff[h + 1];
      pst = 1;
      wst = 5;
    }
    if (g < 5 * cnt) {
      double v = fwd ? row_from_recs<true>(pre, prev, pst, wst, dsv, cnt)
                     : row_from_recs<false>(pre, prev, pst, wst, dsv, cnt);
      if (fwd)
        B.dqs[8 * base + pre.row * cnt + pre.node] = v;
      else
        B.dq[5 * (base + pre.node) + pre.row] = v;
    }
    for (int t = g + G; t < 5 * cnt; t += G) {
      const int row = row_of(t, cnt);
      const int node = t - row * cnt;
      if (fwd)
        B.dqs[8 * base + row * cnt + node] = lusgs_row_l2<true, R>(rec, sca, dsv, cnt, node, row, prev, pst, wst);
      else
        B.dq[5 * (base + node) + row] = lusgs_row_l2<false, R>(rec, sca, dsv, cnt, node, row, prev, pst, wst);
    }
    asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
    preload(gs + 1);
    asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
  }
}
__global__ void __launch_bounds__(512, 1) k_lusgs_sweep_cluster(const BlockView* __restrict__ blocks) {
  lusgs_cluster_body<double>(blocks);
}
__global__ void __launch_bounds__(512, 1) k_lusgs_sweep_cluster_f32(const BlockView* __restrict__ blocks) {
  lusgs_cluster_body<float>(blocks);
}

namespace {

// Shared-memory address of CTA `rank` of the cluster for a local address.
__device__ __forceinline__ unsigned map_rank(unsigned local, unsigned rank) {
  unsigned r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}
// Bulk copy from this CTA's shared memory into another CTA's of the cluster,
// completion counted in bytes on the destination CTA's mbarrier (no
// multicast).  Addresses 16-byte aligned, size a multiple of 16.
__device__ __forceinline__ void bulk_to_cluster(unsigned dst, unsigned src, unsigned bytes, unsigned mbar) {
  asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   dst),
               "r"(src), "r"(bytes), "r"(mbar)
               : "memory");
}
__device__ __forceinline__ bool mbar_wait_bounded(unsigned long long* bar, unsigned parity) {
  return wait_bounded([&] { return mbar_try_wait(bar, parity); });
}
// "no wait has run out" in the bulk sweep's failure stamp
constexpr unsigned kNoFailure = 0xffffffffu;
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// lusgs_rows' arithmetic for one row from preloaded records, the previous
// plane's values read from this CTA's ring in row-major item order
// (row c of node w at c*cnt_prev + w).
template <bool FWD>
__device__ __forceinline__ double row_from_ring(const RowRecs& r, const double* prev, int cnt_prev, const double* dsv,
                                                int cnt) {
  double acc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int w = nbr_local(r.packed, d);
    double sd = 0.0;
    if (w >= 0) {
      const double* x = prev + w;
      sd = r.m[5 * d] * x[0];
      sd = sd + r.m[5 * d + 1] * x[cnt_prev];
      sd = sd + r.m[5 * d + 2] * x[2 * cnt_prev];
      sd = sd + r.m[5 * d + 3] * x[3 * cnt_prev];
      sd = sd + r.m[5 * d + 4] * x[4 * cnt_prev];
    }
    acc[d] = sd;
  }
  const bool bok = !nbr_slow_div(r.packed);  // divisors in div2_rn's fast range
  if (FWD) return div2_rn(r.rhs + (acc[0] + acc[1] + acc[2]), r.diag, r.rdiag, r.invj, r.rinvj, bok);
  return __ldcg(dsv + r.row * cnt + r.node) - div2_rn(acc[0] + acc[1] + acc[2], r.invj, r.rinvj, r.diag, r.rdiag, bok);
}

}  // namespace

// The cluster sweeps with the plane-to-plane exchange by bulk copies between
// the CTAs' shared memories.  Item t of a plane (row t / cnt of node t % cnt)
// belongs to thread t of the cluster (5 * pmax <= cluster threads), so CTA r
// computes the contiguous slice [r*T, (r+1)*T) of the plane's values.  Each CTA
// writes its slice into a two-plane ring in its own shared memory (row-major
// item order), and after a CTA barrier lane r of warp 0 copies the slice into
// the same place in CTA r with cp.async.bulk, the bytes counted on the receiver's mbarrier
// for that ring half; a CTA arms its mbarrier with the bytes it expects and its
// threads wait (bounded) for the previous plane's bytes before reading the
// neighbours from local shared memory.  No cluster barrier or global memory
// is on the plane-to-plane path; one cluster barrier at the pass boundary
// publishes the forward dq* (global) to the backward pass, and a last one keeps
// every CTA resident until the copies into it have landed.  A CTA copies plane
// gs+2 into a ring half only after every CTA has sent it plane gs+1, i.e. after
// all have finished reading that half.  The arithmetic per row is lusgs_rows'.
//
// Failure (a wait that runs out) is contained by these rules:
//  * a CTA arms a ring half for plane gs only while none of its waits has run
//    out, so the half's previous phase (plane gs-2) was seen complete: no half
//    is ever re-armed over an incomplete phase;
//  * once a wait has run out the CTA sends nothing more.  Its peers then run
//    out waiting for its next slice and stop too, so every copy into a CTA
//    belongs to a plane that CTA has armed (no bytes are counted on the wrong
//    phase) and the whole cluster ends in the failed state;
//  * at the end every CTA publishes whether it failed; if any did, each waits
//    again (bounded) for its armed phases and then idles for a bounded time
//    after the last cluster barrier, so copies issued before that barrier land
//    before any CTA leaves.  Without a failure every CTA has seen every byte
//    sent to it before the last barrier, so no copy is in flight at exit.
// The sweep raises ST_TIMEOUT; its values are then meaningless.
template <typename R, int DEPTH>
__device__ __forceinline__ void lusgs_bulk_body(const BlockView* __restrict__ blocks, unsigned* status, int pf) {
  constexpr int W = RecFmt<R>::kWords;
  extern __shared__ __align__(16) double xring[];  // 2 halves x (G + 2) doubles
  __shared__ __align__(8) unsigned long long xbar[2];
  __shared__ unsigned s_failed;  // a wait of this CTA ran out (any thread)
  const unsigned ncta = cluster_size(), me = cluster_rank();
  const BlockView& B = blocks[blockIdx.x / ncta];
  if (B.retired()) return;
  const int H = B.nplanes;
  const long* poff = B.poff;
  const int T = (int)blockDim.x;
  const int G = (int)ncta * T;
  const int HS = G + 2;
  const int g = (int)me * T + (int)threadIdx.x;
  if (threadIdx.x == 0) {
    s_failed = kNoFailure;
    mbar_init(&xbar[0], 1);
    mbar_init(&xbar[1], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  cluster_sync_all();  // every CTA's mbarriers exist before any copy targets them
  const unsigned ring_local = smem_u32(xring), bar_local = smem_u32(xbar);
  auto plane_of = [&](int gs) { return gs < H ? gs : 2 * H - 1 - gs; };
  auto count_of = [&](int gs) {
    const int h = plane_of(gs);
    return (int)(poff[h + 1] - poff[h]);
  };
  auto slice_bytes = [&](int cnt, unsigned r) -> unsigned {
    const int n = min(T, 5 * cnt - (int)r * T);
    return n <= 0 ? 0u : (unsigned)((n * 8 + 15) & ~15);
  };
  // this thread's row of the next DEPTH planes, loaded ahead (records and
  // scalars are read-only during the sweep)
  RowRecs pre0, pre1;
  auto preload = [&](int gs, RowRecs& pre) {
    if (gs >= 2 * H) return;
    const bool fwd = gs < H;
    const long base = poff[plane_of(gs)];
    const int cnt = count_of(gs);
    if (g < 5 * cnt) load_row_recs(recs<R>(B, fwd) + W * base, B.sca + kSca * base, cnt, g, pre);
  };
  // L2 prefetch of plane gs's records and scalars (and, backward, dq*): each
  // CTA asks for its 1/ncta share of each chunk, so the whole chunk is in L2
  // before preload() reads it (pf - 1 planes later, pf >= 2, a kernel argument).  Every chunk starts and ends on a
  // 16-byte boundary (W * sizeof(R), kSca * 8 and 8 * 8 bytes per node are
  // multiples of 16), and so does every share.
  auto prefetch = [&](int gs) {
    if (gs >= 2 * H || threadIdx.x != 32) return;
    const bool fwd = gs < H;
    const long base = poff[plane_of(gs)];
    const long cnt = count_of(gs);
    auto share = [&](const void* chunk, long bytes) {
      const long part = ((bytes + ncta - 1) / ncta + 15) & ~15L;
      const long off = part * me;
      if (off < bytes) bulk_prefetch_l2((const char*)chunk + off, (unsigned)min(part, bytes - off));
    };
    share(recs<R>(B, fwd) + W * base, (long)W * sizeof(R) * cnt);
    share(B.sca + kSca * base, (long)kSca * 8 * cnt);
    if (!fwd) share(B.dqs + 8 * base, 64L * cnt);
  };
  // failures are stamped with the plane whose wait ran out (the smallest
  // such plane is kept), so a test for "a wait of plane <= p ran out" is
  // exact whatever later planes other warps have reached
  volatile unsigned* failed_at = &s_failed;
  auto failed_by = [&](int p) { return p >= 0 && *failed_at <= (unsigned)p; };
  auto fail_at = [&](int p) { atomicMin(&s_failed, (unsigned)p); };
  int armed0 = -1, armed1 = -1;  // thread 0: the last plane armed on ring half 0 / 1
  // one plane step with this thread's row preloaded in `pre`
  auto step = [&](int gs, const RowRecs& pre) {
    const bool fwd = gs < H;
    const long base = poff[plane_of(gs)];
    const int cnt = count_of(gs);
    // arm this plane's half (the bytes of the other CTAs' slices) only if the
    // half's previous phase (plane gs-2, waited for at plane gs-1) completed
    if (threadIdx.x == 0 && !failed_by(gs - 1)) {
      unsigned expect = 0;
      for (unsigned r = 0; r < ncta; ++r)
        if (r != me) expect += slice_bytes(cnt, r);
      mbar_expect_tx(&xbar[gs & 1], expect);
      if (gs & 1)
        armed1 = gs;
      else
        armed0 = gs;
    }
    int cnt_prev = 0;
    if (gs > 0) {
      cnt_prev = count_of(gs - 1);
      if (!failed_by(gs - 1) && !mbar_wait_bounded(&xbar[(gs - 1) & 1], (unsigned)(((gs - 1) >> 1) & 1))) {
        fail_at(gs);
        note_timeout(status, TS_BULK, (int)(blockIdx.x / ncta), (int)me, gs, TW_PLANE);
      }
    }
    if (gs == H) cluster_sync_all();  // the forward dq* stores, for dsv
    const double* prev = xring + ((gs - 1) & 1) * HS;
    double* cur = xring + (gs & 1) * HS;
    if (g < 5 * cnt) {
      const double* dsv = B.dqs + 8 * base;
      const double v = fwd ? row_from_ring<true>(pre, prev, cnt_prev, dsv, cnt)
                           : row_from_ring<false>(pre, prev, cnt_prev, dsv, cnt);
      cur[g] = v;
      if (fwd)
        B.dqs[8 * base + pre.row * cnt + pre.node] = v;
      else
        B.dq[5 * (base + pre.node) + pre.row] = v;
    }
    // the slice is complete once every thread has written and fenced its value;
    // lane r of warp 0 then copies it to CTA r, unless a wait of this CTA up to
    // this plane ran out (every such failure is recorded before the barrier)
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x < ncta && threadIdx.x != me && !failed_by(gs)) {
      const unsigned bytes = slice_bytes(cnt, me);
      const unsigned off = (unsigned)(((gs & 1) * HS + (int)me * T) * sizeof(double));
      const unsigned boff = (unsigned)((gs & 1) * sizeof(unsigned long long));
      if (bytes)
        bulk_to_cluster(map_rank(ring_local + off, threadIdx.x), ring_local + off, bytes,
                        map_rank(bar_local + boff, threadIdx.x));
    }
  };
  // planes 1 .. pf-1 now, then plane gs+pf after each step gs (pf >= 2)
  for (int x = 1; x < pf; ++x) prefetch(x);
  preload(0, pre0);
  if (DEPTH == 2) preload(1, pre1);
  for (int gs = 0; gs < 2 * H; gs += DEPTH) {
    step(gs, pre0);
    prefetch(gs + pf);
    preload(gs + DEPTH, pre0);
    if (DEPTH == 2 && gs + 1 < 2 * H) {
      step(gs + 1, pre1);
      prefetch(gs + 1 + pf);
      preload(gs + 3, pre1);
    }
  }
  // the last plane's bytes
  if (H > 0 && !failed_by(2 * H - 1) &&
      !mbar_wait_bounded(&xbar[(2 * H - 1) & 1], (unsigned)(((2 * H - 1) >> 1) & 1))) {
    fail_at(2 * H);
    note_timeout(status, TS_BULK, (int)(blockIdx.x / ncta), (int)me, 2 * H, TW_LAST_PLANE);
  }
  __syncthreads();
  // every CTA's outcome is final once all have reached the barrier; each
  // reads the others' and no CTA leaves before all have read
  cluster_sync_all();
  unsigned any = (s_failed != kNoFailure) ? 1u : 0u;
  if (threadIdx.x < ncta && threadIdx.x != me) {
    unsigned v;
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(map_rank(smem_u32(&s_failed), threadIdx.x))
                 : "memory");
    any |= v != kNoFailure ? 1u : 0u;
  }
  any = __syncthreads_or(any);
  cluster_sync_all();
  if (any) {
    // copies issued before the last barrier may still be landing in, or
    // reading from, this CTA's shared memory: wait (bounded) for the phases
    // this CTA armed, then idle for a bounded time before leaving
    if (threadIdx.x == 0) {
      for (int h = 0; h < 2; ++h) {
        const int a = h ? armed1 : armed0;
        if (a >= 0)
          wait_bounded([&] { return mbar_try_wait(&xbar[h], (unsigned)((a >> 1) & 1)); });
      }
      for (int s = 0; s < 2000; ++s) __nanosleep(1000);
      if (status) atomicOr(status, (unsigned)ST_TIMEOUT);
      B.raise(ST_TIMEOUT);
    }
    __syncthreads();
  }
}
__global__ void __launch_bounds__(512, 1) k_lusgs_sweep_bulk(const BlockView* __restrict__ blocks, unsigned* status,
                                                             int pf) {
  lusgs_bulk_body<double, 1>(blocks, status, pf);
}
__global__ void __launch_bounds__(512, 1) k_lusgs_sweep_bulk_f32(const BlockView* __restrict__ blocks,
                                                                 unsigned* status, int pf) {
  lusgs_bulk_body<float, 1>(blocks, status, pf);
}
// CTAs of at most 384 threads, two resident per SM (80 registers): for
// batches whose sweep CTAs outnumber the SMs
__global__ void __launch_bounds__(384, 2) k_lusgs_sweep_bulk_o2(const BlockView* __restrict__ blocks,
                                                                unsigned* status, int pf) {
  lusgs_bulk_body<double, 1>(blocks, status, pf);
}
__global__ void __launch_bounds__(384, 2) k_lusgs_sweep_bulk_o2_f32(const BlockView* __restrict__ blocks,
                                                                    unsigned* status, int pf) {
  lusgs_bulk_body<float, 1>(blocks, status, pf);
}
// CTAs of at most 256 threads (a cluster's share of the largest plane's rows):
// each thread's records loaded two planes ahead
__global__ void __launch_bounds__(256, 1) k_lusgs_sweep_bulk2(const BlockView* __restrict__ blocks, unsigned* status,
                                                              int pf) {
  lusgs_bulk_body<double, 2>(blocks, status, pf);
}
__global__ void __launch_bounds__(256, 1) k_lusgs_sweep_bulk2_f32(const BlockView* __restrict__ blocks,
                                                                  unsigned* status, int pf) {
  lusgs_bulk_body<float, 2>(blocks, status, pf);
}

// ------------------------------------------------------------ slab sweeps
namespace {

// What one row of one node of a slab sweep reads besides the previous plane:
// its records, scalars and (backward) dq*.
struct SlabRow {
  double packed, m[15], rhs, diag, invj, rdiag, rinvj, dsv;
  int row, node;
};
template <typename R>
__device__ __forceinline__ void load_slab_row(const BlockView& B, bool fwd, long base, int cnt, int row, int node,
                                              SlabRow& r) {
  constexpr int W = RecFmt<R>::kWords;
  const R* rec = recs<R>(B, fwd) + W * base;
  r.row = row;
  r.node = node;
  const R* rn = rec + node;
  r.packed = RecFmt<R>::packed(rec, cnt, node);
#pragma unroll
  for (int d = 0; d < 3; ++d)
#pragma unroll
    for (int c = 0; c < 5; ++c) r.m[5 * d + c] = (double)rn[(25 * d + 5 * row + c) * cnt];
  const double* sn = B.sca + kSca * base + node;
  r.rhs = sn[row * cnt];
  r.diag = sn[5 * cnt];
  r.invj = sn[6 * cnt];
  r.rdiag = sn[7 * cnt];
  r.rinvj = sn[8 * cnt];
  // dq* of the node, written by this CTA in the forward pass (read from L2;
  // complete once the forward pass has passed the node's plane)
  r.dsv = fwd ? 0.0 : __ldcg(B.dqs + 8 * base + row * cnt + node);
  // (the divisor flag in `packed` is read where the row is computed, so that
  // this load ahead does not wait for its data)
}
// lusgs_rows' arithmetic for one row from preloaded records.  The previous
// plane's values: row c of plane-local node w at own[c*So + w - o0] for the
// slab's own nodes [o0, o0 + no), else (the k-neighbour in the upstream
// slab's edge segment, which starts at eb) at edge[c*L + w - eb].
template <bool FWD>
__device__ __forceinline__ double row_from_slab(const SlabRow& r, const double* own, int o0, int no, int So,
                                                const double* edge, int eb, int L, double dsv) {
  double acc[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int w = nbr_local(r.packed, d);
    double sd = 0.0;
    if (w >= 0) {
      // the i and j neighbours share the node's k-offset, so they are the slab's own
      const bool mine = d < 2 || (unsigned)(w - o0) < (unsigned)no;
      const double* x = mine ? own + (w - o0) : edge + (w - eb);
      const int st = mine ? So : L;
      sd = r.m[5 * d] * x[0];
      sd = sd + r.m[5 * d + 1] * x[st];
      sd = sd + r.m[5 * d + 2] * x[2 * st];
      sd = sd + r.m[5 * d + 3] * x[3 * st];
      sd = sd + r.m[5 * d + 4] * x[4 * st];
    }
    acc[d] = sd;
  }
  const bool bok = !nbr_slow_div(r.packed);  // divisors in div2_rn's fast range
  if (FWD) return div2_rn(r.rhs + (acc[0] + acc[1] + acc[2]), r.diag, r.rdiag, r.invj, r.rinvj, bok);
  return dsv - div2_rn(acc[0] + acc[1] + acc[2], r.invj, r.rinvj, r.diag, r.rdiag, bok);
}

}  // namespace

// The forward and backward sweeps of one block pipelined over a cluster of
// CTAs by k-slabs (grid x = blocks x cluster size, cluster dims (CL,1,1)).
// CTA r owns the nodes of k-offsets [r*nz1/ce, (r+1)*nz1/ce) (slab::Geom); a
// plane lists its nodes by k-offset, so a slab's part of every plane is one
// contiguous range of plane-local indices, which the CTA computes one row of a
// node per thread, in the hyperplane order of the serial sweep.  Within a
// slab every neighbour a node needs from the previous plane is the CTA's own,
// except the k-1 (forward) / k+1 (backward) neighbours of the slab's first /
// last k-segment, which belong to the edge k-segment of the slab below /
// above (the pass's "upstream" slab).  After each plane a CTA stages its own
// edge segment's values and copies them with one cp.async.bulk (no multicast)
// into the downstream CTA's inbox, counted in bytes on the receiver's mbarrier
// for that inbox slot; a CTA waits only on that mbarrier, for the step before
// its own.  So the CTAs run as a pipeline, each a few planes behind its
// upstream neighbour, with no cluster-wide exchange on any plane and no memory
// fence on the plane-to-plane path; what remains per plane is the CTA's own
// work and its record loads, which each thread issues DEPTH steps ahead (two
// register sets for DEPTH 2, which the 256-thread variant has room for) after
// the pass's leading CTA has prefetched the plane's chunks into L2.  Rings,
// inboxes and staging areas hold D planes.  After each step a CTA tells both
// neighbours the last step it completed (a relaxed store into their shared
// memory); a CTA copies step gs into a neighbour's slot only after that
// neighbour has completed step gs-D+1, which waited for the slot's previous
// copy, so no slot is overwritten while in use and no mbarrier phase is armed
// twice.  No CTA can wait forever on another: each wait is for a CTA at an
// earlier step, and every wait is bounded.  A wait that runs out makes the
// CTA stop sending (its neighbours then run out too); slab::finish then keeps
// every CTA resident until no copy can still land in it.  Without a failure
// every copy into a CTA is waited for before the last barrier.  The
// arithmetic per row is lusgs_rows', so the result is the same to the bit.
template <typename R, int DEPTH>
__device__ __forceinline__ void lusgs_slab_body(const BlockView* __restrict__ blocks, unsigned* status, int So,
                                                int L, int D) {
  constexpr int W = RecFmt<R>::kWords;
  extern __shared__ __align__(16) double sdyn[];
  double* stage = sdyn;                // D x 5 x L: this slab's edge values, copied downstream
  double* inbox = stage + D * 5 * L;   // D x 5 x L: the upstream slab's edge values
  double* ring = inbox + D * 5 * L;    // D x 5 x So: this slab's values
  __shared__ __align__(8) unsigned long long full[kSlabSlots];  // inbox slot arrivals
  __shared__ int s_prog[2];  // last step completed by the CTA below / above
  __shared__ int s_fail;
  const int ncta = (int)slab::size();
  const BlockView& B = blocks[blockIdx.x / ncta];
  if (B.retired()) return;
  const slab::Geom G(B, ncta, (int)slab::rank());
  const long* poff = B.poff;
  const int H = G.H, tid = (int)threadIdx.x;
  if (tid == 0) {
    s_prog[0] = -1;
    s_prog[1] = -1;
    s_fail = 0;
    for (int x = 0; x < D; ++x) slab::bar_init(&full[x], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  slab::sync();  // every CTA's counters and mbarriers exist before a neighbour touches them
  const unsigned slot_bytes = (unsigned)(5 * L * sizeof(double));
  if (G.active()) {
    // this CTA's progress lives in the CTA below as its "above" counter and in
    // the CTA above as its "below" counter
    const unsigned at_lo = G.has_lo() ? slab::map(slab::local(&s_prog[1]), G.me - 1) : 0u;
    const unsigned at_hi = G.has_hi() ? slab::map(slab::local(&s_prog[0]), G.me + 1) : 0u;
    const unsigned inbox_l = slab::local(inbox), full_l = slab::local(full), stage_l = slab::local(stage);
    auto preload = [&](int gs, SlabRow& r) {
      if (gs >= 2 * H) return;
      const int h = G.plane(gs);
      const long base = poff[h];
      const int t0 = G.seg(h, G.c0), n = G.seg(h, G.c1) - t0;
      if (tid < 5 * n) {
        const int row = row_of(tid, n);
        load_slab_row<R>(B, gs < H, base, (int)(poff[h + 1] - base), row, t0 + tid - row * n, r);
      }
    };
    // L2 prefetch of step gs's whole chunks (records, scalars and, backward,
    // dq*) by the pass's leading CTA (the one without an upstream slab: every
    // other CTA reaches each step after it), one lane per chunk; the chunks
    // start and end on 16-byte boundaries
    const bool lead_f = G.me == 0, lead_b = G.me == G.ce - 1;
    auto prefetch = [&](int gs) {
      if (gs >= 2 * H || tid >= 35 || tid < 32) return;
      const bool fwd = gs < H;
      if (!(fwd ? lead_f : lead_b)) return;
      const long base = poff[G.plane(gs)];
      const long cnt = poff[G.plane(gs) + 1] - base;
      if (tid == 32) slab::prefetch_span(recs<R>(B, fwd) + W * base, (long)W * (long)sizeof(R) * cnt);
      if (tid == 33) slab::prefetch_span(B.sca + kSca * base, 8L * kSca * cnt);
      if (tid == 34 && !fwd) slab::prefetch_span(B.dqs + 8 * base, 64L * cnt);
    };
    unsigned parity = 0;  // bit x: parity of the next phase of full[x] to wait for
    // one plane step with the row preloaded in `pre`; false (in every thread)
    // when a wait of this CTA ran out
    auto step = [&](int gs, const SlabRow& pre) -> bool {
      const bool fwd = gs < H;
      const int h = G.plane(gs);
      const long base = poff[h];
      const int cnt = (int)(poff[h + 1] - base);
      const int t0 = G.seg(h, G.c0), n = G.seg(h, G.c1) - t0;
      const bool need_dn = G.need_dn(gs);
      const int x = gs % D, xp = (gs + D - 1) % D;
      bool fail = false;
      if (G.need_up(gs)) {
        // the upstream slab's edge values of step gs-1, copied into inbox slot xp
        if (tid == 0) slab::bar_expect(&full[xp], slot_bytes);
        fail = !slab::bar_wait(&full[xp], (parity >> xp) & 1u);
        parity ^= 1u << xp;
        if (fail) note_timeout(status, TS_SLAB, (int)(blockIdx.x / ncta), G.me, gs, TW_PLANE);
      }
      // room downstream: it has completed step gs-D+1, which waited for the
      // previous copy into slot x (so that copy also finished reading stage x)
      if (!fail && need_dn) {
        fail = !slab::wait_for(&s_prog[fwd ? 1 : 0], gs - D + 1);
        if (fail) note_timeout(status, TS_SLAB, (int)(blockIdx.x / ncta), G.me, gs, TW_PROGRESS);
      }
      if (!fail && tid < 5 * n) {  // the launch gives every row of a slab's plane a thread
        const int hp = G.plane(gs > 0 ? gs - 1 : 0);
        const int p0 = G.seg(hp, G.c0), np = G.seg(hp, G.c1) - p0;
        const int eb = G.seg(hp, max(G.c_up(gs), 0));
        const double* own = ring + xp * 5 * So;
        const double* edge = inbox + xp * 5 * L;
        // dq* of the first backward plane (the forward pass's last) is written
        // by the step before, after a two-step-ahead load of it was issued
        const double dsv = (DEPTH > 1 && gs == H) ? __ldcg(B.dqs + 8 * base + pre.row * cnt + pre.node) : pre.dsv;
        const double v = fwd ? row_from_slab<true>(pre, own, p0, np, So, edge, eb, L, dsv)
                             : row_from_slab<false>(pre, own, p0, np, So, edge, eb, L, dsv);
        ring[x * 5 * So + pre.row * So + (pre.node - t0)] = v;
        if (need_dn) {
          const int e0 = G.seg(h, G.c_dn(gs));
          if (pre.node >= e0 && pre.node < G.seg(h, G.c_dn(gs) + 1))
            stage[x * 5 * L + pre.row * L + (pre.node - e0)] = v;
        }
        if (fwd)
          B.dqs[8 * base + pre.row * cnt + pre.node] = v;
        else
          B.dq[5 * (base + pre.node) + pre.row] = v;
      }
      if (need_dn) slab::fence_to_copies();
      if (__syncthreads_or(fail ? 1 : 0)) {
        if (tid == 0) s_fail = 1;
        return false;
      }
      if (tid == 0) {
        if (need_dn) {
          const unsigned r = (unsigned)G.rank_dn(gs);
          const unsigned off = (unsigned)(x * 5 * L * sizeof(double));
          slab::copy_to(slab::map(inbox_l + off, r), stage_l + off, slot_bytes,
                        slab::map(full_l + (unsigned)(x * sizeof(unsigned long long)), r));
        }
        if (G.has_lo()) slab::store_relaxed(at_lo, gs);
        if (G.has_hi()) slab::store_relaxed(at_hi, gs);
      }
      return true;
    };
    constexpr int PF = 4;  // prefetch distance in steps
    for (int gs = 0; gs < PF; ++gs) prefetch(gs);
    SlabRow r0, r1;
    preload(0, r0);
    if (DEPTH == 2) preload(1, r1);
    for (int gs = 0; gs < 2 * H; gs += DEPTH) {
      if (!step(gs, r0)) break;
      prefetch(gs + PF);
      preload(gs + DEPTH, r0);
      if (DEPTH == 2) {
        if (gs + 1 >= 2 * H) break;
        if (!step(gs + 1, r1)) break;
        prefetch(gs + 1 + PF);
        preload(gs + 3, r1);
      }
    }
  }
  slab::finish(s_fail, ncta, status, B);
}
__global__ void __launch_bounds__(512, 1) k_lusgs_sweep_slab(const BlockView* __restrict__ blocks, unsigned* status,
                                                             int So, int L, int D) {
  lusgs_slab_body<double, 1>(blocks, status, So, L, D);
}
__global__ void __launch_bounds__(512, 1) k_lusgs_sweep_slab_f32(const BlockView* __restrict__ blocks,
                                                                 unsigned* status, int So, int L, int D) {
  lusgs_slab_body<float, 1>(blocks, status, So, L, D);
}
// Slabs whose planes have at most 51 nodes (256 rows): record loads two steps ahead.
__global__ void __launch_bounds__(256, 1) k_lusgs_sweep_slab2(const BlockView* __restrict__ blocks,
                                                              unsigned* status, int So, int L, int D) {
  lusgs_slab_body<double, 2>(blocks, status, So, L, D);
}
__global__ void __launch_bounds__(256, 1) k_lusgs_sweep_slab2_f32(const BlockView* __restrict__ blocks,
                                                                  unsigned* status, int So, int L, int D) {
  lusgs_slab_body<float, 2>(blocks, status, So, L, D);
}

// q = q + dq on every updated node (sub_timeadvancement_1stimplicit.f90:568-574).
// q += dq over the updated box, walked in box order so that q is read and
// written along its rows; dq (hyperplane-major, 5 per node) is gathered
// through the position index.
__global__ void k_lusgs_update(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const Box& b1 = B.b1;
  long u = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= b1.size()) return;
  int i = b1.is + (int)(u % b1.nx());
  long r = u / b1.nx();
  int j = b1.js + (int)(r % b1.ny());
  int k = b1.ks + (int)(r / b1.ny());
  long n = B.at(i, j, k);
  const double* dq = B.dq + 5L * B.pidx[u];
#pragma unroll
  for (int x = 1; x <= 5; ++x) B.v(F_Q, x, n) = B.v(F_Q, x, n) + dq[x - 1];
}

}  // namespace aero
