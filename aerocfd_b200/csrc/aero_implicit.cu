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

// The off-diagonal blocks of both sweeps, off the critical path.  For every
// updated node (the provider) and direction d: A = calc_jm at the provider,
// S+ = 0.5*(A + r*I)*inv_j goes to the forward record of the node one step up
// in d, S- = 0.5*(A - r*I)*inv_j to the backward record of the node one step
// down (sub_timeadvancement_1stimplicit.f90:283-301, :459-477, same
// operations).  Each node also stores rhs, diag, inv_j and the positions of
// its six neighbours in the hyperplane-major order.
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
    B.nat[pos] = n;
#pragma unroll
    for (int e = 0; e < 3; ++e) {
      int lo[3] = {a, b, c}, hi[3] = {a, b, c};
      lo[e] -= 1;
      hi[e] += 1;
      B.nbr[6 * pos + e] = off[e] > 0 ? (int)plane_pos(B, lo[0], lo[1], lo[2]) : -1;
      B.nbr[6 * pos + 3 + e] = off[e] < lim[e] - 1 ? (int)plane_pos(B, hi[0], hi[1], hi[2]) : -1;
    }
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
    double* dst = B.rec_f + 75 * plane_pos(B, q[0], q[1], q[2]) + 25 * d;
#pragma unroll
    for (int x = 0; x < 25; ++x) {
      double v = (x % 6 == 0) ? A[x] + rad : A[x];
      dst[x] = 0.5 * v * invj;
    }
  }
  if (down) {
    int q[3] = {a, b, c};
    q[d] -= 1;
    double* dst = B.rec_b + 75 * plane_pos(B, q[0], q[1], q[2]) + 25 * d;
#pragma unroll
    for (int x = 0; x < 25; ++x) {
      double v = (x % 6 == 0) ? A[x] - rad : A[x];
      dst[x] = 0.5 * v * invj;
    }
  }
}

// Forward and backward hyperplane sweeps for one block per CTA.  Thread t of a
// plane handles equation row t%5 of node t/5 of that plane: the row of the
// three neighbour blocks times the neighbours' dq, summed in the reference's
// order (:346-364, :522-540).  The previous plane's results sit in shared
// memory; q += dq is applied as soon as dq is known (the blocks were built
// from the old q before the sweep, so nothing reads q afterwards).
__global__ void k_lusgs_sweep(const BlockView* __restrict__ blocks, CaseConsts cc) {
  const BlockView& B = blocks[blockIdx.x];
  extern __shared__ double sdq[];  // two planes of 5*pmax values
  const int P = B.pmax;
  const int H = B.nplanes;
  // forward
  for (int h = 0; h < H; ++h) {
    long base = B.poff[h];
    int cnt = (int)(B.poff[h + 1] - base);
    long pbase = h > 0 ? B.poff[h - 1] : 0;
    double* prev = sdq + 5 * P * ((h + 1) & 1);
    double* cur = sdq + 5 * P * (h & 1);
    for (int t = threadIdx.x; t < 5 * cnt; t += blockDim.x) {
      int node = t / 5, row = t - 5 * (t / 5);
      long pos = base + node;
      const double* rec = B.rec_f + 75 * pos + 5 * row;
      const int* nb = B.nbr + 6 * pos;
      double acc[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        int p = nb[d];
        if (p < 0) {
          acc[d] = 0.0;
        } else {
          const double* m = rec + 25 * d;
          const double* x = prev + 5 * (p - pbase);
          double s = m[0] * x[0];
          s = s + m[1] * x[1];
          s = s + m[2] * x[2];
          s = s + m[3] * x[3];
          s = s + m[4] * x[4];
          acc[d] = s;
        }
      }
      const double* sc = B.sca + 8 * pos;
      double v = (sc[row] + (acc[0] + acc[1] + acc[2])) / sc[5] / sc[6];
      cur[t] = v;
      B.dqs[5 * pos + row] = v;
    }
    __syncthreads();
  }
  // backward
  for (int h = H - 1; h >= 0; --h) {
    long base = B.poff[h];
    int cnt = (int)(B.poff[h + 1] - base);
    long pbase = h + 1 < H ? B.poff[h + 1] : 0;
    double* prev = sdq + 5 * P * ((h + 1) & 1);
    double* cur = sdq + 5 * P * (h & 1);
    for (int t = threadIdx.x; t < 5 * cnt; t += blockDim.x) {
      int node = t / 5, row = t - 5 * (t / 5);
      long pos = base + node;
      const double* rec = B.rec_b + 75 * pos + 5 * row;
      const int* nb = B.nbr + 6 * pos + 3;
      double acc[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        int p = nb[d];
        if (p < 0) {
          acc[d] = 0.0;
        } else {
          const double* m = rec + 25 * d;
          const double* x = prev + 5 * (p - pbase);
          double s = m[0] * x[0];
          s = s + m[1] * x[1];
          s = s + m[2] * x[2];
          s = s + m[3] * x[3];
          s = s + m[4] * x[4];
          acc[d] = s;
        }
      }
      const double* sc = B.sca + 8 * pos;
      double v = B.dqs[5 * pos + row] - (acc[0] + acc[1] + acc[2]) / sc[6] / sc[5];
      cur[t] = v;
      B.dq[5 * pos + row] = v;
      long n = B.nat[pos];
      B.v(F_Q, row + 1, n) = B.v(F_Q, row + 1, n) + v;
    }
    __syncthreads();
  }
}

}  // namespace aero
