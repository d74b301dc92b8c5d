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

// calc_jm (sub_timeadvancement_jac.f90:17-62) at node nb with the metric row
// starting at component cbase, the spectral radius added (forward, sgn>0) or
// subtracted (backward) on the diagonal, everything scaled by 0.5*inv_j(nb)
// (sub_timeadvancement_1stimplicit.f90:283-301), then multiplied into dqn:
// out[n] = sum_c M(n,c)*dqn[c], summed left to right (:346-350).
__device__ __forceinline__ void lusgs_matvec(const BlockView& B, long nb, int cbase, int radf,
                                             bool plus, double gamma, const double dqn[5],
                                             double out[5]) {
  double rho = B.v(F_Q, 1, nb), mu0 = B.v(F_Q, 2, nb), mv0 = B.v(F_Q, 3, nb);
  double mw0 = B.v(F_Q, 4, nb), e0 = B.v(F_Q, 5, nb);
  double dxidx = B.v(F_DXIDX, cbase, nb), dxidy = B.v(F_DXIDX, cbase + 1, nb);
  double dxidz = B.v(F_DXIDX, cbase + 2, nb);
  double rad = B.s(radf, nb);
  double invj = B.s(F_INVJ, nb);
  double a2 = gamma - 1.0, a3 = gamma - 2.0;
  double uu = (dxidx * mu0 + dxidy * mv0 + dxidz * mw0) / rho;
  double phi = 0.5 * a2 * (p2(mu0) + p2(mv0) + p2(mw0)) / p2(rho);
  double a1 = gamma * e0 / rho - phi;
  double A[25];  // row-major A[r*5+c] = a(r+1,c+1)
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
#pragma unroll
  for (int d = 0; d < 5; ++d) A[d * 6] = plus ? A[d * 6] + rad : A[d * 6] - rad;
#pragma unroll
  for (int x = 0; x < 25; ++x) A[x] = 0.5 * A[x] * invj;
#pragma unroll
  for (int r = 0; r < 5; ++r) {
    double s = A[r * 5 + 0] * dqn[0];
    s = s + A[r * 5 + 1] * dqn[1];
    s = s + A[r * 5 + 2] * dqn[2];
    s = s + A[r * 5 + 3] * dqn[3];
    s = s + A[r * 5 + 4] * dqn[4];
    out[r] = s;
  }
}

// Node `t` of hyperplane h (offsets a+b+c = h inside an nx1 x ny1 x nz1 box);
// returns false when t is past the plane's node count.
__device__ __forceinline__ bool plane_node(int h, long t, int nx1, int ny1, int nz1, int& a, int& b,
                                           int& c) {
  int cmin = max(0, h - (nx1 - 1) - (ny1 - 1));
  int cmax = min(nz1 - 1, h);
  for (c = cmin; c <= cmax; ++c) {
    int r = h - c;
    int bmin = max(0, r - (nx1 - 1));
    int bmax = min(ny1 - 1, r);
    long cnt = bmax - bmin + 1;
    if (cnt <= 0) continue;
    if (t < cnt) {
      b = bmin + (int)t;
      a = r - b;
      return true;
    }
    t -= cnt;
  }
  return false;
}

// Forward and backward sweeps and the update q += dq for one block per CTA
// (sub_timeadvancement_1stimplicit.f90:279-368, :455-545, :568-574).
__global__ void k_lusgs_sweep(const BlockView* __restrict__ blocks, CaseConsts cc) {
  const BlockView& B = blocks[blockIdx.x];
  const Box& b1 = B.b1;
  int nx1 = b1.nx(), ny1 = b1.ny(), nz1 = b1.nz();
  int H = nx1 + ny1 + nz1 - 2;
  const long st[3] = {1, (long)B.nx, (long)B.nx * B.ny};
  double gamma = cc.gamma;
  // forward
  for (int h = 0; h < H; ++h) {
    for (long t = threadIdx.x;; t += blockDim.x) {
      int a, b, c;
      if (!plane_node(h, t, nx1, ny1, nz1, a, b, c)) break;
      long n = B.at(b1.is + a, b1.js + b, b1.ks + c);
      double acc[3][5];
      const int off[3] = {a, b, c};
      const int radf[3] = {F_RA, F_RB, F_RC};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (off[d] == 0) {
#pragma unroll
          for (int x = 0; x < 5; ++x) acc[d][x] = 0.0;
        } else {
          long nb = n - st[d];
          double dqn[5];
#pragma unroll
          for (int x = 0; x < 5; ++x) dqn[x] = B.v(F_DQS, x + 1, nb);
          lusgs_matvec(B, nb, 3 * d + 1, radf[d], true, gamma, dqn, acc[d]);
        }
      }
      double diag = B.s(F_DIAG, n), invj = B.s(F_INVJ, n);
#pragma unroll
      for (int x = 0; x < 5; ++x)
        B.v(F_DQS, x + 1, n) = (B.v(F_RHS, x + 1, n) + (acc[0][x] + acc[1][x] + acc[2][x])) / diag / invj;
    }
    __syncthreads();
  }
  // backward
  for (int h = H - 1; h >= 0; --h) {
    for (long t = threadIdx.x;; t += blockDim.x) {
      int a, b, c;
      if (!plane_node(h, t, nx1, ny1, nz1, a, b, c)) break;
      long n = B.at(b1.is + a, b1.js + b, b1.ks + c);
      double acc[3][5];
      const int off[3] = {nx1 - 1 - a, ny1 - 1 - b, nz1 - 1 - c};
      const int radf[3] = {F_RA, F_RB, F_RC};
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        if (off[d] == 0) {
#pragma unroll
          for (int x = 0; x < 5; ++x) acc[d][x] = 0.0;
        } else {
          long nb = n + st[d];
          double dqn[5];
#pragma unroll
          for (int x = 0; x < 5; ++x) dqn[x] = B.v(F_DQ, x + 1, nb);
          lusgs_matvec(B, nb, 3 * d + 1, radf[d], false, gamma, dqn, acc[d]);
        }
      }
      double diag = B.s(F_DIAG, n), invj = B.s(F_INVJ, n);
#pragma unroll
      for (int x = 0; x < 5; ++x)
        B.v(F_DQ, x + 1, n) = B.v(F_DQS, x + 1, n) - (acc[0][x] + acc[1][x] + acc[2][x]) / invj / diag;
    }
    __syncthreads();
  }
  // q = q + dq on the updated box
  long N1 = b1.size();
  for (long t = threadIdx.x; t < N1; t += blockDim.x) {
    int i = b1.is + (int)(t % nx1);
    long r = t / nx1;
    int j = b1.js + (int)(r % ny1);
    int k = b1.ks + (int)(r / ny1);
    long n = B.at(i, j, k);
#pragma unroll
    for (int x = 1; x <= 5; ++x) B.v(F_Q, x, n) = B.v(F_Q, x, n) + B.v(F_DQ, x, n);
  }
}

}  // namespace aero
