// 2nd-order Crank-Nicolson dual-time advance (crank2nd,
// sub_timeadvancement_2ndcrank.f90:1-466, 3-D) and update_q0 (main.f90:692-711).
//
// crank2nd is an approximately factorised point-implicit update: a forward
// and a backward recurrence along every i line, then every j line, then every
// k line of the updated box.  Lines of one direction are independent, so each
// is one thread walking its line; the per-point arithmetic is the
// reference's.  dq lives in the first five planes of the FVH scratch field
// (natural order, zero outside the updated box).  q0 holds the two earlier
// time levels: component plane (l+1) + 2*(c-1) is q0(l, c), l = -1, 0.
#include <cmath>

#include "aero_device.cuh"
#include "aero_kernels.h"

namespace aero {

namespace {

constexpr double kAlph = 0.5;

__device__ __forceinline__ double& q0v(const BlockView& B, int l, int c, long n) {
  return B.v(F_Q0, 1 + (l + 1) + 2 * (c - 1), n);
}
__device__ __forceinline__ double& dqv(const BlockView& B, int c, long n) {
  return B.f[F_FVH][(long)(c - 1) * B.plane + n];
}

// rou = |U| + c|grad| along the direction whose metric row starts at cb (:92-106)
__device__ __forceinline__ double crank_rou(const BlockView& B, int cb, long n) {
  double u = B.v(F_PRI, 2, n), v = B.v(F_PRI, 3, n), w = B.v(F_PRI, 4, n), c = B.v(F_PRI, 7, n);
  double x0 = B.v(F_DXIDX, cb, n), y0 = B.v(F_DXIDX, cb + 1, n), z0 = B.v(F_DXIDX, cb + 2, n);
  double temp = p2(x0) + p2(y0) + p2(z0);
  temp = sqrt(temp);
  double cu = u * x0 + v * y0 + w * z0;
  return fabs(cu) + fabs(c * temp);
}

// The neighbour term of one recurrence step (:107-161): the flux-Jacobian
// product of neighbour nb with its dq, with +rou (forward) or -rou (backward).
__device__ __forceinline__ void crank_a(const BlockView& B, int cb, long nb, double r, double hdv, double gamma,
                                        bool fwd, double a[5]) {
  double u = B.v(F_PRI, 2, nb), v = B.v(F_PRI, 3, nb), w = B.v(F_PRI, 4, nb), c = B.v(F_PRI, 7, nb);
  double dxidx0 = B.v(F_DXIDX, cb, nb), dxidy0 = B.v(F_DXIDX, cb + 1, nb), dxidz0 = B.v(F_DXIDX, cb + 2, nb);
  double q2 = 0.5 * (p2(u) + p2(v) + p2(w));
  double h = p2(c) / (gamma - 1.0) + q2;
  double cu = dxidx0 * u + dxidy0 * v + dxidz0 * w;
  double s1 = dqv(B, 1, nb), s2 = dqv(B, 2, nb), s3 = dqv(B, 3, nb), s4 = dqv(B, 4, nb), s5 = dqv(B, 5, nb);
  double b1 = hdv * (-(cu * s1) + dxidx0 * s2 + dxidy0 * s3 + dxidz0 * s4);
  double b2 = hdv * (q2 * s1 - u * s2 - v * s3 - w * s4 + s5) * (gamma - 1.0);
  double b3 = fwd ? hdv * (cu + r) : hdv * (cu - r);
  a[0] = b1 + b3 * s1;
  a[1] = b1 * u + b2 * dxidx0 + b3 * s2;
  a[2] = b1 * v + b2 * dxidy0 + b3 * s3;
  a[3] = b1 * w + b2 * dxidz0 + b3 * s4;
  a[4] = b1 * h + b2 * cu + b3 * s5;
}

}  // namespace

// :62-87: rhs = rhsi + rhsv, then the dual-time form with alph = 1/2, on the
// updated nodes.
__global__ void k_crank_rhs(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const Box& b1 = B.b1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b1.size()) return;
  int i = b1.is + (int)(t % b1.nx());
  long r = t / b1.nx();
  int j = b1.js + (int)(r % b1.ny());
  int k = b1.ks + (int)(r / b1.ny());
  long n = B.at(i, j, k);
  const double alph_i = 1.0 / (1.0 + kAlph);
  double dt = B.s(F_DT, n), ij = B.s(F_INVJ, n);
#pragma unroll
  for (int c = 1; c <= 5; ++c) {
    double rhs = B.v(F_RHSI, c, n) + B.v(F_RHSV, c, n);
    B.v(F_RHS, c, n) = alph_i * (rhs * dt - ((1.0 + kAlph) * B.v(F_Q, c, n) - (1.0 + 2.0 * kAlph) * q0v(B, 0, c, n) +
                                             kAlph * q0v(B, -1, c, n)) * ij);
  }
}

// One direction's recurrences: thread = one line of the updated box along
// direction d (0: i, 1: j, 2: k).  The forward recurrence of the k lines
// starts at ks1+1 and the backward one at ke1-1 (:352, :398), as in the
// reference; along i and j they cover the whole line.
__global__ void k_crank_sweep(const BlockView* __restrict__ blocks, int d, double gamma) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const Box& b1 = B.b1;
  const int n1[3] = {b1.nx(), b1.ny(), b1.nz()};
  const int lo[3] = {b1.is, b1.js, b1.ks};
  const int u1 = d == 0 ? 1 : 0, u2 = d == 2 ? 1 : 2;  // the two other directions
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)n1[u1] * n1[u2]) return;
  int ijk[3];
  ijk[u1] = lo[u1] + (int)(t % n1[u1]);
  ijk[u2] = lo[u2] + (int)(t / n1[u1]);
  ijk[d] = lo[d];
  const long st = d == 0 ? 1 : (d == 1 ? (long)B.nx : (long)B.nx * B.ny);
  const long n0 = B.at(ijk[0], ijk[1], ijk[2]);  // first updated node of the line
  const int len = n1[d];
  const int cb = 3 * d + 1;
  const double inv1 = 1.0 + kAlph;
  double a[5];
  // forward
  int f0 = d == 2 ? 1 : 0;
  double rprev = crank_rou(B, cb, n0 + (f0 - 1) * st);
  for (int x = f0; x < len; ++x) {
    long n = n0 + x * st, nb = n - st;
    double r = crank_rou(B, cb, n);
    double dtsub = B.s(F_DT, n) / inv1;
    crank_a(B, cb, nb, rprev, 0.5 * dtsub, gamma, true, a);
    double div = 1.0 / (1.0 + dtsub * r);
#pragma unroll
    for (int c = 1; c <= 5; ++c) {
      double base = d == 0 ? B.v(F_RHS, c, n) : dqv(B, c, n);
      dqv(B, c, n) = div * (base + a[c - 1]);
    }
    rprev = r;
  }
  // backward
  int b0 = d == 2 ? len - 2 : len - 1;
  if (b0 < 0) return;
  rprev = crank_rou(B, cb, n0 + (b0 + 1) * st);
  for (int x = b0; x >= 0; --x) {
    long n = n0 + x * st, nb = n + st;
    double r = crank_rou(B, cb, n);
    double dtsub = B.s(F_DT, n) / inv1;
    crank_a(B, cb, nb, rprev, 0.5 * dtsub, gamma, false, a);
    double div = 1.0 / (1.0 + dtsub * r);
#pragma unroll
    for (int c = 1; c <= 5; ++c) dqv(B, c, n) = dqv(B, c, n) - div * a[c - 1];
    rprev = r;
  }
}

// :455-462: q += dq / inv_j on the updated nodes.
__global__ void k_crank_update(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const Box& b1 = B.b1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b1.size()) return;
  int i = b1.is + (int)(t % b1.nx());
  long r = t / b1.nx();
  int j = b1.js + (int)(r % b1.ny());
  int k = b1.ks + (int)(r / b1.ny());
  long n = B.at(i, j, k);
  double ij = B.s(F_INVJ, n);
#pragma unroll
  for (int c = 1; c <= 5; ++c) B.v(F_Q, c, n) = B.v(F_Q, c, n) + dqv(B, c, n) / ij;
}

// main.f90:692-711 on the physical nodes.
__global__ void k_update_q0(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const Box& b0 = B.b0;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b0.size()) return;
  int i = b0.is + (int)(t % b0.nx());
  long r = t / b0.nx();
  int j = b0.js + (int)(r % b0.ny());
  int k = b0.ks + (int)(r / b0.ny());
  long n = B.at(i, j, k);
#pragma unroll
  for (int c = 1; c <= 5; ++c) {
    q0v(B, -1, c, n) = q0v(B, 0, c, n);
    q0v(B, 0, c, n) = B.v(F_Q, c, n);
  }
}

}  // namespace aero
