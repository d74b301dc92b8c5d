// One-time geometry on the GPU: grid metrics and 1/J (conservative metric form
// of sub_init_gridtransformation.f90), grid spacing (sub_init_spacing.f90) and
// the wall distance (sub_init_walldist.f90).
//
// The reference differentiates on five regions per direction: the "main"
// region (the two other indices physical, the full box along the direction,
// one-sided at the box ends) and four ghost slabs (one other index in a ghost
// layer, the direction's index physical, one-sided at the physical ends).
// Nodes outside every region (ghost corners) are never written.  Here each
// thread decides which region its node is in and applies that region's rule,
// so every written value is computed exactly as the reference computes it.
#include <cmath>

#include "aero_device.cuh"
#include "aero_kernels.h"

namespace aero {

namespace {

__device__ __forceinline__ bool in_range(int x, int lo, int hi) { return x >= lo && x <= hi; }

// Region rule for a derivative along direction d at node (i,j,k): returns
// false when the reference never writes the node, else the ends to use for
// the one-sided differences.
__device__ __forceinline__ bool deriv_region(const BlockView& B, int d, int i, int j, int k, int& lo,
                                             int& hi) {
  const int idx[3] = {i, j, k};
  const int lo0[3] = {B.b0.is, B.b0.js, B.b0.ks}, hi0[3] = {B.b0.ie, B.b0.je, B.b0.ke};
  const int lof[3] = {B.b.is, B.b.js, B.b.ks}, hif[3] = {B.b.ie, B.b.je, B.b.ke};
  int o1 = (d + 1) % 3, o2 = (d + 2) % 3;
  bool p1 = in_range(idx[o1], lo0[o1], hi0[o1]);
  bool p2_ = in_range(idx[o2], lo0[o2], hi0[o2]);
  if (p1 && p2_) {
    lo = lof[d]; hi = hif[d];
    return true;
  }
  if ((p1 != p2_) && in_range(idx[d], lo0[d], hi0[d])) {
    lo = lo0[d]; hi = hi0[d];
    return true;
  }
  return false;
}

__device__ __forceinline__ double dcentral(double fm, double f0, double fp, int pos, int lo, int hi) {
  if (pos == lo) return fp - f0;
  if (pos == hi) return f0 - fm;
  return (fp - fm) / 2.0;
}

}  // namespace

// Pass 1 (sub_init_gridtransformation.f90:107-520): dx/dxi, dx/deta, dx/dzeta
// (3 components each, into the 15-plane scratch field, planes 3*d + c) and
// 1/J on the nodes with at most one index in a ghost layer.
__global__ void k_metric_pass1(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= B.b.size()) return;
  int i = B.b.is + (int)(n % B.nx);
  long r = n / B.nx;
  int j = B.b.js + (int)(r % B.ny);
  int k = B.b.ks + (int)(r / B.ny);
  const long st[3] = {1, (long)B.nx, (long)B.nx * B.ny};
  const int pos[3] = {i, j, k};
  const int lof[3] = {B.b.is, B.b.js, B.b.ks}, hif[3] = {B.b.ie, B.b.je, B.b.ke};
  const double* X[3] = {B.f[F_X], B.f[F_Y], B.f[F_Z]};
  double* D = B.f[F_FVH];
  long P = B.plane;
  double der[3][3];  // der[d][c] = d x_c / d xi_d
  for (int d = 0; d < 3; ++d) {
    if (d == 2 && B.planar()) {  // 2-D (:270-273): d x / d zeta = (0, 0, 1) everywhere
      for (int c = 0; c < 3; ++c) {
        der[2][c] = c == 2 ? 1.0 : 0.0;
        D[(6 + c) * P + n] = der[2][c];
      }
      continue;
    }
    int lo, hi;
    bool on = deriv_region(B, d, i, j, k, lo, hi);
    for (int c = 0; c < 3; ++c) {
      double v = 0.0;
      if (on) {
        double f0 = X[c][n];
        double fp = pos[d] < hif[d] ? X[c][n + st[d]] : 0.0;
        double fm = pos[d] > lof[d] ? X[c][n - st[d]] : 0.0;
        v = dcentral(fm, f0, fp, pos[d], lo, hi);
      }
      der[d][c] = v;
      D[(3 * d + c) * P + n] = v;
    }
  }
  int nout = !in_range(i, B.b0.is, B.b0.ie) + !in_range(j, B.b0.js, B.b0.je) + !in_range(k, B.b0.ks, B.b0.ke);
  if (nout <= 1) {
    double dxdxi0 = der[0][0], dxdeta0 = der[1][0], dxdzeta0 = der[2][0];
    double dydxi0 = der[0][1], dydeta0 = der[1][1], dydzeta0 = der[2][1];
    double dzdxi0 = der[0][2], dzdeta0 = der[1][2], dzdzeta0 = der[2][2];
    B.s(F_INVJ, n) = dxdxi0 * dydeta0 * dzdzeta0 + dxdeta0 * dydzeta0 * dzdxi0 +
                     dxdzeta0 * dydxi0 * dzdeta0 - dxdzeta0 * dydeta0 * dzdxi0 -
                     dxdxi0 * dydzeta0 * dzdeta0 - dxdeta0 * dydxi0 * dzdzeta0;
  }
}

// The six products of one temp array at node m (:559-584):
// which = 0: tempxi, 1: tempeta, 2: tempzeta.
__device__ __forceinline__ void temp_products(const BlockView& B, int which, long m, double t[6]) {
  const double* D = B.f[F_FVH];
  long P = B.plane;
  double x = B.s(F_X, m), y = B.s(F_Y, m), z = B.s(F_Z, m);
  auto der = [&](int d, int c) { return D[(3 * d + c) * P + m]; };
  // first three use d/dzeta (tempxi, tempeta) or d/deta (tempzeta); last three
  // use d/deta (tempxi) or d/dxi (tempeta, tempzeta)
  int da = which == 2 ? 1 : 2;
  int db = which == 0 ? 1 : 0;
  t[0] = der(da, 1) * z;
  t[1] = der(da, 2) * x;
  t[2] = der(da, 0) * y;
  t[3] = der(db, 1) * z;
  t[4] = der(db, 2) * x;
  t[5] = der(db, 0) * y;
}

// Pass 2 (:587-865): derivatives of the temp products along their own
// direction (same five-region rule), the metrics dxidx = difference / (1/J)
// over the full box (2-D: from the in-plane derivatives, :543-557), and
// alpha, beta, gamma.
__global__ void k_metric_pass2(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= B.b.size()) return;
  int i = B.b.is + (int)(n % B.nx);
  long r = n / B.nx;
  int j = B.b.js + (int)(r % B.ny);
  int k = B.b.ks + (int)(r / B.ny);
  double ij = B.s(F_INVJ, n);
  double m[9];
  if (B.planar()) {
    // 2-D (:543-557): the in-plane metrics from dx/dxi and dx/deta (scratch
    // planes 0-2 and 3-5) over the whole box
    const double* D = B.f[F_FVH];
    const long P = B.plane;
    m[0] = D[4 * P + n] / ij;
    m[1] = -D[3 * P + n] / ij;
    m[2] = 0.0;
    m[3] = -D[1 * P + n] / ij;
    m[4] = D[0 * P + n] / ij;
    m[5] = 0.0;
    m[6] = 0.0;
    m[7] = 0.0;
    m[8] = 1.0;
  } else {
  const long st[3] = {1, (long)B.nx, (long)B.nx * B.ny};
  const int pos[3] = {i, j, k};
  const int lof[3] = {B.b.is, B.b.js, B.b.ks}, hif[3] = {B.b.ie, B.b.je, B.b.ke};
  double dd[3][6];  // dd[0] = tempxixi, dd[1] = tempetaeta, dd[2] = tempzetazeta
  for (int d = 0; d < 3; ++d) {
    int lo, hi;
    if (!deriv_region(B, d, i, j, k, lo, hi)) {
      for (int c = 0; c < 6; ++c) dd[d][c] = 0.0;
      continue;
    }
    double t0[6], tp[6], tm[6];
    temp_products(B, d, n, t0);
    if (pos[d] < hif[d]) temp_products(B, d, n + st[d], tp);
    else for (int c = 0; c < 6; ++c) tp[c] = 0.0;
    if (pos[d] > lof[d]) temp_products(B, d, n - st[d], tm);
    else for (int c = 0; c < 6; ++c) tm[c] = 0.0;
    for (int c = 0; c < 6; ++c) dd[d][c] = dcentral(tm[c], t0[c], tp[c], pos[d], lo, hi);
  }
  m[0] = (dd[2][0] - dd[1][0]) / ij;
  m[1] = (dd[2][1] - dd[1][1]) / ij;
  m[2] = (dd[2][2] - dd[1][2]) / ij;
  m[3] = (dd[0][0] - dd[2][3]) / ij;
  m[4] = (dd[0][1] - dd[2][4]) / ij;
  m[5] = (dd[0][2] - dd[2][5]) / ij;
  m[6] = (dd[1][3] - dd[0][3]) / ij;
  m[7] = (dd[1][4] - dd[0][4]) / ij;
  m[8] = (dd[1][5] - dd[0][5]) / ij;
  }
  for (int c = 0; c < 9; ++c) B.v(F_DXIDX, c + 1, n) = m[c];
  double x1 = m[0], x2 = m[1], x3 = m[2], e1 = m[3], e2 = m[4], e3 = m[5], z1 = m[6], z2 = m[7], z3 = m[8];
  B.v(F_ALPHA, 1, n) = (x1 * x1 + x2 * x2 + x3 * x3) * ij;
  B.v(F_ALPHA, 2, n) = (x1 * e1 + x2 * e2 + x3 * e3) * ij;
  B.v(F_ALPHA, 3, n) = (x1 * z1 + x2 * z2 + x3 * z3) * ij;
  B.v(F_BETA, 1, n) = (e1 * x1 + e2 * x2 + e3 * x3) * ij;
  B.v(F_BETA, 2, n) = (e1 * e1 + e2 * e2 + e3 * e3) * ij;
  B.v(F_BETA, 3, n) = (e1 * z1 + e2 * z2 + e3 * z3) * ij;
  B.v(F_GAMMA, 1, n) = (z1 * x1 + z2 * x2 + z3 * x3) * ij;
  B.v(F_GAMMA, 2, n) = (z1 * e1 + z2 * e2 + z3 * e3) * ij;
  B.v(F_GAMMA, 3, n) = (z1 * z1 + z2 * z2 + z3 * z3) * ij;
}

// sub_init_spacing.f90:36-111: the largest node-to-node distance along the
// three directions at every physical node (spacing) .
__global__ void k_spacing(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  const Box& b0 = B.b0;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b0.size()) return;
  int i = b0.is + (int)(t % b0.nx());
  long r = t / b0.nx();
  int j = b0.js + (int)(r % b0.ny());
  int k = b0.ks + (int)(r / b0.ny());
  long n = B.at(i, j, k);
  const long st[3] = {1, (long)B.nx, (long)B.nx * B.ny};
  const int pos[3] = {i, j, k};
  const int hi0[3] = {b0.ie, b0.je, b0.ke};
  double spc[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < 3; ++d) {
    if (d == 2 && b0.ke <= b0.ks) break;  // spck stays 0 for a single k-plane
    long a = pos[d] < hi0[d] ? n : n - st[d];  // last node copies the previous interval
    long c = a + st[d];
    double dx = B.s(F_X, c) - B.s(F_X, a);
    double dy = B.s(F_Y, c) - B.s(F_Y, a);
    double dz = B.s(F_Z, c) - B.s(F_Z, a);
    spc[d] = sqrt(p2(dx) + p2(dy) + p2(dz));
  }
  B.s(F_SPACING, n) = fmax(fmax(spc[0], spc[1]), spc[2]);
}

// Gathers the coordinates of every wall-subface node (sub_init_readbcinfo.f90:
// 286-388 face planes at is0/ie0/js0/je0/ks0/ke0).
__global__ void k_wall_points(const BlockView* __restrict__ blocks, const AvgSrc* __restrict__ wall,
                              long nwall, double* __restrict__ xyz) {
  long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nwall) return;
  const BlockView& B = blocks[wall[e].blk];
  long n = wall[e].n;
  xyz[3 * e + 0] = B.s(F_X, n);
  xyz[3 * e + 1] = B.s(F_Y, n);
  xyz[3 * e + 2] = B.s(F_Z, n);
}

// sub_init_walldist.f90:39-90: distance from each physical node to the nearest
// wall node (brute force).  sqrt is monotone and correctly rounded, so the
// square root of the smallest squared distance equals the smallest distance.
// The wall nodes of block m's case are xyz entries [range[2m], range[2m] +
// range[2m+1]).
__global__ void k_walldist(const BlockView* __restrict__ blocks, const double* __restrict__ xyz,
                           const long* __restrict__ range) {
  const BlockView& B = blocks[blockIdx.y];
  const long first = range[2 * blockIdx.y], nwall = range[2 * blockIdx.y + 1];
  const Box& b0 = B.b0;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  extern __shared__ double tile[];
  bool act = t < b0.size();
  long n = 0;
  double xx = 0, yy = 0, zz = 0;
  if (act) {
    int i = b0.is + (int)(t % b0.nx());
    long r = t / b0.nx();
    int j = b0.js + (int)(r % b0.ny());
    int k = b0.ks + (int)(r / b0.ny());
    n = B.at(i, j, k);
    xx = B.s(F_X, n); yy = B.s(F_Y, n); zz = B.s(F_Z, n);
  }
  double best = INFINITY;
  for (long base = 0; base < nwall; base += blockDim.x) {
    long w = base + threadIdx.x;
    if (w < nwall) {
      tile[3 * threadIdx.x + 0] = xyz[3 * (first + w) + 0];
      tile[3 * threadIdx.x + 1] = xyz[3 * (first + w) + 1];
      tile[3 * threadIdx.x + 2] = xyz[3 * (first + w) + 2];
    }
    __syncthreads();
    long cnt = min((long)blockDim.x, nwall - base);
    if (act)
      for (long q = 0; q < cnt; ++q) {
        double d2 = p2(xx - tile[3 * q]) + p2(yy - tile[3 * q + 1]) + p2(zz - tile[3 * q + 2]);
        best = fmin(best, d2);
      }
    __syncthreads();
  }
  if (act) B.s(F_DIST, n) = nwall > 0 ? fmin(sqrt(best), 1.0e9) : 1.0e9;
}

}  // namespace aero
