// Wall forces and lift / drag of clcd_output (sub_output_forceintegration.f90:
// 8-479, 3-D branch :182-457, 2-D branch :48-180, force_compute :481-509) on
// the device: one thread per wall quad (2-D: wall edge) of every wall
// subface, a fixed-order reduction of the pressure and viscous force
// components, then cl and cd.  The per-quad arithmetic keeps the reference's
// operation order, including its mix of metric components in the wall-normal
// vector and, in 2-D, its 0.25 viscosity average on face 3 (:128); only the
// order of the sums over quads differs from the serial loop.
#include <cmath>

#include "aero_device.cuh"
#include "aero_kernels.h"

namespace aero {

namespace {

// Grid spacing along direction d at node (i,j,k) of the physical box, as
// init_spacing (sub_init_spacing.f90:36-111) stores it: the distance to the
// next node, the last node repeating the previous one; 0 along k when the
// block has a single k-plane.
__device__ __forceinline__ double spacing_at(const BlockView& B, int d, int i, int j, int k) {
  const Box& b0 = B.b0;
  int ijk[3] = {i, j, k};
  const int hi[3] = {b0.ie, b0.je, b0.ke};
  if (d == 2 && b0.ke <= b0.ks) return 0.0;
  if (ijk[d] == hi[d]) ijk[d] -= 1;
  int nx[3] = {ijk[0], ijk[1], ijk[2]};
  nx[d] += 1;
  long a = B.at(ijk[0], ijk[1], ijk[2]), b = B.at(nx[0], nx[1], nx[2]);
  double dx = B.s(F_X, b) - B.s(F_X, a);
  double dy = B.s(F_Y, b) - B.s(F_Y, a);
  double dz = B.s(F_Z, b) - B.s(F_Z, a);
  return sqrt(p2(dx) + p2(dy) + p2(dz));
}

}  // namespace

__global__ void k_forces(const BlockView* __restrict__ blocks, const WallFace* __restrict__ walls, int nwall,
                         long nquad, CaseConsts cc, double* __restrict__ part) {
  long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double f[6] = {0, 0, 0, 0, 0, 0};
  if (q < nquad) {
    int w = 0;
    while (w + 1 < nwall && walls[w + 1].qoff <= q) ++w;
    const WallFace& W = walls[w];
    const BlockView& B = blocks[W.block];
    const int D = (W.face - 1) / 2;
    const bool low = W.face % 2 == 1;
    const int T1 = D == 0 ? 1 : 0, T2 = D == 2 ? 1 : 2;
    long r = q - W.qoff;
    int t1 = W.lo1 + (int)(r % W.n1);
    int t2 = W.lo2 + (int)(r / W.n1);
    const int w0 = W.w0, w1 = low ? w0 + 1 : w0 - 1;
    const int c1 = 3 * D + 1, c2 = 3 * D + 2, c3 = 3 * D + 3;
    if (B.planar()) {
      // 2-D edge (t1, t1+1): velocity and the unit normal from the two nodes
      // one layer in, pressure and viscosity from the two wall nodes, s the
      // edge's spacing along the wall, dn the mean spacing normal to it
      int a[3], b[3];
      a[T1] = t1; a[T2] = t2; a[D] = w1;
      b[T1] = t1 + 1; b[T2] = t2; b[D] = w1;
      const long ia = B.at(a[0], a[1], a[2]), ib = B.at(b[0], b[1], b[2]);
      a[D] = w0; b[D] = w0;
      const long wa = B.at(a[0], a[1], a[2]), wb = B.at(b[0], b[1], b[2]);
      double uc = (B.v(F_PRI, 2, ia) + B.v(F_PRI, 2, ib)) * 0.5;
      double vc = (B.v(F_PRI, 3, ia) + B.v(F_PRI, 3, ib)) * 0.5;
      double wc = 0.0;
      double pc = (B.v(F_PRI, 5, wa) + B.v(F_PRI, 5, wb)) * 0.5;
      double t00 = 1.0 / sqrt(p2(B.v(F_DXIDX, c1, ia)) + p2(B.v(F_DXIDX, c2, ia)) + p2(B.v(F_DXIDX, c3, ia)));
      double t10 = 1.0 / sqrt(p2(B.v(F_DXIDX, c1, ib)) + p2(B.v(F_DXIDX, c2, ib)) + p2(B.v(F_DXIDX, c3, ib)));
      const double sgn = low ? -1.0 : 1.0;
      double n3[3];
#pragma unroll
      for (int x = 0; x < 3; ++x)
        n3[x] = sgn * ((B.v(F_DXIDX, c1 + x, ia) * t00 + B.v(F_DXIDX, c1 + x, ib) * t10) * 0.5);
      double miuc = (B.v(F_AMU, 3, wa) + B.v(F_AMU, 3, wb)) * (W.face == 3 ? 0.25 : 0.5);
      double area = spacing_at(B, T1, a[0], a[1], a[2]);
      double dn = (spacing_at(B, D, a[0], a[1], a[2]) + spacing_at(B, D, b[0], b[1], b[2])) * 0.5;
      double u3[3] = {uc, vc, wc};
      double un = uc * n3[0] + vc * n3[1] + wc * n3[2];
#pragma unroll
      for (int x = 0; x < 3; ++x) {
        f[x] = (pc - cc.p_0) * area * n3[x];
        f[3 + x] = miuc * (u3[x] - un * n3[x]) / dn * area / cc.re;
      }
    } else {
    const int da[4] = {0, 1, 0, 1}, db[4] = {0, 0, 1, 1};  // corners 00, 10, 01, 11
    long ni[4], nw[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      int ijk[3];
      ijk[T1] = t1 + da[c];
      ijk[T2] = t2 + db[c];
      ijk[D] = w1;
      ni[c] = B.at(ijk[0], ijk[1], ijk[2]);
      ijk[D] = w0;
      nw[c] = B.at(ijk[0], ijk[1], ijk[2]);
    }
    auto avg = [&](int fid, int comp, const long* nn) {
      return (B.v(fid, comp, nn[0]) + B.v(fid, comp, nn[1]) + B.v(fid, comp, nn[2]) + B.v(fid, comp, nn[3])) *
             0.25;
    };
    double uc = avg(F_PRI, 2, ni), vc = avg(F_PRI, 3, ni), wc = avg(F_PRI, 4, ni);
    double pc = avg(F_PRI, 5, nw);
    double t[4];
#pragma unroll
    for (int c = 0; c < 4; ++c)
      t[c] = 1.0 / sqrt(p2(B.v(F_DXIDX, c1, ni[c])) + p2(B.v(F_DXIDX, c2, ni[c])) + p2(B.v(F_DXIDX, c3, ni[c])));
    auto mix = [&](int ca, int cb) {
      return (B.v(F_DXIDX, ca, ni[0]) * t[0] + B.v(F_DXIDX, ca, ni[1]) * t[1] + B.v(F_DXIDX, cb, ni[2]) * t[2] +
              B.v(F_DXIDX, cb, ni[3]) * t[3]) *
             0.25;
    };
    const double sgn = low ? -1.0 : 1.0;
    double n3[3] = {sgn * mix(c1, c2), sgn * mix(c3, c1), sgn * mix(c2, c3)};
    double miuc = avg(F_AMU, 3, nw);
    int ijk[3];
    ijk[T1] = t1;
    ijk[T2] = t2;
    ijk[D] = w0;
    double area = spacing_at(B, T1, ijk[0], ijk[1], ijk[2]) * spacing_at(B, T2, ijk[0], ijk[1], ijk[2]);
    double dn = spacing_at(B, D, ijk[0], ijk[1], ijk[2]);
    double u3[3] = {uc, vc, wc};
    double un = uc * n3[0] + vc * n3[1] + wc * n3[2];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
      f[x] = (pc - cc.p_0) * area * n3[x];
      f[3 + x] = miuc * (u3[x] - un * n3[x]) / dn * area / cc.re;
    }
    }
  }
  __shared__ double sm[6][32];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double x = f[c];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sm[c][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    int nwp = blockDim.x >> 5;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      double x = threadIdx.x < nwp ? sm[c][threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (threadIdx.x == 0) part[6 * blockIdx.x + c] = x;
    }
  }
}

// Sums the partials in a fixed order and forms cl, cd (:463-466).
__global__ void k_forces_final(const double* __restrict__ part, int npart, CaseConsts cc, double sref,
                               double* __restrict__ out8) {
  __shared__ double sm[6][256];
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int p = threadIdx.x; p < npart; p += blockDim.x)
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] += part[6 * p + c];
#pragma unroll
  for (int c = 0; c < 6; ++c) sm[c][threadIdx.x] = v[c];
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int c = 0; c < 6; ++c) sm[c][threadIdx.x] += sm[c][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double fp[3] = {sm[0][0], sm[1][0], sm[2][0]}, fv[3] = {sm[3][0], sm[4][0], sm[5][0]};
    double div = 1.0 / (0.5 * cc.d_0 * cc.u_0 * cc.u_0 * sref);
    for (int x = 0; x < 3; ++x) {
      out8[x] = fp[x];
      out8[3 + x] = fv[x];
    }
    out8[6] = ((fp[1] + fv[1]) * cc.cos_aoa - (fp[0] + fv[0]) * cc.sin_aoa) * div;
    out8[7] = ((fp[1] + fv[1]) * cc.sin_aoa + (fp[0] + fv[0]) * cc.cos_aoa) * div;
  }
}

// surface_output (sub_output_surface.f90:8-118): x, y, z and the pressure
// coefficient cp = (p - p0) / qinf, p0 = d_0 t_0 / gamma / ma^2 and
// qinf = 0.5 d_0 u_0^2 (:25-26), at every node of every wall subface, in the
// reference's write order (block, subface, then k, j, i).  One thread per
// node writes its four values contiguously, so the host copy is the file's
// row order.
__global__ void k_surface_cp(const BlockView* __restrict__ blocks, const SurfZone* __restrict__ zones, int nzone,
                             long nnode, CaseConsts cc_launch, double* __restrict__ out) {
  long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nnode) return;
  int z = 0;
  while (z + 1 < nzone && zones[z + 1].off <= q) ++z;
  const SurfZone& Z = zones[z];
  const BlockView& B = blocks[Z.block];
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
  long r = q - Z.off;
  int i = Z.is + (int)(r % Z.nx);
  r /= Z.nx;
  int j = Z.js + (int)(r % Z.ny);
  int k = Z.ks + (int)(r / Z.ny);
  long n = B.at(i, j, k);
  double p0 = cc.p_0;  // formed as d_0 * t_0 / gamma / ma / ma, as at :25
  double qinf = 0.5 * cc.d_0 * p2(cc.u_0);
  double p = B.v(F_PRI, 5, n);
  out[4 * q + 0] = B.s(F_X, n);
  out[4 * q + 1] = B.s(F_Y, n);
  out[4 * q + 2] = B.s(F_Z, n);
  out[4 * q + 3] = (p - p0) / qinf;
}

}  // namespace aero
