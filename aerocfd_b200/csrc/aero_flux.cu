// Residual kernels: primitive variables, inviscid flux (WENO3 + Roe), viscous
// flux and the local time step.  Every kernel keeps the reference's operation
// order (this file is compiled with -fmad=false in the parity build), so the FP64
// path reproduces the CPU result to the last bit except in libm functions.
#include <cmath>

#include "aero_device.cuh"
#include "aero_kernels.h"

namespace aero {

// ----------------------------------------------------------------- primitives
// sub_getpri_v.f90:19-62, over the full box of every block.
__global__ void k_getpri(const BlockView* __restrict__ blocks, CaseConsts cc_launch, unsigned* status) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
  long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long N = B.b.size();
  if (n >= N) return;
  double d = B.v(F_Q, 1, n);
  double u = B.v(F_Q, 2, n) / d;
  double v = B.v(F_Q, 3, n) / d;
  double w = B.v(F_Q, 4, n) / d;
  double q2 = 0.5 * (u * u + v * v + w * w);
  double e = B.v(F_Q, 5, n) / d;
  double t = (e - q2) / cc.cv;
  double p = (B.v(F_Q, 5, n) - q2 * d) * (cc.gamma - 1.0);
  double c = sqrt(cc.gamma * p / d);
  B.v(F_PRI, 1, n) = d;
  B.v(F_PRI, 2, n) = u;
  B.v(F_PRI, 3, n) = v;
  B.v(F_PRI, 4, n) = w;
  B.v(F_PRI, 5, n) = p;
  B.v(F_PRI, 6, n) = t;
  B.v(F_PRI, 7, n) = c;
  if (d < 0.0) {
    if (status) atomicOr(status, (unsigned)ST_NEG_DENSITY);
    B.raise(ST_NEG_DENSITY);
  }
}

// -------------------------------------------------------------- inviscid flux
// WENO3 weights and state (sub_inviscid_upwind.f90:32-41 right, :57-66 left).
// The reference's four divisions per state are formed with fewer: the
// smoothness weight of a difference d, 1 / (3 (eps + d^2)^2), is one
// reciprocal (correctly rounded, as 1.0 / x), the reference's 2 / x is twice
// it (exact: scaling by 2 commutes with rounding for these normal values,
// x >= 3e-12), and the two normalisations w = a / (a1 + a2) share the
// reciprocal of the sum through div_rn_lean, which equals the quotient to
// the bit.  (d^2 is the same for d and -d, so weno_faces' shared weights are
// the reference's s1 / s2 of either state.)
__device__ __forceinline__ double weno_weight(double d) {
  const double eps = 1.0e-6;
  return 1.0 / (3.0 * p2(eps + p2(d)));
}
// w1 (c1) + w2 (c2) with w = a / (a1 + a2)
__device__ __forceinline__ double weno_mix(double a1, double a2, double c1, double c2) {
  const double sum = a1 + a2, rs = 1.0 / sum;
  return div_rn_lean(a1, sum, rs) * c1 + div_rn_lean(a2, sum, rs) * c2;
}
__device__ __forceinline__ double weno_right(double u1, double u2, double u3) {
  const double a1 = weno_weight(u2 - u3);
  const double a2 = 2.0 * weno_weight(u1 - u2);
  return weno_mix(a1, a2, -u3 / 2.0 + 3.0 * u2 / 2.0, u2 / 2.0 + u1 / 2.0);
}
__device__ __forceinline__ double weno_left(double u1, double u2, double u3) {
  const double a1 = weno_weight(u2 - u1);
  const double a2 = 2.0 * weno_weight(u3 - u2);
  return weno_mix(a1, a2, -u1 / 2.0 + 3.0 * u2 / 2.0, u2 / 2.0 + u3 / 2.0);
}

// Roe flux at face (node n, node n+s) along `coord` from primitive left/right
// states d, u, v, w, p (sub_inviscid_splitting.f90:65-162).
__device__ __forceinline__ void roe_prim(const BlockView& B, int coord, long n, long ns, double dl, double ul,
                                         double vl, double wl, double pl, double dr, double ur, double vr, double wr,
                                         double pr, double gamma, double flux[5]) {
  int c1 = coord * 3 - 2;
  double ja = B.s(F_INVJ, n), jb = B.s(F_INVJ, ns);
  double dxidx1 = 0.5 * (B.v(F_DXIDX, c1, n) * ja + B.v(F_DXIDX, c1, ns) * jb);
  double dxidy1 = 0.5 * (B.v(F_DXIDX, c1 + 1, n) * ja + B.v(F_DXIDX, c1 + 1, ns) * jb);
  double dxidz1 = 0.5 * (B.v(F_DXIDX, c1 + 2, n) * ja + B.v(F_DXIDX, c1 + 2, ns) * jb);
  // the divisions that share a divisor go through its reciprocal and
  // div_rn_lean (each quotient the same to the bit)
  double temp = sqrt(p2(dxidx1) + p2(dxidy1) + p2(dxidz1));
  const double rtemp = 1.0 / temp;
  double dxidx0 = div_rn_lean(dxidx1, temp, rtemp), dxidy0 = div_rn_lean(dxidy1, temp, rtemp);
  double dxidz0 = div_rn_lean(dxidz1, temp, rtemp);

  double hl = gamma * pl / ((gamma - 1.0) * dl) + 0.5 * (p2(ul) + p2(vl) + p2(wl));
  double hr = gamma * pr / ((gamma - 1.0) * dr) + 0.5 * (p2(ur) + p2(vr) + p2(wr));
  double uul = ul * dxidx1 + vl * dxidy1 + wl * dxidz1;
  double uur = ur * dxidx1 + vr * dxidy1 + wr * dxidz1;
  double ubarl = div_rn_lean(uul, temp, rtemp), ubarr = div_rn_lean(uur, temp, rtemp);

  double fl0 = dl * uul, fl1 = dl * ul * uul + dxidx1 * pl, fl2 = dl * vl * uul + dxidy1 * pl;
  double fl3 = dl * wl * uul + dxidz1 * pl, fl4 = dl * hl * uul;
  double fr0 = dr * uur, fr1 = dr * ur * uur + dxidx1 * pr, fr2 = dr * vr * uur + dxidy1 * pr;
  double fr3 = dr * wr * uur + dxidz1 * pr, fr4 = dr * hr * uur;

  double tmpp = sqrt(dr / dl);
  double avd = sqrt(dl * dr);
  const double op = 1.0 + tmpp, rop = 1.0 / op;
  double avu = div_rn_lean(ul + ur * tmpp, op, rop);
  double avv = div_rn_lean(vl + vr * tmpp, op, rop);
  double avw = div_rn_lean(wl + wr * tmpp, op, rop);
  double avh = div_rn_lean(hl + hr * tmpp, op, rop);
  double ava = sqrt((gamma - 1.0) * (avh - 0.5 * (p2(avu) + p2(avv) + p2(avw))));
  double avuu = avu * dxidx0 + avv * dxidy0 + avw * dxidz0;

  const double delt = 0.06;
  constexpr double kTwoDelt = 2.0 * 0.06, kRcpTwoDelt = 1.0 / (2.0 * 0.06);
  double lam[5] = {fabs(avuu - ava), fabs(avuu), fabs(avuu), fabs(avuu), fabs(avuu + ava)};
#pragma unroll
  for (int m = 0; m < 5; ++m) {  // Harten entropy fix (sub_inviscid_splitting.f90:122-130)
    double tmp = copysign(1.0, delt - lam[m]);
    double tmp1 = 0.5 * (1.0 - tmp);
    double tmp2 = 0.5 * (1.0 + tmp);
    double harten = div_rn_lean(p2(lam[m]) + p2(delt), kTwoDelt, kRcpTwoDelt);
    lam[m] = tmp1 * lam[m] + tmp2 * harten;
  }
  double deltad = dr - dl, deltap = pr - pl;
  double deltau = ur - ul, deltav = vr - vl, deltaw = wr - wl;
  double deltauu = ubarr - ubarl;
  // p2(ava) and 2 p2(ava) (exactly twice it, so 1/(2 p2(ava)) is exactly half
  // of 1/p2(ava)) as divisors
  const double ava2 = p2(ava), rava2 = 1.0 / ava2;
  double alpha1 = lam[1] * (deltad - div_rn_lean(deltap, ava2, rava2));
  double alpha2 = div_rn_lean(lam[4] * (deltap + avd * ava * deltauu), 2.0 * ava2, 0.5 * rava2);
  double alpha3 = div_rn_lean(lam[0] * (deltap - avd * ava * deltauu), 2.0 * ava2, 0.5 * rava2);
  double alpha4 = alpha1 + alpha2 + alpha3;
  double alpha5 = ava * (alpha2 - alpha3);
  double alpha6 = lam[1] * (avd * deltau - avd * deltauu * dxidx0);
  double alpha7 = lam[1] * (avd * deltav - avd * deltauu * dxidy0);
  double alpha8 = lam[1] * (avd * deltaw - avd * deltauu * dxidz0);
  double f0 = alpha4;
  double f1 = avu * alpha4 + alpha5 * dxidx0 + alpha6;
  double f2 = avv * alpha4 + alpha5 * dxidy0 + alpha7;
  double f3 = avw * alpha4 + alpha5 * dxidz0 + alpha8;
  double f4 = avh * alpha4 + avuu * alpha5 + avu * alpha6 + avv * alpha7 + avw * alpha8 -
              p2(ava) * alpha1 / (gamma - 1.0);
  flux[0] = 0.5 * (fl0 + fr0 - temp * f0);
  flux[1] = 0.5 * (fl1 + fr1 - temp * f1);
  flux[2] = 0.5 * (fl2 + fr2 - temp * f2);
  flux[3] = 0.5 * (fl3 + fr3 - temp * f3);
  flux[4] = 0.5 * (fl4 + fr4 - temp * f4);
}
// The same from conservative left/right states, converted to primitives as
// sub_inviscid1.f90:58-74 does.
__device__ __forceinline__ void roe_face(const BlockView& B, int coord, long n, long ns,
                                         const double ulc[5], const double urc[5], double gamma,
                                         double flux[5]) {
  // the four divisions by the density of each side through its reciprocal
  const double rl = 1.0 / ulc[0], rr = 1.0 / urc[0];
  double dl = ulc[0], ul = div_rn_lean(ulc[1], dl, rl), vl = div_rn_lean(ulc[2], dl, rl);
  double wl = div_rn_lean(ulc[3], dl, rl);
  double pl = (ulc[4] - div_rn_lean(0.5 * (p2(ulc[1]) + p2(ulc[2]) + p2(ulc[3])), dl, rl)) * (gamma - 1.0);
  double dr = urc[0], ur = div_rn_lean(urc[1], dr, rr), vr = div_rn_lean(urc[2], dr, rr);
  double wr = div_rn_lean(urc[3], dr, rr);
  double pr = (urc[4] - div_rn_lean(0.5 * (p2(urc[1]) + p2(urc[2]) + p2(urc[3])), dr, rr)) * (gamma - 1.0);
  roe_prim(B, coord, n, ns, dl, ul, vl, wl, pl, dr, ur, vr, wr, pr, gamma, flux);
}

// Flux through face pos+1/2 along `coord` starting at node (i,j,k); pos is the
// node's index along coord, lo/hi the full-box bounds along coord, st the
// linear stride along coord.
// q(c, m) supplies q's component c at node index m (global memory, or a
// shared-memory copy in the staged face kernel).
template <class Q>
__device__ __forceinline__ void face_flux_q(const BlockView& B, int coord, long n, int pos, int lo, int hi,
                                            long st, double gamma, double flux[5], Q q) {
  double ulc[5], urc[5];
  bool rone = (pos == hi - 1);  // right state one-sided at ie-1 (:25-26)
  bool lone = (pos == lo);      // left state one-sided at is (:50-51)
#pragma unroll
  for (int c = 1; c <= 5; ++c) {
    double f0 = q(c, n);
    double fp = q(c, n + st);
    // the weight of the face's own difference serves both states (the
    // reference's s2 of each)
    const double a_mid = (rone && lone) ? 0.0 : weno_weight(fp - f0);
    if (rone) {
      urc[c - 1] = fp;
    } else {
      double fpp = q(c, n + 2 * st);
      urc[c - 1] = weno_mix(weno_weight(fp - fpp), 2.0 * a_mid, -fpp / 2.0 + 3.0 * fp / 2.0, fp / 2.0 + f0 / 2.0);
    }
    if (lone) {
      ulc[c - 1] = f0;
    } else {
      double fm = q(c, n - st);
      ulc[c - 1] = weno_mix(weno_weight(f0 - fm), 2.0 * a_mid, -fm / 2.0 + 3.0 * f0 / 2.0, f0 / 2.0 + fp / 2.0);
    }
  }
  roe_face(B, coord, n, n + st, ulc, urc, gamma, flux);
}
__device__ __forceinline__ void face_flux(const BlockView& B, int coord, long n, int pos, int lo,
                                          int hi, long st, double gamma, double flux[5]) {
  face_flux_q(B, coord, n, pos, lo, hi, st, gamma, flux, [&](int c, long m) { return B.v(F_Q, c, m); });
}

// ------------------------------------------------ inviscid flux, mixed precision
// The same face flux with FP32 arithmetic where it only forms increments:
// the WENO3 states are written as the centre value (FP64) plus a correction
// w1*(u2-u1)/2 + w2*(u3-u2)/2 evaluated in FP32 from FP64 differences, and the
// Roe flux as the FP64 central part 0.5*(F_L + F_R) minus the FP32 dissipation
// 0.5*|grad xi/J|*|A|*dU, whose inputs are FP64 differences.  Near a
// converged state every FP32 term is proportional to a jump, so its rounding
// error shrinks with the residual instead of setting a floor.
__device__ __forceinline__ double weno_corr(double um, double u0, double up) {
  // the reference's left state weno_left(um, u0, up) =
  //   w1*(-um/2 + 3u0/2) + w2*(u0/2 + up/2) = u0 + w1*(u0-um)/2 + w2*(up-u0)/2
  const float eps = 1.0e-6f;
  float d1 = (float)(u0 - um), d2 = (float)(up - u0);
  float a1 = 1.0f / (3.0f * (eps + d1 * d1) * (eps + d1 * d1));
  float a2 = 2.0f / (3.0f * (eps + d2 * d2) * (eps + d2 * d2));
  float w1 = a1 / (a1 + a2), w2 = a2 / (a1 + a2);
  return (double)(0.5f * (w1 * d1 + w2 * d2));
}

__device__ __forceinline__ void roe_face_mixed(const BlockView& B, int coord, long n, long ns,
                                               const double ulc[5], const double urc[5], double gamma,
                                               double flux[5]) {
  // primitives with one FP64 reciprocal of the density per side (the FP64
  // path divides each component, as the reference)
  const double rl = 1.0 / ulc[0], rr = 1.0 / urc[0];
  double dl = ulc[0], ul = ulc[1] * rl, vl = ulc[2] * rl, wl = ulc[3] * rl;
  double pl = (ulc[4] - 0.5 * (p2(ulc[1]) + p2(ulc[2]) + p2(ulc[3])) * rl) * (gamma - 1.0);
  double dr = urc[0], ur = urc[1] * rr, vr = urc[2] * rr, wr = urc[3] * rr;
  double pr = (urc[4] - 0.5 * (p2(urc[1]) + p2(urc[2]) + p2(urc[3])) * rr) * (gamma - 1.0);
  int c1 = coord * 3 - 2;
  double ja = B.s(F_INVJ, n), jb = B.s(F_INVJ, ns);
  double dxidx1 = 0.5 * (B.v(F_DXIDX, c1, n) * ja + B.v(F_DXIDX, c1, ns) * jb);
  double dxidy1 = 0.5 * (B.v(F_DXIDX, c1 + 1, n) * ja + B.v(F_DXIDX, c1 + 1, ns) * jb);
  double dxidz1 = 0.5 * (B.v(F_DXIDX, c1 + 2, n) * ja + B.v(F_DXIDX, c1 + 2, ns) * jb);
  const double gg = gamma / (gamma - 1.0);
  double hl = gg * pl * rl + 0.5 * (p2(ul) + p2(vl) + p2(wl));
  double hr = gg * pr * rr + 0.5 * (p2(ur) + p2(vr) + p2(wr));
  double uul = ul * dxidx1 + vl * dxidy1 + wl * dxidz1;
  double uur = ur * dxidx1 + vr * dxidy1 + wr * dxidz1;
  // central part (FP64)
  double fc[5];
  fc[0] = dl * uul + dr * uur;
  fc[1] = dl * ul * uul + dxidx1 * pl + (dr * ur * uur + dxidx1 * pr);
  fc[2] = dl * vl * uul + dxidy1 * pl + (dr * vr * uur + dxidy1 * pr);
  fc[3] = dl * wl * uul + dxidz1 * pl + (dr * wr * uur + dxidz1 * pr);
  fc[4] = dl * hl * uul + dr * hr * uur;
  // dissipation (FP32 on FP64 differences)
  const float g = (float)gamma;
  float mx = (float)dxidx1, my = (float)dxidy1, mz = (float)dxidz1;
  float temp = sqrtf(mx * mx + my * my + mz * mz);
  float nx = mx / temp, ny = my / temp, nz = mz / temp;
  float fdl = (float)dl, fdr = (float)dr;
  float tmpp = sqrtf(fdr / fdl);
  float avd = sqrtf(fdl * fdr);
  float inv1 = 1.0f / (1.0f + tmpp);
  float avu = ((float)ul + (float)ur * tmpp) * inv1;
  float avv = ((float)vl + (float)vr * tmpp) * inv1;
  float avw = ((float)wl + (float)wr * tmpp) * inv1;
  float avh = ((float)hl + (float)hr * tmpp) * inv1;
  float ava2 = (g - 1.0f) * (avh - 0.5f * (avu * avu + avv * avv + avw * avw));
  float ava = sqrtf(ava2);
  float avuu = avu * nx + avv * ny + avw * nz;
  const float delt = 0.06f;
  float lam[5] = {fabsf(avuu - ava), fabsf(avuu), fabsf(avuu), fabsf(avuu), fabsf(avuu + ava)};
#pragma unroll
  for (int m = 0; m < 5; ++m)  // Harten entropy fix
    if (lam[m] < delt) lam[m] = (lam[m] * lam[m] + delt * delt) / (2.0f * delt);
  float deltad = (float)(dr - dl), deltap = (float)(pr - pl);
  float deltau = (float)(ur - ul), deltav = (float)(vr - vl), deltaw = (float)(wr - wl);
  float deltauu = (float)(uur - uul) / temp;
  float alpha1 = lam[1] * (deltad - deltap / ava2);
  float alpha2 = lam[4] * (deltap + avd * ava * deltauu) / (2.0f * ava2);
  float alpha3 = lam[0] * (deltap - avd * ava * deltauu) / (2.0f * ava2);
  float alpha4 = alpha1 + alpha2 + alpha3;
  float alpha5 = ava * (alpha2 - alpha3);
  float alpha6 = lam[1] * avd * (deltau - deltauu * nx);
  float alpha7 = lam[1] * avd * (deltav - deltauu * ny);
  float alpha8 = lam[1] * avd * (deltaw - deltauu * nz);
  float fd[5];
  fd[0] = alpha4;
  fd[1] = avu * alpha4 + alpha5 * nx + alpha6;
  fd[2] = avv * alpha4 + alpha5 * ny + alpha7;
  fd[3] = avw * alpha4 + alpha5 * nz + alpha8;
  fd[4] = avh * alpha4 + avuu * alpha5 + avu * alpha6 + avv * alpha7 + avw * alpha8 - ava2 * alpha1 / (g - 1.0f);
#pragma unroll
  for (int c = 0; c < 5; ++c) flux[c] = 0.5 * fc[c] - (double)(0.5f * temp * fd[c]);
}

__device__ __forceinline__ void face_flux_mixed(const BlockView& B, int coord, long n, int pos, int lo, int hi,
                                                long st, double gamma, double flux[5]) {
  double ulc[5], urc[5];
  bool rone = (pos == hi - 1);
  bool lone = (pos == lo);
#pragma unroll
  for (int c = 1; c <= 5; ++c) {
    double f0 = B.v(F_Q, c, n);
    double fp = B.v(F_Q, c, n + st);
    // right state = weno_right(f0, fp, fpp) = weno_left(fpp, fp, f0) (mirror)
    urc[c - 1] = rone ? fp : fp + weno_corr(B.v(F_Q, c, n + 2 * st), fp, f0);
    ulc[c - 1] = lone ? f0 : f0 + weno_corr(B.v(F_Q, c, n - st), f0, fp);
  }
  roe_face_mixed(B, coord, n, n + st, ulc, urc, gamma, flux);
}

template <bool MIXED, int TILE>
__device__ __forceinline__ void inviscid_body(const BlockView* __restrict__ blocks, CaseConsts cc) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const Box& b1 = B.b1;
  __shared__ double dsm[3][5][TILE];
  long t = (long)blockIdx.x * TILE + threadIdx.x;
  long N1 = b1.size();
  int d = threadIdx.y;
  int ndir = cc.dimension == IFLAG_3D ? 3 : 2;
  long n = 0;
  if (t < N1) {
    int i = b1.is + (int)(t % b1.nx());
    long r = t / b1.nx();
    int j = b1.js + (int)(r % b1.ny());
    int k = b1.ks + (int)(r / b1.ny());
    n = B.at(i, j, k);
    if (d < ndir) {
      const long st = d == 0 ? 1 : (d == 1 ? (long)B.nx : (long)B.nx * B.ny);
      const int pos = d == 0 ? i : (d == 1 ? j : k);
      const int lo = d == 0 ? B.b.is : (d == 1 ? B.b.js : B.b.ks);
      const int hi = d == 0 ? B.b.ie : (d == 1 ? B.b.je : B.b.ke);
      double fm[5], fp[5];
      if (MIXED) {
        face_flux_mixed(B, d + 1, n - st, pos - 1, lo, hi, st, cc.gamma, fm);
        face_flux_mixed(B, d + 1, n, pos, lo, hi, st, cc.gamma, fp);
      } else {
        face_flux(B, d + 1, n - st, pos - 1, lo, hi, st, cc.gamma, fm);
        face_flux(B, d + 1, n, pos, lo, hi, st, cc.gamma, fp);
      }
#pragma unroll
      for (int c = 0; c < 5; ++c) dsm[d][c][threadIdx.x] = fp[c] - fm[c];
    }
  }
  __syncthreads();
  if (d == 0 && t < N1) {
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      double acc = -dsm[0][c][threadIdx.x];
      acc = acc - dsm[1][c][threadIdx.x];
      if (ndir == 3) acc = acc - dsm[2][c][threadIdx.x];
      B.v(F_RHSI, c + 1, n) = acc;
    }
  }
}

// sub_inviscid1.f90:8-189: rhsi on the updated nodes.  A CTA covers TILE
// nodes x 3 directions (TILE = 32, 64 or 128, picked by the autotuner); thread
// (x, d) computes the flux difference of direction d at its node (both
// faces), and the three differences are combined in the reference's order:
// rhsi = -dF; rhsi -= dG; rhsi -= dH.  The _mixed kernels use face_flux_mixed.
__global__ void k_inviscid_32(const BlockView* __restrict__ blocks, CaseConsts cc) { inviscid_body<false, 32>(blocks, cc); }
__global__ void k_inviscid_64(const BlockView* __restrict__ blocks, CaseConsts cc) { inviscid_body<false, 64>(blocks, cc); }
__global__ void k_inviscid_128(const BlockView* __restrict__ blocks, CaseConsts cc) { inviscid_body<false, 128>(blocks, cc); }
__global__ void k_inviscid_mixed_32(const BlockView* __restrict__ blocks, CaseConsts cc) { inviscid_body<true, 32>(blocks, cc); }
__global__ void k_inviscid_mixed_64(const BlockView* __restrict__ blocks, CaseConsts cc) { inviscid_body<true, 64>(blocks, cc); }
__global__ void k_inviscid_mixed_128(const BlockView* __restrict__ blocks, CaseConsts cc) { inviscid_body<true, 128>(blocks, cc); }

// Face-based variant of the same residual: every face flux once.
// k_inviscid_faces: thread = one face along direction d = blockIdx.z, the face
// between node n and its neighbour up in d, for every n of the updated box
// grown by one node down in d; the flux goes to plane 5*d + c of the FIH
// scratch (its own, so the viscous kernels may run at the same time).  k_inviscid_combine then forms
// rhsi = -dF; rhsi -= dG; rhsi -= dH as the per-node kernels do.
template <bool MIXED>
__device__ __forceinline__ void faces_body(const BlockView* __restrict__ blocks, CaseConsts cc) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const int d = blockIdx.z;
  if (d >= (cc.dimension == IFLAG_3D && !B.planar() ? 3 : 2)) return;
  const Box& b1 = B.b1;
  Box e = b1;
  if (d == 0) e.is -= 1; else if (d == 1) e.js -= 1; else e.ks -= 1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= e.size()) return;
  int i = e.is + (int)(t % e.nx());
  long r = t / e.nx();
  int j = e.js + (int)(r % e.ny());
  int k = e.ks + (int)(r / e.ny());
  long n = B.at(i, j, k);
  const long st = d == 0 ? 1 : (d == 1 ? (long)B.nx : (long)B.nx * B.ny);
  const int pos = d == 0 ? i : (d == 1 ? j : k);
  const int lo = d == 0 ? B.b.is : (d == 1 ? B.b.js : B.b.ks);
  const int hi = d == 0 ? B.b.ie : (d == 1 ? B.b.je : B.b.ke);
  double f[5];
  if (MIXED)
    face_flux_mixed(B, d + 1, n, pos, lo, hi, st, cc.gamma, f);
  else
    face_flux(B, d + 1, n, pos, lo, hi, st, cc.gamma, f);
  double* out = B.f[F_FIH] + (long)(5 * d) * B.plane + n;
#pragma unroll
  for (int c = 0; c < 5; ++c) out[(long)c * B.plane] = f[c];
}
__global__ void k_inviscid_faces(const BlockView* __restrict__ blocks, CaseConsts cc) { faces_body<false>(blocks, cc); }
// The same under register bounds for 6 or 8 resident CTAs of 128 threads per
// SM (more warps to hide the FP64 latency, at the cost of a few spills); the
// autotuner chooses.
__global__ void __launch_bounds__(128, 6) k_inviscid_faces_o6(const BlockView* __restrict__ blocks, CaseConsts cc) {
  faces_body<false>(blocks, cc);
}
__global__ void __launch_bounds__(128, 8) k_inviscid_faces_o8(const BlockView* __restrict__ blocks, CaseConsts cc) {
  faces_body<false>(blocks, cc);
}
// The mixed-precision face kernel under a register bound for 10 resident CTAs
// of 128 threads per SM (48 registers, a few spills).
__global__ void __launch_bounds__(128, 10) k_inviscid_faces_mixed_o10(const BlockView* __restrict__ blocks,
                                                                     CaseConsts cc) {
  faces_body<true>(blocks, cc);
}
__global__ void k_inviscid_faces_mixed(const BlockView* __restrict__ blocks, CaseConsts cc) { faces_body<true>(blocks, cc); }

// The FP64 face kernel with its WENO stencil values staged in shared memory
// (inviscid tile -10).  A CTA's 128 faces are consecutive in the face box (i
// fastest), so the nodes their stencils read (n - st .. n + 2 st) lie in one
// index range of the block, from the first face's node - st to the last
// face's node + 2 st, clamped to the block: about 150 nodes along i and 230
// along j on the plate's blocks.  The CTA copies that range of the five q
// components once, coalesced, and each face reads its four values per
// component from there; the metrics come from global memory as before.
// Where the range exceeds kStageSpan nodes (the k faces, whose stride is a
// whole plane, and long j strides) the faces read global memory.  The
// arithmetic is face_flux's, so the results are the same bits.
constexpr int kStageSpan = 512;
__global__ void __launch_bounds__(128, 8) k_inviscid_faces_staged(const BlockView* __restrict__ blocks,
                                                                 CaseConsts cc) {
  __shared__ double sq[5][kStageSpan];
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const int d = blockIdx.z;
  if (d >= (cc.dimension == IFLAG_3D && !B.planar() ? 3 : 2)) return;
  const Box& b1 = B.b1;
  Box e = b1;
  if (d == 0) e.is -= 1; else if (d == 1) e.js -= 1; else e.ks -= 1;
  const long nf = e.size();
  const long t0 = (long)blockIdx.x * blockDim.x;
  if (t0 >= nf) return;  // the whole CTA
  auto node_of = [&](long t) {
    int i = e.is + (int)(t % e.nx());
    long r = t / e.nx();
    int j = e.js + (int)(r % e.ny());
    int k = e.ks + (int)(r / e.ny());
    return B.at(i, j, k);
  };
  const long st = d == 0 ? 1 : (d == 1 ? (long)B.nx : (long)B.nx * B.ny);
  const long first = max(node_of(t0) - st, 0L);
  const long last = min(node_of(min(t0 + (long)blockDim.x, nf) - 1) + 2 * st, B.b.size() - 1);
  const long span = last - first + 1;
  const bool staged = span <= kStageSpan;  // the same for every thread of the CTA
  if (staged) {
    for (long x = threadIdx.x; x < 5 * span; x += blockDim.x) {
      const int c = (int)(x / span);
      const long o = x - c * span;
      sq[c][o] = B.v(F_Q, c + 1, first + o);
    }
    __syncthreads();
  }
  const long t = t0 + threadIdx.x;
  if (t >= nf) return;
  int i = e.is + (int)(t % e.nx());
  long r = t / e.nx();
  int j = e.js + (int)(r % e.ny());
  int k = e.ks + (int)(r / e.ny());
  long n = B.at(i, j, k);
  const int pos = d == 0 ? i : (d == 1 ? j : k);
  const int lo = d == 0 ? B.b.is : (d == 1 ? B.b.js : B.b.ks);
  const int hi = d == 0 ? B.b.ie : (d == 1 ? B.b.je : B.b.ke);
  double f[5];
  if (staged)
    face_flux_q(B, d + 1, n, pos, lo, hi, st, cc.gamma, f, [&](int c, long m) { return sq[c - 1][m - first]; });
  else
    face_flux(B, d + 1, n, pos, lo, hi, st, cc.gamma, f);
  double* out = B.f[F_FIH] + (long)(5 * d) * B.plane + n;
#pragma unroll
  for (int c = 0; c < 5; ++c) out[(long)c * B.plane] = f[c];
}

__global__ void k_inviscid_combine(const BlockView* __restrict__ blocks, CaseConsts cc) {
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
  const long st[3] = {1, (long)B.nx, (long)B.nx * B.ny};
  const int ndir = cc.dimension == IFLAG_3D ? 3 : 2;
  const double* F = B.f[F_FIH];
  const long P = B.plane;
#pragma unroll
  for (int c = 0; c < 5; ++c) {
    double acc = -(F[(long)c * P + n] - F[(long)c * P + n - st[0]]);
    acc = acc - (F[(long)(5 + c) * P + n] - F[(long)(5 + c) * P + n - st[1]]);
    if (ndir == 3) acc = acc - (F[(long)(10 + c) * P + n] - F[(long)(10 + c) * P + n - st[2]]);
    B.v(F_RHSI, c + 1, n) = acc;
  }
}

// ----------------------------------- the reconstruction and the Riemann solver
// thirdorder_weno (sub_inviscid_upwind.f90:1-179) and roe_3d
// (sub_inviscid_splitting.f90:1-172) as stand-alone routines over one block
// (view 0), for the drop-in entry points aero_thirdorder_weno / aero_roe_3d.
// Face i stands for i+1/2 along coord, for the faces of r0 grown by one node
// down along coord (the routines' loops); the states and fluxes are those of
// face_flux and roe_face, the same operations.
__device__ __forceinline__ bool face_node(const Box& r0, int coord, long t, int& i, int& j, int& k) {
  Box e = r0;
  if (coord == 1) e.is -= 1; else if (coord == 2) e.js -= 1; else e.ks -= 1;
  if (t >= e.size()) return false;
  i = e.is + (int)(t % e.nx());
  long r = t / e.nx();
  j = e.js + (int)(r % e.ny());
  k = e.ks + (int)(r / e.ny());
  return true;
}
// f in the F_Q slot, df (left state for direction -1, right for +1) in F_RHSI
__global__ void k_weno3_states(const BlockView* __restrict__ blocks, int coord, int direction, Box r0) {
  const BlockView& B = blocks[0];
  int i, j, k;
  if (!face_node(r0, coord, (long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const long n = B.at(i, j, k);
  const long st = coord == 1 ? 1 : (coord == 2 ? (long)B.nx : (long)B.nx * B.ny);
  const int pos = coord == 1 ? i : (coord == 2 ? j : k);
  const int lo = coord == 1 ? B.b.is : (coord == 2 ? B.b.js : B.b.ks);
  const int hi = coord == 1 ? B.b.ie : (coord == 2 ? B.b.je : B.b.ke);
#pragma unroll
  for (int c = 1; c <= 5; ++c) {
    double v;
    if (direction == 1)
      v = pos == hi - 1 ? B.v(F_Q, c, n + st) : weno_right(B.v(F_Q, c, n), B.v(F_Q, c, n + st), B.v(F_Q, c, n + 2 * st));
    else
      v = pos == lo ? B.v(F_Q, c, n) : weno_left(B.v(F_Q, c, n - st), B.v(F_Q, c, n), B.v(F_Q, c, n + st));
    B.v(F_RHSI, c, n) = v;
  }
}
// primitive ql in the F_Q slot, qr in F_RHSI, the flux to F_RHSV
__global__ void k_roe_states(const BlockView* __restrict__ blocks, int coord, Box r0, double gamma) {
  const BlockView& B = blocks[0];
  int i, j, k;
  if (!face_node(r0, coord, (long)blockIdx.x * blockDim.x + threadIdx.x, i, j, k)) return;
  const long n = B.at(i, j, k);
  const long st = coord == 1 ? 1 : (coord == 2 ? (long)B.nx : (long)B.nx * B.ny);
  double f[5];
  roe_prim(B, coord, n, n + st, B.v(F_Q, 1, n), B.v(F_Q, 2, n), B.v(F_Q, 3, n), B.v(F_Q, 4, n), B.v(F_Q, 5, n),
           B.v(F_RHSI, 1, n), B.v(F_RHSI, 2, n), B.v(F_RHSI, 3, n), B.v(F_RHSI, 4, n), B.v(F_RHSI, 5, n), gamma, f);
#pragma unroll
  for (int c = 0; c < 5; ++c) B.v(F_RHSV, c + 1, n) = f[c];
}

// ------------------------------------------- extension inviscid schemes
// The reference defines iflag_5thweno = 5 and iflag_5thwcns = 8
// (module_flags.f90:68, 71) but has no code for them (GetBufferLength stops on
// any scheme but the 3rd-order WENO, main.f90:636-653).  These are the
// published methods, on three ghost layers, in FP64:
//  * 5: Steger-Warming flux-vector splitting (J. Comput. Phys. 40, 1981) of
//    the contravariant flux at the nodes, the split fluxes reconstructed at
//    the faces with the WENO5 of Jiang & Shu (J. Comput. Phys. 126, 1996);
//  * 8: WCNS5 (Deng & Zhang, J. Comput. Phys. 165, 2000): 5th-order weighted
//    nonlinear interpolation of the conservative variables to the faces
//    (linear weights 1/16, 10/16, 5/16, Jiang-Shu smoothness indicators), the
//    reference's Roe flux there, and the 4th-order hybrid face/node
//    difference F'_i = 4/3 (F_i+1/2 - F_i-1/2) - 1/6 (F_i+1 - F_i-1), written
//    as the face flux G = 4/3 F_i+1/2 - (F_i + F_i+1)/6 so that the combine
//    kernel's difference applies.  For uniform flow G equals the reference's
//    face flux, so freestream preservation is the reference scheme's.
// Near a physical boundary, where a stencil would leave the box, the WENO5
// reconstructions drop to WENO3 and then 1st order, and WCNS5 uses the
// reference's WENO3 + Roe face.
namespace {

constexpr double kEps5 = 1.0e-6;

// WENO5 value at the right edge of v2 from v0..v4 (Jiang & Shu).
__device__ __forceinline__ double weno5_edge(double v0, double v1, double v2, double v3, double v4) {
  double b0 = 13.0 / 12.0 * p2(v0 - 2.0 * v1 + v2) + 0.25 * p2(v0 - 4.0 * v1 + 3.0 * v2);
  double b1 = 13.0 / 12.0 * p2(v1 - 2.0 * v2 + v3) + 0.25 * p2(v1 - v3);
  double b2 = 13.0 / 12.0 * p2(v2 - 2.0 * v3 + v4) + 0.25 * p2(3.0 * v2 - 4.0 * v3 + v4);
  double a0 = 0.1 / p2(kEps5 + b0);
  double a1 = 0.6 / p2(kEps5 + b1);
  double a2 = 0.3 / p2(kEps5 + b2);
  double q0 = (2.0 * v0 - 7.0 * v1 + 11.0 * v2) / 6.0;
  double q1 = (-v1 + 5.0 * v2 + 2.0 * v3) / 6.0;
  double q2 = (2.0 * v2 + 5.0 * v3 - v4) / 6.0;
  return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
}
// WENO3 value at the right edge of v1 from v0..v2 (Jiang & Shu).
__device__ __forceinline__ double weno3_edge(double v0, double v1, double v2) {
  double b0 = p2(v1 - v0);
  double b1 = p2(v2 - v1);
  double a0 = (1.0 / 3.0) / p2(kEps5 + b0);
  double a1 = (2.0 / 3.0) / p2(kEps5 + b1);
  double q0 = (3.0 * v1 - v0) / 2.0;
  double q1 = (v1 + v2) / 2.0;
  return (a0 * q0 + a1 * q1) / (a0 + a1);
}
// WCNS5 interpolation at the right edge of v2 from v0..v4 (Deng & Zhang).
__device__ __forceinline__ double wcns5_edge(double v0, double v1, double v2, double v3, double v4) {
  double b0 = 13.0 / 12.0 * p2(v0 - 2.0 * v1 + v2) + 0.25 * p2(v0 - 4.0 * v1 + 3.0 * v2);
  double b1 = 13.0 / 12.0 * p2(v1 - 2.0 * v2 + v3) + 0.25 * p2(v1 - v3);
  double b2 = 13.0 / 12.0 * p2(v2 - 2.0 * v3 + v4) + 0.25 * p2(3.0 * v2 - 4.0 * v3 + v4);
  double a0 = 0.0625 / p2(kEps5 + b0);
  double a1 = 0.625 / p2(kEps5 + b1);
  double a2 = 0.3125 / p2(kEps5 + b2);
  double q0 = (3.0 * v0 - 10.0 * v1 + 15.0 * v2) / 8.0;
  double q1 = (-v1 + 6.0 * v2 + 3.0 * v3) / 8.0;
  double q2 = (3.0 * v2 + 6.0 * v3 - v4) / 8.0;
  return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
}

// Steger-Warming part of the contravariant flux along `coord` at node n
// (metric K = grad xi * inv_j): PLUS takes the eigenvalues' positive parts,
// otherwise the negative parts.
template <bool PLUS>
__device__ __forceinline__ void sw_part(const BlockView& B, int coord, long n, double gamma, double f[5]) {
  double rho = B.v(F_Q, 1, n);
  double u = B.v(F_Q, 2, n) / rho, v = B.v(F_Q, 3, n) / rho, w = B.v(F_Q, 4, n) / rho;
  double q2 = 0.5 * (u * u + v * v + w * w);
  double p = (B.v(F_Q, 5, n) - rho * q2) * (gamma - 1.0);
  double c = sqrt(gamma * p / rho);
  const int c1 = 3 * coord - 2;
  double ij = B.s(F_INVJ, n);
  double kx = B.v(F_DXIDX, c1, n) * ij, ky = B.v(F_DXIDX, c1 + 1, n) * ij, kz = B.v(F_DXIDX, c1 + 2, n) * ij;
  double kn = sqrt(kx * kx + ky * ky + kz * kz);
  double nx = kx / kn, ny = ky / kn, nz = kz / kn;
  double uu = kx * u + ky * v + kz * w;
  double ub = nx * u + ny * v + nz * w;
  double l1 = uu, l4 = uu + c * kn, l5 = uu - c * kn;
  if (PLUS) {
    l1 = 0.5 * (l1 + fabs(l1));
    l4 = 0.5 * (l4 + fabs(l4));
    l5 = 0.5 * (l5 + fabs(l5));
  } else {
    l1 = 0.5 * (l1 - fabs(l1));
    l4 = 0.5 * (l4 - fabs(l4));
    l5 = 0.5 * (l5 - fabs(l5));
  }
  double h = c * c / (gamma - 1.0) + q2;
  double coef = rho / (2.0 * gamma);
  double a1 = 2.0 * (gamma - 1.0) * l1;
  f[0] = coef * (a1 + l4 + l5);
  f[1] = coef * (a1 * u + l4 * (u + c * nx) + l5 * (u - c * nx));
  f[2] = coef * (a1 * v + l4 * (v + c * ny) + l5 * (v - c * ny));
  f[3] = coef * (a1 * w + l4 * (w + c * nz) + l5 * (w - c * nz));
  f[4] = coef * (a1 * q2 + l4 * (h + c * ub) + l5 * (h - c * ub));
}

// Contravariant flux along `coord` at node n with the node's metric, the
// left-state expressions of roe_face.
__device__ __forceinline__ void node_flux(const BlockView& B, int coord, long n, double gamma, double f[5]) {
  double d = B.v(F_Q, 1, n);
  double u = B.v(F_Q, 2, n) / d, v = B.v(F_Q, 3, n) / d, w = B.v(F_Q, 4, n) / d;
  double p = (B.v(F_Q, 5, n) - 0.5 * (p2(B.v(F_Q, 2, n)) + p2(B.v(F_Q, 3, n)) + p2(B.v(F_Q, 4, n))) / d) *
             (gamma - 1.0);
  const int c1 = 3 * coord - 2;
  double ij = B.s(F_INVJ, n);
  double kx = B.v(F_DXIDX, c1, n) * ij, ky = B.v(F_DXIDX, c1 + 1, n) * ij, kz = B.v(F_DXIDX, c1 + 2, n) * ij;
  double h = gamma * p / ((gamma - 1.0) * d) + 0.5 * (p2(u) + p2(v) + p2(w));
  double uu = u * kx + v * ky + w * kz;
  f[0] = d * uu;
  f[1] = d * u * uu + kx * p;
  f[2] = d * v * uu + ky * p;
  f[3] = d * w * uu + kz * p;
  f[4] = d * h * uu;
}

// The face pos+1/2 of node n along direction d (blockIdx.z) for every n of the
// updated box grown by one node down in d, as faces_body: the geometry of one
// thread.
struct FaceAt {
  long n, st;
  int pos, lo, hi;
};
__device__ __forceinline__ bool face_at(const BlockView& B, int d, FaceAt& F) {
  if (d == 2 && B.planar()) return false;  // 2-D: no zeta faces (sub_inviscid1.f90:137)
  Box e = B.b1;
  if (d == 0) e.is -= 1; else if (d == 1) e.js -= 1; else e.ks -= 1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= e.size()) return false;
  int i = e.is + (int)(t % e.nx());
  long r = t / e.nx();
  int j = e.js + (int)(r % e.ny());
  int k = e.ks + (int)(r / e.ny());
  F.n = B.at(i, j, k);
  F.st = d == 0 ? 1 : (d == 1 ? (long)B.nx : (long)B.nx * B.ny);
  F.pos = d == 0 ? i : (d == 1 ? j : k);
  F.lo = d == 0 ? B.b.is : (d == 1 ? B.b.js : B.b.ks);
  F.hi = d == 0 ? B.b.ie : (d == 1 ? B.b.je : B.b.ke);
  return true;
}

// Mixed precision of the extension schemes: every reconstructed value is the
// FP64 centre value plus an FP32 correction built from FP64 differences
// (q_k - v2 and the smoothness indicators rewritten in differences), so the
// FP32 rounding scales with the jumps.  a = v0-v1, b = v1-v2, c = v3-v2,
// e = v4-v3 around the centre v2; `lin` selects the WENO5 reconstruction
// (d = 0.1, 0.6, 0.3) or the WCNS5 interpolation (d = 1/16, 10/16, 5/16).
template <bool WCNS>
__device__ __forceinline__ double edge5_corr(double v0, double v1, double v2, double v3, double v4) {
  const float eps = 1.0e-6f;
  float a = (float)(v0 - v1), b = (float)(v1 - v2), c = (float)(v3 - v2), e = (float)(v4 - v3);
  float s0 = a - b, t0 = a - 3.0f * b;
  float s1 = b + c, t1 = b - c;
  float s2 = e - c, t2 = e - 3.0f * c;
  float b0 = 13.0f / 12.0f * s0 * s0 + 0.25f * t0 * t0;
  float b1 = 13.0f / 12.0f * s1 * s1 + 0.25f * t1 * t1;
  float b2 = 13.0f / 12.0f * s2 * s2 + 0.25f * t2 * t2;
  float a0 = (WCNS ? 0.0625f : 0.1f) / ((eps + b0) * (eps + b0));
  float a1 = (WCNS ? 0.625f : 0.6f) / ((eps + b1) * (eps + b1));
  float a2 = (WCNS ? 0.3125f : 0.3f) / ((eps + b2) * (eps + b2));
  float q0, q1, q2;
  if (WCNS) {
    q0 = (3.0f * a - 7.0f * b) / 8.0f;
    q1 = (3.0f * c - b) / 8.0f;
    q2 = (5.0f * c - e) / 8.0f;
  } else {
    q0 = (2.0f * a - 5.0f * b) / 6.0f;
    q1 = (2.0f * c - b) / 6.0f;
    q2 = (4.0f * c - e) / 6.0f;
  }
  return (double)((a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2));
}
// WENO3 (Jiang & Shu) at the right edge of v1 as v1 + FP32 correction.
__device__ __forceinline__ double edge3_corr(double v0, double v1, double v2) {
  const float eps = 1.0e-6f;
  float a = (float)(v1 - v0), c = (float)(v2 - v1);
  float a0 = (1.0f / 3.0f) / ((eps + a * a) * (eps + a * a));
  float a1 = (2.0f / 3.0f) / ((eps + c * c) * (eps + c * c));
  return (double)((a0 * (0.5f * a) + a1 * (0.5f * c)) / (a0 + a1));
}

}  // namespace

// Steger-Warming + WENO5 face fluxes into FIH planes 5*d + c (then
// k_inviscid_combine).  F+ at pos+1/2 from nodes pos-2..pos+2, F- from
// pos-1..pos+3.
template <bool MIXED>
__device__ __forceinline__ void sw_weno5_body(const BlockView* __restrict__ blocks, CaseConsts cc) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const int d = blockIdx.z;
  FaceAt F;
  if (!face_at(B, d, F)) return;
  const int pos = F.pos, lo = F.lo, hi = F.hi;
  const long n = F.n, st = F.st;
  double out[5];
  {
    double v[5][5] = {};  // F+ at pos-2..pos+2 (those inside the box)
#pragma unroll
    for (int x = 0; x < 5; ++x)
      if (pos - 2 + x >= lo && pos - 2 + x <= hi) sw_part<true>(B, d + 1, n + (x - 2) * st, cc.gamma, v[x]);
    const bool five = pos - 2 >= lo && pos + 2 <= hi, three = pos - 1 >= lo && pos + 1 <= hi;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      if (MIXED)
        out[c] = v[2][c] + (five ? edge5_corr<false>(v[0][c], v[1][c], v[2][c], v[3][c], v[4][c])
                                 : (three ? edge3_corr(v[1][c], v[2][c], v[3][c]) : 0.0));
      else
        out[c] = five ? weno5_edge(v[0][c], v[1][c], v[2][c], v[3][c], v[4][c])
                      : (three ? weno3_edge(v[1][c], v[2][c], v[3][c]) : v[2][c]);
    }
  }
  {
    double v[5][5] = {};  // F- at pos-1..pos+3
#pragma unroll
    for (int x = 0; x < 5; ++x)
      if (pos - 1 + x >= lo && pos - 1 + x <= hi) sw_part<false>(B, d + 1, n + (x - 1) * st, cc.gamma, v[x]);
    const bool five = pos - 1 >= lo && pos + 3 <= hi, three = pos >= lo && pos + 2 <= hi;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
      double fm;
      if (MIXED)
        fm = v[2][c] + (five ? edge5_corr<false>(v[4][c], v[3][c], v[2][c], v[1][c], v[0][c])
                             : (three ? edge3_corr(v[3][c], v[2][c], v[1][c]) : 0.0));
      else
        fm = five ? weno5_edge(v[4][c], v[3][c], v[2][c], v[1][c], v[0][c])
                  : (three ? weno3_edge(v[3][c], v[2][c], v[1][c]) : v[2][c]);
      out[c] = out[c] + fm;
    }
  }
  double* o = B.f[F_FIH] + (long)(5 * d) * B.plane + n;
#pragma unroll
  for (int c = 0; c < 5; ++c) o[(long)c * B.plane] = out[c];
}
__global__ void k_faces_sw_weno5(const BlockView* __restrict__ blocks, CaseConsts cc) {
  sw_weno5_body<false>(blocks, cc);
}
__global__ void k_faces_sw_weno5_mixed(const BlockView* __restrict__ blocks, CaseConsts cc) {
  sw_weno5_body<true>(blocks, cc);
}

// WCNS5 face fluxes G into FIH planes 5*d + c (then k_inviscid_combine).
template <bool MIXED>
__device__ __forceinline__ void wcns5_body(const BlockView* __restrict__ blocks, CaseConsts cc) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const int d = blockIdx.z;
  FaceAt F;
  if (!face_at(B, d, F)) return;
  const int pos = F.pos;
  const long n = F.n, st = F.st;
  double out[5];
  if (pos - 2 >= F.lo && pos + 3 <= F.hi) {
    double ul[5], ur[5], fh[5], fa[5], fb[5];
#pragma unroll
    for (int c = 1; c <= 5; ++c) {
      double u0 = B.v(F_Q, c, n - 2 * st), u1 = B.v(F_Q, c, n - st), u2 = B.v(F_Q, c, n);
      double u3 = B.v(F_Q, c, n + st), u4 = B.v(F_Q, c, n + 2 * st), u5 = B.v(F_Q, c, n + 3 * st);
      if (MIXED) {
        ul[c - 1] = u2 + edge5_corr<true>(u0, u1, u2, u3, u4);
        ur[c - 1] = u3 + edge5_corr<true>(u5, u4, u3, u2, u1);
      } else {
        ul[c - 1] = wcns5_edge(u0, u1, u2, u3, u4);
        ur[c - 1] = wcns5_edge(u5, u4, u3, u2, u1);
      }
    }
    if (MIXED)
      roe_face_mixed(B, d + 1, n, n + st, ul, ur, cc.gamma, fh);
    else
      roe_face(B, d + 1, n, n + st, ul, ur, cc.gamma, fh);
    node_flux(B, d + 1, n, cc.gamma, fa);
    node_flux(B, d + 1, n + st, cc.gamma, fb);
#pragma unroll
    for (int c = 0; c < 5; ++c) out[c] = 4.0 / 3.0 * fh[c] - (fa[c] + fb[c]) / 6.0;
  } else if (MIXED) {
    face_flux_mixed(B, d + 1, n, pos, F.lo, F.hi, st, cc.gamma, out);
  } else {
    face_flux(B, d + 1, n, pos, F.lo, F.hi, st, cc.gamma, out);
  }
  double* o = B.f[F_FIH] + (long)(5 * d) * B.plane + n;
#pragma unroll
  for (int c = 0; c < 5; ++c) o[(long)c * B.plane] = out[c];
}
__global__ void k_faces_wcns5(const BlockView* __restrict__ blocks, CaseConsts cc) { wcns5_body<false>(blocks, cc); }
__global__ void k_faces_wcns5_mixed(const BlockView* __restrict__ blocks, CaseConsts cc) {
  wcns5_body<true>(blocks, cc);
}

// Zero-fills one field over the full box of every block (the reference's
// `rhsi = 0.d0`, sub_inviscid1.f90:40, and similar whole-array assignments).
__global__ void k_fill(const BlockView* __restrict__ blocks, int fid, int nc, double val) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long N = B.b.size();
  if (n >= N || !B.f[fid]) return;
  for (int c = 1; c <= nc; ++c) B.v(fid, c, n) = val;
}

// --------------------------------------------------------------- viscous flux
// Central difference along one direction inside the physical range, one-sided
// at its ends (sub_viscous.f90:106-178 and :296-340).
__device__ __forceinline__ double cdiff(const double* f, long n, long st, int pos, int lo, int hi) {
  if (pos == lo) return f[n + st] - f[n];
  if (pos == hi) return f[n] - f[n - st];
  return (f[n + st] - f[n - st]) / 2.0;
}

// sub_viscous.f90:187-293: gradients, Sutherland viscosity, stresses, heat flux,
// vorticity and the contravariant viscous fluxes on the physical nodes.  The
// fluxes fv,gv,hv (components 2..5 each) go to the FVH scratch field.
__device__ __forceinline__ void viscous_a_body(const BlockView* __restrict__ blocks, CaseConsts cc_launch, int store_dudx_tao) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
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
  const int lo[3] = {b0.is, b0.js, b0.ks};
  const int hi[3] = {b0.ie, b0.je, b0.ke};
  const double* pu = B.f[F_PRI] + 1 * B.plane;
  const double* pv = B.f[F_PRI] + 2 * B.plane;
  const double* pw = B.f[F_PRI] + 3 * B.plane;
  const double* pt = B.f[F_PRI] + 5 * B.plane;
  double gt[3] = {0, 0, 0}, gu[3] = {0, 0, 0}, gv[3] = {0, 0, 0}, gw[3] = {0, 0, 0};
  int ndir = cc.dimension == IFLAG_3D ? 3 : 2;
  for (int d = 0; d < ndir; ++d) {
    gt[d] = cdiff(pt, n, st[d], pos[d], lo[d], hi[d]);
    gu[d] = cdiff(pu, n, st[d], pos[d], lo[d], hi[d]);
    gv[d] = cdiff(pv, n, st[d], pos[d], lo[d], hi[d]);
    gw[d] = cdiff(pw, n, st[d], pos[d], lo[d], hi[d]);
  }
  double u0 = pu[n], v0 = pv[n], w0 = pw[n], t0 = pt[n];
  double amu1 = (1.0 + 124.0 / cc.tinf) / (t0 + 124.0 / cc.tinf) * crm::pow(t0, 1.5);
  double amu2 = B.v(F_AMU, 2, n);
  double amu3 = amu1 + amu2;
  B.v(F_AMU, 1, n) = amu1;
  B.v(F_AMU, 3, n) = amu3;
  double ki = cc.gamma * cc.cv * (amu1 / cc.prl + amu2 / cc.prt);
  double m[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) m[c] = B.v(F_DXIDX, c + 1, n);
  double tx = gt[0] * m[0] + gt[1] * m[3] + gt[2] * m[6];
  double ty = gt[0] * m[1] + gt[1] * m[4] + gt[2] * m[7];
  double tz = gt[0] * m[2] + gt[1] * m[5] + gt[2] * m[8];
  double du[9];
  const double* g[3] = {gu, gv, gw};
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) du[3 * a + c] = g[a][0] * m[c] + g[a][1] * m[c + 3] + g[a][2] * m[c + 6];
  double ta[6];
  ta[0] = amu3 * (4.0 / 3.0 * du[0] - 2.0 / 3.0 * (du[4] + du[8]));
  ta[1] = amu3 * (du[1] + du[3]);
  ta[2] = amu3 * (du[6] + du[2]);
  ta[3] = amu3 * (4.0 / 3.0 * du[4] - 2.0 / 3.0 * (du[0] + du[8]));
  ta[4] = amu3 * (du[7] + du[5]);
  ta[5] = amu3 * (4.0 / 3.0 * du[8] - 2.0 / 3.0 * (du[0] + du[4]));
  double bx = u0 * ta[0] + v0 * ta[1] + w0 * ta[2] + ki * tx;
  double by = u0 * ta[1] + v0 * ta[3] + w0 * ta[4] + ki * ty;
  double bz = u0 * ta[2] + v0 * ta[4] + w0 * ta[5] + ki * tz;
  B.s(F_VOR, n) = sqrt(p2(du[5] - du[7]) + p2(du[2] - du[6]) + p2(du[1] - du[3]));
  if (store_dudx_tao) {
#pragma unroll
    for (int c = 0; c < 9; ++c) B.v(F_DUDX, c + 1, n) = du[c];
#pragma unroll
    for (int c = 0; c < 6; ++c) B.v(F_TAO, c + 1, n) = ta[c];
  }
  double ij = B.s(F_INVJ, n);
  double* fvh = B.f[F_FVH];
  long P = B.plane;
  // fv/gv/hv components 2..5 -> FVH planes 0..3 (fv), 4..7 (gv), 8..11 (hv)
#pragma unroll
  for (int dd = 0; dd < 3; ++dd) {
    double x1 = m[3 * dd], x2 = m[3 * dd + 1], x3 = m[3 * dd + 2];
    fvh[(4 * dd + 0) * P + n] = (x1 * ta[0] + x2 * ta[1] + x3 * ta[2]) * ij;
    fvh[(4 * dd + 1) * P + n] = (x1 * ta[1] + x2 * ta[3] + x3 * ta[4]) * ij;
    fvh[(4 * dd + 2) * P + n] = (x1 * ta[2] + x2 * ta[4] + x3 * ta[5]) * ij;
    fvh[(4 * dd + 3) * P + n] = (x1 * bx + x2 * by + x3 * bz) * ij;
  }
}
// k_viscous_a_bound: the same under a register bound of 64 per thread (at
// most 256 threads per CTA, 4 CTAs of 256 per SM; a few spills); the
// autotuner chooses.
__global__ void k_viscous_a(const BlockView* __restrict__ blocks, CaseConsts cc_launch, int store_dudx_tao) {
  viscous_a_body(blocks, cc_launch, store_dudx_tao);
}
__global__ void __launch_bounds__(256, 4) k_viscous_a_bound(const BlockView* __restrict__ blocks, CaseConsts cc_launch,
                                                             int store_dudx_tao) {
  viscous_a_body(blocks, cc_launch, store_dudx_tao);
}


// Mixed-precision variant of k_viscous_a: the gradients are FP64 central
// differences, the viscosity (Sutherland) stays FP64 since the local time step
// reads it; the velocity-gradient chain rule, stresses, heat flux, vorticity
// and the contravariant fluxes are FP32.
__global__ void k_viscous_a_mixed(const BlockView* __restrict__ blocks, CaseConsts cc_launch, int store_dudx_tao) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
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
  const int lo[3] = {b0.is, b0.js, b0.ks};
  const int hi[3] = {b0.ie, b0.je, b0.ke};
  const double* pu = B.f[F_PRI] + 1 * B.plane;
  const double* pv = B.f[F_PRI] + 2 * B.plane;
  const double* pw = B.f[F_PRI] + 3 * B.plane;
  const double* pt = B.f[F_PRI] + 5 * B.plane;
  float gt[3] = {0, 0, 0}, gu[3] = {0, 0, 0}, gv[3] = {0, 0, 0}, gw[3] = {0, 0, 0};
  int ndir = cc.dimension == IFLAG_3D ? 3 : 2;
  for (int d = 0; d < ndir; ++d) {
    gt[d] = (float)cdiff(pt, n, st[d], pos[d], lo[d], hi[d]);
    gu[d] = (float)cdiff(pu, n, st[d], pos[d], lo[d], hi[d]);
    gv[d] = (float)cdiff(pv, n, st[d], pos[d], lo[d], hi[d]);
    gw[d] = (float)cdiff(pw, n, st[d], pos[d], lo[d], hi[d]);
  }
  double t0 = pt[n];
  double amu1 = (1.0 + 124.0 / cc.tinf) / (t0 + 124.0 / cc.tinf) * crm::pow(t0, 1.5);
  double amu2 = B.v(F_AMU, 2, n);
  double amu3d = amu1 + amu2;
  B.v(F_AMU, 1, n) = amu1;
  B.v(F_AMU, 3, n) = amu3d;
  float amu3 = (float)amu3d;
  float ki = (float)(cc.gamma * cc.cv * (amu1 / cc.prl + amu2 / cc.prt));
  float u0 = (float)pu[n], v0 = (float)pv[n], w0 = (float)pw[n];
  float m[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) m[c] = (float)B.v(F_DXIDX, c + 1, n);
  float tx = gt[0] * m[0] + gt[1] * m[3] + gt[2] * m[6];
  float ty = gt[0] * m[1] + gt[1] * m[4] + gt[2] * m[7];
  float tz = gt[0] * m[2] + gt[1] * m[5] + gt[2] * m[8];
  float du[9];
  const float* gg[3] = {gu, gv, gw};
#pragma unroll
  for (int a = 0; a < 3; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c) du[3 * a + c] = gg[a][0] * m[c] + gg[a][1] * m[c + 3] + gg[a][2] * m[c + 6];
  float ta[6];
  ta[0] = amu3 * (4.0f / 3.0f * du[0] - 2.0f / 3.0f * (du[4] + du[8]));
  ta[1] = amu3 * (du[1] + du[3]);
  ta[2] = amu3 * (du[6] + du[2]);
  ta[3] = amu3 * (4.0f / 3.0f * du[4] - 2.0f / 3.0f * (du[0] + du[8]));
  ta[4] = amu3 * (du[7] + du[5]);
  ta[5] = amu3 * (4.0f / 3.0f * du[8] - 2.0f / 3.0f * (du[0] + du[4]));
  float bx = u0 * ta[0] + v0 * ta[1] + w0 * ta[2] + ki * tx;
  float by = u0 * ta[1] + v0 * ta[3] + w0 * ta[4] + ki * ty;
  float bz = u0 * ta[2] + v0 * ta[4] + w0 * ta[5] + ki * tz;
  float a1 = du[5] - du[7], a2 = du[2] - du[6], a3 = du[1] - du[3];
  B.s(F_VOR, n) = (double)sqrtf(a1 * a1 + a2 * a2 + a3 * a3);
  if (store_dudx_tao) {
#pragma unroll
    for (int c = 0; c < 9; ++c) B.v(F_DUDX, c + 1, n) = (double)du[c];
#pragma unroll
    for (int c = 0; c < 6; ++c) B.v(F_TAO, c + 1, n) = (double)ta[c];
  }
  float ij = (float)B.s(F_INVJ, n);
  double* fvh = B.f[F_FVH];
  long P = B.plane;
#pragma unroll
  for (int dd = 0; dd < 3; ++dd) {
    float x1 = m[3 * dd], x2 = m[3 * dd + 1], x3 = m[3 * dd + 2];
    fvh[(4 * dd + 0) * P + n] = (double)((x1 * ta[0] + x2 * ta[1] + x3 * ta[2]) * ij);
    fvh[(4 * dd + 1) * P + n] = (double)((x1 * ta[1] + x2 * ta[3] + x3 * ta[4]) * ij);
    fvh[(4 * dd + 2) * P + n] = (double)((x1 * ta[2] + x2 * ta[4] + x3 * ta[5]) * ij);
    fvh[(4 * dd + 3) * P + n] = (double)((x1 * bx + x2 * by + x3 * bz) * ij);
  }
}

// sub_viscous.f90:296-365: rhsv = (d fv/dxi + d gv/deta + d hv/dzeta)/re.
__global__ void k_viscous_b(const BlockView* __restrict__ blocks, CaseConsts cc_launch) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
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
  const int lo[3] = {b0.is, b0.js, b0.ks};
  const int hi[3] = {b0.ie, b0.je, b0.ke};
  const double* fvh = B.f[F_FVH];
  long P = B.plane;
  bool three = cc.dimension == IFLAG_3D;
  B.v(F_RHSV, 1, n) = 0.0;  // fv(1)=gv(1)=hv(1)=0: ((0+0)+0)/re
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    double a = cdiff(fvh + (0 + c) * P, n, st[0], pos[0], lo[0], hi[0]);
    double b = cdiff(fvh + (4 + c) * P, n, st[1], pos[1], lo[1], hi[1]);
    double h = three ? cdiff(fvh + (8 + c) * P, n, st[2], pos[2], lo[2], hi[2]) : 0.0;
    B.v(F_RHSV, c + 2, n) = (a + b + h) / cc.re;
  }
}

// ------------------------------------------------------------------ time step
// sub_timeadvancement_finddt.f90:52-88 (steady).  Besides dt, each CTA writes
// the maximum of its dt values (NaN skipped) for the quirk-exact dtmax/dtmin
// reduction in k_dt_minmax.
__global__ void k_find_dt(const BlockView* __restrict__ blocks, CaseConsts cc_launch, double* cta_max) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
  long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  long N = B.b.size();
  double dt = nan("");
  if (n < N) {
    double m[9];
#pragma unroll
    for (int c = 0; c < 9; ++c) m[c] = B.v(F_DXIDX, c + 1, n);
    double tempxi = sqrt(p2(m[0]) + p2(m[1]) + p2(m[2]));
    double tempeta = sqrt(p2(m[3]) + p2(m[4]) + p2(m[5]));
    double tempzeta = sqrt(p2(m[6]) + p2(m[7]) + p2(m[8]));
    double d0 = B.v(F_PRI, 1, n), u0 = B.v(F_PRI, 2, n), v0 = B.v(F_PRI, 3, n);
    double w0 = B.v(F_PRI, 4, n), c0 = B.v(F_PRI, 7, n);
    double uu = (m[0] * u0 + m[1] * v0 + m[2] * w0) / tempxi;
    double vv = (m[3] * u0 + m[4] * v0 + m[5] * w0) / tempeta;
    double ww = (m[6] * u0 + m[7] * v0 + m[8] * w0) / tempzeta;
    double m3 = B.v(F_AMU, 3, n);
    double t1 = fabs(uu) + c0 + 2.0 * tempxi * m3 * 4.0 / 3.0 / cc.re / d0;
    double t2 = fabs(vv) + c0 + 2.0 * tempeta * m3 * 4.0 / 3.0 / cc.re / d0;
    double t3 = fabs(ww) + c0 + 2.0 * tempzeta * m3 * 4.0 / 3.0 / cc.re / d0;
    dt = cc.cfl / (tempxi * t1 + tempeta * t2 + tempzeta * t3);
    B.s(F_DT, n) = dt;
  }
  if (cta_max) {
    // block-wide max ignoring NaN
    __shared__ double sm[32];
    double v = (dt == dt) ? dt : -INFINITY;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
      v = (threadIdx.x < (blockDim.x >> 5)) ? sm[threadIdx.x] : -INFINITY;
      for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
      if (threadIdx.x == 0) cta_max[(long)blockIdx.y * gridDim.x + blockIdx.x] = v;
    }
  }
}

// Reproduces find_dt's running `if (dt >= dtmax) ... else if (dt <= dtmin)`
// (sub_timeadvancement_finddt.f90:81-85) for block `m` with one CTA: dtmax is
// the plain maximum; dtmin is the minimum over nodes that did not set a new
// running maximum when visited in (k,j,i) order.  Each thread scans a
// contiguous chunk seeded with the exclusive prefix maximum of the chunk
// maxima, so the result equals the serial loop.
__global__ void k_dt_minmax(const BlockView* __restrict__ blocks, int m, const double* cta_max,
                            int ncta, int cta_size, double* out2) {
  const BlockView& B = blocks[m];
  long N = B.b.size();
  __shared__ double pref[1024];
  __shared__ double red[1024];
  int T = blockDim.x;
  long chunk = (N + T - 1) / T;
  // chunk maxima
  double cm = -INFINITY;
  long lo = (long)threadIdx.x * chunk, hi = min(N, lo + chunk);
  for (long n = lo; n < hi; ++n) {
    double v = B.s(F_DT, n);
    if (v == v) cm = fmax(cm, v);
  }
  (void)cta_max; (void)ncta; (void)cta_size;
  pref[threadIdx.x] = cm;
  __syncthreads();
  // inclusive scan (max), Hillis-Steele
  for (int o = 1; o < T; o <<= 1) {
    double x = pref[threadIdx.x];
    if (threadIdx.x >= o) x = fmax(x, pref[threadIdx.x - o]);
    __syncthreads();
    pref[threadIdx.x] = x;
    __syncthreads();
  }
  double run = (threadIdx.x == 0) ? 0.0 : fmax(0.0, pref[threadIdx.x - 1]);  // dtmax starts at 0
  double mn = INFINITY;
  for (long n = lo; n < hi; ++n) {
    double v = B.s(F_DT, n);
    if (v >= run) run = v;           // NaN compares false on both branches
    else if (v == v) mn = fmin(mn, v);
  }
  red[threadIdx.x] = mn;
  __syncthreads();
  for (int o = T / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] = fmin(red[threadIdx.x], red[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out2[0] = fmax(0.0, pref[T - 1]);
    out2[1] = fmin(1.0e10, red[0]);  // dtmin starts at 1e10 and only moves down
  }
}

}  // namespace aero
