// TEST INFRASTRUCTURE ONLY (see oracle_common.h): per-block routines of the
// hot path restated from the reference Fortran, loop by loop.
#include "oracle_blockops.h"

#include <algorithm>
#include <cmath>

namespace oracle {

Flags g_flags;
Consts g_consts;

// sub_getpri_v.f90:19-62
long get_primitivevariables(int mm, V pri_v, V q, double gamma, double cv, const Box& b) {
  (void)mm;
  long nneg = 0;
  for (int k = b.ks; k <= b.ke; ++k)
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) {
        double d = q(1, i, j, k);
        double u = q(2, i, j, k) / d;
        double v = q(3, i, j, k) / d;
        double w = q(4, i, j, k) / d;
        double q2 = 0.5 * (u * u + v * v + w * w);
        double e = q(5, i, j, k) / d;
        double t = (e - q2) / cv;
        double p = (q(5, i, j, k) - q2 * d) * (gamma - 1.0);
        double c = std::sqrt(gamma * p / d);
        pri_v(1, i, j, k) = d;
        pri_v(2, i, j, k) = u;
        pri_v(3, i, j, k) = v;
        pri_v(4, i, j, k) = w;
        pri_v(5, i, j, k) = p;
        pri_v(6, i, j, k) = t;
        pri_v(7, i, j, k) = c;
        if (d < 0.0) ++nneg;  // :54-56 prints "Negative density found!!!"
      }
  return nneg;
}

// sub_inviscid_upwind.f90:1-179.  r0 is the caller's is1..ke1 box (the routine's
// dummy is0..ke0), coord 1/2/3, direction +1 (right state at face i+1/2) or -1
// (left state at face i+1/2).  Faces run from r0 lower-1 to r0 upper along coord.
void thirdorder_weno(V df, V f, const Box& b, const Box& r0, int coord, int direction) {
  const double eps = 1.0e-6;  // :17
  int di = coord == 1, dj = coord == 2, dk = coord == 3;
  for (int k = r0.ks - dk; k <= r0.ke; ++k)
    for (int j = r0.js - dj; j <= r0.je; ++j)
      for (int i = r0.is - di; i <= r0.ie; ++i) {
        int pos = coord == 1 ? i : (coord == 2 ? j : k);
        if (direction == 1) {
          int lim = coord == 1 ? b.ie : (coord == 2 ? b.je : b.ke);
          if (pos == lim - 1) {  // :25-26 one-sided copy next to the block end
            for (int n = 1; n <= 5; ++n) df(n, i, j, k) = f(n, i + di, j + dj, k + dk);
          } else {
            for (int n = 1; n <= 5; ++n) {
              double u1 = f(n, i, j, k);
              double u2 = f(n, i + di, j + dj, k + dk);
              double u3 = f(n, i + 2 * di, j + 2 * dj, k + 2 * dk);
              double s1 = p2(u2 - u3);
              double s2 = p2(u1 - u2);
              double a1 = 1.0 / (3.0 * p2(eps + s1));
              double a2 = 2.0 / (3.0 * p2(eps + s2));
              double w1 = a1 / (a1 + a2);
              double w2 = a2 / (a1 + a2);
              df(n, i, j, k) = w1 * (-u3 / 2.0 + 3.0 * u2 / 2.0) + w2 * (u2 / 2.0 + u1 / 2.0);  // :41
            }
          }
        } else {
          int lim = coord == 1 ? b.is : (coord == 2 ? b.js : b.ks);
          if (pos == lim) {  // :50-51
            for (int n = 1; n <= 5; ++n) df(n, i, j, k) = f(n, i, j, k);
          } else {
            for (int n = 1; n <= 5; ++n) {
              double u1 = f(n, i - di, j - dj, k - dk);
              double u2 = f(n, i, j, k);
              double u3 = f(n, i + di, j + dj, k + dk);
              double s1 = p2(u2 - u1);
              double s2 = p2(u3 - u2);
              double a1 = 1.0 / (3.0 * p2(eps + s1));
              double a2 = 2.0 / (3.0 * p2(eps + s2));
              double w1 = a1 / (a1 + a2);
              double w2 = a2 / (a1 + a2);
              df(n, i, j, k) = w1 * (-u1 / 2.0 + 3.0 * u2 / 2.0) + w2 * (u2 / 2.0 + u3 / 2.0);  // :66
            }
          }
        }
      }
}

// sub_inviscid_splitting.f90:1-172 (Roe flux-difference splitting, Harten fix).
// Face i stands for i+1/2 along coord; faces from r0 lower-1 to r0 upper.
void roe_3d(V ql, V qr, V flux, V dxidx, V inv_j, double gamma, const Box& b, const Box& r0,
            int coord) {
  (void)b;
  const double delt = 0.06;  // :42
  int ii = coord == 1, jj = coord == 2, kk = coord == 3;
  int c1 = coord * 3 - 2, c2 = coord * 3 - 1, c3 = coord * 3;
  for (int k = r0.ks - kk; k <= r0.ke; ++k)
    for (int j = r0.js - jj; j <= r0.je; ++j)
      for (int i = r0.is - ii; i <= r0.ie; ++i) {
        double ja = inv_j(i, j, k), jb = inv_j(i + ii, j + jj, k + kk);
        double dxidx1 = 0.5 * (dxidx(c1, i, j, k) * ja + dxidx(c1, i + ii, j + jj, k + kk) * jb);
        double dxidy1 = 0.5 * (dxidx(c2, i, j, k) * ja + dxidx(c2, i + ii, j + jj, k + kk) * jb);
        double dxidz1 = 0.5 * (dxidx(c3, i, j, k) * ja + dxidx(c3, i + ii, j + jj, k + kk) * jb);
        double temp = std::sqrt(p2(dxidx1) + p2(dxidy1) + p2(dxidz1));
        double dxidx0 = dxidx1 / temp, dxidy0 = dxidy1 / temp, dxidz0 = dxidz1 / temp;

        double dl = ql(1, i, j, k), dr = qr(1, i, j, k);
        double ul = ql(2, i, j, k), ur = qr(2, i, j, k);
        double vl = ql(3, i, j, k), vr = qr(3, i, j, k);
        double wl = ql(4, i, j, k), wr = qr(4, i, j, k);
        double pl = ql(5, i, j, k), pr = qr(5, i, j, k);

        double hl = gamma * pl / ((gamma - 1.0) * dl) + 0.5 * (p2(ul) + p2(vl) + p2(wl));
        double hr = gamma * pr / ((gamma - 1.0) * dr) + 0.5 * (p2(ur) + p2(vr) + p2(wr));
        double uul = ul * dxidx1 + vl * dxidy1 + wl * dxidz1;
        double uur = ur * dxidx1 + vr * dxidy1 + wr * dxidz1;
        double ubarl = uul / temp, ubarr = uur / temp;

        double fl[5], fr[5];
        fl[0] = dl * uul;
        fl[1] = dl * ul * uul + dxidx1 * pl;
        fl[2] = dl * vl * uul + dxidy1 * pl;
        fl[3] = dl * wl * uul + dxidz1 * pl;
        fl[4] = dl * hl * uul;
        fr[0] = dr * uur;
        fr[1] = dr * ur * uur + dxidx1 * pr;
        fr[2] = dr * vr * uur + dxidy1 * pr;
        fr[3] = dr * wr * uur + dxidz1 * pr;
        fr[4] = dr * hr * uur;

        double tmpp = std::sqrt(dr / dl);
        double avd = std::sqrt(dl * dr);
        double avu = (ul + ur * tmpp) / (1.0 + tmpp);
        double avv = (vl + vr * tmpp) / (1.0 + tmpp);
        double avw = (wl + wr * tmpp) / (1.0 + tmpp);
        double avh = (hl + hr * tmpp) / (1.0 + tmpp);
        double ava = std::sqrt((gamma - 1.0) * (avh - 0.5 * (p2(avu) + p2(avv) + p2(avw))));
        double avuu = avu * dxidx0 + avv * dxidy0 + avw * dxidz0;

        double lam[5];
        lam[0] = std::fabs(avuu - ava);
        lam[1] = std::fabs(avuu);
        lam[2] = std::fabs(avuu);
        lam[3] = std::fabs(avuu);
        lam[4] = std::fabs(avuu + ava);
        for (int n = 0; n < 5; ++n) {  // :122-130
          double tmp = fsign1(delt - lam[n]);
          double tmp1 = 0.5 * (1.0 - tmp);
          double tmp2 = 0.5 * (1.0 + tmp);
          double harten = (p2(lam[n]) + p2(delt)) / (2.0 * delt);
          lam[n] = tmp1 * lam[n] + tmp2 * harten;
        }
        double deltad = dr - dl, deltap = pr - pl;
        double deltau = ur - ul, deltav = vr - vl, deltaw = wr - wl;
        double deltauu = ubarr - ubarl;

        double alpha1 = lam[1] * (deltad - deltap / p2(ava));
        double alpha2 = lam[4] * (deltap + avd * ava * deltauu) / (2.0 * p2(ava));
        double alpha3 = lam[0] * (deltap - avd * ava * deltauu) / (2.0 * p2(ava));
        double alpha4 = alpha1 + alpha2 + alpha3;
        double alpha5 = ava * (alpha2 - alpha3);
        double alpha6 = lam[1] * (avd * deltau - avd * deltauu * dxidx0);
        double alpha7 = lam[1] * (avd * deltav - avd * deltauu * dxidy0);
        double alpha8 = lam[1] * (avd * deltaw - avd * deltauu * dxidz0);

        double ff[5];
        ff[0] = alpha4;
        ff[1] = avu * alpha4 + alpha5 * dxidx0 + alpha6;
        ff[2] = avv * alpha4 + alpha5 * dxidy0 + alpha7;
        ff[3] = avw * alpha4 + alpha5 * dxidz0 + alpha8;
        ff[4] = avh * alpha4 + avuu * alpha5 + avu * alpha6 + avv * alpha7 + avw * alpha8 -
                p2(ava) * alpha1 / (gamma - 1.0);
        for (int n = 0; n < 5; ++n) flux(n + 1, i, j, k) = 0.5 * (fl[n] + fr[n] - temp * ff[n]);  // :158-162
      }
}

// sub_inviscid1.f90:8-189
void inviscid_flux_1(V rhsi, V q, V dxidx, V inv_j, const Box& b, const Box& b0, const Box& b1,
                     double gamma) {
  (void)b0;
  Tmp ql(5, b), qr(5, b), ul(5, b), ur(5, b), flux(5, b);
  for (long n = 0; n < 5 * b.size(); ++n) rhsi.p[n] = 0.0;  // :40
  int ndir = g_flags.dimension == IFLAG_3D ? 3 : 2;
  for (int coord = 1; coord <= ndir; ++coord) {
    ql.zero(); qr.zero(); ul.zero(); ur.zero(); flux.zero();  // :42-48, :91-97, :138-144
    thirdorder_weno(ur.view, q, b, b1, coord, 1);   // right
    thirdorder_weno(ul.view, q, b, b1, coord, -1);  // left
    int di = coord == 1, dj = coord == 2, dk = coord == 3;
    for (int k = b1.ks - dk; k <= b1.ke; ++k)  // :58-74 conservative -> primitive at faces
      for (int j = b1.js - dj; j <= b1.je; ++j)
        for (int i = b1.is - di; i <= b1.ie; ++i) {
          ql(1, i, j, k) = ul(1, i, j, k);
          ql(2, i, j, k) = ul(2, i, j, k) / ul(1, i, j, k);
          ql(3, i, j, k) = ul(3, i, j, k) / ul(1, i, j, k);
          ql(4, i, j, k) = ul(4, i, j, k) / ul(1, i, j, k);
          ql(5, i, j, k) = (ul(5, i, j, k) - 0.5 * (p2(ul(2, i, j, k)) + p2(ul(3, i, j, k)) +
                                                    p2(ul(4, i, j, k))) / ul(1, i, j, k)) *
                           (gamma - 1.0);
          qr(1, i, j, k) = ur(1, i, j, k);
          qr(2, i, j, k) = ur(2, i, j, k) / ur(1, i, j, k);
          qr(3, i, j, k) = ur(3, i, j, k) / ur(1, i, j, k);
          qr(4, i, j, k) = ur(4, i, j, k) / ur(1, i, j, k);
          qr(5, i, j, k) = (ur(5, i, j, k) - 0.5 * (p2(ur(2, i, j, k)) + p2(ur(3, i, j, k)) +
                                                    p2(ur(4, i, j, k))) / ur(1, i, j, k)) *
                           (gamma - 1.0);
        }
    roe_3d(ql.view, qr.view, flux.view, dxidx, inv_j, gamma, b, b1, coord);
    for (int k = b1.ks; k <= b1.ke; ++k)  // :82-88, :128-134, :175-181
      for (int j = b1.js; j <= b1.je; ++j)
        for (int i = b1.is; i <= b1.ie; ++i)
          for (int n = 1; n <= 5; ++n) {
            double d = flux(n, i, j, k) - flux(n, i - di, j - dj, k - dk);
            if (coord == 1)
              rhsi(n, i, j, k) = -d;
            else
              rhsi(n, i, j, k) = rhsi(n, i, j, k) - d;
          }
  }
}

// ------------------------------------------- extension inviscid schemes
// iflag_inviscid = 5 (Steger-Warming splitting + WENO5) and 8 (WCNS5 + Roe):
// flag values of the reference (module_flags.f90:68, 71) that it stops on
// (main.f90:636-653), so there is no reference code to follow.  Restated from
// the published methods: Steger & Warming, J. Comput. Phys. 40 (1981) 263;
// Jiang & Shu, J. Comput. Phys. 126 (1996) 202; Deng & Zhang, J. Comput.
// Phys. 165 (2000) 22.  Three ghost layers at interfaces; near a physical
// boundary WENO5 drops to WENO3 and then 1st order, and WCNS5 to the
// reference's WENO3 + Roe face.  The WCNS5 face flux is
// G = 4/3 F(i+1/2) - (F(i) + F(i+1))/6 with node fluxes F(i), the 4th-order
// hybrid face/node difference in conservative form.
namespace {

const double kEps5 = 1.0e-6;

double w5_edge(double v0, double v1, double v2, double v3, double v4) {
  double b0 = 13.0 / 12.0 * p2(v0 - 2.0 * v1 + v2) + 0.25 * p2(v0 - 4.0 * v1 + 3.0 * v2);
  double b1 = 13.0 / 12.0 * p2(v1 - 2.0 * v2 + v3) + 0.25 * p2(v1 - v3);
  double b2 = 13.0 / 12.0 * p2(v2 - 2.0 * v3 + v4) + 0.25 * p2(3.0 * v2 - 4.0 * v3 + v4);
  double a0 = 0.1 / p2(kEps5 + b0), a1 = 0.6 / p2(kEps5 + b1), a2 = 0.3 / p2(kEps5 + b2);
  double q0 = (2.0 * v0 - 7.0 * v1 + 11.0 * v2) / 6.0;
  double q1 = (-v1 + 5.0 * v2 + 2.0 * v3) / 6.0;
  double q2 = (2.0 * v2 + 5.0 * v3 - v4) / 6.0;
  return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
}

double w3_edge(double v0, double v1, double v2) {
  double b0 = p2(v1 - v0), b1 = p2(v2 - v1);
  double a0 = (1.0 / 3.0) / p2(kEps5 + b0), a1 = (2.0 / 3.0) / p2(kEps5 + b1);
  double q0 = (3.0 * v1 - v0) / 2.0, q1 = (v1 + v2) / 2.0;
  return (a0 * q0 + a1 * q1) / (a0 + a1);
}

double c5_edge(double v0, double v1, double v2, double v3, double v4) {
  double b0 = 13.0 / 12.0 * p2(v0 - 2.0 * v1 + v2) + 0.25 * p2(v0 - 4.0 * v1 + 3.0 * v2);
  double b1 = 13.0 / 12.0 * p2(v1 - 2.0 * v2 + v3) + 0.25 * p2(v1 - v3);
  double b2 = 13.0 / 12.0 * p2(v2 - 2.0 * v3 + v4) + 0.25 * p2(3.0 * v2 - 4.0 * v3 + v4);
  double a0 = 0.0625 / p2(kEps5 + b0), a1 = 0.625 / p2(kEps5 + b1), a2 = 0.3125 / p2(kEps5 + b2);
  double q0 = (3.0 * v0 - 10.0 * v1 + 15.0 * v2) / 8.0;
  double q1 = (-v1 + 6.0 * v2 + 3.0 * v3) / 8.0;
  double q2 = (3.0 * v2 + 6.0 * v3 - v4) / 8.0;
  return (a0 * q0 + a1 * q1 + a2 * q2) / (a0 + a1 + a2);
}

// Steger-Warming split contravariant flux (positive or negative eigenvalue
// parts) at node (i,j,k) along coord, metric K = grad xi * inv_j.
void sw_flux(bool plus, V q, V dxidx, V inv_j, int coord, int i, int j, int k, double gamma, double f[5]) {
  double rho = q(1, i, j, k);
  double u = q(2, i, j, k) / rho, v = q(3, i, j, k) / rho, w = q(4, i, j, k) / rho;
  double q2 = 0.5 * (u * u + v * v + w * w);
  double p = (q(5, i, j, k) - rho * q2) * (gamma - 1.0);
  double c = std::sqrt(gamma * p / rho);
  int c1 = 3 * coord - 2;
  double ij = inv_j(i, j, k);
  double kx = dxidx(c1, i, j, k) * ij, ky = dxidx(c1 + 1, i, j, k) * ij, kz = dxidx(c1 + 2, i, j, k) * ij;
  double kn = std::sqrt(kx * kx + ky * ky + kz * kz);
  double nx = kx / kn, ny = ky / kn, nz = kz / kn;
  double uu = kx * u + ky * v + kz * w;
  double ub = nx * u + ny * v + nz * w;
  double lam[3] = {uu, uu + c * kn, uu - c * kn};
  for (double& l : lam) l = plus ? 0.5 * (l + std::fabs(l)) : 0.5 * (l - std::fabs(l));
  double h = c * c / (gamma - 1.0) + q2;
  double coef = rho / (2.0 * gamma);
  double a1 = 2.0 * (gamma - 1.0) * lam[0];
  f[0] = coef * (a1 + lam[1] + lam[2]);
  f[1] = coef * (a1 * u + lam[1] * (u + c * nx) + lam[2] * (u - c * nx));
  f[2] = coef * (a1 * v + lam[1] * (v + c * ny) + lam[2] * (v - c * ny));
  f[3] = coef * (a1 * w + lam[1] * (w + c * nz) + lam[2] * (w - c * nz));
  f[4] = coef * (a1 * q2 + lam[1] * (h + c * ub) + lam[2] * (h - c * ub));
}

// Physical contravariant flux at node (i,j,k) with its own metric.
void phys_flux(V q, V dxidx, V inv_j, int coord, int i, int j, int k, double gamma, double f[5]) {
  double d = q(1, i, j, k);
  double u = q(2, i, j, k) / d, v = q(3, i, j, k) / d, w = q(4, i, j, k) / d;
  double p = (q(5, i, j, k) - 0.5 * (p2(q(2, i, j, k)) + p2(q(3, i, j, k)) + p2(q(4, i, j, k))) / d) *
             (gamma - 1.0);
  int c1 = 3 * coord - 2;
  double ij = inv_j(i, j, k);
  double kx = dxidx(c1, i, j, k) * ij, ky = dxidx(c1 + 1, i, j, k) * ij, kz = dxidx(c1 + 2, i, j, k) * ij;
  double h = gamma * p / ((gamma - 1.0) * d) + 0.5 * (p2(u) + p2(v) + p2(w));
  double uu = u * kx + v * ky + w * kz;
  f[0] = d * uu;
  f[1] = d * u * uu + kx * p;
  f[2] = d * v * uu + ky * p;
  f[3] = d * w * uu + kz * p;
  f[4] = d * h * uu;
}

// rhsi from face fluxes flux(i) = F(i+1/2) along coord, as sub_inviscid1.f90:82-88.
void difference_faces(V rhsi, Tmp& flux, const Box& b1, int coord) {
  int di = coord == 1, dj = coord == 2, dk = coord == 3;
  for (int k = b1.ks; k <= b1.ke; ++k)
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i)
        for (int n = 1; n <= 5; ++n) {
          double d = flux(n, i, j, k) - flux(n, i - di, j - dj, k - dk);
          if (coord == 1)
            rhsi(n, i, j, k) = -d;
          else
            rhsi(n, i, j, k) = rhsi(n, i, j, k) - d;
        }
}

}  // namespace

void inviscid_flux_sw_weno5(V rhsi, V q, V dxidx, V inv_j, const Box& b, const Box& b1, double gamma) {
  for (long n = 0; n < 5 * b.size(); ++n) rhsi.p[n] = 0.0;
  int ndir = g_flags.dimension == IFLAG_3D ? 3 : 2;
  for (int coord = 1; coord <= ndir; ++coord) {
    Tmp flux(5, b);
    int di = coord == 1, dj = coord == 2, dk = coord == 3;
    int lo = coord == 1 ? b.is : (coord == 2 ? b.js : b.ks);
    int hi = coord == 1 ? b.ie : (coord == 2 ? b.je : b.ke);
    for (int k = b1.ks - dk; k <= b1.ke; ++k)
      for (int j = b1.js - dj; j <= b1.je; ++j)
        for (int i = b1.is - di; i <= b1.ie; ++i) {
          int pos = coord == 1 ? i : (coord == 2 ? j : k);
          double fp[5][5], fm[5][5];  // node pos-2+x (plus), pos-1+x (minus)
          for (int x = 0; x < 5; ++x) {
            int o = x - 2;
            if (pos + o >= lo && pos + o <= hi)
              sw_flux(true, q, dxidx, inv_j, coord, i + o * di, j + o * dj, k + o * dk, gamma, fp[x]);
            o = x - 1;
            if (pos + o >= lo && pos + o <= hi)
              sw_flux(false, q, dxidx, inv_j, coord, i + o * di, j + o * dj, k + o * dk, gamma, fm[x]);
          }
          bool p5 = pos - 2 >= lo && pos + 2 <= hi, p3 = pos - 1 >= lo && pos + 1 <= hi;
          bool m5 = pos - 1 >= lo && pos + 3 <= hi, m3 = pos >= lo && pos + 2 <= hi;
          for (int n = 0; n < 5; ++n) {
            double a = p5 ? w5_edge(fp[0][n], fp[1][n], fp[2][n], fp[3][n], fp[4][n])
                          : (p3 ? w3_edge(fp[1][n], fp[2][n], fp[3][n]) : fp[2][n]);
            double m = m5 ? w5_edge(fm[4][n], fm[3][n], fm[2][n], fm[1][n], fm[0][n])
                          : (m3 ? w3_edge(fm[3][n], fm[2][n], fm[1][n]) : fm[2][n]);
            flux(n + 1, i, j, k) = a + m;
          }
        }
    difference_faces(rhsi, flux, b1, coord);
  }
}

void inviscid_flux_wcns5(V rhsi, V q, V dxidx, V inv_j, const Box& b, const Box& b1, double gamma) {
  for (long n = 0; n < 5 * b.size(); ++n) rhsi.p[n] = 0.0;
  int ndir = g_flags.dimension == IFLAG_3D ? 3 : 2;
  for (int coord = 1; coord <= ndir; ++coord) {
    Tmp ul(5, b), ur(5, b), ql(5, b), qr(5, b), flux(5, b);
    thirdorder_weno(ur.view, q, b, b1, coord, 1);
    thirdorder_weno(ul.view, q, b, b1, coord, -1);
    int di = coord == 1, dj = coord == 2, dk = coord == 3;
    int lo = coord == 1 ? b.is : (coord == 2 ? b.js : b.ks);
    int hi = coord == 1 ? b.ie : (coord == 2 ? b.je : b.ke);
    auto wcns = [&](int i, int j, int k) {
      int pos = coord == 1 ? i : (coord == 2 ? j : k);
      return pos - 2 >= lo && pos + 3 <= hi;
    };
    for (int k = b1.ks - dk; k <= b1.ke; ++k)
      for (int j = b1.js - dj; j <= b1.je; ++j)
        for (int i = b1.is - di; i <= b1.ie; ++i) {
          if (wcns(i, j, k))
            for (int n = 1; n <= 5; ++n) {
              double u[6];
              for (int x = 0; x < 6; ++x) u[x] = q(n, i + (x - 2) * di, j + (x - 2) * dj, k + (x - 2) * dk);
              ul(n, i, j, k) = c5_edge(u[0], u[1], u[2], u[3], u[4]);
              ur(n, i, j, k) = c5_edge(u[5], u[4], u[3], u[2], u[1]);
            }
          ql(1, i, j, k) = ul(1, i, j, k);
          ql(2, i, j, k) = ul(2, i, j, k) / ul(1, i, j, k);
          ql(3, i, j, k) = ul(3, i, j, k) / ul(1, i, j, k);
          ql(4, i, j, k) = ul(4, i, j, k) / ul(1, i, j, k);
          ql(5, i, j, k) = (ul(5, i, j, k) - 0.5 * (p2(ul(2, i, j, k)) + p2(ul(3, i, j, k)) +
                                                    p2(ul(4, i, j, k))) / ul(1, i, j, k)) * (gamma - 1.0);
          qr(1, i, j, k) = ur(1, i, j, k);
          qr(2, i, j, k) = ur(2, i, j, k) / ur(1, i, j, k);
          qr(3, i, j, k) = ur(3, i, j, k) / ur(1, i, j, k);
          qr(4, i, j, k) = ur(4, i, j, k) / ur(1, i, j, k);
          qr(5, i, j, k) = (ur(5, i, j, k) - 0.5 * (p2(ur(2, i, j, k)) + p2(ur(3, i, j, k)) +
                                                    p2(ur(4, i, j, k))) / ur(1, i, j, k)) * (gamma - 1.0);
        }
    roe_3d(ql.view, qr.view, flux.view, dxidx, inv_j, gamma, b, b1, coord);
    for (int k = b1.ks - dk; k <= b1.ke; ++k)
      for (int j = b1.js - dj; j <= b1.je; ++j)
        for (int i = b1.is - di; i <= b1.ie; ++i) {
          if (!wcns(i, j, k)) continue;
          double fa[5], fb[5];
          phys_flux(q, dxidx, inv_j, coord, i, j, k, gamma, fa);
          phys_flux(q, dxidx, inv_j, coord, i + di, j + dj, k + dk, gamma, fb);
          for (int n = 0; n < 5; ++n) flux(n + 1, i, j, k) = 4.0 / 3.0 * flux(n + 1, i, j, k) - (fa[n] + fb[n]) / 6.0;
        }
    difference_faces(rhsi, flux, b1, coord);
  }
}

void inviscid_flux(V rhsi, V q, V dxidx, V inv_j, const Box& b, const Box& b0, const Box& b1, double gamma) {
  if (g_flags.inviscid == IFLAG_5THWENO)
    inviscid_flux_sw_weno5(rhsi, q, dxidx, inv_j, b, b1, gamma);
  else if (g_flags.inviscid == IFLAG_5THWCNS)
    inviscid_flux_wcns5(rhsi, q, dxidx, inv_j, b, b1, gamma);
  else
    inviscid_flux_1(rhsi, q, dxidx, inv_j, b, b0, b1, gamma);
}

// sub_viscous.f90:9-378 (3-D branch).
void viscous_flux(V rhsv, V pri_v, V amu, V vor, V dudx, V tao, V dxidx, V inv_j, double tinf,
                  double prl, double prt, double gamma, double cv, double re, const Box& b,
                  const Box& b0, const Box& b1) {
  Tmp u(1, b), v(1, b), w(1, b), t(1, b);
  Tmp txi(1, b), teta(1, b), tzeta(1, b), uxi(1, b), ueta(1, b), uzeta(1, b);
  Tmp vxi(1, b), veta(1, b), vzeta(1, b), wxi(1, b), weta(1, b), wzeta(1, b);
  Tmp bx(1, b), by(1, b), bz(1, b);
  Tmp fv(5, b), gv(5, b), hv(5, b), fvxi(5, b), gveta(5, b), hvzeta(5, b);
  bool three = g_flags.dimension == IFLAG_3D;

  const int kx = three ? 1 : 0;  // 2-D: the plane k = 1 only (:93-101)
  for (int k = b1.ks - kx; k <= b1.ke + kx; ++k)  // :82-92
    for (int j = b1.js - 1; j <= b1.je + 1; ++j)
      for (int i = b1.is - 1; i <= b1.ie + 1; ++i) {
        u(i, j, k) = pri_v(2, i, j, k);
        v(i, j, k) = pri_v(3, i, j, k);
        w(i, j, k) = pri_v(4, i, j, k);
        t(i, j, k) = pri_v(6, i, j, k);
      }
  // One-sided at the ends of the physical range, central elsewhere (:106-178).
  auto grad = [&](Tmp& src, Tmp& dst, int di, int dj, int dk) {
    for (int k = b0.ks; k <= b0.ke; ++k)
      for (int j = b0.js; j <= b0.je; ++j)
        for (int i = b0.is; i <= b0.ie; ++i) {
          int pos = di ? i : (dj ? j : k);
          int lo = di ? b0.is : (dj ? b0.js : b0.ks);
          int hi = di ? b0.ie : (dj ? b0.je : b0.ke);
          if (pos == lo)
            dst(i, j, k) = src(i + di, j + dj, k + dk) - src(i, j, k);
          else if (pos == hi)
            dst(i, j, k) = src(i, j, k) - src(i - di, j - dj, k - dk);
          else
            dst(i, j, k) = (src(i + di, j + dj, k + dk) - src(i - di, j - dj, k - dk)) / 2.0;
        }
  };
  grad(t, txi, 1, 0, 0); grad(u, uxi, 1, 0, 0); grad(v, vxi, 1, 0, 0); grad(w, wxi, 1, 0, 0);
  grad(t, teta, 0, 1, 0); grad(u, ueta, 0, 1, 0); grad(v, veta, 0, 1, 0); grad(w, weta, 0, 1, 0);
  if (three) {
    grad(t, tzeta, 0, 0, 1); grad(u, uzeta, 0, 0, 1); grad(v, vzeta, 0, 0, 1); grad(w, wzeta, 0, 0, 1);
  }
  for (int k = b0.ks; k <= b0.ke; ++k)  // :187-254
    for (int j = b0.js; j <= b0.je; ++j)
      for (int i = b0.is; i <= b0.ie; ++i) {
        double u0 = u(i, j, k), v0 = v(i, j, k), w0 = w(i, j, k), t0 = t(i, j, k);
        amu(1, i, j, k) = (1.0 + 124.0 / tinf) / (t0 + 124.0 / tinf) * xpow(t0, 1.5);
        amu(3, i, j, k) = amu(1, i, j, k) + amu(2, i, j, k);
        double ki = gamma * cv * (amu(1, i, j, k) / prl + amu(2, i, j, k) / prt);
        double tx = txi(i, j, k) * dxidx(1, i, j, k) + teta(i, j, k) * dxidx(4, i, j, k) +
                    tzeta(i, j, k) * dxidx(7, i, j, k);
        double ty = txi(i, j, k) * dxidx(2, i, j, k) + teta(i, j, k) * dxidx(5, i, j, k) +
                    tzeta(i, j, k) * dxidx(8, i, j, k);
        double tz = txi(i, j, k) * dxidx(3, i, j, k) + teta(i, j, k) * dxidx(6, i, j, k) +
                    tzeta(i, j, k) * dxidx(9, i, j, k);
        Tmp* gx[3] = {&uxi, &vxi, &wxi};
        Tmp* ge[3] = {&ueta, &veta, &weta};
        Tmp* gz[3] = {&uzeta, &vzeta, &wzeta};
        for (int a = 0; a < 3; ++a)
          for (int c = 0; c < 3; ++c)
            dudx(3 * a + c + 1, i, j, k) = (*gx[a])(i, j, k) * dxidx(c + 1, i, j, k) +
                                           (*ge[a])(i, j, k) * dxidx(c + 4, i, j, k) +
                                           (*gz[a])(i, j, k) * dxidx(c + 7, i, j, k);
        double m3 = amu(3, i, j, k);
        tao(1, i, j, k) = m3 * (4.0 / 3.0 * dudx(1, i, j, k) - 2.0 / 3.0 * (dudx(5, i, j, k) + dudx(9, i, j, k)));
        tao(2, i, j, k) = m3 * (dudx(2, i, j, k) + dudx(4, i, j, k));
        tao(3, i, j, k) = m3 * (dudx(7, i, j, k) + dudx(3, i, j, k));
        tao(4, i, j, k) = m3 * (4.0 / 3.0 * dudx(5, i, j, k) - 2.0 / 3.0 * (dudx(1, i, j, k) + dudx(9, i, j, k)));
        tao(5, i, j, k) = m3 * (dudx(8, i, j, k) + dudx(6, i, j, k));
        tao(6, i, j, k) = m3 * (4.0 / 3.0 * dudx(9, i, j, k) - 2.0 / 3.0 * (dudx(1, i, j, k) + dudx(5, i, j, k)));
        bx(i, j, k) = u0 * tao(1, i, j, k) + v0 * tao(2, i, j, k) + w0 * tao(3, i, j, k) + ki * tx;
        by(i, j, k) = u0 * tao(2, i, j, k) + v0 * tao(4, i, j, k) + w0 * tao(5, i, j, k) + ki * ty;
        bz(i, j, k) = u0 * tao(3, i, j, k) + v0 * tao(5, i, j, k) + w0 * tao(6, i, j, k) + ki * tz;
      }
  for (int k = b0.ks; k <= b0.ke; ++k)  // :258-266
    for (int j = b0.js; j <= b0.je; ++j)
      for (int i = b0.is; i <= b0.ie; ++i)
        vor(i, j, k) = std::sqrt(p2(dudx(6, i, j, k) - dudx(8, i, j, k)) +
                                 p2(dudx(3, i, j, k) - dudx(7, i, j, k)) +
                                 p2(dudx(2, i, j, k) - dudx(4, i, j, k)));
  for (int k = b0.ks; k <= b0.ke; ++k)  // :269-293
    for (int j = b0.js; j <= b0.je; ++j)
      for (int i = b0.is; i <= b0.ie; ++i) {
        double ij = inv_j(i, j, k);
        double x1 = dxidx(1, i, j, k), x2 = dxidx(2, i, j, k), x3 = dxidx(3, i, j, k);
        double e1 = dxidx(4, i, j, k), e2 = dxidx(5, i, j, k), e3 = dxidx(6, i, j, k);
        double z1 = dxidx(7, i, j, k), z2 = dxidx(8, i, j, k), z3 = dxidx(9, i, j, k);
        double t1 = tao(1, i, j, k), t2 = tao(2, i, j, k), t3 = tao(3, i, j, k);
        double t4 = tao(4, i, j, k), t5 = tao(5, i, j, k), t6 = tao(6, i, j, k);
        double bxx = bx(i, j, k), byy = by(i, j, k), bzz = bz(i, j, k);
        fv(1, i, j, k) = 0.0; gv(1, i, j, k) = 0.0; hv(1, i, j, k) = 0.0;
        fv(2, i, j, k) = (x1 * t1 + x2 * t2 + x3 * t3) * ij;
        gv(2, i, j, k) = (e1 * t1 + e2 * t2 + e3 * t3) * ij;
        hv(2, i, j, k) = (z1 * t1 + z2 * t2 + z3 * t3) * ij;
        fv(3, i, j, k) = (x1 * t2 + x2 * t4 + x3 * t5) * ij;
        gv(3, i, j, k) = (e1 * t2 + e2 * t4 + e3 * t5) * ij;
        hv(3, i, j, k) = (z1 * t2 + z2 * t4 + z3 * t5) * ij;
        fv(4, i, j, k) = (x1 * t3 + x2 * t5 + x3 * t6) * ij;
        gv(4, i, j, k) = (e1 * t3 + e2 * t5 + e3 * t6) * ij;
        hv(4, i, j, k) = (z1 * t3 + z2 * t5 + z3 * t6) * ij;
        fv(5, i, j, k) = (x1 * bxx + x2 * byy + x3 * bzz) * ij;
        gv(5, i, j, k) = (e1 * bxx + e2 * byy + e3 * bzz) * ij;
        hv(5, i, j, k) = (z1 * bxx + z2 * byy + z3 * bzz) * ij;
      }
  auto div = [&](Tmp& src, Tmp& dst, int di, int dj, int dk) {  // :296-340
    for (int k = b0.ks; k <= b0.ke; ++k)
      for (int j = b0.js; j <= b0.je; ++j)
        for (int i = b0.is; i <= b0.ie; ++i) {
          int pos = di ? i : (dj ? j : k);
          int lo = di ? b0.is : (dj ? b0.js : b0.ks);
          int hi = di ? b0.ie : (dj ? b0.je : b0.ke);
          for (int n = 1; n <= 5; ++n) {
            if (pos == lo)
              dst(n, i, j, k) = src(n, i + di, j + dj, k + dk) - src(n, i, j, k);
            else if (pos == hi)
              dst(n, i, j, k) = src(n, i, j, k) - src(n, i - di, j - dj, k - dk);
            else
              dst(n, i, j, k) = (src(n, i + di, j + dj, k + dk) - src(n, i - di, j - dj, k - dk)) / 2.0;
          }
        }
  };
  div(fv, fvxi, 1, 0, 0);
  div(gv, gveta, 0, 1, 0);
  if (three) div(hv, hvzeta, 0, 0, 1);
  for (int k = b0.ks; k <= b0.ke; ++k)  // :359-365
    for (int j = b0.js; j <= b0.je; ++j)
      for (int i = b0.is; i <= b0.ie; ++i)
        for (int n = 1; n <= 5; ++n)
          rhsv(n, i, j, k) = (fvxi(n, i, j, k) + gveta(n, i, j, k) + hvzeta(n, i, j, k)) / re;
}

// sub_timeadvancement_finddt.f90:24-130.  cfl is overwritten in the unsteady
// branch (:116), exactly like the Fortran dummy argument.
void find_dt(V dt, double* dtmax, double* dtmin, double* cflmax, double* cflmin, V pri_v, V amu,
             V dxidx, double re, double* cfl, const Box& b, int iflag_time) {
  *dtmin = 1.0e10; *dtmax = 0.0; *cflmin = 1.0e10; *cflmax = 0.0;
  for (int k = b.ks; k <= b.ke; ++k)
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) {
        double x1 = dxidx(1, i, j, k), x2 = dxidx(2, i, j, k), x3 = dxidx(3, i, j, k);
        double e1 = dxidx(4, i, j, k), e2 = dxidx(5, i, j, k), e3 = dxidx(6, i, j, k);
        double z1 = dxidx(7, i, j, k), z2 = dxidx(8, i, j, k), z3 = dxidx(9, i, j, k);
        double tempxi = std::sqrt(p2(x1) + p2(x2) + p2(x3));
        double tempeta = std::sqrt(p2(e1) + p2(e2) + p2(e3));
        double tempzeta = std::sqrt(p2(z1) + p2(z2) + p2(z3));
        double d0 = pri_v(1, i, j, k), u0 = pri_v(2, i, j, k), v0 = pri_v(3, i, j, k);
        double w0 = pri_v(4, i, j, k), c0 = pri_v(7, i, j, k);
        double uu = (x1 * u0 + x2 * v0 + x3 * w0) / tempxi;
        double vv = (e1 * u0 + e2 * v0 + e3 * w0) / tempeta;
        double ww = (z1 * u0 + z2 * v0 + z3 * w0) / tempzeta;
        double m3 = amu(3, i, j, k);
        double t1 = std::fabs(uu) + c0 + 2.0 * tempxi * m3 * 4.0 / 3.0 / re / d0;
        double t2 = std::fabs(vv) + c0 + 2.0 * tempeta * m3 * 4.0 / 3.0 / re / d0;
        double t3 = std::fabs(ww) + c0 + 2.0 * tempzeta * m3 * 4.0 / 3.0 / re / d0;
        if (iflag_time == IFLAG_STEADY) {
          dt(i, j, k) = *cfl / (tempxi * t1 + tempeta * t2 + tempzeta * t3);
          if (dt(i, j, k) >= *dtmax)  // :81-85 (else-if min/max)
            *dtmax = dt(i, j, k);
          else if (dt(i, j, k) <= *dtmin)
            *dtmin = dt(i, j, k);
        } else {
          *cfl = dt(i, j, k) * (tempxi * t1 + tempeta * t2 + tempzeta * t3);
          if (*cfl >= *cflmax)
            *cflmax = *cfl;
          else if (*cfl <= *cflmin)
            *cflmin = *cfl;
        }
      }
}

// sub_timeadvancement_jac.f90:7-62.  a is a 5x5 column-major (Fortran) matrix.
void calc_jm(double a[25], double q1, double q2, double q3, double q4, double q5, double dxidx,
             double dxidy, double dxidz, double gamma) {
#define A(r, c) a[((c) - 1) * 5 + ((r) - 1)]
  double a2 = gamma - 1.0, a3 = gamma - 2.0;
  double rho = q1, mu0 = q2, mv0 = q3, mw0 = q4, e0 = q5;
  double uu = (dxidx * mu0 + dxidy * mv0 + dxidz * mw0) / rho;
  double phi = 0.5 * a2 * (p2(mu0) + p2(mv0) + p2(mw0)) / p2(rho);
  double a1 = gamma * e0 / rho - phi;
  A(1, 1) = 0.0; A(1, 2) = dxidx; A(1, 3) = dxidy; A(1, 4) = dxidz; A(1, 5) = 0.0;
  A(2, 1) = phi * dxidx - uu * mu0 / rho;
  A(2, 2) = uu - a3 * dxidx * mu0 / rho;
  A(2, 3) = dxidy * mu0 / rho - a2 * dxidx * mv0 / rho;
  A(2, 4) = dxidz * mu0 / rho - a2 * dxidx * mw0 / rho;
  A(2, 5) = a2 * dxidx;
  A(3, 1) = phi * dxidy - uu * mv0 / rho;
  A(3, 2) = dxidx * mv0 / rho - a2 * dxidy * mu0 / rho;
  A(3, 3) = uu - a3 * dxidy * mv0 / rho;
  A(3, 4) = dxidz * mv0 / rho - a2 * dxidy * mw0 / rho;
  A(3, 5) = a2 * dxidy;
  A(4, 1) = phi * dxidz - uu * mw0 / rho;
  A(4, 2) = dxidx * mw0 / rho - a2 * dxidz * mu0 / rho;
  A(4, 3) = dxidy * mw0 / rho - a2 * dxidz * mv0 / rho;
  A(4, 4) = uu - a3 * dxidz * mw0 / rho;
  A(4, 5) = a2 * dxidz;
  A(5, 1) = (phi - a1) * uu;
  A(5, 2) = a1 * dxidx - a2 * uu * mu0 / rho;
  A(5, 3) = a1 * dxidy - a2 * uu * mv0 / rho;
  A(5, 4) = a1 * dxidz - a2 * uu * mw0 / rho;
  A(5, 5) = gamma * uu;
#undef A
}

// One off-diagonal LU-SGS block: calc_jm at the neighbour, +/- spectral radius on
// the diagonal, whole matrix scaled by 0.5*inv_j of the neighbour
// (sub_timeadvancement_1stimplicit.f90:283-301 and :459-477).
static void lusgs_block(double m[25], V q, V dxidx, double rad, double invj, int cbase, int i,
                        int j, int k, double gamma, double sgn) {
  calc_jm(m, q(1, i, j, k), q(2, i, j, k), q(3, i, j, k), q(4, i, j, k), q(5, i, j, k),
          dxidx(cbase, i, j, k), dxidx(cbase + 1, i, j, k), dxidx(cbase + 2, i, j, k), gamma);
  for (int n = 0; n < 5; ++n) {
    if (sgn > 0)
      m[n * 5 + n] = m[n * 5 + n] + rad;
    else
      m[n * 5 + n] = m[n * 5 + n] - rad;
  }
  for (int n = 0; n < 25; ++n) m[n] = 0.5 * m[n] * invj;
}

static double matrow(const double m[25], int n, V dq, int i, int j, int k) {
  // tempa = jm(n,1)*dq(1) + ... + jm(n,5)*dq(5), left to right (:346-350)
  double s = m[0 * 5 + n] * dq(1, i, j, k);
  s = s + m[1 * 5 + n] * dq(2, i, j, k);
  s = s + m[2 * 5 + n] * dq(3, i, j, k);
  s = s + m[3 * 5 + n] * dq(4, i, j, k);
  s = s + m[4 * 5 + n] * dq(5, i, j, k);
  return s;
}

// sub_timeadvancement_1stimplicit.f90:7-585 (3-D and 2-D branches).
void implicit1st(V q, V dt, V pri_v, V rhs, V rhsi, V rhsv, V dxidx, V inv_j, const Box& b,
                 const Box& b0, const Box& b1, double gamma, double cfl) {
  (void)b0;
  Tmp diag(1, b), ra(1, b), rb(1, b), rc(1, b), dqstar(5, b), dq(5, b);
  for (int k = b1.ks; k <= b1.ke; ++k)  // :72-78
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i)
        for (int n = 1; n <= 5; ++n) rhs(n, i, j, k) = rhsi(n, i, j, k) + rhsv(n, i, j, k);
  double phi = cfl >= 1.0e3 ? 0.0 : 1.0;  // :98-102
  // 2-D (:157-210, :213-278, :388-453): the plane k = 1, no zeta radius in
  // the diagonal and no zeta neighbour in the sweeps
  const bool three = g_flags.dimension == IFLAG_3D;
  const int kx = three ? 1 : 0;
  for (int k = b1.ks - kx; k <= b1.ke + kx; ++k)  // :110-156
    for (int j = b1.js - 1; j <= b1.je + 1; ++j)
      for (int i = b1.is - 1; i <= b1.ie + 1; ++i) {
        double u = pri_v(2, i, j, k), v = pri_v(3, i, j, k), w = pri_v(4, i, j, k);
        double c = pri_v(7, i, j, k);
        double r3[3];
        for (int dd = 0; dd < 3; ++dd) {
          double x0 = dxidx(3 * dd + 1, i, j, k), y0 = dxidx(3 * dd + 2, i, j, k),
                 z0 = dxidx(3 * dd + 3, i, j, k);
          double temp = p2(x0) + p2(y0) + p2(z0);
          temp = std::sqrt(temp);
          double cu = x0 * u + y0 * v + z0 * w;
          r3[dd] = std::fabs(cu) + std::fabs(c * temp);
        }
        ra(i, j, k) = r3[0]; rb(i, j, k) = r3[1]; rc(i, j, k) = r3[2];
        if (three)
          diag(i, j, k) = phi * 1.0 / dt(i, j, k) + ra(i, j, k) + rb(i, j, k) + rc(i, j, k);
        else
          diag(i, j, k) = phi * 1.0 / dt(i, j, k) + ra(i, j, k) + rb(i, j, k);
      }
  double ma[25], mb[25], mc[25];
  for (int k = b1.ks; k <= b1.ke; ++k)  // forward sweep :279-368
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i) {
        lusgs_block(ma, q, dxidx, ra(i - 1, j, k), inv_j(i - 1, j, k), 1, i - 1, j, k, gamma, +1);
        lusgs_block(mb, q, dxidx, rb(i, j - 1, k), inv_j(i, j - 1, k), 4, i, j - 1, k, gamma, +1);
        if (three) lusgs_block(mc, q, dxidx, rc(i, j, k - 1), inv_j(i, j, k - 1), 7, i, j, k - 1, gamma, +1);
        for (int n = 0; n < 5; ++n) {
          double ta = matrow(ma, n, dqstar.view, i - 1, j, k);
          double tb = matrow(mb, n, dqstar.view, i, j - 1, k);
          if (!three) {
            dqstar(n + 1, i, j, k) = (rhs(n + 1, i, j, k) + (ta + tb)) / diag(i, j, k) / inv_j(i, j, k);
            continue;
          }
          double tc = matrow(mc, n, dqstar.view, i, j, k - 1);
          dqstar(n + 1, i, j, k) = (rhs(n + 1, i, j, k) + (ta + tb + tc)) / diag(i, j, k) / inv_j(i, j, k);
        }
      }
  for (int k = b1.ke; k >= b1.ks; --k)  // backward sweep :455-545
    for (int j = b1.je; j >= b1.js; --j)
      for (int i = b1.ie; i >= b1.is; --i) {
        lusgs_block(ma, q, dxidx, ra(i + 1, j, k), inv_j(i + 1, j, k), 1, i + 1, j, k, gamma, -1);
        lusgs_block(mb, q, dxidx, rb(i, j + 1, k), inv_j(i, j + 1, k), 4, i, j + 1, k, gamma, -1);
        if (three) lusgs_block(mc, q, dxidx, rc(i, j, k + 1), inv_j(i, j, k + 1), 7, i, j, k + 1, gamma, -1);
        for (int n = 0; n < 5; ++n) {
          double ta = matrow(ma, n, dq.view, i + 1, j, k);
          double tb = matrow(mb, n, dq.view, i, j + 1, k);
          if (!three) {
            dq(n + 1, i, j, k) = dqstar(n + 1, i, j, k) - (ta + tb) / inv_j(i, j, k) / diag(i, j, k);
            continue;
          }
          double tc = matrow(mc, n, dq.view, i, j, k + 1);
          dq(n + 1, i, j, k) = dqstar(n + 1, i, j, k) - (ta + tb + tc) / inv_j(i, j, k) / diag(i, j, k);
        }
      }
  for (int k = b1.ks; k <= b1.ke; ++k)  // :568-574
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i)
        for (int n = 1; n <= 5; ++n) q(n, i, j, k) = q(n, i, j, k) + dq(n, i, j, k);
}

// sub_tur_sa.f90:130-212
static void sa_rhs1(V sa_rhs, V nut, V pri_v, V dxidx, const Box& b1) {
  bool three = g_flags.dimension == IFLAG_3D;
  for (int k = b1.ks; k <= b1.ke; ++k)
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i) {
        double u = pri_v(2, i, j, k), v = pri_v(3, i, j, k), w = pri_v(4, i, j, k);
        double res[3] = {0.0, 0.0, 0.0};
        for (int dd = 0; dd < (three ? 3 : 2); ++dd) {
          int di = dd == 0, dj = dd == 1, dk = dd == 2;
          double uu = dxidx(3 * dd + 1, i, j, k) * u + dxidx(3 * dd + 2, i, j, k) * v +
                      dxidx(3 * dd + 3, i, j, k) * w;
          double nutp = nut(i + di, j + dj, k + dk), nutc = nut(i, j, k),
                 nutm = nut(i - di, j - dj, k - dk);
          res[dd] = -(0.5 * (uu + std::fabs(uu)) * (nutc - nutm) + 0.5 * (uu - std::fabs(uu)) * (nutp - nutc));
        }
        sa_rhs(i, j, k) = res[0] + res[1] + res[2];
      }
}

// sub_tur_sa.f90:220-523
static void sa_rhs2(V sa_rhs, V nut, V amu, V pri_v, V dxidx, V inv_j, V alpha, V beta, V gamma,
                    double re, const Box& b, const Box& b0, const Box& b1) {
  bool three = g_flags.dimension == IFLAG_3D;
  Tmp dnutdxi(1, b), dnutdeta(1, b), dnutdzeta(1, b);
  Tmp tempalpha(1, b), tempbeta(1, b), tempgamma(1, b);
  Tmp tempa(1, b), tempb(1, b), tempc(1, b), temp(1, b);
  Tmp tempxi(1, b), tempeta(1, b), tempzeta(1, b);
  Tmp tempx(1, b), tempy(1, b), tempz(1, b);
  // Differences on is1..ie1, one-sided when the node is the physical end is0/ie0.
  auto d1 = [&](V src, V dst, int di, int dj, int dk) {
    for (int k = b1.ks; k <= b1.ke; ++k)
      for (int j = b1.js; j <= b1.je; ++j)
        for (int i = b1.is; i <= b1.ie; ++i) {
          int pos = di ? i : (dj ? j : k);
          int lo = di ? b0.is : (dj ? b0.js : b0.ks);
          int hi = di ? b0.ie : (dj ? b0.je : b0.ke);
          if (pos == lo)
            dst(i, j, k) = src(i + di, j + dj, k + dk) - src(i, j, k);
          else if (pos == hi)
            dst(i, j, k) = src(i, j, k) - src(i - di, j - dj, k - dk);
          else
            dst(i, j, k) = (src(i + di, j + dj, k + dk) - src(i - di, j - dj, k - dk)) / 2.0;
        }
  };
  d1(nut, dnutdxi.view, 1, 0, 0);  // :294-306
  d1(nut, dnutdeta.view, 0, 1, 0);
  if (three) d1(nut, dnutdzeta.view, 0, 0, 1);
  for (int k = b1.ks; k <= b1.ke; ++k)  // :340-356
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i) {
        tempalpha(i, j, k) = alpha(1, i, j, k) * dnutdxi(i, j, k) + alpha(2, i, j, k) * dnutdeta(i, j, k) +
                             alpha(3, i, j, k) * dnutdzeta(i, j, k);
        tempbeta(i, j, k) = beta(1, i, j, k) * dnutdxi(i, j, k) + beta(2, i, j, k) * dnutdeta(i, j, k) +
                            beta(3, i, j, k) * dnutdzeta(i, j, k);
        tempgamma(i, j, k) = gamma(1, i, j, k) * dnutdxi(i, j, k) + gamma(2, i, j, k) * dnutdeta(i, j, k) +
                             gamma(3, i, j, k) * dnutdzeta(i, j, k);
      }
  d1(tempalpha.view, tempa.view, 1, 0, 0);  // :359-403
  d1(tempbeta.view, tempb.view, 0, 1, 0);
  if (three) d1(tempgamma.view, tempc.view, 0, 0, 1);
  for (int k = b1.ks; k <= b1.ke; ++k)  // :405-413
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i) {
        double nut0 = nut(i, j, k);
        double nu0 = amu(1, i, j, k) / pri_v(1, i, j, k);
        temp(i, j, k) = nu0 + (1.0 + SA_CB2) * nut0;
      }
  d1(temp.view, tempxi.view, 1, 0, 0);  // :416-460
  d1(temp.view, tempeta.view, 0, 1, 0);
  if (three) d1(temp.view, tempzeta.view, 0, 0, 1);
  for (int k = b1.ks; k <= b1.ke; ++k)  // :462-480
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i) {
        tempx(i, j, k) = tempxi(i, j, k) * dxidx(1, i, j, k) + tempeta(i, j, k) * dxidx(4, i, j, k) +
                         tempzeta(i, j, k) * dxidx(7, i, j, k);
        tempy(i, j, k) = tempxi(i, j, k) * dxidx(2, i, j, k) + tempeta(i, j, k) * dxidx(5, i, j, k) +
                         tempzeta(i, j, k) * dxidx(8, i, j, k);
        tempz(i, j, k) = tempxi(i, j, k) * dxidx(3, i, j, k) + tempeta(i, j, k) * dxidx(6, i, j, k) +
                         tempzeta(i, j, k) * dxidx(9, i, j, k);
      }
  for (int k = b1.ks; k <= b1.ke; ++k)  // :482-512
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i) {
        double nut0 = nut(i, j, k);
        double inv_j0 = inv_j(i, j, k);
        double deltanut = (tempa(i, j, k) + tempb(i, j, k) + tempc(i, j, k)) / inv_j0;
        double dnutdx = dnutdxi(i, j, k) * dxidx(1, i, j, k) + dnutdeta(i, j, k) * dxidx(4, i, j, k) +
                        dnutdzeta(i, j, k) * dxidx(7, i, j, k);
        double dnutdy = dnutdxi(i, j, k) * dxidx(2, i, j, k) + dnutdeta(i, j, k) * dxidx(5, i, j, k) +
                        dnutdzeta(i, j, k) * dxidx(8, i, j, k);
        double dnutdz = dnutdxi(i, j, k) * dxidx(3, i, j, k) + dnutdeta(i, j, k) * dxidx(6, i, j, k) +
                        dnutdzeta(i, j, k) * dxidx(9, i, j, k);
        double diff = -(SA_CB2 / (re * SA_DTA)) * nut0 * deltanut +
                      (1.0 / (re * SA_DTA)) * (temp(i, j, k) * deltanut + tempx(i, j, k) * dnutdx +
                                               tempy(i, j, k) * dnutdy + tempz(i, j, k) * dnutdz);
        sa_rhs(i, j, k) = sa_rhs(i, j, k) + diff;
      }
}

// sub_tur_sa.f90:532-629 (reference mode: r = nut0*div, :579).
static void sa_rhs3(V sa_rhs, V nut, V pri_v, V amu, V vor, V length, V diasd, double re,
                    const Box& b1) {
  for (int k = b1.ks; k <= b1.ke; ++k)
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i) {
        double d = pri_v(1, i, j, k);
        double nut0 = nut(i, j, k);
        double nu0 = amu(1, i, j, k) / d;
        double omega = std::fabs(vor(i, j, k));
        double dist0 = length(i, j, k);
        double leix = std::max(nut0 / nu0, 0.001);
        double fv1 = p3(leix) / (p3(leix) + SA_CV13);
        double fv2 = 1.0 - leix / (1.0 + leix * fv1);
        double s = omega + nut0 * fv2 / (re * SA_KAR2 * p2(dist0));
        s = std::max(s, 0.3 * omega);
        double div = s * re * SA_KAR2 * p2(dist0);
        div = std::max(div, 1.0e-6);
        double r = nut0 * div;
        r = std::min(r, 10.0);
        double g = r + SA_CW2 * (p6(r) - r);
        double fw = g * xpow((1.0 + 64.0) / (p6(g) + 64.0), 1.0 / 6.0);
        double ft2 = SA_CT3 * xexp(-SA_CT4 * p2(leix));
        double aaa = SA_CB1 * ((1.0 - ft2) * fv2 + ft2) / SA_KAR2;
        double bbb = SA_CW1 * fw;
        double ccc = nut0 / p2(dist0);
        double sd1 = (aaa - bbb) * ccc / re;
        double sd = sd1 * nut0;
        double sp = SA_CB1 * (1.0 - ft2) * omega * nut0;
        sa_rhs(i, j, k) = sa_rhs(i, j, k) + sd + sp;

        double leixn = 1.0 / nu0;
        double fv1n = (3.0 * p2(leix) * leixn * (p3(leix) + SA_CV13) - p3(leix) * (3.0 * p2(leix) * leixn)) /
                      p2(p3(leix) + SA_CV13);
        double fv2n = (leixn * (1.0 + leix * fv1) - leix * (leixn * fv1 + leix * fv1n)) / p2(1.0 + leix * fv1);
        double ft2n = -(2.0 * SA_CT4 * leix * leixn * ft2);
        double sn = 1.0 / (re * SA_KAR2 * p2(dist0)) * (fv2 + fv2n * nut0);
        div = p2(s) * (re * SA_KAR2 * p2(dist0));
        div = std::max(div, 1.0e-6);
        double rn = (s - sn * nut0) / div;
        double gn = (1.0 + SA_CW2 * 6.0 * p5(r) - SA_CW2) * rn;
        const double cw3m6 = 0.015625;  // cw3**(-6.d0), folded
        double fwn = -((1.0 / 6.0) * xpow((xpow(g, -6.0) + cw3m6) / (1.0 + cw3m6), -7.0 / 6.0));
        fwn = fwn / (1.0 + cw3m6) * (-(6.0 * xpow(g, -7.0))) * gn;
        double spn = SA_CB1 * (1.0 - ft2) * omega + SA_CB1 * (-ft2n) * omega * nut0;
        double sdn = (1.0 / re) * (SA_CB1 * (fv2 - ft2 * fv2 + ft2) / SA_KAR2 - SA_CW1 * fw) * 2.0 * nut0 / p2(dist0);
        sdn = (1.0 / re) * (SA_CB1 * (fv2n - ft2n * fv2 - ft2 * fv2n + ft2n) / SA_KAR2 - SA_CW1 * fwn) *
                  (p2(nut0) / p2(dist0)) + sdn;
        diasd(i, j, k) = std::min(spn + sdn, 0.0);
      }
}

// sub_tur_sa.f90:638-825 (3-D branch).
static void sa_lusgs(V nut, V dt, V sa_rhs, V pri_v, V dxidx, V diasd, double re, double cfl,
                     const Box& b, const Box& b1) {
  Tmp dnut(1, b), dnut1(1, b), diag(1, b), contrau(1, b), contrav(1, b), contraw(1, b);
  double phi = (cfl >= 1.0e3 && g_flags.time == IFLAG_STEADY) ? 0.0 : 1.0;
  // 2-D (:683-717, :785-806): the plane k = 1, sweeps without the zeta term
  const bool three = g_flags.dimension == IFLAG_3D;
  const int kx = three ? 1 : 0;
  for (int k = b1.ks - kx; k <= b1.ke + kx; ++k)  // :719-753
    for (int j = b1.js - 1; j <= b1.je + 1; ++j)
      for (int i = b1.is - 1; i <= b1.ie + 1; ++i) {
        double u = pri_v(2, i, j, k), v = pri_v(3, i, j, k), w = pri_v(4, i, j, k);
        double x0 = dxidx(1, i, j, k), y0 = dxidx(2, i, j, k), z0 = dxidx(3, i, j, k);
        double d2 = x0 * x0 + y0 * y0 + z0 * z0;
        contrau(i, j, k) = x0 * u + y0 * v + z0 * w;
        x0 = dxidx(4, i, j, k); y0 = dxidx(5, i, j, k); z0 = dxidx(6, i, j, k);
        d2 = d2 + x0 * x0 + y0 * y0 + z0 * z0;
        contrav(i, j, k) = x0 * u + y0 * v + z0 * w;
        x0 = dxidx(7, i, j, k); y0 = dxidx(8, i, j, k); z0 = dxidx(9, i, j, k);
        d2 = d2 + x0 * x0 + y0 * y0 + z0 * z0;
        contraw(i, j, k) = x0 * u + y0 * v + z0 * w;
        double tm = 4.0 * d2 * nut(i, j, k) / re;
        diag(i, j, k) = 1.0 / dt(i, j, k) * phi + std::fabs(contrau(i, j, k)) + std::fabs(contrav(i, j, k)) +
                        std::fabs(contraw(i, j, k)) + tm - diasd(i, j, k);
      }
  for (int k = b1.ks; k <= b1.ke; ++k)  // :759-769
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i) {
        double ta = 0.5 * (contrau(i, j, k) + std::fabs(contrau(i, j, k))) * dnut1(i - 1, j, k);
        double tb = 0.5 * (contrav(i, j, k) + std::fabs(contrav(i, j, k))) * dnut1(i, j - 1, k);
        if (!three) {
          dnut1(i, j, k) = (sa_rhs(i, j, k) + (ta + tb)) / diag(i, j, k);
          continue;
        }
        double tc = 0.5 * (contraw(i, j, k) + std::fabs(contraw(i, j, k))) * dnut1(i, j, k - 1);
        dnut1(i, j, k) = (sa_rhs(i, j, k) + (ta + tb + tc)) / diag(i, j, k);
      }
  for (int k = b1.ke; k >= b1.ks; --k)  // :773-783
    for (int j = b1.je; j >= b1.js; --j)
      for (int i = b1.ie; i >= b1.is; --i) {
        double ta = 0.5 * (contrau(i, j, k) - std::fabs(contrau(i, j, k))) * dnut(i + 1, j, k);
        double tb = 0.5 * (contrav(i, j, k) - std::fabs(contrav(i, j, k))) * dnut(i, j + 1, k);
        if (!three) {
          dnut(i, j, k) = dnut1(i, j, k) - (ta + tb) / diag(i, j, k);
          continue;
        }
        double tc = 0.5 * (contraw(i, j, k) - std::fabs(contraw(i, j, k))) * dnut(i, j, k + 1);
        dnut(i, j, k) = dnut1(i, j, k) - (ta + tb + tc) / diag(i, j, k);
      }
  for (int k = b1.ks; k <= b1.ke; ++k)  // :812-818
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i) nut(i, j, k) = nut(i, j, k) + dnut(i, j, k);
}

// sub_tur_sa.f90:7-122.  dxidx and dudx keep their (9,...) storage; DDES reads
// dudx through the reference's (3,...,3) declaration (:29, :78-80).
void sa_model(V nut, V sa_rhs, V dt, V pri_v, V amu, V dudx, V vor, V dxidx, V inv_j, V alpha,
              V beta, V gamma, V length, V dist, V spac, double re, double cfl, const Box& b,
              const Box& b0, const Box& b1) {
  const double cdes = 0.65;
  Tmp diasd(1, b);
  for (long n = 0; n < b.size(); ++n) sa_rhs.p[n] = 0.0;  // :48
  for (int k = b.ks; k <= b.ke; ++k)
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) length(i, j, k) = dist(i, j, k);
  if (g_flags.des == IFLAG_DES97) {
    for (int k = b.ks; k <= b.ke; ++k)
      for (int j = b.js; j <= b.je; ++j)
        for (int i = b.is; i <= b.ie; ++i)
          length(i, j, k) = std::min(dist(i, j, k), cdes * spac(i, j, k));
  } else if (g_flags.des == IFLAG_DDES) {
    long N = b.size();
    for (int k = b.ks; k <= b.ke; ++k)
      for (int j = b.js; j <= b.je; ++j)
        for (int i = b.is; i <= b.ie; ++i) {
          long node = b.at(i, j, k);
          auto g3 = [&](int a, int c) { return dudx.p[(a - 1) + 3 * node + 3 * N * (c - 1)]; };
          double uy = g3(1, 2), uz = g3(1, 3), vx = g3(2, 1), vz = g3(2, 3), wx = g3(3, 1), wy = g3(3, 2);
          double d0 = pri_v(1, i, j, k), nut0 = nut(i, j, k), nu0 = amu(1, i, j, k) / d0;
          double dist0 = dist(i, j, k), spac0 = spac(i, j, k);
          double temp = p2(uy) + p2(uz) + p2(vx) + p2(vz) + p2(wx) + p2(wy);
          temp = std::sqrt(temp);
          double rd = (nu0 + nut0) / (temp * re * SA_KAR2 * p2(dist0));
          double fd = 1.0 - std::tanh(p3(8.0 * rd));
          length(i, j, k) = dist0 - fd * std::max(0.0, dist0 - cdes * spac0);
        }
  }
  sa_rhs1(sa_rhs, nut, pri_v, dxidx, b1);
  sa_rhs2(sa_rhs, nut, amu, pri_v, dxidx, inv_j, alpha, beta, gamma, re, b, b0, b1);
  sa_rhs3(sa_rhs, nut, pri_v, amu, vor, length, diasd.view, re, b1);
  sa_lusgs(nut, dt, sa_rhs, pri_v, dxidx, diasd.view, re, cfl, b, b1);
}

}  // namespace oracle

namespace oracle {

// q0(l, c, i, j, k) with l = -1, 0 (sub_init_allocatememory.f90:285): the
// time level is the fastest index, then the component.
static inline double& Q0(V q0, int l, int c, int i, int j, int k) { return q0(1 + (l + 1) + 2 * (c - 1), i, j, k); }

// One point of the factorised sweep (sub_timeadvancement_2ndcrank.f90:129-161
// and its j, k twins): a = the flux-Jacobian product of neighbour node nb
// with its dq, plus/minus the spectral radius (sgn = +1 forward, -1
// backward); cb = first metric component of the direction.
static inline void crank_a(V pri_v, V dxidx, double r, int cb, double hdv, double gamma, const double s[5],
                           double sgn, int i, int j, int k, double a[5]) {
  double u = pri_v(2, i, j, k), v = pri_v(3, i, j, k), w = pri_v(4, i, j, k), c = pri_v(7, i, j, k);
  double dxidx0 = dxidx(cb, i, j, k), dxidy0 = dxidx(cb + 1, i, j, k), dxidz0 = dxidx(cb + 2, i, j, k);
  double q2 = 0.5 * (p2(u) + p2(v) + p2(w));
  double h = p2(c) / (gamma - 1.0) + q2;
  double cu = dxidx0 * u + dxidy0 * v + dxidz0 * w;
  double b1 = hdv * (-(cu * s[0]) + dxidx0 * s[1] + dxidy0 * s[2] + dxidz0 * s[3]);
  double b2 = hdv * (q2 * s[0] - u * s[1] - v * s[2] - w * s[3] + s[4]) * (gamma - 1.0);
  double b3 = sgn > 0 ? hdv * (cu + r) : hdv * (cu - r);
  a[0] = b1 + b3 * s[0];
  a[1] = b1 * u + b2 * dxidx0 + b3 * s[1];
  a[2] = b1 * v + b2 * dxidy0 + b3 * s[2];
  a[3] = b1 * w + b2 * dxidz0 + b3 * s[3];
  a[4] = b1 * h + b2 * cu + b3 * s[4];
}

static inline double crank_rou(V pri_v, V dxidx, int cb, int i, int j, int k) {
  double u = pri_v(2, i, j, k), v = pri_v(3, i, j, k), w = pri_v(4, i, j, k), c = pri_v(7, i, j, k);
  double x0 = dxidx(cb, i, j, k), y0 = dxidx(cb + 1, i, j, k), z0 = dxidx(cb + 2, i, j, k);
  double temp = p2(x0) + p2(y0) + p2(z0);
  temp = std::sqrt(temp);
  double cu = u * x0 + v * y0 + w * z0;
  return std::fabs(cu) + std::fabs(c * temp);
}

// sub_timeadvancement_2ndcrank.f90:1-466 (crank2nd, 3-D): the dual-time
// right-hand side with alph = 1/2, then the approximately factorised
// point-implicit sweeps along i, j and k lines and q += dq/inv_j.  The forward
// k recurrence starts at ks1+1, as in the reference (:352).
void crank2nd(V q, V q0, V dt, V pri_v, V rhs, V rhsi, V rhsv, V dxidx, V inv_j, const Box& b, const Box& b0,
              const Box& b1, double gamma) {
  (void)b0;
  for (int k = b1.ks; k <= b1.ke; ++k)
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i)
        for (int c = 1; c <= 5; ++c) rhs(c, i, j, k) = rhsi(c, i, j, k) + rhsv(c, i, j, k);
  const double alph = 0.5;
  const double alph_i = 1.0 / (1.0 + alph);
  for (int k = b1.ks; k <= b1.ke; ++k)
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i)
        for (int c = 1; c <= 5; ++c)
          rhs(c, i, j, k) = alph_i * (rhs(c, i, j, k) * dt(i, j, k) -
                                      ((1.0 + alph) * q(c, i, j, k) - (1.0 + 2.0 * alph) * Q0(q0, 0, c, i, j, k) +
                                       alph * Q0(q0, -1, c, i, j, k)) * inv_j(i, j, k));
  std::vector<double> dtsub_s(b.size(), 0.0), rou_s(b.size(), 0.0), dq_s(5 * (size_t)b.size(), 0.0);
  V dtsub{dtsub_s.data(), 1, b}, rou{rou_s.data(), 1, b}, dq{dq_s.data(), 5, b};
  // 2-D (sub_timeadvancement_2ndcrank.f90:84-99, :335): the plane k = 1, no k lines
  const bool three = g_flags.dimension == IFLAG_3D;
  const int kx = three ? 1 : 0;
  for (int k = b1.ks - kx; k <= b1.ke + kx; ++k)
    for (int j = b1.js - 1; j <= b1.je + 1; ++j)
      for (int i = b1.is - 1; i <= b1.ie + 1; ++i) dtsub(i, j, k) = dt(i, j, k) / (1.0 + alph);
  double s[5], a[5];
  auto load = [&](int i, int j, int k) {
    for (int c = 0; c < 5; ++c) s[c] = dq(c + 1, i, j, k);
  };
  // i lines
  for (int k = b1.ks; k <= b1.ke; ++k)
    for (int j = b1.js; j <= b1.je; ++j) {
      for (int i = b1.is - 1; i <= b1.ie + 1; ++i) rou(i, j, k) = crank_rou(pri_v, dxidx, 1, i, j, k);
      for (int i = b1.is; i <= b1.ie; ++i) {
        load(i - 1, j, k);
        crank_a(pri_v, dxidx, rou(i - 1, j, k), 1, 0.5 * dtsub(i, j, k), gamma, s, 1.0, i - 1, j, k, a);
        double div = 1.0 / (1.0 + dtsub(i, j, k) * rou(i, j, k));
        for (int c = 0; c < 5; ++c) dq(c + 1, i, j, k) = div * (rhs(c + 1, i, j, k) + a[c]);
      }
      for (int i = b1.ie; i >= b1.is; --i) {
        load(i + 1, j, k);
        crank_a(pri_v, dxidx, rou(i + 1, j, k), 1, 0.5 * dtsub(i, j, k), gamma, s, -1.0, i + 1, j, k, a);
        double div = 1.0 / (1.0 + dtsub(i, j, k) * rou(i, j, k));
        for (int c = 0; c < 5; ++c) dq(c + 1, i, j, k) = dq(c + 1, i, j, k) - div * a[c];
      }
    }
  // j lines
  for (int k = b1.ks; k <= b1.ke; ++k)
    for (int i = b1.is; i <= b1.ie; ++i) {
      for (int j = b1.js - 1; j <= b1.je + 1; ++j) rou(i, j, k) = crank_rou(pri_v, dxidx, 4, i, j, k);
      for (int j = b1.js; j <= b1.je; ++j) {
        load(i, j - 1, k);
        crank_a(pri_v, dxidx, rou(i, j - 1, k), 4, 0.5 * dtsub(i, j, k), gamma, s, 1.0, i, j - 1, k, a);
        double div = 1.0 / (1.0 + dtsub(i, j, k) * rou(i, j, k));
        for (int c = 0; c < 5; ++c) dq(c + 1, i, j, k) = div * (dq(c + 1, i, j, k) + a[c]);
      }
      for (int j = b1.je; j >= b1.js; --j) {
        load(i, j + 1, k);
        crank_a(pri_v, dxidx, rou(i, j + 1, k), 4, 0.5 * dtsub(i, j, k), gamma, s, -1.0, i, j + 1, k, a);
        double div = 1.0 / (1.0 + dtsub(i, j, k) * rou(i, j, k));
        for (int c = 0; c < 5; ++c) dq(c + 1, i, j, k) = dq(c + 1, i, j, k) - div * a[c];
      }
    }
  // k lines
  for (int j = b1.js; j <= b1.je && three; ++j)
    for (int i = b1.is; i <= b1.ie; ++i) {
      for (int k = b1.ks - 1; k <= b1.ke + 1; ++k) rou(i, j, k) = crank_rou(pri_v, dxidx, 7, i, j, k);
      for (int k = b1.ks + 1; k <= b1.ke; ++k) {
        load(i, j, k - 1);
        crank_a(pri_v, dxidx, rou(i, j, k - 1), 7, 0.5 * dtsub(i, j, k), gamma, s, 1.0, i, j, k - 1, a);
        double div = 1.0 / (1.0 + dtsub(i, j, k) * rou(i, j, k));
        for (int c = 0; c < 5; ++c) dq(c + 1, i, j, k) = div * (dq(c + 1, i, j, k) + a[c]);
      }
      for (int k = b1.ke - 1; k >= b1.ks; --k) {
        load(i, j, k + 1);
        crank_a(pri_v, dxidx, rou(i, j, k + 1), 7, 0.5 * dtsub(i, j, k), gamma, s, -1.0, i, j, k + 1, a);
        double div = 1.0 / (1.0 + dtsub(i, j, k) * rou(i, j, k));
        for (int c = 0; c < 5; ++c) dq(c + 1, i, j, k) = dq(c + 1, i, j, k) - div * a[c];
      }
    }
  for (int k = b1.ks; k <= b1.ke; ++k)
    for (int j = b1.js; j <= b1.je; ++j)
      for (int i = b1.is; i <= b1.ie; ++i)
        for (int c = 1; c <= 5; ++c) q(c, i, j, k) = q(c, i, j, k) + dq(c, i, j, k) / inv_j(i, j, k);
}

// main.f90:692-711: q0(-1) = q0(0), q0(0) = q on the physical nodes.
void update_q0(V q0, V q, const Box& b0) {
  for (int k = b0.ks; k <= b0.ke; ++k)
    for (int j = b0.js; j <= b0.je; ++j)
      for (int i = b0.is; i <= b0.ie; ++i)
        for (int c = 1; c <= 5; ++c) {
          Q0(q0, -1, c, i, j, k) = Q0(q0, 0, c, i, j, k);
          Q0(q0, 0, c, i, j, k) = q(c, i, j, k);
        }
}

}  // namespace oracle
