// Spalart-Allmaras one-equation model (sub_tur_sa.f90): residual of the
// advection, diffusion and source terms plus the scalar LU-SGS update, loosely
// coupled after the mean-flow update as in main.f90:414-419.
//
// sa_rhs2 works on zero-filled temporaries written only on the updated box, so
// a second difference next to a physical boundary reads a zero neighbour
// (sub_tur_sa.f90:259-291, :359-403).  The SA scratch planes here are written
// only on the updated box and are zero elsewhere, which reproduces that.
#include <cmath>

#include "aero_device.cuh"
#include "aero_kernels.h"

namespace aero {

namespace {

// One-sided at the physical ends is0/ie0, central elsewhere (sub_tur_sa.f90:297-303).
__device__ __forceinline__ double d1(const double* f, long n, long st, int pos, int lo0, int hi0) {
  if (pos == lo0) return f[n + st] - f[n];
  if (pos == hi0) return f[n] - f[n - st];
  return (f[n + st] - f[n - st]) / 2.0;
}

__device__ __forceinline__ void node_of(const Box& bx, long t, int& i, int& j, int& k) {
  i = bx.is + (int)(t % bx.nx());
  long r = t / bx.nx();
  j = bx.js + (int)(r % bx.ny());
  k = bx.ks + (int)(r / bx.ny());
}

}  // namespace

// Pass A over the updated box: dnut/dxi, dnut/deta, dnut/dzeta, the alpha/beta/
// gamma contractions and nu + (1+cb2)*nut (sub_tur_sa.f90:294-413) into SA
// scratch planes 0..6.
__global__ void k_sa_a(const BlockView* __restrict__ blocks, CaseConsts cc_launch) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
  const Box& b1 = B.b1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b1.size()) return;
  int i, j, k;
  node_of(b1, t, i, j, k);
  long n = B.at(i, j, k);
  const long st[3] = {1, (long)B.nx, (long)B.nx * B.ny};
  const int pos[3] = {i, j, k};
  const int lo0[3] = {B.b0.is, B.b0.js, B.b0.ks}, hi0[3] = {B.b0.ie, B.b0.je, B.b0.ke};
  const double* nut = B.f[F_NUT];
  double g[3] = {0.0, 0.0, 0.0};
  int ndir = cc.dimension == IFLAG_3D ? 3 : 2;
  for (int d = 0; d < ndir; ++d) g[d] = d1(nut, n, st[d], pos[d], lo0[d], hi0[d]);
  double* S = B.f[F_SAS];
  long P = B.plane;
  S[0 * P + n] = g[0];
  S[1 * P + n] = g[1];
  S[2 * P + n] = g[2];
  S[3 * P + n] = B.v(F_ALPHA, 1, n) * g[0] + B.v(F_ALPHA, 2, n) * g[1] + B.v(F_ALPHA, 3, n) * g[2];
  S[4 * P + n] = B.v(F_BETA, 1, n) * g[0] + B.v(F_BETA, 2, n) * g[1] + B.v(F_BETA, 3, n) * g[2];
  S[5 * P + n] = B.v(F_GAMMA, 1, n) * g[0] + B.v(F_GAMMA, 2, n) * g[1] + B.v(F_GAMMA, 3, n) * g[2];
  double nu0 = B.v(F_AMU, 1, n) / B.v(F_PRI, 1, n);
  S[6 * P + n] = nu0 + (1.0 + SA_CB2) * nut[n];
}

// Pass B over the updated box: sa_rhs = advection (sa_rhs1) + diffusion
// (sa_rhs2) + production/destruction (sa_rhs3), in that order, and the source
// linearisation diasd (sub_tur_sa.f90:152-208, :359-512, :561-625).
__device__ __forceinline__ void sa_b_body(const BlockView* __restrict__ blocks, CaseConsts cc_launch) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
  const Box& b1 = B.b1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b1.size()) return;
  int i, j, k;
  node_of(b1, t, i, j, k);
  long n = B.at(i, j, k);
  const long st[3] = {1, (long)B.nx, (long)B.nx * B.ny};
  const int pos[3] = {i, j, k};
  const int lo0[3] = {B.b0.is, B.b0.js, B.b0.ks}, hi0[3] = {B.b0.ie, B.b0.je, B.b0.ke};
  const double* nut = B.f[F_NUT];
  const double* S = B.f[F_SAS];
  long P = B.plane;
  bool three = cc.dimension == IFLAG_3D;
  double re = cc.re;
  double m[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) m[c] = B.v(F_DXIDX, c + 1, n);
  double u = B.v(F_PRI, 2, n), v = B.v(F_PRI, 3, n), w = B.v(F_PRI, 4, n);
  double nut0 = nut[n];
  // sa_rhs1: first-order upwind advection on the contravariant velocities
  double adv[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < (three ? 3 : 2); ++d) {
    double uu = m[3 * d] * u + m[3 * d + 1] * v + m[3 * d + 2] * w;
    double nutp = nut[n + st[d]], nutm = nut[n - st[d]];
    adv[d] = -(0.5 * (uu + fabs(uu)) * (nut0 - nutm) + 0.5 * (uu - fabs(uu)) * (nutp - nut0));
  }
  double rhs = adv[0] + adv[1] + adv[2];
  // sa_rhs2: diffusion
  double ta = d1(S + 3 * P, n, st[0], pos[0], lo0[0], hi0[0]);
  double tb = d1(S + 4 * P, n, st[1], pos[1], lo0[1], hi0[1]);
  double tc = three ? d1(S + 5 * P, n, st[2], pos[2], lo0[2], hi0[2]) : 0.0;
  double txi = d1(S + 6 * P, n, st[0], pos[0], lo0[0], hi0[0]);
  double teta = d1(S + 6 * P, n, st[1], pos[1], lo0[1], hi0[1]);
  double tzeta = three ? d1(S + 6 * P, n, st[2], pos[2], lo0[2], hi0[2]) : 0.0;
  double tx = txi * m[0] + teta * m[3] + tzeta * m[6];
  double ty = txi * m[1] + teta * m[4] + tzeta * m[7];
  double tz = txi * m[2] + teta * m[5] + tzeta * m[8];
  double inv_j0 = B.s(F_INVJ, n);
  double deltanut = (ta + tb + tc) / inv_j0;
  double gx = S[0 * P + n], ge = S[1 * P + n], gz = S[2 * P + n];
  double dnutdx = gx * m[0] + ge * m[3] + gz * m[6];
  double dnutdy = gx * m[1] + ge * m[4] + gz * m[7];
  double dnutdz = gx * m[2] + ge * m[5] + gz * m[8];
  double temp = S[6 * P + n];
  double diff = -(SA_CB2 / (re * SA_DTA)) * nut0 * deltanut +
                (1.0 / (re * SA_DTA)) * (temp * deltanut + tx * dnutdx + ty * dnutdy + tz * dnutdz);
  rhs = rhs + diff;
  // sa_rhs3: production / destruction and the derivative of the source
  double d = B.v(F_PRI, 1, n);
  double nu0 = B.v(F_AMU, 1, n) / d;
  double omega = fabs(B.s(F_VOR, n));
  double dist0 = B.s(F_LENGTH, n);
  double leix = fmax(nut0 / nu0, 0.001);
  double fv1 = p3(leix) / (p3(leix) + SA_CV13);
  double fv2 = 1.0 - leix / (1.0 + leix * fv1);
  double s = omega + nut0 * fv2 / (re * SA_KAR2 * p2(dist0));
  s = fmax(s, 0.3 * omega);
  double dv = s * re * SA_KAR2 * p2(dist0);
  dv = fmax(dv, 1.0e-6);
  double r = nut0 * dv;  // the reference's r (sub_tur_sa.f90:579)
  r = fmin(r, 10.0);
  double g = r + SA_CW2 * (p6(r) - r);
  double fw = g * crm::pow((1.0 + 64.0) / (p6(g) + 64.0), 1.0 / 6.0);
  double ft2 = SA_CT3 * crm::exp(-SA_CT4 * p2(leix));
  double aaa = SA_CB1 * ((1.0 - ft2) * fv2 + ft2) / SA_KAR2;
  double bbb = SA_CW1 * fw;
  double ccc = nut0 / p2(dist0);
  double sd1 = (aaa - bbb) * ccc / re;
  double sd = sd1 * nut0;
  double sp = SA_CB1 * (1.0 - ft2) * omega * nut0;
  rhs = rhs + sd + sp;
  B.s(F_SARHS, n) = rhs;
  double leixn = 1.0 / nu0;
  double fv1n = (3.0 * p2(leix) * leixn * (p3(leix) + SA_CV13) - p3(leix) * (3.0 * p2(leix) * leixn)) /
                p2(p3(leix) + SA_CV13);
  double fv2n = (leixn * (1.0 + leix * fv1) - leix * (leixn * fv1 + leix * fv1n)) / p2(1.0 + leix * fv1);
  double ft2n = -(2.0 * SA_CT4 * leix * leixn * ft2);
  double sn = 1.0 / (re * SA_KAR2 * p2(dist0)) * (fv2 + fv2n * nut0);
  dv = p2(s) * (re * SA_KAR2 * p2(dist0));
  dv = fmax(dv, 1.0e-6);
  double rn = (s - sn * nut0) / dv;
  double gn = (1.0 + SA_CW2 * 6.0 * p5(r) - SA_CW2) * rn;
  const double cw3m6 = 0.015625;  // cw3**(-6)
  double fwn = -((1.0 / 6.0) * crm::pow((crm::pow(g, -6.0) + cw3m6) / (1.0 + cw3m6), -7.0 / 6.0));
  fwn = fwn / (1.0 + cw3m6) * (-(6.0 * crm::pow(g, -7.0))) * gn;
  double spn = SA_CB1 * (1.0 - ft2) * omega + SA_CB1 * (-ft2n) * omega * nut0;
  double sdn = (1.0 / re) * (SA_CB1 * (fv2 - ft2 * fv2 + ft2) / SA_KAR2 - SA_CW1 * fw) * 2.0 * nut0 / p2(dist0);
  sdn = (1.0 / re) * (SA_CB1 * (fv2n - ft2n * fv2 - ft2 * fv2n + ft2n) / SA_KAR2 - SA_CW1 * fwn) *
            (p2(nut0) / p2(dist0)) + sdn;
  B.s(F_DIASD, n) = fmin(spn + sdn, 0.0);
}
__global__ void k_sa_b(const BlockView* __restrict__ blocks, CaseConsts cc_launch) { sa_b_body(blocks, cc_launch); }


// k_sa_b for mixed precision (aero_set_precision(1)): the same three terms
// with their arithmetic in FP32 -- the advection products of FP32 contravariant
// velocities with FP64 differences of nut, the diffusion products of FP64
// differences of the scratch planes with FP32 metrics, and the production /
// destruction closure (fv1, fv2, fw, ft2) -- summed into the FP64 sa_rhs in the
// order of k_sa_b; diasd likewise.  nut, the metrics, the diagonal and the
// sweep stay FP64 (the scalar LU-SGS sees only sa_rhs and diasd).
__global__ void k_sa_b_mixed(const BlockView* __restrict__ blocks, CaseConsts cc_launch) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
  const Box& b1 = B.b1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b1.size()) return;
  int i, j, k;
  node_of(b1, t, i, j, k);
  long n = B.at(i, j, k);
  const long st[3] = {1, (long)B.nx, (long)B.nx * B.ny};
  const int pos[3] = {i, j, k};
  const int lo0[3] = {B.b0.is, B.b0.js, B.b0.ks}, hi0[3] = {B.b0.ie, B.b0.je, B.b0.ke};
  const double* nut = B.f[F_NUT];
  const double* S = B.f[F_SAS];
  long P = B.plane;
  bool three = cc.dimension == IFLAG_3D;
  const float re = (float)cc.re;
  float m[9];
#pragma unroll
  for (int c = 0; c < 9; ++c) m[c] = (float)B.v(F_DXIDX, c + 1, n);
  const float u = (float)B.v(F_PRI, 2, n), v = (float)B.v(F_PRI, 3, n), w = (float)B.v(F_PRI, 4, n);
  const double nut0d = nut[n];
  const float nut0 = (float)nut0d;
  // sa_rhs1: first-order upwind advection
  float adv[3] = {0.0f, 0.0f, 0.0f};
  for (int d = 0; d < (three ? 3 : 2); ++d) {
    float uu = m[3 * d] * u + m[3 * d + 1] * v + m[3 * d + 2] * w;
    float dm = (float)(nut0d - nut[n - st[d]]), dp = (float)(nut[n + st[d]] - nut0d);
    adv[d] = -(0.5f * (uu + fabsf(uu)) * dm + 0.5f * (uu - fabsf(uu)) * dp);
  }
  double rhs = (double)adv[0] + (double)adv[1] + (double)adv[2];
  // sa_rhs2: diffusion
  float ta = (float)d1(S + 3 * P, n, st[0], pos[0], lo0[0], hi0[0]);
  float tb = (float)d1(S + 4 * P, n, st[1], pos[1], lo0[1], hi0[1]);
  float tc = three ? (float)d1(S + 5 * P, n, st[2], pos[2], lo0[2], hi0[2]) : 0.0f;
  float txi = (float)d1(S + 6 * P, n, st[0], pos[0], lo0[0], hi0[0]);
  float teta = (float)d1(S + 6 * P, n, st[1], pos[1], lo0[1], hi0[1]);
  float tzeta = three ? (float)d1(S + 6 * P, n, st[2], pos[2], lo0[2], hi0[2]) : 0.0f;
  float tx = txi * m[0] + teta * m[3] + tzeta * m[6];
  float ty = txi * m[1] + teta * m[4] + tzeta * m[7];
  float tz = txi * m[2] + teta * m[5] + tzeta * m[8];
  const float inv_j0 = (float)B.s(F_INVJ, n);
  float deltanut = (ta + tb + tc) / inv_j0;
  float gx = (float)S[0 * P + n], ge = (float)S[1 * P + n], gz = (float)S[2 * P + n];
  float dnutdx = gx * m[0] + ge * m[3] + gz * m[6];
  float dnutdy = gx * m[1] + ge * m[4] + gz * m[7];
  float dnutdz = gx * m[2] + ge * m[5] + gz * m[8];
  float temp = (float)S[6 * P + n];
  const float rd = 1.0f / (re * (float)SA_DTA);
  float diff = -((float)SA_CB2 * rd) * nut0 * deltanut + rd * (temp * deltanut + tx * dnutdx + ty * dnutdy + tz * dnutdz);
  rhs = rhs + (double)diff;
  // sa_rhs3: production / destruction
  const float kar2 = (float)SA_KAR2, cv13 = (float)SA_CV13, cw2 = (float)SA_CW2, cb1 = (float)SA_CB1;
  const float ct3 = (float)SA_CT3, ct4 = (float)SA_CT4, cw1 = (float)SA_CW1;
  float nu0 = (float)(B.v(F_AMU, 1, n) / B.v(F_PRI, 1, n));
  float omega = fabsf((float)B.s(F_VOR, n));
  float dist2 = (float)p2(B.s(F_LENGTH, n));
  float leix = fmaxf(nut0 / nu0, 0.001f);
  float l3 = leix * leix * leix;
  float fv1 = l3 / (l3 + cv13);
  float fv2 = 1.0f - leix / (1.0f + leix * fv1);
  float sv = omega + nut0 * fv2 / (re * kar2 * dist2);
  sv = fmaxf(sv, 0.3f * omega);
  float dv = fmaxf(sv * re * kar2 * dist2, 1.0e-6f);
  float r = fminf(nut0 * dv, 10.0f);  // the reference's r (sub_tur_sa.f90:579)
  float r2 = r * r, r6 = r2 * r2 * r2;
  float g = r + cw2 * (r6 - r);
  float g2 = g * g, g6 = g2 * g2 * g2;
  float fw = g * powf(65.0f / (g6 + 64.0f), 1.0f / 6.0f);
  float ft2 = ct3 * expf(-ct4 * leix * leix);
  float aaa = cb1 * ((1.0f - ft2) * fv2 + ft2) / kar2;
  float bbb = cw1 * fw;
  float ccc = nut0 / dist2;
  float sd = (aaa - bbb) * ccc / re * nut0;
  float sp = cb1 * (1.0f - ft2) * omega * nut0;
  rhs = rhs + (double)sd + (double)sp;
  B.s(F_SARHS, n) = rhs;
  float leixn = 1.0f / nu0;
  float fv1n = (3.0f * leix * leix * leixn * (l3 + cv13) - l3 * (3.0f * leix * leix * leixn)) / ((l3 + cv13) * (l3 + cv13));
  float fv2n = (leixn * (1.0f + leix * fv1) - leix * (leixn * fv1 + leix * fv1n)) / ((1.0f + leix * fv1) * (1.0f + leix * fv1));
  float ft2n = -(2.0f * ct4 * leix * leixn * ft2);
  float sn = 1.0f / (re * kar2 * dist2) * (fv2 + fv2n * nut0);
  dv = fmaxf(sv * sv * (re * kar2 * dist2), 1.0e-6f);
  float rn = (sv - sn * nut0) / dv;
  float r5 = r2 * r2 * r;
  float gn = (1.0f + cw2 * 6.0f * r5 - cw2) * rn;
  const float cw3m6 = 0.015625f;
  float fwn = -((1.0f / 6.0f) * powf((powf(g, -6.0f) + cw3m6) / (1.0f + cw3m6), -7.0f / 6.0f));
  fwn = fwn / (1.0f + cw3m6) * (-(6.0f * powf(g, -7.0f))) * gn;
  float spn = cb1 * (1.0f - ft2) * omega + cb1 * (-ft2n) * omega * nut0;
  float sdn = (1.0f / re) * (cb1 * (fv2 - ft2 * fv2 + ft2) / kar2 - cw1 * fw) * 2.0f * nut0 / dist2;
  sdn = (1.0f / re) * (cb1 * (fv2n - ft2n * fv2 - ft2 * fv2n + ft2n) / kar2 - cw1 * fwn) * (nut0 * nut0 / dist2) + sdn;
  B.s(F_DIASD, n) = (double)fminf(spn + sdn, 0.0f);
}

// sa_lusgs diagonal and upwind coefficients of every updated node
// (sub_tur_sa.f90:676-750, :762-778) in the plane-local layout of the sweep:
// the records of hyperplane h form one chunk at kSaRec*poff[h], element x of
// plane-local node t at x*cnt + t, so a warp's loads are consecutive words.
// x = 0..2: 0.5*(U+|U|) per direction, 3..5: 0.5*(U-|U|), 6: sa_rhs, 7: diag,
// 8 / 9: the packed forward / backward neighbours, 10: 1/diag (the sweeps'
// exact division by diag uses it), 11: unused (keeps 16-byte chunks).
__global__ void k_sa_recs(const BlockView* __restrict__ blocks, CaseConsts cc_launch) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
  const Box& b1 = B.b1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= b1.size()) return;
  long pos = t;  // the t-th node in hyperplane-major order
  long n = B.nat[pos];
  long r = n / B.nx;
  const int i = B.b.is + (int)(n - r * B.nx);
  const int j = B.b.js + (int)(r % B.ny);
  const int k = B.b.ks + (int)(r / B.ny);
  const int h = (i - b1.is) + (j - b1.js) + (k - b1.ks);
  const long base = B.poff[h], cnt = B.poff[h + 1] - base;
  double phi = (cc.cfl >= 1.0e3 && cc.time == IFLAG_STEADY) ? 0.0 : 1.0;
  double u = B.v(F_PRI, 2, n), v = B.v(F_PRI, 3, n), w = B.v(F_PRI, 4, n);
  double x0 = B.v(F_DXIDX, 1, n), y0 = B.v(F_DXIDX, 2, n), z0 = B.v(F_DXIDX, 3, n);
  double d2 = x0 * x0 + y0 * y0 + z0 * z0;
  double cu = x0 * u + y0 * v + z0 * w;
  x0 = B.v(F_DXIDX, 4, n); y0 = B.v(F_DXIDX, 5, n); z0 = B.v(F_DXIDX, 6, n);
  d2 = d2 + x0 * x0 + y0 * y0 + z0 * z0;
  double cv = x0 * u + y0 * v + z0 * w;
  x0 = B.v(F_DXIDX, 7, n); y0 = B.v(F_DXIDX, 8, n); z0 = B.v(F_DXIDX, 9, n);
  d2 = d2 + x0 * x0 + y0 * y0 + z0 * z0;
  double cw = x0 * u + y0 * v + z0 * w;
  double tm = 4.0 * d2 * B.s(F_NUT, n) / cc.re;
  double diag = 1.0 / B.s(F_DT, n) * phi + fabs(cu) + fabs(cv) + fabs(cw) + tm - B.s(F_DIASD, n);
  double* rec = B.sa_rec + kSaRec * base + (pos - base);
  rec[0] = 0.5 * (cu + fabs(cu));
  rec[cnt] = 0.5 * (cv + fabs(cv));
  rec[2 * cnt] = 0.5 * (cw + fabs(cw));
  rec[3 * cnt] = 0.5 * (cu - fabs(cu));
  rec[4 * cnt] = 0.5 * (cv - fabs(cv));
  rec[5 * cnt] = 0.5 * (cw - fabs(cw));
  rec[6 * cnt] = B.s(F_SARHS, n);
  rec[7 * cnt] = diag;
  const int* nb = B.nbr + 6 * pos;
  rec[8 * cnt] = pack_nbrs(nb, h > 0 ? B.poff[h - 1] : 0);
  rec[9 * cnt] = pack_nbrs(nb + 3, h + 1 < B.nplanes ? B.poff[h + 1] : 0);
  rec[10 * cnt] = 1.0 / diag;
}

namespace {

struct SaFwd {
  double a[3], rhs, diag, rdiag, packed;
};
struct SaBwd {
  double b[3], diag, rdiag, packed, dqs, nut;
  long nat;
};
__device__ __forceinline__ void sa_load_fwd(const BlockView& B, int h, int t, SaFwd& f) {
  const long base = B.poff[h];
  const int cnt = (int)(B.poff[h + 1] - base);
  const double* r = B.sa_rec + kSaRec * base + t;
  f.a[0] = r[0];
  f.a[1] = r[cnt];
  f.a[2] = r[2 * cnt];
  f.rhs = r[6 * cnt];
  f.diag = r[7 * cnt];
  f.rdiag = r[10 * cnt];
  f.packed = r[8 * cnt];
}
__device__ __forceinline__ void sa_load_bwd(const BlockView& B, int h, int t, SaBwd& f) {
  const long base = B.poff[h];
  const int cnt = (int)(B.poff[h + 1] - base);
  const double* r = B.sa_rec + kSaRec * base + t;
  f.b[0] = r[3 * cnt];
  f.b[1] = r[4 * cnt];
  f.b[2] = r[5 * cnt];
  f.diag = r[7 * cnt];
  f.rdiag = r[10 * cnt];
  f.packed = r[9 * cnt];
  f.dqs = B.sa_dq[base + t];
  f.nat = B.nat[base + t];
  f.nut = B.s(F_NUT, f.nat);  // loaded with the records, off the plane-to-plane chain
}

}  // namespace

// L2 prefetch of the SA records of plane h (kSaRec * 8 bytes per node, a
// multiple of 16, so the chunk starts and ends on 16-byte boundaries).
__device__ __forceinline__ void sa_prefetch(const BlockView& B, int h) {
  if (h < 0 || h >= B.nplanes) return;
  const long base = B.poff[h];
  const unsigned bytes = (unsigned)((B.poff[h + 1] - base) * kSaRec * 8);
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(B.sa_rec + kSaRec * base), "r"(bytes) : "memory");
}

// Scalar LU-SGS sweeps of the SA equation and nut += dnut, one CTA per block,
// one thread per node of a hyperplane (sub_tur_sa.f90:759-818).  Each thread
// loads the records of its node of the next plane while it computes the
// current one (one thread prefetches the plane after that into L2), so the
// plane-to-plane path is the shared-memory neighbours, one division (div_rn_lean
// with the reciprocal stored in the records: the correctly rounded quotient,
// as a / b) and the barrier.
__device__ __forceinline__ void sa_sweep_body(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.x];
  if (B.retired()) return;
  extern __shared__ double sdn[];  // two planes of pmax values
  const int P = B.pmax;
  const int H = B.nplanes;
  const int T = blockDim.x, tid = threadIdx.x;
  auto cnt_of = [&](int h) { return (int)(B.poff[h + 1] - B.poff[h]); };
  {
    SaFwd nx{};
    if (H > 0 && tid < cnt_of(0)) sa_load_fwd(B, 0, tid, nx);
    if (tid == 32) sa_prefetch(B, 1);
    for (int h = 0; h < H; ++h) {
      const SaFwd cu = nx;
      if (tid == 32) sa_prefetch(B, h + 2);
      if (h + 1 < H && tid < cnt_of(h + 1)) sa_load_fwd(B, h + 1, tid, nx);
      const long base = B.poff[h];
      const int cnt = (int)(B.poff[h + 1] - base);
      const double* prev = sdn + P * ((h + 1) & 1);
      double* cur = sdn + P * (h & 1);
      for (int t = tid; t < cnt; t += T) {
        SaFwd f = cu;
        if (t != tid) sa_load_fwd(B, h, t, f);
        double tt[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          int w = nbr_local(f.packed, d);
          tt[d] = w < 0 ? 0.0 : f.a[d] * prev[w];
        }
        double v = div_rn_lean(f.rhs + (tt[0] + tt[1] + tt[2]), f.diag, f.rdiag);
        cur[t] = v;
        B.sa_dq[base + t] = v;
      }
      __syncthreads();
    }
  }
  SaBwd nx{};
  if (H > 0 && tid < cnt_of(H - 1)) sa_load_bwd(B, H - 1, tid, nx);
  if (tid == 32) sa_prefetch(B, H - 2);
  for (int h = H - 1; h >= 0; --h) {
    const SaBwd cu = nx;
    if (tid == 32) sa_prefetch(B, h - 2);
    if (h > 0 && tid < cnt_of(h - 1)) sa_load_bwd(B, h - 1, tid, nx);
    const long base = B.poff[h];
    const int cnt = (int)(B.poff[h + 1] - base);
    const double* prev = sdn + P * ((h + 1) & 1);
    double* cur = sdn + P * (h & 1);
    for (int t = tid; t < cnt; t += T) {
      SaBwd f = cu;
      if (t != tid) sa_load_bwd(B, h, t, f);
      double tt[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        int w = nbr_local(f.packed, d);
        tt[d] = w < 0 ? 0.0 : f.b[d] * prev[w];
      }
      double v = f.dqs - div_rn_lean(tt[0] + tt[1] + tt[2], f.diag, f.rdiag);
      cur[t] = v;
      B.s(F_NUT, f.nat) = f.nut + v;
    }
    __syncthreads();
  }
}

// Two register budgets: up to 1024 threads (64 registers each) and up to 768
// (80 registers, no spills), the launch picking the second when planes fit.
__global__ void __launch_bounds__(1024) k_sa_sweep(const BlockView* __restrict__ blocks) { sa_sweep_body(blocks); }
__global__ void __launch_bounds__(768) k_sa_sweep_768(const BlockView* __restrict__ blocks) { sa_sweep_body(blocks); }

// The SA sweeps pipelined over a cluster of CTAs by k-slabs, as
// k_lusgs_sweep_slab pipelines the mean-flow sweeps (slab::Geom: CTA r owns
// the nodes of one range of k-offsets; after each plane a CTA copies its edge
// k-segment's values into the downstream CTA's inbox with one bulk copy,
// counted on that CTA's mbarrier; relaxed progress counters keep the D-plane
// slots from being overwritten while in use; every wait is bounded, and
// slab::finish keeps every CTA resident until no copy can still land in it).
// One node per thread, its records loaded two steps ahead.  The arithmetic
// per node is sa_sweep_body's, so the result is the same to the bit.
__global__ void __launch_bounds__(512, 1) k_sa_sweep_slab(const BlockView* __restrict__ blocks, unsigned* status,
                                                          int So, int L, int D) {
  extern __shared__ __align__(16) double sdyn[];
  double* stage = sdyn;            // D x L: this slab's edge values, copied downstream
  double* inbox = stage + D * L;   // D x L: the upstream slab's edge values
  double* ring = inbox + D * L;    // D x So: this slab's values
  __shared__ __align__(8) unsigned long long full[kSlabSlots];
  __shared__ int s_prog[2];  // last step completed by the CTA below / above
  __shared__ int s_fail;
  const int ncta = (int)slab::size();
  const BlockView& B = blocks[blockIdx.x / ncta];
  if (B.retired()) return;
  const slab::Geom G(B, ncta, (int)slab::rank());
  const int H = G.H, tid = (int)threadIdx.x;
  if (tid == 0) {
    s_prog[0] = -1;
    s_prog[1] = -1;
    s_fail = 0;
    for (int x = 0; x < D; ++x) slab::bar_init(&full[x], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  slab::sync();  // every CTA's counters and mbarriers exist before a neighbour touches them
  const unsigned slot_bytes = (unsigned)(L * sizeof(double));
  if (G.active()) {
    const unsigned at_lo = G.has_lo() ? slab::map(slab::local(&s_prog[1]), G.me - 1) : 0u;
    const unsigned at_hi = G.has_hi() ? slab::map(slab::local(&s_prog[0]), G.me + 1) : 0u;
    const unsigned inbox_l = slab::local(inbox), full_l = slab::local(full), stage_l = slab::local(stage);
    // the records of this thread's node, loaded two steps ahead (even and odd steps)
    SaFwd pf[2] = {};
    SaBwd pb[2] = {};
    auto preload = [&](int gs, SaFwd& f, SaBwd& bw) {
      if (gs >= 2 * H) return;
      const int h = G.plane(gs);
      const int t0 = G.seg(h, G.c0), n = G.seg(h, G.c1) - t0;
      if (tid < n) {
        if (gs < H)
          sa_load_fwd(B, h, t0 + tid, f);
        else
          sa_load_bwd(B, h, t0 + tid, bw);
      }
    };
    // L2 prefetch of step gs's whole chunks (records and, backward, sa_dq and
    // the natural indices) by the pass's leading CTA (the one without an
    // upstream slab: every other CTA reaches each step after it)
    const bool lead_f = G.me == 0, lead_b = G.me == G.ce - 1;
    auto prefetch = [&](int gs) {
      if (gs >= 2 * H || tid >= 35 || tid < 32) return;
      const bool fwd = gs < H;
      if (!(fwd ? lead_f : lead_b)) return;
      const long base = B.poff[G.plane(gs)];
      const long cnt = B.poff[G.plane(gs) + 1] - base;
      if (tid == 32) slab::prefetch_span(B.sa_rec + kSaRec * base, 8L * kSaRec * cnt);
      if (tid == 33 && !fwd) slab::prefetch_span(B.sa_dq + base, 8L * cnt);
      if (tid == 34 && !fwd) slab::prefetch_span(B.nat + base, 8L * cnt);
    };
    unsigned parity = 0;  // bit x: parity of the next phase of full[x] to wait for
    // one plane step; false (in every thread) when a wait of this CTA ran out
    auto step = [&](int gs, const SaFwd& pre_f, const SaBwd& pre_b) -> bool {
      const bool fwd = gs < H;
      const int h = G.plane(gs);
      const long base = B.poff[h];
      const int t0 = G.seg(h, G.c0), n = G.seg(h, G.c1) - t0;
      const bool need_dn = G.need_dn(gs);
      const int x = gs % D, xp = (gs + D - 1) % D;
      bool fail = false;
      if (G.need_up(gs)) {
        if (tid == 0) slab::bar_expect(&full[xp], slot_bytes);
        fail = !slab::bar_wait(&full[xp], (parity >> xp) & 1u);
        parity ^= 1u << xp;
        if (fail) note_timeout(status, TS_SA_SLAB, (int)(blockIdx.x / ncta), G.me, gs, TW_PLANE);
      }
      if (!fail && need_dn) {
        fail = !slab::wait_for(&s_prog[fwd ? 1 : 0], gs - D + 1);
        if (fail) note_timeout(status, TS_SA_SLAB, (int)(blockIdx.x / ncta), G.me, gs, TW_PROGRESS);
      }
      if (!fail && tid < n) {  // the launch gives every node of a slab's plane a thread
        const int hp = G.plane(gs > 0 ? gs - 1 : 0);
        const int p0 = G.seg(hp, G.c0), np = G.seg(hp, G.c1) - p0;
        const int eb = G.seg(hp, max(G.c_up(gs), 0));
        const double* own = ring + xp * So;
        const double* edge = inbox + xp * L;
        auto prev = [&](int w, int d) {
          // the i and j neighbours share the node's k-offset, so they are the slab's own
          return (d < 2 || (unsigned)(w - p0) < (unsigned)np) ? own[w - p0] : edge[w - eb];
        };
        const int t = t0 + tid;
        double tt[3], v;
        if (fwd) {
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const int w = nbr_local(pre_f.packed, d);
            tt[d] = w < 0 ? 0.0 : pre_f.a[d] * prev(w, d);
          }
          v = div_rn_lean(pre_f.rhs + (tt[0] + tt[1] + tt[2]), pre_f.diag, pre_f.rdiag);
          B.sa_dq[base + t] = v;
        } else {
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const int w = nbr_local(pre_b.packed, d);
            tt[d] = w < 0 ? 0.0 : pre_b.b[d] * prev(w, d);
          }
          // sa_dq of the first backward plane (the forward pass's last) is
          // written by the step before, after its two-step-ahead load was issued
          const double dqs = gs == H ? __ldcg(B.sa_dq + base + t) : pre_b.dqs;
          v = dqs - div_rn_lean(tt[0] + tt[1] + tt[2], pre_b.diag, pre_b.rdiag);
          B.s(F_NUT, pre_b.nat) = pre_b.nut + v;
        }
        ring[x * So + tid] = v;
        if (need_dn) {
          const int e0 = G.seg(h, G.c_dn(gs));
          if (t >= e0 && t < G.seg(h, G.c_dn(gs) + 1)) stage[x * L + (t - e0)] = v;
        }
      }
      if (need_dn) slab::fence_to_copies();
      if (__syncthreads_or(fail ? 1 : 0)) {
        if (tid == 0) s_fail = 1;
        return false;
      }
      if (tid == 0) {
        if (need_dn) {
          const unsigned r = (unsigned)G.rank_dn(gs);
          const unsigned off = (unsigned)(x * L * sizeof(double));
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
    preload(0, pf[0], pb[0]);
    preload(1, pf[1], pb[1]);
    for (int gs = 0; gs < 2 * H; gs += 2) {
      if (!step(gs, pf[0], pb[0])) break;
      prefetch(gs + PF);
      preload(gs + 2, pf[0], pb[0]);
      if (gs + 1 >= 2 * H) break;
      if (!step(gs + 1, pf[1], pb[1])) break;
      prefetch(gs + 1 + PF);
      preload(gs + 3, pf[1], pb[1]);
    }
  }
  slab::finish(s_fail, ncta, status, B);
}

// length = dist over the full box (sub_tur_sa.f90:51-57; no DES).
// With iflag_des = 1 (DES97) length = min(dist, cdes*spacing); with 2 (DDES)
// length = dist - fd*max(0, dist - cdes*spacing), fd = 1 - tanh((8 rd)^3),
// rd = (nu + nut) / (|S'| Re kar^2 dist^2) with |S'| formed from the
// off-diagonal velocity gradients (sub_tur_sa.f90:51-97).  The reference
// declares dudx as (3, is:ie, js:je, ks:ke, 3) over its (9, ...) array, so
// dudx(a, node, c) reads word (a-1) + 3*node + 3*N*(c-1) of the (9, node)
// layout, N the box size; that is reproduced.
__global__ void k_sa_length(const BlockView* __restrict__ blocks, CaseConsts cc_launch) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
  long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long N = B.b.size();
  if (n >= N) return;
  const double cdes = 0.65;
  double dist0 = B.s(F_DIST, n);
  double len = dist0;
  if (cc.des == IFLAG_DES97) {
    double a = cdes * B.s(F_SPACING, n);
    len = a < dist0 ? a : dist0;  // min(dist0, cdes*spac0)
  } else if (cc.des == IFLAG_DDES) {
    auto g3 = [&](int a, int c) {
      long w = (a - 1) + 3 * n + 3 * N * (c - 1);  // word of the (9, node) array
      long node = w / 9;
      return B.v(F_DUDX, (int)(w - 9 * node) + 1, node);
    };
    double uy = g3(1, 2), uz = g3(1, 3), vx = g3(2, 1), vz = g3(2, 3), wx = g3(3, 1), wy = g3(3, 2);
    double d0 = B.v(F_PRI, 1, n), nut0 = B.s(F_NUT, n), nu0 = B.v(F_AMU, 1, n) / d0;
    double spac0 = B.s(F_SPACING, n);
    double temp = p2(uy) + p2(uz) + p2(vx) + p2(vz) + p2(wx) + p2(wy);
    temp = sqrt(temp);
    double rd = (nu0 + nut0) / (temp * cc.re * SA_KAR2 * p2(dist0));
    double fd = 1.0 - tanh(p3(8.0 * rd));
    double e = dist0 - cdes * spac0;
    len = dist0 - fd * (0.0 < e ? e : 0.0);
  }
  B.s(F_LENGTH, n) = len;
  B.s(F_SARHS, n) = 0.0;
}

}  // namespace aero
