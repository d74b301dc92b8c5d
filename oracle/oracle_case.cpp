// TEST INFRASTRUCTURE ONLY (see oracle_common.h): module-state routines
// (physical BCs, block-interface halo and averaging, residual, freestream init,
// wall distance) and the per-iteration driver of main.f90:343-447, restated with
// a single "rank" that owns every block, so every interface takes the reference's
// same-rank copy branch (sub_bc_updatebuffer.f90:155-171).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "oracle_blockops.h"

namespace oracle {

enum Field {
  F_Q, F_PRI, F_RHSI, F_RHSV, F_RHS, F_DT, F_DXIDX, F_INVJ, F_AMU, F_NUT, F_SARHS,
  F_X, F_Y, F_Z, F_DIST, F_ALPHA, F_BETA, F_GAMMA, F_DUDX, F_TAO, F_VOR, F_LENGTH, F_SPACING, F_Q0,
  F_COUNT
};
static const int kNc[F_COUNT] = {5, 7, 5, 5, 5, 1, 9, 1, 3, 1, 1, 1, 1, 1, 1, 3, 3, 3, 9, 6, 1, 1, 1, 10};

struct Sub {
  int f_no, face, is, ie, js, je, ks, ke, blk_t, subface_t, ori;
  Box box() const { return Box{is, ie, js, je, ks, ke}; }
  std::vector<double> send, recv, buf;  // buffer_send, buffer_recv, buffer
};

struct Block {
  bool used = false;
  Box b, b0, b1;
  std::vector<Sub> bc;
  double* f[F_COUNT] = {};
  V v(int fid) const { return V{f[fid], kNc[fid], b}; }
};

static std::vector<Block> g_blk;  // index m-1
static double g_last_dtmax = 0, g_last_dtmin = 0, g_last_cflmax = 0, g_last_cflmin = 0;

static Block& blk(int m) {
  if (m < 1 || m > (int)g_blk.size() || !g_blk[m - 1].used) {
    std::fprintf(stderr, "oracle: block %d is not registered\n", m);
    std::abort();
  }
  return g_blk[m - 1];
}

static void alloc_buffers() {
  // sub_init_readbcinfo.f90:440-475: send/buffer over the own subface box,
  // recv over the donor subface box; zero-filled.
  int BL = g_flags.bufferLength;
  for (auto& B : g_blk)
    for (auto& s : B.bc)
      if (s.blk_t > 0) {
        const Sub& d = blk(s.blk_t).bc.at(s.subface_t - 1);
        s.send.assign((size_t)BL * 9 * s.box().size(), 0.0);
        s.buf.assign((size_t)9 * s.box().size(), 0.0);
        s.recv.assign((size_t)BL * 9 * d.box().size(), 0.0);
      }
}

static inline double& S5(std::vector<double>& v, const Box& bx, int BL, int nb, int ind, int i, int j,
                         int k) {
  return v[(size_t)(nb - 1) + (size_t)BL * ((ind - 1) + 9 * (size_t)bx.at(i, j, k))];
}

// ---------------------------------------------------------------- physical BCs
struct FaceGeom {
  int dir;   // 0,1,2 = i,j,k
  int sgn;   // +1 interior is at plane+1 (low face), -1 at plane-1 (high face)
};
static FaceGeom face_geom(int face) { return FaceGeom{(face - 1) / 2, (face % 2 == 1) ? 1 : -1}; }

// Loops over the subface nodes of face `face`, where the subface box is
// (is,ie,js,je,ks,ke) exactly as the BC routine receives it; the boundary plane
// index is the lower bound of the box for low faces and the upper bound for
// high faces (sub_bc_-50_inflow.f90:21-231 and siblings).
template <class Fn>
static void for_face(int face, const Box& sb, Fn fn) {
  FaceGeom g = face_geom(face);
  if (g.dir == 0) {
    int i = g.sgn > 0 ? sb.is : sb.ie;
    for (int k = sb.ks; k <= sb.ke; ++k)
      for (int j = sb.js; j <= sb.je; ++j) fn(i, j, k, 1, 0, 0, g.sgn);
  } else if (g.dir == 1) {
    int j = g.sgn > 0 ? sb.js : sb.je;
    for (int k = sb.ks; k <= sb.ke; ++k)
      for (int i = sb.is; i <= sb.ie; ++i) fn(i, j, k, 0, 1, 0, g.sgn);
  } else {
    int k = g.sgn > 0 ? sb.ks : sb.ke;
    for (int j = sb.js; j <= sb.je; ++j)
      for (int i = sb.is; i <= sb.ie; ++i) fn(i, j, k, 0, 0, 1, g.sgn);
  }
}

static void bc_inflow(Block& B, const Box& sb, int face) {  // sub_bc_-50_inflow.f90:7-139
  V q = B.v(F_Q), tur = B.v(F_NUT);
  const Consts& c = g_consts;
  for_face(face, sb, [&](int i, int j, int k, int, int, int, int) {
    q(1, i, j, k) = c.d_0;
    q(2, i, j, k) = c.d_0 * c.u_0 * std::cos(c.aoa);
    q(3, i, j, k) = c.d_0 * c.u_0 * std::sin(c.aoa);
    q(4, i, j, k) = 0.0;
    q(5, i, j, k) = c.p_0 / (c.gamma - 1.0) + 0.5 * p2(c.u_0);
    if (g_flags.turbulence >= 1) tur(i, j, k) = c.nutinf;
  });
}

static void bc_outflow(Block& B, const Box& sb, int face) {  // sub_bc_-40_outflow.f90:9-129
  V q = B.v(F_Q), tur = B.v(F_NUT);
  for_face(face, sb, [&](int i, int j, int k, int di, int dj, int dk, int s) {
    int ii = i + s * di, jj = j + s * dj, kk = k + s * dk;
    for (int n = 1; n <= 5; ++n) q(n, i, j, k) = q(n, ii, jj, kk);
    if (g_flags.turbulence >= 1) tur(i, j, k) = tur(ii, jj, kk);
  });
}

// Symmetry plane and slip wall share the same update (sub_bc_-30_symm.f90:8-211,
// sub_bc_-20_solidwall.f90:10-211).
static void bc_mirror(Block& B, const Box& sb, int face) {
  V q = B.v(F_Q), tur = B.v(F_NUT), dxidx = B.v(F_DXIDX);
  for_face(face, sb, [&](int i, int j, int k, int di, int dj, int dk, int s) {
    int c0 = 3 * (di ? 0 : (dj ? 1 : 2)) + 1;
    double x0 = dxidx(c0, i, j, k), y0 = dxidx(c0 + 1, i, j, k), z0 = dxidx(c0 + 2, i, j, k);
    double temp = p2(x0) + p2(y0) + p2(z0);
    temp = std::sqrt(temp);
    if (s > 0) {
      x0 = -x0 / temp; y0 = -y0 / temp; z0 = -z0 / temp;
    } else {
      x0 = x0 / temp; y0 = y0 / temp; z0 = z0 / temp;
    }
    int ii = i + s * di, jj = j + s * dj, kk = k + s * dk;
    double cu = q(2, ii, jj, kk) * x0 + q(3, ii, jj, kk) * y0 + q(4, ii, jj, kk) * z0;
    q(1, i, j, k) = q(1, ii, jj, kk);
    q(2, i, j, k) = q(2, ii, jj, kk) - cu * x0;
    q(3, i, j, k) = q(3, ii, jj, kk) - cu * y0;
    q(4, i, j, k) = q(4, ii, jj, kk) - cu * z0;
    q(5, i, j, k) = q(5, ii, jj, kk);
    if (g_flags.turbulence >= 1) tur(i, j, k) = tur(ii, jj, kk);
  });
}

static void bc_nonslipwall(Block& B, const Box& sb, int face) {  // sub_bc_-20_solidwall.f90:213-327
  V q = B.v(F_Q), tur = B.v(F_NUT);
  for_face(face, sb, [&](int i, int j, int k, int di, int dj, int dk, int s) {
    int a1 = i + s * di, b1 = j + s * dj, c1 = k + s * dk;
    int a2 = i + 2 * s * di, b2 = j + 2 * s * dj, c2 = k + 2 * s * dk;
    int a3 = i + 3 * s * di, b3 = j + 3 * s * dj, c3 = k + 3 * s * dk;
    q(1, i, j, k) = (11.0 * q(1, a1, b1, c1) - 7.0 * q(1, a2, b2, c2) + 2.0 * q(1, a3, b3, c3)) / 6.0;
    q(2, i, j, k) = 0.0;
    q(3, i, j, k) = 0.0;
    q(4, i, j, k) = 0.0;
    q(5, i, j, k) = (11.0 * q(5, a1, b1, c1) - 7.0 * q(5, a2, b2, c2) + 2.0 * q(5, a3, b3, c3)) / 6.0;
    if (g_flags.turbulence >= 1) tur(i, j, k) = 0.0;
  });
}

static void bc_farfield(Block& B, const Box& sb, int face) {  // sub_bc_-10_farfield.f90:7-460
  V q = B.v(F_Q), tur = B.v(F_NUT), dxidx = B.v(F_DXIDX);
  const Consts& c = g_consts;
  double gamma = c.gamma;
  double d_inf = c.d_0, u_inf = c.u_0 * std::cos(c.aoa), v_inf = c.u_0 * std::sin(c.aoa), w_inf = 0.0;
  double p_inf = c.p_0;
  double s_inf = c.p_0 / xpow(c.d_0, gamma);
  double c_inf = c.c_0;
  (void)d_inf; (void)p_inf;
  for_face(face, sb, [&](int i, int j, int k, int di, int dj, int dk, int s) {
    int c0 = 3 * (di ? 0 : (dj ? 1 : 2)) + 1;
    double x0 = dxidx(c0, i, j, k), y0 = dxidx(c0 + 1, i, j, k), z0 = dxidx(c0 + 2, i, j, k);
    double temp = p2(x0) + p2(y0) + p2(z0);
    temp = std::sqrt(temp);
    if (s > 0) {
      x0 = -x0 / temp; y0 = -y0 / temp; z0 = -z0 / temp;
    } else {
      x0 = x0 / temp; y0 = y0 / temp; z0 = z0 / temp;
    }
    int ii = i + s * di, jj = j + s * dj, kk = k + s * dk;
    double d_p = q(1, ii, jj, kk);
    double u_p = q(2, ii, jj, kk) / d_p;
    double v_p = q(3, ii, jj, kk) / d_p;
    double w_p = q(4, ii, jj, kk) / d_p;
    double p_p = (q(5, ii, jj, kk) - 0.5 * d_p * (p2(u_p) + p2(v_p) + p2(w_p))) * (gamma - 1.0);
    double c_p = std::sqrt(gamma * p_p / d_p);
    double s_p = p_p / xpow(d_p, gamma);
    double vn_inf = u_inf * x0 + v_inf * y0 + w_inf * z0;
    double vn_p = u_p * x0 + v_p * y0 + w_p * z0;
    double rm = vn_inf - 2.0 * c_inf / (gamma - 1.0);
    double rp = vn_p + 2.0 * c_p / (gamma - 1.0);
    double vn_b = 0.5 * (rp + rm);
    double s_b = 0, u_ref = 0, v_ref = 0, w_ref = 0, turVal = 0;
    if (vn_b < 0.0) {
      s_b = s_inf; u_ref = u_inf; v_ref = v_inf; w_ref = w_inf; turVal = c.nutinf;
    }
    if (vn_b >= 0.0) {
      s_b = s_p; u_ref = u_p; v_ref = v_p; w_ref = w_p; turVal = tur(ii, jj, kk);
    }
    double u_ref_t = u_ref * x0 + v_ref * y0 + w_ref * z0;
    double u_b = u_ref + (vn_b - u_ref_t) * x0;
    double v_b = v_ref + (vn_b - u_ref_t) * y0;
    double w_b = w_ref + (vn_b - u_ref_t) * z0;
    double d_b = xpow(c_p * c_p / (gamma * s_b), 1.0 / (gamma - 1.0));  // c_p, as the reference (:93)
    double p_b = s_b * xpow(d_b, gamma);
    q(1, i, j, k) = d_b;
    q(2, i, j, k) = d_b * u_b;
    q(3, i, j, k) = d_b * v_b;
    q(4, i, j, k) = d_b * w_b;
    q(5, i, j, k) = p_b / (gamma - 1.0) + 0.5 * d_b * (p2(u_b) + p2(v_b) + p2(w_b));
    if (g_flags.turbulence >= 1) tur(i, j, k) = turVal;
  });
}

// sub_bc.f90:9-90
void physical_bc() {
  for (auto& B : g_blk) {
    if (!B.used) continue;
    for (auto& s : B.bc) {
      Box sb = s.box();
      if (s.blk_t == BC_INFLOW) bc_inflow(B, sb, s.face);
      else if (s.blk_t == BC_OUTFLOW) bc_outflow(B, sb, s.face);
      else if (s.blk_t == BC_SYMM) bc_mirror(B, sb, s.face);
      else if (s.blk_t == BC_WALL) {
        if (g_flags.solver == IFLAG_NSSOLVER) bc_nonslipwall(B, sb, s.face);
        else if (g_flags.solver == IFLAG_EULERSOLVER) bc_mirror(B, sb, s.face);
      } else if (s.blk_t == BC_FARFIELD) {
        Box fb = sb;
        fb.js = B.b.js;  // the reference passes the block's js here (sub_bc.f90:59)
        bc_farfield(B, fb, s.face);
      }
    }
  }
  if (g_flags.turbulence == IFLAG_SA && g_flags.solver == IFLAG_NSSOLVER) {  // :65-87
    for (auto& B : g_blk) {
      if (!B.used) continue;
      V pri = B.v(F_PRI), nutv = B.v(F_NUT), amu = B.v(F_AMU);
      const Box& b = B.b;
      for (int k = b.ks; k <= b.ke; ++k)
        for (int j = b.js; j <= b.je; ++j)
          for (int i = b.is; i <= b.ie; ++i) {
            double d = pri(1, i, j, k);
            double nut = nutv(i, j, k);
            double leix = nutv(i, j, k) / amu(1, i, j, k) * d;
            leix = std::max(leix, 0.001);
            double fv1 = p3(leix) / (p3(leix) + SA_CV13);
            nutv(i, j, k) = std::max(nut, 0.0001);
            nutv(i, j, k) = std::min(nut, 1.0e6);  // overwrites the lower clip (:80-81)
            amu(2, i, j, k) = nutv(i, j, k) * fv1 * d;
          }
    }
  }
}

// ------------------------------------------------------------------ halo
// 2-D mode (UpdateBuffer2d, UpdateBufferCoordinate2d, average2d1 in
// sub_bc_updatebuffer2d.f90, sub_bc_updatebuffercoordinate2d.f90,
// sub_bc_updatebufferaverage2d.f90): a face is a line, ua(ll) runs along it
// (j on faces 1/2, i on faces 3/4) with nn = max(n11, n12) of the donor
// subface (:218-222), ori 2 keeps the order and ori 3 reverses it (:284-293);
// every map below takes (l, m) = (ll, 1) there.
static bool two_d() { return g_flags.dimension == IFLAG_2D; }

// Donor-face (l,m) indexing of a received subface (sub_bc_updatebuffer.f90:265-354).
static void donor_lm(const Sub& d, int& l1, int& m1) {
  int n11 = d.ie - d.is + 1, n12 = d.je - d.js + 1, n13 = d.ke - d.ks + 1;
  if (two_d()) {
    l1 = std::max(n11, n12);
    m1 = 1;
    return;
  }
  switch (d.face) {
    case 1: l1 = n13; m1 = n12; break;
    case 2: l1 = n12; m1 = n13; break;
    case 3: l1 = n11; m1 = n13; break;
    case 4: l1 = n13; m1 = n11; break;
    case 5: l1 = n12; m1 = n11; break;
    default: l1 = n11; m1 = n12; break;
  }
}
static void donor_node(const Sub& d, int ll0, int mm0, int& i, int& j, int& k) {
  if (two_d()) {
    k = d.ks;
    switch (d.face) {
      case 1: i = d.is; j = d.js + ll0 - 1; break;
      case 2: i = d.ie; j = d.js + ll0 - 1; break;
      case 3: i = d.is + ll0 - 1; j = d.js; break;
      default: i = d.is + ll0 - 1; j = d.je; break;
    }
    return;
  }
  switch (d.face) {
    case 1: i = d.is; j = d.js + mm0 - 1; k = d.ks + ll0 - 1; break;
    case 2: i = d.ie; j = d.js + ll0 - 1; k = d.ks + mm0 - 1; break;
    case 3: i = d.is + ll0 - 1; j = d.js; k = d.ks + mm0 - 1; break;
    case 4: i = d.is + mm0 - 1; j = d.je; k = d.ks + ll0 - 1; break;
    case 5: i = d.is + mm0 - 1; j = d.js + ll0 - 1; k = d.ks; break;
    default: i = d.is + ll0 - 1; j = d.js + mm0 - 1; k = d.ke; break;
  }
}
// Reorientation by ori (:358-395): element (ll,mm) of ua2 comes from ua(la,ma).
static void ori_map(int ori, int l1, int m1, int& l2, int& m2) {
  if (two_d()) { l2 = l1; m2 = m1; return; }
  if (ori == 2 || ori == 4) { l2 = m1; m2 = l1; } else { l2 = l1; m2 = m1; }
}
static void ori_src(int ori, int l1, int m1, int ll, int mm, int& la, int& ma) {
  if (two_d()) {
    if (ori != 2 && ori != 3) {
      std::fprintf(stderr, "oracle: 2-D interface orientation %d (only 2 and 3 are defined)\n", ori);
      std::abort();
    }
    la = ori == 2 ? ll : l1 - ll + 1;
    ma = mm;
    return;
  }
  switch (ori) {
    case 1: la = ll; ma = m1 - mm + 1; break;
    case 2: la = mm; ma = ll; break;
    case 3: la = l1 - ll + 1; ma = mm; break;
    default: la = l1 - mm + 1; ma = m1 - ll + 1; break;
  }
}
// Own-face node written by element (a,b) of ua2 (:398-540), plus the outward step.
static void own_node(const Sub& s, int a, int bidx, int& i, int& j, int& k, int& di, int& dj, int& dk) {
  di = dj = dk = 0;
  if (two_d()) {
    k = s.ks;
    switch (s.face) {
      case 1: i = s.is; j = s.js + a - 1; di = -1; break;
      case 2: i = s.ie; j = s.js + a - 1; di = 1; break;
      case 3: i = s.is + a - 1; j = s.js; dj = -1; break;
      default: i = s.is + a - 1; j = s.je; dj = 1; break;
    }
    return;
  }
  switch (s.face) {
    case 1: i = s.is; j = s.js + bidx - 1; k = s.ks + a - 1; di = -1; break;
    case 2: i = s.ie; j = s.js + a - 1; k = s.ks + bidx - 1; di = 1; break;
    case 3: i = s.is + a - 1; j = s.js; k = s.ks + bidx - 1; dj = -1; break;
    case 4: i = s.is + bidx - 1; j = s.je; k = s.ks + a - 1; dj = 1; break;
    case 5: i = s.is + bidx - 1; j = s.js + a - 1; k = s.ks; dk = -1; break;
    default: i = s.is + a - 1; j = s.js + bidx - 1; k = s.ke; dk = 1; break;
  }
}

// Generic exchange used by UpdateBuffer (nvar q+nut, layers 1..BL inward),
// UpdateBufferCoordinate (x,y,z) and average1 (layer 0 = the interface plane).
// get(m, slot, i,j,k) reads the source value, put(...) writes the ghost.
template <class Get, class Put>
static void exchange(int nlayers, bool plane_only, Get get, Put put) {
  const int BL = g_flags.bufferLength;  // buffer layout (bufferLength,9,...) shared by all exchanges
  // pack (:47-140)
  for (size_t mi = 0; mi < g_blk.size(); ++mi) {
    Block& B = g_blk[mi];
    if (!B.used) continue;
    for (auto& s : B.bc) {
      if (s.blk_t < 0) continue;
      Box sb = s.box();
      FaceGeom g = face_geom(s.face);
      for (int k = sb.ks; k <= sb.ke; ++k)
        for (int j = sb.js; j <= sb.je; ++j)
          for (int i = sb.is; i <= sb.ie; ++i)
            for (int nb = 1; nb <= nlayers; ++nb) {
              int off = plane_only ? 0 : g.sgn * nb;
              int ii = i + (g.dir == 0 ? off : 0), jj = j + (g.dir == 1 ? off : 0),
                  kk = k + (g.dir == 2 ? off : 0);
              for (int slot = 1; slot <= 6; ++slot) {
                double val;
                if (get((int)mi + 1, slot, ii, jj, kk, val)) S5(s.send, sb, BL, nb, slot, i, j, k) = val;
              }
            }
    }
  }
  // same-rank copy (:155-171): receiver's buffer_recv <- sender's buffer_send
  for (size_t mi = 0; mi < g_blk.size(); ++mi) {
    Block& B = g_blk[mi];
    if (!B.used) continue;
    for (size_t ks = 0; ks < B.bc.size(); ++ks) {
      Sub& s = B.bc[ks];
      if (s.blk_t < 0) continue;
      Sub& r = blk(s.blk_t).bc.at(s.subface_t - 1);
      if (r.recv.size() != s.send.size()) {
        std::fprintf(stderr, "oracle: interface %d/%zu <-> %d/%d box mismatch\n", (int)mi + 1, ks + 1,
                     s.blk_t, s.subface_t);
        std::abort();
      }
      std::memcpy(r.recv.data(), s.send.data(), s.send.size() * sizeof(double));
    }
  }
  // unpack (:233-545)
  for (size_t mi = 0; mi < g_blk.size(); ++mi) {
    Block& B = g_blk[mi];
    if (!B.used) continue;
    for (auto& s : B.bc) {
      if (s.blk_t < 0) continue;
      const Sub& d = blk(s.blk_t).bc.at(s.subface_t - 1);
      Box db = d.box();
      int l1, m1, l2, m2;
      donor_lm(d, l1, m1);
      ori_map(s.ori, l1, m1, l2, m2);
      for (int b2 = 1; b2 <= m2; ++b2)
        for (int a2 = 1; a2 <= l2; ++a2) {
          int la, ma;
          ori_src(s.ori, l1, m1, a2, b2, la, ma);
          int di_, dj_, dk_, si, sj, sk;
          donor_node(d, la, ma, si, sj, sk);
          int oi, oj, ok;
          own_node(s, a2, b2, oi, oj, ok, di_, dj_, dk_);
          for (int nb = 1; nb <= nlayers; ++nb) {
            int off = plane_only ? 0 : nb;
            for (int slot = 1; slot <= 9; ++slot)
              put((int)mi + 1, s, slot, oi + di_ * off, oj + dj_ * off, ok + dk_ * off,
                  S5(s.recv, db, BL, nb, slot, si, sj, sk));
          }
        }
    }
  }
}

// sub_bc_updatebuffer.f90:10-548
void updatebuffer() {
  bool sa = g_flags.turbulence == IFLAG_SA;
  exchange(
      g_flags.bufferLength, false,
      [&](int m, int slot, int i, int j, int k, double& val) {
        Block& B = blk(m);
        if (slot <= 5) { val = B.v(F_Q)(slot, i, j, k); return true; }
        if (slot == 6 && sa) { val = B.v(F_NUT)(i, j, k); return true; }
        return false;
      },
      [&](int m, Sub&, int slot, int i, int j, int k, double val) {
        Block& B = blk(m);
        if (slot <= 5) B.v(F_Q)(slot, i, j, k) = val;
        else if (slot == 6 && sa) B.v(F_NUT)(i, j, k) = val;
      });
}

// sub_bc_updatebuffercoordinate.f90:10-473
void updatebuffercoordinate() {
  exchange(
      g_flags.bufferLength, false,
      [&](int m, int slot, int i, int j, int k, double& val) {
        Block& B = blk(m);
        if (slot >= 1 && slot <= 3) { val = B.v(F_X + slot - 1)(i, j, k); return true; }
        return false;
      },
      [&](int m, Sub&, int slot, int i, int j, int k, double val) {
        Block& B = blk(m);
        if (slot >= 1 && slot <= 3) B.v(F_X + slot - 1)(i, j, k) = val;
      });
}

// sub_bc_updatebufferaverage.f90:10-439: the neighbour's copy of the shared
// plane lands in the subface's `buffer` (9 slots, own subface indexing).
void average1() {
  bool sa = g_flags.turbulence == IFLAG_SA;
  exchange(
      1, true,
      [&](int m, int slot, int i, int j, int k, double& val) {
        Block& B = blk(m);
        if (slot <= 5) { val = B.v(F_Q)(slot, i, j, k); return true; }
        if (slot == 6 && sa) { val = B.v(F_NUT)(i, j, k); return true; }
        return false;
      },
      [&](int, Sub& s, int slot, int i, int j, int k, double val) {
        s.buf[(size_t)(slot - 1) + 9 * (size_t)s.box().at(i, j, k)] = val;
      });
}

// sub_bc_updatebufferaverage.f90:442-561
void average2() {
  bool sa = g_flags.turbulence == IFLAG_SA;
  for (auto& B : g_blk) {
    if (!B.used) continue;
    V q = B.v(F_Q), nut = B.v(F_NUT);
    for (auto& s : B.bc) {
      if (s.blk_t < 0) continue;
      Box sb = s.box();
      for (int k = sb.ks; k <= sb.ke; ++k)
        for (int j = sb.js; j <= sb.je; ++j)
          for (int i = sb.is; i <= sb.ie; ++i) {
            size_t o = 9 * (size_t)sb.at(i, j, k);
            for (int n = 1; n <= 5; ++n) q(n, i, j, k) = (q(n, i, j, k) + s.buf[o + n - 1]) * 0.5;
            if (sa) nut(i, j, k) = (nut(i, j, k) + s.buf[o + 5]) * 0.5;
          }
    }
  }
}

// sub_output_residual.f90:8-69 (returns the 7 printed values).
void residual(double out[7]) {
  double rms[5] = {0, 0, 0, 0, 0}, tur[2] = {0, 0};
  long totalnodes = 0;
  for (auto& B : g_blk) {
    if (!B.used) continue;
    totalnodes += B.b0.size();
    V rhs = B.v(F_RHS), dt = B.v(F_DT), invj = B.v(F_INVJ), sarhs = B.v(F_SARHS);
    const Box& b1 = B.b1;
    for (int k = b1.ks; k <= b1.ke; ++k)
      for (int j = b1.js; j <= b1.je; ++j)
        for (int i = b1.is; i <= b1.ie; ++i) {
          for (int n = 0; n < 5; ++n) rms[n] = rms[n] + p2(rhs(n + 1, i, j, k) * dt(i, j, k) / invj(i, j, k));
          tur[0] = tur[0] + p2(sarhs(i, j, k) * dt(i, j, k));
        }
  }
  for (int n = 0; n < 5; ++n) out[n] = std::sqrt(rms[n] / (double)totalnodes);
  out[5] = std::sqrt(tur[0] / (double)totalnodes);
  out[6] = std::sqrt(tur[1] / (double)totalnodes);
}

// sub_output_forceintegration.f90:8-479, 3-D branch (:182-457) with
// force_compute (:481-509): pressure and viscous forces summed over every
// quad of every wall subface (blk_t = -20) in the reference's loop order, then
// cl and cd.  out: fp(3), fv(3), cl, cd, and (test use) the sums of |f_prs|
// and |f_vis| per component.  The wall-normal unit vector keeps the
// reference's component mix (e.g. face 1: x from dxidx(1) at the first two
// corners and dxidx(2) at the last two).
void clcd_output(double sref, double out[14]) {
  const Consts& c = g_consts;
  double pinf = c.p_0;
  double div = 1.0 / (0.5 * c.d_0 * c.u_0 * c.u_0 * sref);
  double fp[3] = {0, 0, 0}, fv[3] = {0, 0, 0}, ap[3] = {0, 0, 0}, av[3] = {0, 0, 0};
  for (auto& B : g_blk) {
    if (!B.used) continue;
    size_t N = (size_t)B.b.size();
    std::vector<double> si(N), sj(N), sk(N), spc(N), vol(N);
    init_spacing(V{si.data(), 1, B.b}, V{sj.data(), 1, B.b}, V{sk.data(), 1, B.b}, V{spc.data(), 1, B.b},
                 V{vol.data(), 1, B.b}, B.v(F_X), B.v(F_Y), B.v(F_Z), B.b, B.b0);
    V spcv[3] = {V{si.data(), 1, B.b}, V{sj.data(), 1, B.b}, V{sk.data(), 1, B.b}};
    V pri = B.v(F_PRI), m = B.v(F_DXIDX), amu = B.v(F_AMU);
    for (auto& s : B.bc) {
      if (s.blk_t != BC_WALL) continue;
      if (two_d()) {
        // sub_output_forceintegration.f90:48-180: the wall is a line; each
        // edge (t, t+1) averages velocity and the unit normal over the two
        // nodes one layer in, pressure and viscosity over the two wall nodes
        // (face 3 averages the viscosity with 0.25, :128), s = the edge's
        // spacing along the wall, dn = the mean spacing normal to it
        const int k = s.ks;
        const bool iface = s.face <= 2;
        const bool low = s.face % 2 == 1;
        const double sgn = low ? -1.0 : 1.0;
        const int w = iface ? (low ? s.is : s.ie) : (low ? s.js : s.je);
        const int w1 = low ? w + 1 : w - 1;
        const int lo = iface ? s.js : s.is, hi = iface ? s.je : s.ie;
        const int c1 = iface ? 1 : 4;
        const double mfac = s.face == 3 ? 0.25 : 0.5;
        for (int t = lo; t <= hi - 1; ++t) {
          const int ia = iface ? w1 : t, ja = iface ? t : w1, ib = iface ? w1 : t + 1, jb = iface ? t + 1 : w1;
          const int iwa = iface ? w : t, jwa = iface ? t : w, iwb = iface ? w : t + 1, jwb = iface ? t + 1 : w;
          double uc = (pri(2, ia, ja, k) + pri(2, ib, jb, k)) * 0.5;
          double vc = (pri(3, ia, ja, k) + pri(3, ib, jb, k)) * 0.5;
          double wc = 0.0;
          double pc = (pri(5, iwa, jwa, k) + pri(5, iwb, jwb, k)) * 0.5;
          double t00 = 1.0 / std::sqrt(p2(m(c1, ia, ja, k)) + p2(m(c1 + 1, ia, ja, k)) + p2(m(c1 + 2, ia, ja, k)));
          double t10 = 1.0 / std::sqrt(p2(m(c1, ib, jb, k)) + p2(m(c1 + 1, ib, jb, k)) + p2(m(c1 + 2, ib, jb, k)));
          double n3[3];
          for (int x = 0; x < 3; ++x) n3[x] = sgn * ((m(c1 + x, ia, ja, k) * t00 + m(c1 + x, ib, jb, k) * t10) * 0.5);
          double miuc = (amu(3, iwa, jwa, k) + amu(3, iwb, jwb, k)) * mfac;
          double area = iface ? spcv[1](1, w, t, k) : spcv[0](1, t, w, k);
          double dn = iface ? 0.5 * (spcv[0](1, w, t, k) + spcv[0](1, w, t + 1, k))
                            : (spcv[1](1, t, w, k) + spcv[1](1, t + 1, w, k)) * 0.5;
          double u3[3] = {uc, vc, wc};
          double un = uc * n3[0] + vc * n3[1] + wc * n3[2];
          for (int x = 0; x < 3; ++x) {
            double f_prs = (pc - pinf) * area * n3[x];
            double f_vis = miuc * (u3[x] - un * n3[x]) / dn * area / c.re;
            fp[x] = fp[x] + f_prs;
            fv[x] = fv[x] + f_vis;
            ap[x] += std::fabs(f_prs);
            av[x] += std::fabs(f_vis);
          }
        }
        continue;
      }
      const int D = (s.face - 1) / 2;
      const bool low = s.face % 2 == 1;
      const int lo[3] = {s.is, s.js, s.ks}, hi[3] = {s.ie, s.je, s.ke};
      const int T1 = D == 0 ? 1 : 0, T2 = D == 2 ? 1 : 2;  // inner, outer loop directions
      const int w0 = low ? lo[D] : hi[D], w1 = low ? w0 + 1 : w0 - 1;
      const int c1 = 3 * D + 1, c2 = 3 * D + 2, c3 = 3 * D + 3;
      const double sgn = low ? -1.0 : 1.0;
      for (int t2 = lo[T2]; t2 <= hi[T2] - 1; ++t2)
        for (int t1 = lo[T1]; t1 <= hi[T1] - 1; ++t1) {
          // node at (tangential a, tangential b, layer)
          auto at = [&](int a, int b, int layer, int& i, int& j, int& k) {
            int ijk[3];
            ijk[D] = layer; ijk[T1] = a; ijk[T2] = b;
            i = ijk[0]; j = ijk[1]; k = ijk[2];
          };
          int I[4], J[4], K[4], Iw[4], Jw[4], Kw[4];
          const int da[4] = {0, 1, 0, 1}, db[4] = {0, 0, 1, 1};  // corners 00, 10, 01, 11
          for (int q = 0; q < 4; ++q) {
            at(t1 + da[q], t2 + db[q], w1, I[q], J[q], K[q]);
            at(t1 + da[q], t2 + db[q], w0, Iw[q], Jw[q], Kw[q]);
          }
          auto avg = [&](V f, int comp, const int* Ii, const int* Jj, const int* Kk) {
            return (f(comp, Ii[0], Jj[0], Kk[0]) + f(comp, Ii[1], Jj[1], Kk[1]) + f(comp, Ii[2], Jj[2], Kk[2]) +
                    f(comp, Ii[3], Jj[3], Kk[3])) * 0.25;
          };
          double uc = avg(pri, 2, I, J, K), vc = avg(pri, 3, I, J, K), wc = avg(pri, 4, I, J, K);
          double pc = avg(pri, 5, Iw, Jw, Kw);
          double t[4];
          for (int q = 0; q < 4; ++q)
            t[q] = 1.0 / std::sqrt(p2(m(c1, I[q], J[q], K[q])) + p2(m(c2, I[q], J[q], K[q])) +
                                   p2(m(c3, I[q], J[q], K[q])));
          auto mix = [&](int ca, int cb) {
            return (m(ca, I[0], J[0], K[0]) * t[0] + m(ca, I[1], J[1], K[1]) * t[1] +
                    m(cb, I[2], J[2], K[2]) * t[2] + m(cb, I[3], J[3], K[3]) * t[3]) * 0.25;
          };
          double nx = sgn * mix(c1, c2), ny = sgn * mix(c3, c1), nz = sgn * mix(c2, c3);
          double miuc = avg(amu, 3, Iw, Jw, Kw);
          int i0, j0, k0;
          at(t1, t2, w0, i0, j0, k0);
          // element area: the two tangential spacings in i, j, k order
          double area = spcv[T1](1, i0, j0, k0) * spcv[T2](1, i0, j0, k0);
          double dn = spcv[D](1, i0, j0, k0);
          double n3[3] = {nx, ny, nz}, u3[3] = {uc, vc, wc};
          double un = uc * nx + vc * ny + wc * nz;
          for (int x = 0; x < 3; ++x) {
            double f_prs = (pc - pinf) * area * n3[x];
            double f_vis = miuc * (u3[x] - un * n3[x]) / dn * area / c.re;
            fp[x] = fp[x] + f_prs;
            fv[x] = fv[x] + f_vis;
            ap[x] += std::fabs(f_prs);
            av[x] += std::fabs(f_vis);
          }
        }
    }
  }
  for (int x = 0; x < 3; ++x) {
    out[x] = fp[x];
    out[3 + x] = fv[x];
    out[8 + x] = ap[x];
    out[11 + x] = av[x];
  }
  out[6] = ((fp[1] + fv[1]) * std::cos(c.aoa) - (fp[0] + fv[0]) * std::sin(c.aoa)) * div;
  out[7] = ((fp[1] + fv[1]) * std::sin(c.aoa) + (fp[0] + fv[0]) * std::cos(c.aoa)) * div;
}

// sub_init_flowfield.f90:29-111 (freestream start, iflag_init = 0).  ma, aoa in
// degrees and dt come from Control.in; the nondimensional constants are derived
// here exactly as the reference does.
void init_flowfield(double ma, double aoa_deg, double dt) {
  Consts& c = g_consts;
  const double pi = 3.1415926535897932;
  c.ma = ma;
  c.d_0 = 1.0; c.u_0 = 1.0; c.t_0 = 1.0;
  c.p_0 = c.d_0 * c.t_0 / c.gamma / ma / ma;
  c.c_0 = std::sqrt(c.t_0) / ma;
  c.cv = 1.0 / c.gamma / (c.gamma - 1.0) / ma / ma;
  c.cp = 1.0 / (c.gamma - 1.0) / ma / ma;
  c.aoa = aoa_deg * pi / 180.0;
  c.dt = dt;
  for (auto& B : g_blk) {
    if (!B.used) continue;
    long N = B.b.size();
    for (int fid : {F_DUDX, F_VOR, F_TAO, F_RHSV, F_RHSI, F_RHS})
      if (B.f[fid]) std::fill(B.f[fid], B.f[fid] + kNc[fid] * N, 0.0);
    V q = B.v(F_Q), pri = B.v(F_PRI), dtv = B.v(F_DT), amu = B.v(F_AMU);
    for (long n = 0; n < N; ++n) {
      q.p[5 * n + 0] = c.d_0;
      q.p[5 * n + 1] = c.d_0 * c.u_0 * std::cos(c.aoa);
      q.p[5 * n + 2] = c.d_0 * c.u_0 * std::sin(c.aoa);
      q.p[5 * n + 3] = 0.0;
      q.p[5 * n + 4] = c.d_0 * c.t_0 * c.cv + 0.5 * c.d_0 * c.u_0 * c.u_0;
      if (B.f[F_Q0])  // q0(:, c) = q(c) at both time levels (:78-82)
        for (int x = 0; x < 10; ++x) B.f[F_Q0][10 * n + x] = q.p[5 * n + x / 2];
      pri.p[7 * n + 0] = c.d_0;
      pri.p[7 * n + 1] = c.u_0 * std::cos(c.aoa);
      pri.p[7 * n + 2] = c.u_0 * std::sin(c.aoa);
      pri.p[7 * n + 3] = 0.0;
      pri.p[7 * n + 4] = c.p_0;
      pri.p[7 * n + 5] = c.t_0;
      pri.p[7 * n + 6] = c.c_0;
      dtv.p[n] = dt;
      if (g_flags.turbulence == IFLAG_SA) {
        B.f[F_NUT][n] = c.nutinf;
        amu.p[3 * n + 1] = 0.009;
        B.f[F_SARHS][n] = 0.0;
      } else {
        amu.p[3 * n + 1] = 0.0;
      }
      amu.p[3 * n + 0] = 1.0;
      amu.p[3 * n + 2] = amu.p[3 * n + 0] + amu.p[3 * n + 1];
    }
  }
}

// sub_init_walldist.f90:9-123 (brute force over every wall-subface node).
void init_walldist() {
  struct P { double x, y, z; };
  std::vector<P> wall;
  for (auto& B : g_blk) {  // sub_init_readbcinfo.f90:286-388 face coordinates
    if (!B.used) continue;
    V x = B.v(F_X), y = B.v(F_Y), z = B.v(F_Z);
    for (auto& s : B.bc) {
      if (s.blk_t != BC_WALL) continue;
      for (int k = s.ks; k <= s.ke; ++k)
        for (int j = s.js; j <= s.je; ++j)
          for (int i = s.is; i <= s.ie; ++i) {
            int ii = i, jj = j, kk = k;
            if (s.face == 1) ii = B.b0.is;
            if (s.face == 2) ii = B.b0.ie;
            if (s.face == 3) jj = B.b0.js;
            if (s.face == 4) jj = B.b0.je;
            if (s.face == 5) kk = B.b0.ks;
            if (s.face == 6) kk = B.b0.ke;
            wall.push_back(P{x(ii, jj, kk), y(ii, jj, kk), z(ii, jj, kk)});
          }
    }
  }
  for (auto& B : g_blk) {
    if (!B.used) continue;
    V x = B.v(F_X), y = B.v(F_Y), z = B.v(F_Z), dist = B.v(F_DIST);
    const Box& b0 = B.b0;
    for (int k = b0.ks; k <= b0.ke; ++k)
      for (int j = b0.js; j <= b0.je; ++j)
        for (int i = b0.is; i <= b0.ie; ++i) {
          double xx = x(i, j, k), yy = y(i, j, k), zz = z(i, j, k);
          double walldist = 1.0e9;
          for (const P& w : wall) {
            double temp = std::sqrt(p2(xx - w.x) + p2(yy - w.y) + p2(zz - w.z));
            if (temp <= walldist) walldist = temp;
          }
          dist(i, j, k) = walldist;
        }
  }
}

// Per-block part of one 1st-order implicit iteration (main.f90:344-419).
static void block_update(Block& B, int m, double* dtmax, double* dtmin, double* cflmax,
                         double* cflmin) {
  const Consts& c = g_consts;
  const Box &b = B.b, &b0 = B.b0, &b1 = B.b1;
  get_primitivevariables(m, B.v(F_PRI), B.v(F_Q), c.gamma, c.cv, b);
  inviscid_flux(B.v(F_RHSI), B.v(F_Q), B.v(F_DXIDX), B.v(F_INVJ), b, b0, b1, c.gamma);
  if (g_flags.solver == IFLAG_NSSOLVER)
    viscous_flux(B.v(F_RHSV), B.v(F_PRI), B.v(F_AMU), B.v(F_VOR), B.v(F_DUDX), B.v(F_TAO),
                 B.v(F_DXIDX), B.v(F_INVJ), c.tinf, c.prl, c.prt, c.gamma, c.cv, c.re, b, b0, b1);
  double cfl = c.cfl;
  find_dt(B.v(F_DT), dtmax, dtmin, cflmax, cflmin, B.v(F_PRI), B.v(F_AMU), B.v(F_DXIDX), c.re, &cfl,
          b, g_flags.time);
  implicit1st(B.v(F_Q), B.v(F_DT), B.v(F_PRI), B.v(F_RHS), B.v(F_RHSI), B.v(F_RHSV), B.v(F_DXIDX),
              B.v(F_INVJ), b, b0, b1, c.gamma, cfl);
  if (g_flags.turbulence == IFLAG_SA && g_flags.solver == IFLAG_NSSOLVER)
    sa_model(B.v(F_NUT), B.v(F_SARHS), B.v(F_DT), B.v(F_PRI), B.v(F_AMU), B.v(F_DUDX), B.v(F_VOR),
             B.v(F_DXIDX), B.v(F_INVJ), B.v(F_ALPHA), B.v(F_BETA), B.v(F_GAMMA), B.v(F_LENGTH),
             B.v(F_DIST), B.v(F_SPACING), c.re, cfl, b, b0, b1);
}

// main.f90:342-448 and the residual of :603, for nsteps iterations.  The
// per-block phase runs one host thread per block (at most nthreads at a
// time), as the reference runs one MPI rank per block group.
// main.f90:450-573 (iflag_timeadvance = 2nd Crank-Nicolson) and the
// residual of :603 for nsteps physical time steps: three dual-time
// sub-iterations of [physical_bc, halo, averaging, then per block getpri,
// inviscid, viscous, find_dt, crank2nd], then update_q0 and SA per block, and
// the closing BCs, halo, averaging and primitives.
void iterate_crank(int nsteps, double* resid_hist) {
  const Consts& c = g_consts;
  for (int step = 0; step < nsteps; ++step) {
    for (int sub = 1; sub <= 3; ++sub) {
      physical_bc();
      updatebuffer();
      average1();
      average2();
      for (auto& B : g_blk) {
        if (!B.used) continue;
        const Box &b = B.b, &b0 = B.b0, &b1 = B.b1;
        get_primitivevariables(0, B.v(F_PRI), B.v(F_Q), c.gamma, c.cv, b);
        inviscid_flux(B.v(F_RHSI), B.v(F_Q), B.v(F_DXIDX), B.v(F_INVJ), b, b0, b1, c.gamma);
        if (g_flags.solver == IFLAG_NSSOLVER)
          viscous_flux(B.v(F_RHSV), B.v(F_PRI), B.v(F_AMU), B.v(F_VOR), B.v(F_DUDX), B.v(F_TAO), B.v(F_DXIDX),
                       B.v(F_INVJ), c.tinf, c.prl, c.prt, c.gamma, c.cv, c.re, b, b0, b1);
        double cfl = c.cfl;
        find_dt(B.v(F_DT), &g_last_dtmax, &g_last_dtmin, &g_last_cflmax, &g_last_cflmin, B.v(F_PRI),
                B.v(F_AMU), B.v(F_DXIDX), c.re, &cfl, b, g_flags.time);
        crank2nd(B.v(F_Q), B.v(F_Q0), B.v(F_DT), B.v(F_PRI), B.v(F_RHS), B.v(F_RHSI), B.v(F_RHSV),
                 B.v(F_DXIDX), B.v(F_INVJ), b, b0, b1, c.gamma);
      }
    }
    for (auto& B : g_blk)
      if (B.used) update_q0(B.v(F_Q0), B.v(F_Q), B.b0);
    if (g_flags.turbulence == IFLAG_SA && g_flags.solver == IFLAG_NSSOLVER)
      for (auto& B : g_blk)
        if (B.used)
          sa_model(B.v(F_NUT), B.v(F_SARHS), B.v(F_DT), B.v(F_PRI), B.v(F_AMU), B.v(F_DUDX), B.v(F_VOR),
                   B.v(F_DXIDX), B.v(F_INVJ), B.v(F_ALPHA), B.v(F_BETA), B.v(F_GAMMA), B.v(F_LENGTH),
                   B.v(F_DIST), B.v(F_SPACING), c.re, c.cfl, B.b, B.b0, B.b1);
    physical_bc();
    updatebuffer();
    average1();
    average2();
    for (auto& B : g_blk)
      if (B.used) get_primitivevariables(0, B.v(F_PRI), B.v(F_Q), c.gamma, c.cv, B.b);
    if (resid_hist) residual(resid_hist + 7 * step);
  }
}

void iterate(int nsteps, int nthreads, double* resid_hist) {
  int nb = (int)g_blk.size();
  std::vector<double> dmx(nb), dmn(nb), cmx(nb), cmn(nb);
  for (int step = 0; step < nsteps; ++step) {
    auto work = [&](int lo, int hi) {
      for (int m = lo; m < hi; ++m)
        if (g_blk[m].used) block_update(g_blk[m], m + 1, &dmx[m], &dmn[m], &cmx[m], &cmn[m]);
    };
    if (nthreads <= 1 || nb == 1) {
      work(0, nb);
    } else {
      std::vector<std::thread> th;
      int T = std::min(nthreads, nb);
      for (int t = 0; t < T; ++t) th.emplace_back([&, t] {
        for (int m = t; m < nb; m += T)
          if (g_blk[m].used) block_update(g_blk[m], m + 1, &dmx[m], &dmn[m], &cmx[m], &cmn[m]);
      });
      for (auto& x : th) x.join();
    }
    // dtmax/dtmin are module variables that each find_dt call resets: the rank
    // reports the values of its last block.
    for (int m = nb - 1; m >= 0; --m)
      if (g_blk[m].used) {
        g_last_dtmax = dmx[m]; g_last_dtmin = dmn[m]; g_last_cflmax = cmx[m]; g_last_cflmin = cmn[m];
        break;
      }
    physical_bc();
    updatebuffer();
    average1();
    average2();
    for (int m = 0; m < nb; ++m)
      if (g_blk[m].used)
        get_primitivevariables(m + 1, g_blk[m].v(F_PRI), g_blk[m].v(F_Q), g_consts.gamma, g_consts.cv,
                               g_blk[m].b);
    if (resid_hist) residual(resid_hist + 7 * step);
  }
}

}  // namespace oracle

// ============================================================ extern "C" API
using namespace oracle;

static Box mkbox(const int* is, const int* ie, const int* js, const int* je, const int* ks,
                 const int* ke) {
  return Box{*is, *ie, *js, *je, *ks, *ke};
}
#define BOX6(p) mkbox(p##is, p##ie, p##js, p##je, p##ks, p##ke)
#define ARGS6(p) const int *p##is, const int *p##ie, const int *p##js, const int *p##je, \
                 const int *p##ks, const int *p##ke

extern "C" {

// iflags: dimension, solver, time, timeadvance, turbulence, des, bufferLength, inviscid
void oracle_configure(const int* iflags, const double* params) {
  g_flags.dimension = iflags[0]; g_flags.solver = iflags[1]; g_flags.time = iflags[2];
  g_flags.timeadvance = iflags[3]; g_flags.turbulence = iflags[4]; g_flags.des = iflags[5];
  g_flags.bufferLength = iflags[6]; g_flags.inviscid = iflags[7];
  // params: ma, re, tinf, aoa_deg, cfl, dt, nutinf
  g_consts.ma = params[0]; g_consts.re = params[1]; g_consts.tinf = params[2];
  g_consts.cfl = params[4]; g_consts.dt = params[5]; g_consts.nutinf = params[6];
  const double pi = 3.1415926535897932;
  g_consts.aoa = params[3] * pi / 180.0;
}

void oracle_reset() { g_blk.clear(); }

// box18: is,ie,js,je,ks,ke, is0..ke0, is1..ke1; sub11 per subface:
// f_no,face,is,ie,js,je,ks,ke,blk_t,subface_t,ori
void oracle_register_block(int m, const int* box18, int nsub, const int* sub11) {
  if ((int)g_blk.size() < m) g_blk.resize(m);
  Block& B = g_blk[m - 1];
  B.used = true;
  B.b = Box{box18[0], box18[1], box18[2], box18[3], box18[4], box18[5]};
  B.b0 = Box{box18[6], box18[7], box18[8], box18[9], box18[10], box18[11]};
  B.b1 = Box{box18[12], box18[13], box18[14], box18[15], box18[16], box18[17]};
  B.bc.clear();
  for (int s = 0; s < nsub; ++s) {
    const int* r = sub11 + 11 * s;
    Sub x;
    x.f_no = r[0]; x.face = r[1]; x.is = r[2]; x.ie = r[3]; x.js = r[4]; x.je = r[5];
    x.ks = r[6]; x.ke = r[7]; x.blk_t = r[8]; x.subface_t = r[9]; x.ori = r[10];
    B.bc.push_back(x);
  }
}

void oracle_bind_field(int m, int fid, double* ptr) { blk(m).f[fid] = ptr; }
void oracle_finish_setup() { alloc_buffers(); }

void oracle_get_primitivevariables(const int* mm, double* pri_v, double* q, const double* gamma,
                                   const double* cv, ARGS6()) {
  Box b = BOX6();
  get_primitivevariables(*mm, V{pri_v, 7, b}, V{q, 5, b}, *gamma, *cv, b);
}

void oracle_thirdorder_weno(double* df, double* f, ARGS6(), ARGS6(r), const int* coord,
                            const int* direction) {
  Box b = BOX6(), r = BOX6(r);
  thirdorder_weno(V{df, 5, b}, V{f, 5, b}, b, r, *coord, *direction);
}

void oracle_roe_3d(double* ql, double* qr, double* flux, double* dxidx, double* inv_j,
                   const double* gamma, ARGS6(), ARGS6(r), const int* coord) {
  Box b = BOX6(), r = BOX6(r);
  roe_3d(V{ql, 5, b}, V{qr, 5, b}, V{flux, 5, b}, V{dxidx, 9, b}, V{inv_j, 1, b}, *gamma, b, r, *coord);
}

void oracle_inviscid_flux_1(double* rhsi, double* q, double* dxidx, double* inv_j, ARGS6(),
                            ARGS6(z), ARGS6(o), const double* gamma) {
  Box b = BOX6(), b0 = BOX6(z), b1 = BOX6(o);
  inviscid_flux_1(V{rhsi, 5, b}, V{q, 5, b}, V{dxidx, 9, b}, V{inv_j, 1, b}, b, b0, b1, *gamma);
}

void oracle_inviscid_flux_weno5(double* rhsi, double* q, double* dxidx, double* inv_j, ARGS6(),
                                ARGS6(z), ARGS6(o), const double* gamma) {
  Box b = BOX6(), b1 = BOX6(o);
  (void)zis; (void)zie; (void)zjs; (void)zje; (void)zks; (void)zke;
  inviscid_flux_sw_weno5(V{rhsi, 5, b}, V{q, 5, b}, V{dxidx, 9, b}, V{inv_j, 1, b}, b, b1, *gamma);
}

void oracle_inviscid_flux_wcns5(double* rhsi, double* q, double* dxidx, double* inv_j, ARGS6(),
                                ARGS6(z), ARGS6(o), const double* gamma) {
  Box b = BOX6(), b1 = BOX6(o);
  (void)zis; (void)zie; (void)zjs; (void)zje; (void)zks; (void)zke;
  inviscid_flux_wcns5(V{rhsi, 5, b}, V{q, 5, b}, V{dxidx, 9, b}, V{inv_j, 1, b}, b, b1, *gamma);
}

void oracle_viscous_flux(double* rhsv, double* pri_v, double* amu, double* vor, double* dudx,
                         double* tao, double* dxidx, double* inv_j, const double* tinf,
                         const double* prl, const double* prt, const double* gamma,
                         const double* cv, const double* re, ARGS6(), ARGS6(z), ARGS6(o),
                         const int* mm) {
  (void)mm;
  Box b = BOX6(), b0 = BOX6(z), b1 = BOX6(o);
  viscous_flux(V{rhsv, 5, b}, V{pri_v, 7, b}, V{amu, 3, b}, V{vor, 1, b}, V{dudx, 9, b},
               V{tao, 6, b}, V{dxidx, 9, b}, V{inv_j, 1, b}, *tinf, *prl, *prt, *gamma, *cv, *re,
               b, b0, b1);
}

void oracle_find_dt(double* dt, double* dtmax, double* dtmin, double* cflmax, double* cflmin,
                    double* pri_v, double* amu, double* dxidx, const double* re, double* cfl,
                    ARGS6(), const int* iflag_time, const int* iflag_steady,
                    const int* iflag_unsteady) {
  (void)iflag_steady; (void)iflag_unsteady;
  Box b = BOX6();
  find_dt(V{dt, 1, b}, dtmax, dtmin, cflmax, cflmin, V{pri_v, 7, b}, V{amu, 3, b}, V{dxidx, 9, b},
          *re, cfl, b, *iflag_time);
}

void oracle_calc_jm(double* a, const double* q1, const double* q2, const double* q3,
                    const double* q4, const double* q5, const double* dxidx, const double* dxidy,
                    const double* dxidz, const double* gamma) {
  calc_jm(a, *q1, *q2, *q3, *q4, *q5, *dxidx, *dxidy, *dxidz, *gamma);
}

void oracle_implicit1st(double* q, double* dt, double* pri_v, double* rhs, double* rhsi,
                        double* rhsv, double* dxidx, double* inv_j, ARGS6(), ARGS6(z), ARGS6(o),
                        const double* gamma, const double* cfl, double* xx, double* yy, double* zz) {
  (void)xx; (void)yy; (void)zz;
  Box b = BOX6(), b0 = BOX6(z), b1 = BOX6(o);
  implicit1st(V{q, 5, b}, V{dt, 1, b}, V{pri_v, 7, b}, V{rhs, 5, b}, V{rhsi, 5, b}, V{rhsv, 5, b},
              V{dxidx, 9, b}, V{inv_j, 1, b}, b, b0, b1, *gamma, *cfl);
}

void oracle_sa_model(double* nut, double* sa_rhs, double* dt, double* pri_v, double* amu,
                     double* dudx, double* vor, double* dxidx, double* inv_j, double* alpha,
                     double* beta, double* gamma, double* length, double* dist, double* spac,
                     const double* re, const double* cfl, ARGS6(), ARGS6(z), ARGS6(o)) {
  Box b = BOX6(), b0 = BOX6(z), b1 = BOX6(o);
  sa_model(V{nut, 1, b}, V{sa_rhs, 1, b}, V{dt, 1, b}, V{pri_v, 7, b}, V{amu, 3, b}, V{dudx, 9, b},
           V{vor, 1, b}, V{dxidx, 9, b}, V{inv_j, 1, b}, V{alpha, 3, b}, V{beta, 3, b},
           V{gamma, 3, b}, V{length, 1, b}, V{dist, 1, b}, V{spac, 1, b}, *re, *cfl, b, b0, b1);
}

void oracle_gridtransformation(double* dxidx, double* inv_j, double* alpha, double* beta,
                               double* gamma, double* x, double* y, double* z, ARGS6(), ARGS6(z),
                               const int* m0) {
  (void)m0;
  Box b = BOX6(), b0 = BOX6(z);
  gridtransformation(V{dxidx, 9, b}, V{inv_j, 1, b}, V{alpha, 3, b}, V{beta, 3, b}, V{gamma, 3, b},
                     V{x, 1, b}, V{y, 1, b}, V{z, 1, b}, b, b0);
}

void oracle_init_spacing(double* spci, double* spcj, double* spck, double* spacing, double* vol,
                         double* x, double* y, double* z, ARGS6(), ARGS6(z)) {
  Box b = BOX6(), b0 = BOX6(z);
  init_spacing(V{spci, 1, b}, V{spcj, 1, b}, V{spck, 1, b}, V{spacing, 1, b}, V{vol, 1, b},
               V{x, 1, b}, V{y, 1, b}, V{z, 1, b}, b, b0);
}

void oracle_physical_bc() { physical_bc(); }
void oracle_updatebuffer() { updatebuffer(); }
void oracle_updatebuffercoordinate() { updatebuffercoordinate(); }
void oracle_average1() { average1(); }
void oracle_average2() { average2(); }
void oracle_residual(double* out7) { residual(out7); }
void oracle_clcd_output(double sref, double* out14) { clcd_output(sref, out14); }
void oracle_init_flowfield(const double* ma, const double* aoa_deg, const double* dt) {
  init_flowfield(*ma, *aoa_deg, *dt);
}
void oracle_init_walldist() { init_walldist(); }
void oracle_iterate(int nsteps, int nthreads, double* resid_hist) {
  if (g_flags.timeadvance == IFLAG_2NDCRANK)
    iterate_crank(nsteps, resid_hist);
  else
    iterate(nsteps, nthreads, resid_hist);
}
void oracle_crank2nd(double* q, double* q0, double* dt, double* pri_v, double* rhs, double* rhsi, double* rhsv,
                     double* dxidx, double* inv_j, const int* box18, double gamma) {
  Box b{box18[0], box18[1], box18[2], box18[3], box18[4], box18[5]};
  Box b0{box18[6], box18[7], box18[8], box18[9], box18[10], box18[11]};
  Box b1{box18[12], box18[13], box18[14], box18[15], box18[16], box18[17]};
  crank2nd(V{q, 5, b}, V{q0, 10, b}, V{dt, 1, b}, V{pri_v, 7, b}, V{rhs, 5, b}, V{rhsi, 5, b}, V{rhsv, 5, b},
           V{dxidx, 9, b}, V{inv_j, 1, b}, b, b0, b1, gamma);
}
void oracle_update_q0(double* q0, double* q, const int* box18) {
  Box b{box18[0], box18[1], box18[2], box18[3], box18[4], box18[5]};
  Box b0{box18[6], box18[7], box18[8], box18[9], box18[10], box18[11]};
  update_q0(V{q0, 10, b}, V{q, 5, b}, b0);
}
void oracle_last_dt_minmax(double* out4) {
  out4[0] = g_last_dtmax; out4[1] = g_last_dtmin; out4[2] = g_last_cflmax; out4[3] = g_last_cflmin;
}
// Derived freestream constants (d_0,u_0,t_0,p_0,c_0,cv,cp,aoa_rad,gamma,nutinf).
void oracle_get_consts(double* out10) {
  const Consts& c = g_consts;
  double v[10] = {c.d_0, c.u_0, c.t_0, c.p_0, c.c_0, c.cv, c.cp, c.aoa, c.gamma, c.nutinf};
  std::memcpy(out10, v, sizeof v);
}

}  // extern "C"
