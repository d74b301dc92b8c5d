// TEST INFRASTRUCTURE ONLY (see oracle_common.h): one-time geometry
// precompute restated from sub_init_gridtransformation.f90 and sub_init_spacing.f90.
#include <algorithm>
#include <cmath>

#include "oracle_blockops.h"

namespace oracle {

namespace {

struct Range { int lo, hi; };

// Differentiates src (nc components) along direction dir (0=xi,1=eta,2=zeta)
// over the five regions the reference uses for every metric derivative
// (sub_init_gridtransformation.f90:107-175 for xi, :189-257 eta, :276-344 zeta):
//   main region: full box along dir, physical range in the two other directions,
//                one-sided at the full-box ends;
//   four slabs:  ghost layers of one other direction x physical ranges,
//                one-sided at the physical ends along dir.
void region_derivative(V src, V dst, int nc, int dir, const Box& b, const Box& b0) {
  Range full[3] = {{b.is, b.ie}, {b.js, b.je}, {b.ks, b.ke}};
  Range phys[3] = {{b0.is, b0.ie}, {b0.js, b0.je}, {b0.ks, b0.ke}};
  auto run = [&](Range r[3], Range ends) {
    for (int k = r[2].lo; k <= r[2].hi; ++k)
      for (int j = r[1].lo; j <= r[1].hi; ++j)
        for (int i = r[0].lo; i <= r[0].hi; ++i) {
          int idx[3] = {i, j, k};
          int di = dir == 0, dj = dir == 1, dk = dir == 2;
          int pos = idx[dir];
          for (int c = 1; c <= nc; ++c) {
            if (pos == ends.lo)
              dst(c, i, j, k) = src(c, i + di, j + dj, k + dk) - src(c, i, j, k);
            else if (pos == ends.hi)
              dst(c, i, j, k) = src(c, i, j, k) - src(c, i - di, j - dj, k - dk);
            else
              dst(c, i, j, k) = (src(c, i + di, j + dj, k + dk) - src(c, i - di, j - dj, k - dk)) / 2.0;
          }
        }
  };
  // main region
  Range r[3];
  for (int a = 0; a < 3; ++a) r[a] = (a == dir) ? full[a] : phys[a];
  run(r, full[dir]);
  // slabs: for each other direction o, the low and high ghost layers
  for (int o = 0; o < 3; ++o) {
    if (o == dir) continue;
    for (int side = 0; side < 2; ++side) {
      Range s[3];
      for (int a = 0; a < 3; ++a) s[a] = phys[a];
      s[o] = side == 0 ? Range{full[o].lo, phys[o].lo - 1} : Range{phys[o].hi + 1, full[o].hi};
      run(s, phys[dir]);
    }
  }
}

}  // namespace

// sub_init_gridtransformation.f90:27-874 (3-D and 2-D branches).  Nodes with two or more
// indices in ghost layers (block corners/edges of the overlap) are never
// written by the reference; inv_j, dxidx, alpha, beta, gamma keep whatever the
// caller stored there (zero-filled arrays give 0 for inv_j and NaN = 0/0 for the
// metrics there).  Scratch arrays are zero-filled.
void gridtransformation(V dxidx, V inv_j, V alpha, V beta, V gamma, V x, V y, V z, const Box& b,
                        const Box& b0) {
  Tmp xyz(3, b), dxdxi(3, b), dxdeta(3, b), dxdzeta(3, b);
  Tmp tempxi(6, b), tempeta(6, b), tempzeta(6, b);
  Tmp tempxixi(6, b), tempetaeta(6, b), tempzetazeta(6, b);
  for (int k = b.ks; k <= b.ke; ++k)  // :81-89
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) {
        xyz(1, i, j, k) = x(i, j, k);
        xyz(2, i, j, k) = y(i, j, k);
        xyz(3, i, j, k) = z(i, j, k);
      }
  region_derivative(xyz.view, dxdxi.view, 3, 0, b, b0);
  region_derivative(xyz.view, dxdeta.view, 3, 1, b, b0);
  const bool two = g_flags.dimension == IFLAG_2D;
  if (two) {  // :270-273: the zeta direction is the unit z vector everywhere
    for (int k = b.ks; k <= b.ke; ++k)
      for (int j = b.js; j <= b.je; ++j)
        for (int i = b.is; i <= b.ie; ++i) {
          dxdzeta(1, i, j, k) = 0.0;
          dxdzeta(2, i, j, k) = 0.0;
          dxdzeta(3, i, j, k) = 1.0;
        }
  } else {
    region_derivative(xyz.view, dxdzeta.view, 3, 2, b, b0);
  }

  auto jac = [&](int i, int j, int k) {  // :366-371
    double dxdxi0 = dxdxi(1, i, j, k), dxdeta0 = dxdeta(1, i, j, k), dxdzeta0 = dxdzeta(1, i, j, k);
    double dydxi0 = dxdxi(2, i, j, k), dydeta0 = dxdeta(2, i, j, k), dydzeta0 = dxdzeta(2, i, j, k);
    double dzdxi0 = dxdxi(3, i, j, k), dzdeta0 = dxdeta(3, i, j, k), dzdzeta0 = dxdzeta(3, i, j, k);
    inv_j(i, j, k) = dxdxi0 * dydeta0 * dzdzeta0 + dxdeta0 * dydzeta0 * dzdxi0 +
                     dxdzeta0 * dydxi0 * dzdeta0 - dxdzeta0 * dydeta0 * dzdxi0 -
                     dxdxi0 * dydzeta0 * dzdeta0 - dxdeta0 * dydxi0 * dzdzeta0;
  };
  // :359-520: physical core, then each ghost slab including the face plane.
  for (int k = b0.ks; k <= b0.ke; ++k)
    for (int j = b0.js; j <= b0.je; ++j)
      for (int i = b0.is; i <= b0.ie; ++i) jac(i, j, k);
  for (int k = b0.ks; k <= b0.ke; ++k)
    for (int j = b0.js; j <= b0.je; ++j) {
      for (int i = b.is; i <= b0.is; ++i) jac(i, j, k);
      for (int i = b0.ie; i <= b.ie; ++i) jac(i, j, k);
    }
  for (int k = b0.ks; k <= b0.ke; ++k)
    for (int i = b0.is; i <= b0.ie; ++i) {
      for (int j = b.js; j <= b0.js; ++j) jac(i, j, k);
      for (int j = b0.je; j <= b.je; ++j) jac(i, j, k);
    }
  for (int j = b0.js; j <= b0.je; ++j)
    for (int i = b0.is; i <= b0.ie; ++i) {
      for (int k = b.ks; k <= b0.ks; ++k) jac(i, j, k);
      for (int k = b0.ke; k <= b.ke; ++k) jac(i, j, k);
    }

  if (two) {  // :543-557: in-plane metrics from the in-plane derivatives
    for (int k = b.ks; k <= b.ke; ++k)
      for (int j = b.js; j <= b.je; ++j)
        for (int i = b.is; i <= b.ie; ++i) {
          double ij = inv_j(i, j, k);
          dxidx(1, i, j, k) = dxdeta(2, i, j, k) / ij;
          dxidx(2, i, j, k) = -dxdeta(1, i, j, k) / ij;
          dxidx(3, i, j, k) = 0.0;
          dxidx(4, i, j, k) = -dxdxi(2, i, j, k) / ij;
          dxidx(5, i, j, k) = dxdxi(1, i, j, k) / ij;
          dxidx(6, i, j, k) = 0.0;
          dxidx(7, i, j, k) = 0.0;
          dxidx(8, i, j, k) = 0.0;
          dxidx(9, i, j, k) = 1.0;
        }
  }
  for (int k = b.ks; k <= b.ke && !two; ++k)  // :559-584
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) {
        double X = xyz(1, i, j, k), Y = xyz(2, i, j, k), Z = xyz(3, i, j, k);
        tempxi(1, i, j, k) = dxdzeta(2, i, j, k) * Z;
        tempxi(2, i, j, k) = dxdzeta(3, i, j, k) * X;
        tempxi(3, i, j, k) = dxdzeta(1, i, j, k) * Y;
        tempxi(4, i, j, k) = dxdeta(2, i, j, k) * Z;
        tempxi(5, i, j, k) = dxdeta(3, i, j, k) * X;
        tempxi(6, i, j, k) = dxdeta(1, i, j, k) * Y;
        tempeta(1, i, j, k) = dxdzeta(2, i, j, k) * Z;
        tempeta(2, i, j, k) = dxdzeta(3, i, j, k) * X;
        tempeta(3, i, j, k) = dxdzeta(1, i, j, k) * Y;
        tempeta(4, i, j, k) = dxdxi(2, i, j, k) * Z;
        tempeta(5, i, j, k) = dxdxi(3, i, j, k) * X;
        tempeta(6, i, j, k) = dxdxi(1, i, j, k) * Y;
        tempzeta(1, i, j, k) = dxdeta(2, i, j, k) * Z;
        tempzeta(2, i, j, k) = dxdeta(3, i, j, k) * X;
        tempzeta(3, i, j, k) = dxdeta(1, i, j, k) * Y;
        tempzeta(4, i, j, k) = dxdxi(2, i, j, k) * Z;
        tempzeta(5, i, j, k) = dxdxi(3, i, j, k) * X;
        tempzeta(6, i, j, k) = dxdxi(1, i, j, k) * Y;
      }
  if (!two) {
    region_derivative(tempxi.view, tempxixi.view, 6, 0, b, b0);        // :587-655
    region_derivative(tempeta.view, tempetaeta.view, 6, 1, b, b0);     // :658-726
    region_derivative(tempzeta.view, tempzetazeta.view, 6, 2, b, b0);  // :729-797
  }

  for (int k = b.ks; k <= b.ke && !two; ++k)  // :799-831
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) {
        double ij = inv_j(i, j, k);
        dxidx(1, i, j, k) = (tempzetazeta(1, i, j, k) - tempetaeta(1, i, j, k)) / ij;
        dxidx(2, i, j, k) = (tempzetazeta(2, i, j, k) - tempetaeta(2, i, j, k)) / ij;
        dxidx(3, i, j, k) = (tempzetazeta(3, i, j, k) - tempetaeta(3, i, j, k)) / ij;
        dxidx(4, i, j, k) = (tempxixi(1, i, j, k) - tempzetazeta(4, i, j, k)) / ij;
        dxidx(5, i, j, k) = (tempxixi(2, i, j, k) - tempzetazeta(5, i, j, k)) / ij;
        dxidx(6, i, j, k) = (tempxixi(3, i, j, k) - tempzetazeta(6, i, j, k)) / ij;
        dxidx(7, i, j, k) = (tempetaeta(4, i, j, k) - tempxixi(4, i, j, k)) / ij;
        dxidx(8, i, j, k) = (tempetaeta(5, i, j, k) - tempxixi(5, i, j, k)) / ij;
        dxidx(9, i, j, k) = (tempetaeta(6, i, j, k) - tempxixi(6, i, j, k)) / ij;
      }
  for (int k = b.ks; k <= b.ke; ++k)  // :838-865
    for (int j = b.js; j <= b.je; ++j)
      for (int i = b.is; i <= b.ie; ++i) {
        double x1 = dxidx(1, i, j, k), x2 = dxidx(2, i, j, k), x3 = dxidx(3, i, j, k);
        double e1 = dxidx(4, i, j, k), e2 = dxidx(5, i, j, k), e3 = dxidx(6, i, j, k);
        double z1 = dxidx(7, i, j, k), z2 = dxidx(8, i, j, k), z3 = dxidx(9, i, j, k);
        double ij = inv_j(i, j, k);
        alpha(1, i, j, k) = (x1 * x1 + x2 * x2 + x3 * x3) * ij;
        alpha(2, i, j, k) = (x1 * e1 + x2 * e2 + x3 * e3) * ij;
        alpha(3, i, j, k) = (x1 * z1 + x2 * z2 + x3 * z3) * ij;
        beta(1, i, j, k) = (e1 * x1 + e2 * x2 + e3 * x3) * ij;
        beta(2, i, j, k) = (e1 * e1 + e2 * e2 + e3 * e3) * ij;
        beta(3, i, j, k) = (e1 * z1 + e2 * z2 + e3 * z3) * ij;
        gamma(1, i, j, k) = (z1 * x1 + z2 * x2 + z3 * x3) * ij;
        gamma(2, i, j, k) = (z1 * e1 + z2 * e2 + z3 * e3) * ij;
        gamma(3, i, j, k) = (z1 * z1 + z2 * z2 + z3 * z3) * ij;
      }
}

// sub_init_spacing.f90:16-113
void init_spacing(V spci, V spcj, V spck, V spacing, V vol, V x, V y, V z, const Box& b,
                  const Box& b0) {
  for (long n = 0; n < b.size(); ++n) {
    spci.p[n] = 0.0; spcj.p[n] = 0.0; spck.p[n] = 0.0; spacing.p[n] = 0.0; vol.p[n] = 0.0;
  }
  auto len = [&](int i, int j, int k, int di, int dj, int dk) {
    double dx = x(i + di, j + dj, k + dk) - x(i, j, k);
    double dy = y(i + di, j + dj, k + dk) - y(i, j, k);
    double dz = z(i + di, j + dj, k + dk) - z(i, j, k);
    return std::sqrt(p2(dx) + p2(dy) + p2(dz));
  };
  for (int k = b0.ks; k <= b0.ke; ++k)
    for (int j = b0.js; j <= b0.je; ++j) {
      for (int i = b0.is; i <= b0.ie - 1; ++i) spci(i, j, k) = len(i, j, k, 1, 0, 0);
      spci(b0.ie, j, k) = spci(b0.ie - 1, j, k);
    }
  for (int k = b0.ks; k <= b0.ke; ++k) {
    for (int j = b0.js; j <= b0.je - 1; ++j)
      for (int i = b0.is; i <= b0.ie; ++i) spcj(i, j, k) = len(i, j, k, 0, 1, 0);
    for (int i = b0.is; i <= b0.ie; ++i) spcj(i, b0.je, k) = spcj(i, b0.je - 1, k);
  }
  if (b0.ke > b0.ks) {
    for (int k = b0.ks; k <= b0.ke - 1; ++k)
      for (int j = b0.js; j <= b0.je; ++j)
        for (int i = b0.is; i <= b0.ie; ++i) spck(i, j, k) = len(i, j, k, 0, 0, 1);
    for (int j = b0.js; j <= b0.je; ++j)
      for (int i = b0.is; i <= b0.ie; ++i) spck(i, j, b0.ke) = spck(i, j, b0.ke - 1);
  }
  for (int k = b0.ks; k <= b0.ke; ++k)
    for (int j = b0.js; j <= b0.je; ++j)
      for (int i = b0.is; i <= b0.ie; ++i) {
        spacing(i, j, k) = std::max(std::max(spci(i, j, k), spcj(i, j, k)), spck(i, j, k));
        if (b0.ke == b0.ks)
          vol(i, j, k) = spci(i, j, k) * spcj(i, j, k);
        else
          vol(i, j, k) = spci(i, j, k) * spcj(i, j, k) * spck(i, j, k);
      }
}

}  // namespace oracle
