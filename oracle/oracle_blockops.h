// TEST INFRASTRUCTURE ONLY (see oracle_common.h).
#pragma once
#include "oracle_common.h"

namespace oracle {

long get_primitivevariables(int mm, V pri_v, V q, double gamma, double cv, const Box& b);
void thirdorder_weno(V df, V f, const Box& b, const Box& r0, int coord, int direction);
void roe_3d(V ql, V qr, V flux, V dxidx, V inv_j, double gamma, const Box& b, const Box& r0,
            int coord);
void inviscid_flux_sw_weno5(V rhsi, V q, V dxidx, V inv_j, const Box& b, const Box& b1, double gamma);
void inviscid_flux_wcns5(V rhsi, V q, V dxidx, V inv_j, const Box& b, const Box& b1, double gamma);
// inviscid_flux_1 or the extension scheme g_flags.inviscid names
void inviscid_flux(V rhsi, V q, V dxidx, V inv_j, const Box& b, const Box& b0, const Box& b1, double gamma);
void inviscid_flux_1(V rhsi, V q, V dxidx, V inv_j, const Box& b, const Box& b0, const Box& b1,
                     double gamma);
void viscous_flux(V rhsv, V pri_v, V amu, V vor, V dudx, V tao, V dxidx, V inv_j, double tinf,
                  double prl, double prt, double gamma, double cv, double re, const Box& b,
                  const Box& b0, const Box& b1);
void find_dt(V dt, double* dtmax, double* dtmin, double* cflmax, double* cflmin, V pri_v, V amu,
             V dxidx, double re, double* cfl, const Box& b, int iflag_time);
void calc_jm(double a[25], double q1, double q2, double q3, double q4, double q5, double dxidx,
             double dxidy, double dxidz, double gamma);
void crank2nd(V q, V q0, V dt, V pri_v, V rhs, V rhsi, V rhsv, V dxidx, V inv_j, const Box& b, const Box& b0,
              const Box& b1, double gamma);
void update_q0(V q0, V q, const Box& b0);
void implicit1st(V q, V dt, V pri_v, V rhs, V rhsi, V rhsv, V dxidx, V inv_j, const Box& b,
                 const Box& b0, const Box& b1, double gamma, double cfl);
void sa_model(V nut, V sa_rhs, V dt, V pri_v, V amu, V dudx, V vor, V dxidx, V inv_j, V alpha,
              V beta, V gamma, V length, V dist, V spac, double re, double cfl, const Box& b,
              const Box& b0, const Box& b1);
void gridtransformation(V dxidx, V inv_j, V alpha, V beta, V gamma, V x, V y, V z, const Box& b,
                        const Box& b0);
void init_spacing(V spci, V spcj, V spck, V spacing, V vol, V x, V y, V z, const Box& b,
                  const Box& b0);

}  // namespace oracle
