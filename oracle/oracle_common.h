// TEST INFRASTRUCTURE ONLY -- the CPU oracle for aerocfd's per-iteration residual
// and update path.  Nothing in the product (aerocfd_b200/, include/) links or calls
// this code; tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it
// as the checker.
//
// Parity status: UNPINNED against the reference's own outputs.  The reference is
// Fortran-90 + MPI and there is no Fortran compiler or MPI in this image, and the
// reference ships no tests, fixtures or golden vectors.  The restatement is pinned
// instead by known-answer tests derived from the mathematics (freestream
// preservation, Roe consistency, WENO3 exactness on linear data, calc_jm versus a
// finite-difference Jacobian, LU-SGS identities, halo orientation round trips,
// SA source at zero viscosity, residual of a known field): tests/test_oracle_kat.py.
//
// Every routine restates the Fortran loop by loop, keeps the 1-based index boxes
// (is..ie incl. overlap ghosts, is0..ie0 physical nodes, is1..ie1 updated nodes),
// the (component, i, j, k) column-major layout and the Fortran operation order
// (left-to-right evaluation, x**2 -> x*x, integer powers by GCC's powi chain).
// Build with -ffp-contract=off so no multiply-add is fused.
//
// x**y and exp(x): the reference gets them from the platform libm, which is
// not specified to the last bit (glibc's pow and exp return a result one ulp
// off the correctly rounded one on about 1 in 1,200 arguments; CUDA's differ on
// others).  The oracle builds used as the checker and the FP64 GPU kernels
// both call the correctly rounded crm::pow / crm::exp of
// aerocfd_b200/csrc/aero_crmath.h (a header of plain arithmetic, host and
// device), so that libm choices do not separate them; tests/test_crmath.py
// checks those functions against exact values (Python's decimal) and against
// glibc on the arguments the solver produces.  The build timed as the CPU
// baseline (liboracle_libm.so) calls glibc's pow and exp instead, as the
// reference does, so its speed is the reference's.
#pragma once
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "../aerocfd_b200/csrc/aero_crmath.h"

namespace oracle {
// x**y and exp(x) of the restatement: the shared correctly rounded functions,
// or, in the build timed as the CPU baseline (ORACLE_PLATFORM_LIBM), the
// platform libm that the reference's own build calls.
inline double xpow(double x, double y) {
#ifdef ORACLE_PLATFORM_LIBM
  return std::pow(x, y);
#else
  return crm::pow(x, y);
#endif
}
inline double xexp(double x) {
#ifdef ORACLE_PLATFORM_LIBM
  return std::exp(x);
#else
  return crm::exp(x);
#endif
}
}  // namespace oracle

namespace oracle {

// Index box is:ie, js:je, ks:ke of one Fortran array.
struct Box {
  int is, ie, js, je, ks, ke;
  long nx() const { return (long)ie - is + 1; }
  long ny() const { return (long)je - js + 1; }
  long nz() const { return (long)ke - ks + 1; }
  long size() const { return nx() * ny() * nz(); }
  long at(int i, int j, int k) const {
#ifdef ORACLE_BOUNDS
    if (i < is || i > ie || j < js || j > je || k < ks || k > ke) {
      std::fprintf(stderr, "oracle: index (%d,%d,%d) outside (%d:%d,%d:%d,%d:%d)\n", i, j, k,
                   is, ie, js, je, ks, ke);
      std::abort();
    }
#endif
    return (long)(i - is) + nx() * ((long)(j - js) + ny() * (long)(k - ks));
  }
};

// View of a Fortran array a(nc, is:ie, js:je, ks:ke); component index is 1-based.
struct V {
  double* p;
  int nc;
  Box b;
  double& operator()(int c, int i, int j, int k) const {
#ifdef ORACLE_BOUNDS
    if (c < 1 || c > nc) {
      std::fprintf(stderr, "oracle: component %d outside 1:%d\n", c, nc);
      std::abort();
    }
#endif
    return p[(c - 1) + (long)nc * b.at(i, j, k)];
  }
  double& operator()(int i, int j, int k) const { return p[b.at(i, j, k)]; }
};

// Owning scratch array with the same indexing, zero-filled (the reference
// allocates and zero-fills its temporaries explicitly in every routine).
struct Tmp {
  std::vector<double> v;
  V view;
  Tmp(int nc, const Box& b) : v((size_t)nc * b.size(), 0.0) { view = V{v.data(), nc, b}; }
  double& operator()(int c, int i, int j, int k) { return view(c, i, j, k); }
  double& operator()(int i, int j, int k) { return view(i, j, k); }
  void zero() { std::fill(v.begin(), v.end(), 0.0); }
};

// Integer powers as gfortran expands them (GCC powi addition chains).
inline double p2(double x) { return x * x; }
inline double p3(double x) { double x2 = x * x; return x2 * x; }
inline double p5(double x) { double x2 = x * x; double x3 = x2 * x; return x3 * x2; }
inline double p6(double x) { double x2 = x * x; double x3 = x2 * x; return x3 * x3; }

// Fortran SIGN(1.d0, b): +1 for b >= +0, -1 for negative b (incl. -0).
inline double fsign1(double b) { return std::copysign(1.0, b); }

// Module flag_var values (module_flags.f90:30-87).
enum {
  IFLAG_2D = 2, IFLAG_3D = 3,
  IFLAG_NSSOLVER = 0, IFLAG_EULERSOLVER = 1,
  IFLAG_STEADY = 0, IFLAG_UNSTEADY = 1,
  IFLAG_1STIMPLICIT = 2, IFLAG_2NDCRANK = 3,
  IFLAG_3RDWENO = 4, IFLAG_5THWENO = 5, IFLAG_5THWCNS = 8,
  IFLAG_LAMINAR = 0, IFLAG_SA = 2,
  IFLAG_DES97 = 1, IFLAG_DDES = 2,
  BC_INFLOW = -50, BC_OUTFLOW = -40, BC_SYMM = -30, BC_WALL = -20, BC_FARFIELD = -10,
};

// Spalart-Allmaras constants (module_tursa.f90:4-10).
const double SA_DTA = 2.0 / 3.0, SA_KAR = 0.41;
const double SA_CB1 = 0.1355, SA_CB2 = 0.622;
const double SA_CW1 = SA_CB1 / SA_KAR / SA_KAR + (1.0 + SA_CB2) / SA_DTA;
const double SA_CW2 = 0.3, SA_CW3 = 2.0;
const double SA_CT3 = 1.2, SA_CT4 = 0.5;
const double SA_CV1 = 7.1;
// Constant-folded parameter powers (gfortran folds cv1**3 and kar**2 exactly
// once; both equal the runtime products for these values).
const double SA_KAR2 = SA_KAR * SA_KAR;
const double SA_CV13 = SA_CV1 * SA_CV1 * SA_CV1;

struct Flags {
  int dimension = IFLAG_3D, solver = IFLAG_NSSOLVER, time = IFLAG_STEADY;
  int timeadvance = IFLAG_1STIMPLICIT, turbulence = IFLAG_LAMINAR, des = 0;
  int bufferLength = 2, inviscid = 4;
};

struct Consts {
  double ma = 0.5, re = 1e6, tinf = 288.15, aoa = 0.0;  // aoa in radians
  double cfl = 5.0, dt = 1.0;
  double d_0 = 1, u_0 = 1, t_0 = 1, p_0 = 0, c_0 = 0, cv = 0, cp = 0;
  double gamma = 1.4, prl = 0.72, prt = 0.90;
  double nutinf = 1.341946;
};

extern Flags g_flags;
extern Consts g_consts;

}  // namespace oracle
