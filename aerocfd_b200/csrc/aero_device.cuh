// Device-side data layout and helpers shared by every kernel of the aerocfd
// residual-and-update path.
//
// Layout in HBM: one arena per case.  Each block owns, for every field, a
// structure-of-arrays set of component planes over its full index box
// is..ie x js..je x ks..ke (overlap ghosts included), i fastest, then j, then k.
// Component c (1-based, as in the reference) of node (i,j,k) of field f lives at
//   f + (c-1)*plane + (i-is) + nx*((j-js) + ny*(k-ks)),
// with `plane` the box size rounded up to 32 doubles so every plane starts on a
// 256-byte boundary.  The reference's host arrays are (component, i, j, k)
// column-major; the transfer kernels in aero_transfer.cu convert between the two.
#pragma once
#include <cstdint>

#include "aero_crmath.h"

namespace aero {

// Field ids of the C-ABI (AERO_F_* in include/aerocfd_gpu.h).
enum FieldId {
  F_Q = 0, F_PRI, F_RHSI, F_RHSV, F_RHS, F_DT, F_DXIDX, F_INVJ, F_AMU, F_NUT, F_SARHS,
  F_X, F_Y, F_Z, F_DIST, F_ALPHA, F_BETA, F_GAMMA, F_DUDX, F_TAO, F_VOR, F_LENGTH, F_SPACING, F_Q0,
  // device-only scratch
  F_RA, F_RB, F_RC, F_DIAG, F_FVH, F_DIASD, F_SAS,
  F_FIH,  // inviscid face fluxes of the face-based kernels (5 per direction)
  F_NUM
};
__host__ __device__ constexpr int field_nc(int f) {
  return f == F_Q ? 5 : f == F_PRI ? 7 : f == F_RHSI ? 5 : f == F_RHSV ? 5 : f == F_RHS ? 5
       : f == F_DXIDX ? 9 : f == F_AMU ? 3 : f == F_ALPHA ? 3 : f == F_BETA ? 3 : f == F_GAMMA ? 3
       : f == F_DUDX ? 9 : f == F_TAO ? 6 : f == F_FVH ? 15 : f == F_SAS ? 7 : f == F_Q0 ? 10
       : f == F_FIH ? 15 : 1;
}
constexpr int kNumPublicFields = F_Q0 + 1;

struct Box {
  int is, ie, js, je, ks, ke;
  __host__ __device__ int nx() const { return ie - is + 1; }
  __host__ __device__ int ny() const { return je - js + 1; }
  __host__ __device__ int nz() const { return ke - ks + 1; }
  __host__ __device__ long size() const { return (long)nx() * ny() * nz(); }
  __host__ __device__ bool contains(int i, int j, int k) const {
    return i >= is && i <= ie && j >= js && j <= je && k >= ks && k <= ke;
  }
};

// Per-case scalars (module ns_const / flag_var values the path reads).
struct CaseConsts {
  double gamma, cv, re, tinf, prl, prt, cfl;
  double d_0, u_0, p_0, c_0, aoa, nutinf;
  // cos(aoa) and sin(aoa) from the host's libm (the reference's cos and sin
  // on its CPU), so every kernel uses the same values as the CPU path
  double cos_aoa, sin_aoa;
  int dimension, solver, time, turbulence, des, bufferLength;
  int inviscid;  // iflag_inviscid: 4 Roe + WENO3, 5 Steger-Warming + WENO5, 8 WCNS5 + Roe
};

// Everything a kernel needs to address one block's fields.
struct BlockView {
  Box b, b0, b1;
  int nx, ny;
  long plane;            // doubles between component planes
  double* f[F_NUM];      // base of component 1 of each field (nullptr if absent)
  // LU-SGS workspace, indexed by the hyperplane-major position of an updated
  // node (nodes of plane h = (i-is1)+(j-js1)+(k-ks1) are contiguous):
  int nplanes, pmax;     // number of hyperplanes, largest plane
  long* poff;            // nplanes+1 plane offsets
  double* rec_f;         // kRec per node: forward blocks from the i-1, j-1, k-1 neighbours
  double* rec_b;         // kRec per node: backward blocks from the i+1, j+1, k+1 neighbours
  double* sca;           // kSca per node: rhs(5), diag, inv_j, 1/diag, 1/inv_j, unused
  int* nbr;              // 6 per node: hyperplane-major positions of those neighbours (-1: outside)
  long* nat;             // natural (box) index of the node
  int* pidx;             // per updated-box node in box order: its hyperplane-major position
  double* sa_rec;        // kSaRec per node: SA sweep records (plane-local layout)
  double* sa_dq;         // 1 per node: SA forward-sweep increment
  double* dqs;           // 8 per node: dq* (forward result), padded to 64 bytes
  double* dq;            // 5 per node: dq (backward result)
  // Case constants of this block when blocks of different cases share one
  // launch (a batch); nullptr: the launch's constants apply.
  const CaseConsts* ccb;
  // Registered blocks: this block's own status word (the ST_* bits its
  // kernels raised, besides the global word) and its live flag, refreshed from
  // the status word at the start of every step while retirement is on
  // (aero_set_retirement); a block whose flag is 0 is skipped by every kernel
  // of the step, so its state stays as it was when it failed.  Both nullptr
  // for the drop-in entry points' temporary views.
  unsigned* bstat;
  const int* live;
  __device__ __forceinline__ bool retired() const { return live && *live == 0; }
  __device__ __forceinline__ void raise(unsigned bits) const {
#if defined(__CUDA_ARCH__)
    if (bstat) atomicOr(bstat, bits);
#else
    (void)bits;  // host builds of this header (tests) never call it
#endif
  }

  __device__ __forceinline__ long at(int i, int j, int k) const {
    return (long)(i - b.is) + (long)nx * ((long)(j - b.js) + (long)ny * (long)(k - b.ks));
  }
  __device__ __forceinline__ double& v(int fid, int c, long n) const { return f[fid][(long)(c - 1) * plane + n]; }
  __device__ __forceinline__ double& s(int fid, long n) const { return f[fid][n]; }
};

// LU-SGS record stride: three 5x5 blocks (75 doubles) plus the packed
// neighbour positions, 608 bytes (bulk-copy alignment: multiples of 16).
constexpr int kRec = 76;
// LU-SGS per-node scalars: rhs(5), diag, inv_j, 1/diag, 1/inv_j, unused.
constexpr int kSca = 10;
// SA sweep records per node: 0.5*(U+|U|) x3, 0.5*(U-|U|) x3, sa_rhs, diag,
// packed forward and backward neighbours.
constexpr int kSaRec = 12;

// Three plane-local indices (+1; 0 = no neighbour) in one 64-bit word: the
// neighbours' positions in their hyperplane relative to its first node.  Bit
// 63, unused by the indices, marks an LU-SGS node whose divisors fall outside
// div2_rn's fast range.
constexpr int kNbrBits = 21;
#ifdef __CUDACC__
__device__ __forceinline__ double pack_nbrs(const int* nb, long prev_base, bool slow_div = false) {
  unsigned long long u = slow_div ? 1ull << 63 : 0ull;
#pragma unroll
  for (int e = 0; e < 3; ++e) {
    unsigned long long f = nb[e] < 0 ? 0ull : (unsigned long long)(nb[e] - prev_base + 1);
    u |= f << (kNbrBits * e);
  }
  return __longlong_as_double((long long)u);
}
__device__ __forceinline__ int nbr_local(double packed, int e) {
  unsigned long long u = (unsigned long long)__double_as_longlong(packed);
  return (int)((u >> (kNbrBits * e)) & ((1ull << kNbrBits) - 1)) - 1;
}
__device__ __forceinline__ bool nbr_slow_div(double packed) { return __double2hiint(packed) < 0; }
#endif


// ---------------------------------------------------------------- arithmetic
// Integer powers follow gfortran's powi expansion; x**2 is x*x.
__device__ __forceinline__ double p2(double x) { return x * x; }
__device__ __forceinline__ double p3(double x) { double x2 = x * x; return x2 * x; }
__device__ __forceinline__ double p5(double x) { double x2 = x * x; double x3 = x2 * x; return x3 * x2; }
__device__ __forceinline__ double p6(double x) { double x2 = x * x; double x3 = x2 * x; return x3 * x3; }

// a / b rounded to nearest, given rb = 1/b rounded to nearest: Markstein's
// correction (P. Markstein, IBM J. Res. Dev. 34(1), 1990, Theorem 1: with rb
// correctly rounded and q within one ulp of a/b, q + (a - b*q)*rb rounded once
// is the correctly rounded quotient).  The first correction makes a*rb
// faithful, the second rounds it correctly; each remainder a - b*q is exact
// in one fma.  The theorem needs normal operands and quotient with room for the
// remainder, so values outside [2^-960, 2^960] (and a = 0, whose sign the
// corrections would lose) take the IEEE division.  The result is bit-identical
// to a / b.
__device__ __forceinline__ double div_newton(double a, double b, double rb) {
  double q = a * rb;
  double r = fma(-q, b, a);
  q = fma(r, rb, q);
  r = fma(-q, b, a);
  return fma(r, rb, q);
}
__device__ __forceinline__ double div_rn(double a, double b, double rb) {
  double q = div_newton(a, b, rb);
  double aa = fabs(a), ab = fabs(b), aq = fabs(q);
  if (!(aa > 0x1p-960 && aa < 0x1p960 && ab > 0x1p-960 && ab < 0x1p960 && aq > 0x1p-960 && aq < 0x1p960))
    q = a / b;
  return q;
}
// div_rn with the IEEE division of the rare out-of-range case in a function
// of its own, which keeps the division's long code (and its registers) out of
// a sweep loop.  Bit-identical to a / b, as div_rn.
inline __device__ __noinline__ double div1_ieee(double a, double b) { return a / b; }
__device__ __forceinline__ double div_rn_lean(double a, double b, double rb) {
  double q = div_newton(a, b, rb);
  double aa = fabs(a), ab = fabs(b), aq = fabs(q);
  if (!(aa > 0x1p-960 && aa < 0x1p960 && ab > 0x1p-960 && ab < 0x1p960 && aq > 0x1p-960 && aq < 0x1p960))
    q = div1_ieee(a, b);
  return q;
}

// The two divisions of a sweep row, (a / b1) / b2, with the stored
// reciprocals rb1, rb2.  div_rn's corrections are exact while a, b and the
// quotient lie within (2^-960, 2^960).  With both divisors within
// (2^-200, 2^200) (divisors_ok, tested once per node when its records are
// made) and |a| within (2^-500, 2^500), the first quotient lies within
// (2^-700, 2^700) and the second within (2^-900, 2^900), so only a is tested
// on the plane-to-plane chain.  Every other case, zero included, takes the
// IEEE divisions in a function of its own, which keeps the division's long
// code out of the sweep loop.  The result equals a / b1 / b2 bit for bit.
inline __device__ __noinline__ double div2_ieee(double a, double b1, double b2) { return a / b1 / b2; }
__device__ __forceinline__ bool divisors_ok(double b1, double b2) {
  const double x1 = fabs(b1), x2 = fabs(b2);
  return x1 > 0x1p-200 && x1 < 0x1p200 && x2 > 0x1p-200 && x2 < 0x1p200;
}
__device__ __forceinline__ double div2_rn(double a, double b1, double rb1, double b2, double rb2, bool bok) {
  double q = div_newton(div_newton(a, b1, rb1), b2, rb2);
  const double aa = fabs(a);
  if (!(bok && aa > 0x1p-500 && aa < 0x1p500)) q = div2_ieee(a, b1, b2);
  return q;
}

// Spalart-Allmaras constants (module_tursa.f90:4-10).
constexpr double SA_DTA = 2.0 / 3.0, SA_KAR = 0.41;
constexpr double SA_CB1 = 0.1355, SA_CB2 = 0.622;
constexpr double SA_CW1 = SA_CB1 / SA_KAR / SA_KAR + (1.0 + SA_CB2) / SA_DTA;
constexpr double SA_CW2 = 0.3, SA_CW3 = 2.0;
constexpr double SA_CT3 = 1.2, SA_CT4 = 0.5;
constexpr double SA_CV1 = 7.1;
constexpr double SA_KAR2 = SA_KAR * SA_KAR;
constexpr double SA_CV13 = SA_CV1 * SA_CV1 * SA_CV1;

// Reference flag values (module_flags.f90:30-87).
enum {
  IFLAG_2D = 2, IFLAG_3D = 3, IFLAG_NSSOLVER = 0, IFLAG_EULERSOLVER = 1,
  IFLAG_STEADY = 0, IFLAG_UNSTEADY = 1, IFLAG_LAMINAR = 0, IFLAG_SA = 2,
  IFLAG_1STIMPLICIT = 2, IFLAG_2NDCRANK = 3,
  IFLAG_3RDWENO = 4, IFLAG_5THWENO = 5, IFLAG_5THWCNS = 8,
  IFLAG_DES97 = 1, IFLAG_DDES = 2,
  BC_INFLOW = -50, BC_OUTFLOW = -40, BC_SYMM = -30, BC_WALL = -20, BC_FARFIELD = -10,
};

// Device status word bits (aero_get_status).
enum StatusBits : unsigned {
  ST_NEG_DENSITY = 1u, ST_NONFINITE_RESIDUAL = 2u, ST_NEG_PRESSURE = 4u, ST_TIMEOUT = 8u,
};

}  // namespace aero
