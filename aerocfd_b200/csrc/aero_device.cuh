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
  // nplanes x (nz1+2) k-segment starts: entry h*(nz1+2) + c+1 counts the
  // nodes of plane h with k-offset below c (c = -1 .. nz1), i.e. where the
  // nodes of k-offset c begin inside the plane (a plane lists its nodes by
  // k-offset, then j); the slab sweeps address their k-slabs by it
  int* seg;
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
  // 2-D mode (iflag_dimension = 2): the block is the single plane k = 1 (a
  // 3-D block has at least three k-planes)
  __host__ __device__ __forceinline__ bool planar() const { return b.ks == b.ke; }
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


// The updated box grown by one node on every side, where the implicit
// schemes form their radii and diagonals (sub_timeadvancement_1stimplicit.f90:
// 110-156); in 2-D only in i and j (:157-210), the block having one plane.
__host__ __device__ __forceinline__ Box grown_box(const Box& b, const Box& b1) {
  const int kx = b.ks == b.ke ? 0 : 1;
  return Box{b1.is - 1, b1.ie + 1, b1.js - 1, b1.je + 1, b1.ks - kx, b1.ke + kx};
}
__host__ __device__ __forceinline__ Box grown_box(const BlockView& B) { return grown_box(B.b, B.b1); }
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

#ifdef __CUDACC__
// ------------------------------------------- thread-block cluster primitives
// (the slab sweeps: a CTA's progress counters and ring slots are written by
// its neighbours in the cluster)
// Ring, inbox and staging slots (planes) of a slab sweep, at most.
constexpr int kSlabSlots = 8;
// Nanoseconds of the GPU's global timer.
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bound of every wait of the cluster sweeps: a wait not satisfied within
// kWaitNs of the global timer (or, as a second bound, within 2^30 polls)
// gives up, and the sweep ends with ST_TIMEOUT.  A plane step takes
// microseconds, so the bound only ends a wait that cannot finish.
constexpr unsigned long long kWaitNs = 1000000000ull;
// Polls `done` until it holds (true) or the bound passes (false); the timer is
// read every 64 polls.
template <class Done>
__device__ __forceinline__ bool wait_bounded(Done done) {
  if (done()) return true;
  const unsigned long long t0 = global_ns();
  for (unsigned n = 1; n < (1u << 30); ++n) {
    if (done()) return true;
    if ((n & 63u) == 0u && global_ns() - t0 > kWaitNs) return false;
  }
  return false;
}
// Sweep codes and wait kinds of the first wait that gave up, recorded in
// status words 1..6 (aero_timeout_site): word 1 claims the record, then the
// sweep, the block, the CTA's rank in its cluster, the step and the wait.
enum TimeoutSweep { TS_BULK = 1, TS_SLAB = 2, TS_SA_SLAB = 3, TS_STAGED = 4 };
enum TimeoutWait { TW_PLANE = 1, TW_PROGRESS = 2, TW_LAST_PLANE = 3 };
__device__ __forceinline__ void note_timeout(unsigned* status, int sweep, int block, int rank, int step,
                                             int wait) {
  if (!status || atomicCAS(status + 1, 0u, 1u) != 0u) return;
  status[2] = (unsigned)sweep;
  status[3] = (unsigned)block;
  status[4] = (unsigned)rank;
  status[5] = (unsigned)step;
  status[6] = (unsigned)wait;
}

namespace slab {
__device__ __forceinline__ unsigned rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned size() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
  return r;
}
__device__ __forceinline__ unsigned local(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
// address of the same shared-memory word in CTA `r` of the cluster
__device__ __forceinline__ unsigned map(unsigned addr, unsigned r) {
  unsigned out;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(addr), "r"(r));
  return out;
}
// full cluster barrier (release / acquire): orders every shared::cluster
// store issued before it
__device__ __forceinline__ void sync() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// relaxed store of a counter into another CTA's shared memory (no fence: the
// counters only say that a slot's earlier contents have been read)
__device__ __forceinline__ void store_relaxed(unsigned remote, int v) {
  asm volatile("st.relaxed.cluster.shared::cluster.u32 [%0], %1;" ::"r"(remote), "r"(v) : "memory");
}
__device__ __forceinline__ int load_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.cluster.shared::cta.u32 %0, [%1];" : "=r"(v) : "r"(local(p)) : "memory");
  return v;
}
// mbarriers of this CTA
__device__ __forceinline__ void bar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(local(bar)), "r"(count) : "memory");
}
// this CTA's arrival on `bar` with `bytes` more to come from copies
__device__ __forceinline__ void bar_expect(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(local(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool bar_try(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(local(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait for the phase of `bar` with this parity; false when it did
// not complete within the wait bound (wait_bounded)
__device__ __forceinline__ bool bar_wait(unsigned long long* bar, unsigned parity) {
  return wait_bounded([&] { return bar_try(bar, parity); });
}
// bulk copy of `bytes` from this CTA's shared memory into another CTA's of the
// cluster, counted in bytes on the receiver's mbarrier (no multicast); both
// addresses 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void copy_to(unsigned dst, unsigned src, unsigned bytes, unsigned remote_bar) {
  asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   dst),
               "r"(src), "r"(bytes), "r"(remote_bar)
               : "memory");
}
// this thread's shared-memory writes visible to the bulk copies it issues next
__device__ __forceinline__ void fence_to_copies() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// Bounded wait until a counter of this CTA (written by a neighbour with
// store_relaxed) reaches v; false when it did not within the wait bound.
__device__ __forceinline__ bool wait_for(const int* counter, int v) {
  return wait_bounded([&] { return load_relaxed(counter) >= v; });
}
// L2 prefetch of [p, p + bytes) widened to 16-byte boundaries; the caller
// keeps the widened range inside one allocation
__device__ __forceinline__ void prefetch_span(const void* p, long bytes) {
  if (bytes <= 0) return;
  const unsigned long long a = (unsigned long long)p & ~15ull;
  const unsigned long long e = ((unsigned long long)p + (unsigned long long)bytes + 15ull) & ~15ull;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((unsigned)(e - a)) : "memory");
}

// The k-slab of one CTA of a slab sweep and its links to the neighbouring
// slabs.  The block's k-offsets 0..nz1-1 split into ce = min(cluster size,
// nz1) slabs, slab r = [r*nz1/ce, (r+1)*nz1/ce); CTAs ce.. of the cluster
// idle.  Steps gs = 0..H-1 are the forward pass over planes h = gs, steps
// H..2H-1 the backward pass over h = 2H-1-gs.  A node's k-1 (forward) or k+1
// (backward) neighbour may lie in the slab below or above: the "upstream"
// slab of the pass (below forward, above backward) delivers those values,
// and this CTA delivers its own edge values to the "downstream" slab.
struct Geom {
  const int* segt;
  int SW, nz1, nab, H, ce, me, c0, c1;
  __device__ Geom(const BlockView& B, int ncta, int rank) {
    segt = B.seg;
    nz1 = B.b1.nz();
    SW = nz1 + 2;
    nab = B.b1.nx() + B.b1.ny() - 2;
    H = B.nplanes;
    ce = min(ncta, nz1);
    me = rank;
    c0 = c0_of(me);
    c1 = c0_of(me + 1);
  }
  __device__ bool active() const { return me < ce; }
  __device__ int c0_of(int r) const { return r * nz1 / ce; }
  // nodes of plane h with k-offset below c (c = -1 .. nz1)
  __device__ int seg(int h, int c) const { return segt[h * SW + c + 1]; }
  __device__ int plane(int gs) const { return gs < H ? gs : 2 * H - 1 - gs; }
  __device__ bool has_lo() const { return me > 0 && me < ce; }
  __device__ bool has_hi() const { return me + 1 < ce; }
  // plane h holds nodes of k-offset c
  __device__ bool holds(int h, int c) const { return h - c >= 0 && h - c <= nab; }
  // step gs reads values of the upstream slab (the k-1 / k+1 neighbours of
  // this slab's first / last k-segment)
  __device__ bool need_up(int gs) const {
    const int h = plane(gs);
    return gs < H ? (has_lo() && h >= 1 && holds(h, c0)) : (has_hi() && h + 1 < H && holds(h, c1 - 1));
  }
  // step gs delivers values to the downstream slab; the same condition as
  // the downstream CTA's need_up at step gs + 1
  __device__ bool need_dn(int gs) const {
    const int h = plane(gs);
    return gs < H ? (has_hi() && h + 1 < H && holds(h, c1 - 1)) : (has_lo() && h >= 1 && holds(h, c0));
  }
  // this slab's edge k-segment the downstream slab reads at step gs
  __device__ int c_dn(int gs) const { return gs < H ? c1 - 1 : c0; }
  // the upstream slab's edge k-segment, whose values of step gs-1 step gs reads
  __device__ int c_up(int gs) const { return gs < H ? c0 - 1 : c1; }
  // the downstream CTA's rank at step gs
  __device__ int rank_dn(int gs) const { return gs < H ? me + 1 : me - 1; }
};

// End of a slab sweep for every CTA of the cluster: the CTAs exchange their
// failure flags (s_fail, shared); if any CTA failed, each idles for a bounded
// time after the last cluster barrier, so that copies issued before that
// barrier land before any CTA leaves, and a CTA that failed raises
// ST_TIMEOUT for its block.
__device__ __forceinline__ void finish(const int& s_fail, int ncta, unsigned* status, const BlockView& B) {
  __syncthreads();
  sync();
  unsigned any = s_fail ? 1u : 0u;
  if ((int)threadIdx.x < ncta && threadIdx.x != rank()) {
    unsigned v;
    asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(map(local(&s_fail), threadIdx.x)) : "memory");
    any |= v != 0u ? 1u : 0u;
  }
  any = __syncthreads_or(any);
  sync();
  if (any) {
    if (threadIdx.x == 0) {
      for (int x = 0; x < 2000; ++x) __nanosleep(1000);
      if (s_fail) {
        if (status) atomicOr(status, (unsigned)ST_TIMEOUT);
        B.raise(ST_TIMEOUT);
      }
    }
    __syncthreads();
  }
}
}  // namespace slab
#endif

}  // namespace aero
