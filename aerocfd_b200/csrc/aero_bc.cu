// Physical boundary conditions (sub_bc.f90 and the five sub_bc_-*.f90
// routines), the block-interface halo of q/nut and of the coordinates
// (sub_bc_updatebuffer.f90, sub_bc_updatebuffercoordinate.f90), the interface
// averaging (sub_bc_updatebufferaverage.f90) and the residual norm
// (sub_output_residual.f90).
//
// The reference's MPI pack / isend / irecv / unpack becomes a gather through
// index maps built once on the host (aero_topology.cpp): all blocks of a case
// live in this GPU's memory, so every interface is the reference's same-rank
// branch, done by one kernel for all interfaces of all blocks.
#include <cmath>

#include "aero_device.cuh"
#include "aero_kernels.h"

namespace aero {

// Face node `t` of a BC op: the boundary plane index along the face normal and
// the two tangential indices, plus the unit step toward the interior.
__device__ __forceinline__ bool bc_node(const BcOp& op, long t, int& i, int& j, int& k, int& di,
                                        int& dj, int& dk, int& s) {
  const Box& sb = op.sb;
  int dir = (op.face - 1) / 2;
  s = (op.face % 2 == 1) ? 1 : -1;
  di = dj = dk = 0;
  if (dir == 0) {
    long n1 = sb.ny(), n2 = sb.nz();
    if (t >= n1 * n2) return false;
    i = s > 0 ? sb.is : sb.ie; j = sb.js + (int)(t % n1); k = sb.ks + (int)(t / n1); di = 1;
  } else if (dir == 1) {
    long n1 = sb.nx(), n2 = sb.nz();
    if (t >= n1 * n2) return false;
    j = s > 0 ? sb.js : sb.je; i = sb.is + (int)(t % n1); k = sb.ks + (int)(t / n1); dj = 1;
  } else {
    long n1 = sb.nx(), n2 = sb.ny();
    if (t >= n1 * n2) return false;
    k = s > 0 ? sb.ks : sb.ke; i = sb.is + (int)(t % n1); j = sb.js + (int)(t / n1); dk = 1;
  }
  return true;
}

__device__ __forceinline__ void unit_normal(const BlockView& B, long n, int dir, int s, double& x0,
                                            double& y0, double& z0) {
  int c0 = 3 * dir + 1;
  x0 = B.v(F_DXIDX, c0, n); y0 = B.v(F_DXIDX, c0 + 1, n); z0 = B.v(F_DXIDX, c0 + 2, n);
  double temp = p2(x0) + p2(y0) + p2(z0);
  temp = sqrt(temp);
  if (s > 0) {
    x0 = -x0 / temp; y0 = -y0 / temp; z0 = -z0 / temp;
  } else {
    x0 = x0 / temp; y0 = y0 / temp; z0 = z0 / temp;
  }
}

// sub_bc.f90:26-62 for the ops of one dependency level (grid y: the level's
// entries), launched level after level: an op that must see what another op
// of its block wrote, or must overwrite it, sits in a later level, as the
// serial reference orders them.  The nodes of one subface are independent
// and spread over the grid's x.
__global__ void k_physical_bc(const BlockView* __restrict__ blocks, const BcOp* __restrict__ ops,
                              const BcEntry* __restrict__ list, int first, CaseConsts cc_launch) {
  const BcEntry e = list[first + blockIdx.y];
  const BlockView& B = blocks[e.blk];
  if (B.retired()) return;
  const CaseConsts& cc = B.ccb ? *B.ccb : cc_launch;
  const BcOp op = ops[e.op];
  bool tur = cc.turbulence >= 1;
  double gamma = cc.gamma;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, k, di, dj, dk, s;
  if (!bc_node(op, t, i, j, k, di, dj, dk, s)) return;
  long n = B.at(i, j, k);
  long st = di ? 1 : (dj ? (long)B.nx : (long)B.nx * B.ny);
  long n1 = n + s * st;
  int dir = di ? 0 : (dj ? 1 : 2);
  if (op.type == BCT_INFLOW) {  // sub_bc_-50_inflow.f90:21-40
    B.v(F_Q, 1, n) = cc.d_0;
    B.v(F_Q, 2, n) = cc.d_0 * cc.u_0 * cc.cos_aoa;
    B.v(F_Q, 3, n) = cc.d_0 * cc.u_0 * cc.sin_aoa;
    B.v(F_Q, 4, n) = 0.0;
    B.v(F_Q, 5, n) = cc.p_0 / (gamma - 1.0) + 0.5 * p2(cc.u_0);
    if (tur) B.s(F_NUT, n) = cc.nutinf;
  } else if (op.type == BCT_OUTFLOW) {  // sub_bc_-40_outflow.f90:21-35
    for (int c = 1; c <= 5; ++c) B.v(F_Q, c, n) = B.v(F_Q, c, n1);
    if (tur) B.s(F_NUT, n) = B.s(F_NUT, n1);
  } else if (op.type == BCT_MIRROR) {  // symmetry plane or slip wall
    double x0, y0, z0;
    unit_normal(B, n, dir, s, x0, y0, z0);
    double cu = B.v(F_Q, 2, n1) * x0 + B.v(F_Q, 3, n1) * y0 + B.v(F_Q, 4, n1) * z0;
    B.v(F_Q, 1, n) = B.v(F_Q, 1, n1);
    B.v(F_Q, 2, n) = B.v(F_Q, 2, n1) - cu * x0;
    B.v(F_Q, 3, n) = B.v(F_Q, 3, n1) - cu * y0;
    B.v(F_Q, 4, n) = B.v(F_Q, 4, n1) - cu * z0;
    B.v(F_Q, 5, n) = B.v(F_Q, 5, n1);
    if (tur) B.s(F_NUT, n) = B.s(F_NUT, n1);
  } else if (op.type == BCT_NOSLIP) {  // no-slip (sub_bc_-20_solidwall.f90:225-240)
    long n2 = n + 2 * s * st, n3 = n + 3 * s * st;
    B.v(F_Q, 1, n) = (11.0 * B.v(F_Q, 1, n1) - 7.0 * B.v(F_Q, 1, n2) + 2.0 * B.v(F_Q, 1, n3)) / 6.0;
    B.v(F_Q, 2, n) = 0.0;
    B.v(F_Q, 3, n) = 0.0;
    B.v(F_Q, 4, n) = 0.0;
    B.v(F_Q, 5, n) = (11.0 * B.v(F_Q, 5, n1) - 7.0 * B.v(F_Q, 5, n2) + 2.0 * B.v(F_Q, 5, n3)) / 6.0;
    if (tur) B.s(F_NUT, n) = 0.0;
  } else if (op.type == BCT_FARFIELD) {  // sub_bc_-10_farfield.f90:30-106
    double u_inf = cc.u_0 * cc.cos_aoa, v_inf = cc.u_0 * cc.sin_aoa, w_inf = 0.0;
    double s_inf = cc.p_0 / crm::pow(cc.d_0, gamma);
    double c_inf = cc.c_0;
    double x0, y0, z0;
    unit_normal(B, n, dir, s, x0, y0, z0);
    double d_p = B.v(F_Q, 1, n1);
    double u_p = B.v(F_Q, 2, n1) / d_p;
    double v_p = B.v(F_Q, 3, n1) / d_p;
    double w_p = B.v(F_Q, 4, n1) / d_p;
    double p_p = (B.v(F_Q, 5, n1) - 0.5 * d_p * (p2(u_p) + p2(v_p) + p2(w_p))) * (gamma - 1.0);
    double c_p = sqrt(gamma * p_p / d_p);
    double s_p = p_p / crm::pow(d_p, gamma);
    double vn_inf = u_inf * x0 + v_inf * y0 + w_inf * z0;
    double vn_p = u_p * x0 + v_p * y0 + w_p * z0;
    double rm = vn_inf - 2.0 * c_inf / (gamma - 1.0);
    double rp = vn_p + 2.0 * c_p / (gamma - 1.0);
    double vn_b = 0.5 * (rp + rm);
    double s_b = 0, u_ref = 0, v_ref = 0, w_ref = 0, turVal = 0;
    if (vn_b < 0.0) { s_b = s_inf; u_ref = u_inf; v_ref = v_inf; w_ref = w_inf; turVal = cc.nutinf; }
    if (vn_b >= 0.0) { s_b = s_p; u_ref = u_p; v_ref = v_p; w_ref = w_p; turVal = tur ? B.s(F_NUT, n1) : 0.0; }
    double u_ref_t = u_ref * x0 + v_ref * y0 + w_ref * z0;
    double u_b = u_ref + (vn_b - u_ref_t) * x0;
    double v_b = v_ref + (vn_b - u_ref_t) * y0;
    double w_b = w_ref + (vn_b - u_ref_t) * z0;
    double d_b = crm::pow(c_p * c_p / (gamma * s_b), 1.0 / (gamma - 1.0));
    double p_b = s_b * crm::pow(d_b, gamma);
    B.v(F_Q, 1, n) = d_b;
    B.v(F_Q, 2, n) = d_b * u_b;
    B.v(F_Q, 3, n) = d_b * v_b;
    B.v(F_Q, 4, n) = d_b * w_b;
    B.v(F_Q, 5, n) = p_b / (gamma - 1.0) + 0.5 * d_b * (p2(u_b) + p2(v_b) + p2(w_b));
    if (tur) B.s(F_NUT, n) = turVal;
  }
}

// sub_bc.f90:65-87: SA clip and eddy viscosity over the full box.  The lower
// clip is overwritten by the upper clip of the unclipped value, as in :80-81.
__global__ void k_sa_clip(const BlockView* __restrict__ blocks) {
  const BlockView& B = blocks[blockIdx.y];
  if (B.retired()) return;
  long n = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= B.b.size()) return;
  double d = B.v(F_PRI, 1, n);
  double nut = B.s(F_NUT, n);
  double leix = nut / B.v(F_AMU, 1, n) * d;
  leix = fmax(leix, 0.001);
  double fv1 = p3(leix) / (p3(leix) + SA_CV13);
  double nn = fmin(nut, 1.0e6);
  B.s(F_NUT, n) = nn;
  B.v(F_AMU, 2, n) = nn * fv1 * d;
}

// UpdateBuffer / UpdateBufferCoordinate: every ghost node copies its donor
// interior node (the map resolves orientation and repeated writes).
__global__ void k_halo(const BlockView* __restrict__ blocks, const HaloEntry* __restrict__ map,
                       long nmap, int mode) {
  long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nmap) return;
  HaloEntry h = map[e];
  const BlockView& D = blocks[h.dst_blk];
  const BlockView& S = blocks[h.src_blk];
  if (mode == HALO_COORD) {
    D.s(F_X, h.dst_n) = S.s(F_X, h.src_n);
    D.s(F_Y, h.dst_n) = S.s(F_Y, h.src_n);
    D.s(F_Z, h.dst_n) = S.s(F_Z, h.src_n);
  } else {
#pragma unroll
    for (int c = 1; c <= 5; ++c) D.v(F_Q, c, h.dst_n) = S.v(F_Q, c, h.src_n);
    if (mode == HALO_Q_NUT) D.s(F_NUT, h.dst_n) = S.s(F_NUT, h.src_n);
  }
}

// average1: the neighbour's copy of every shared interface node, gathered
// before any averaging (buf: 6 values per contribution).
__global__ void k_avg_gather(const BlockView* __restrict__ blocks, const AvgSrc* __restrict__ src,
                             long nsrc, double* __restrict__ buf, int with_nut) {
  long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nsrc) return;
  AvgSrc a = src[e];
  const BlockView& S = blocks[a.blk];
#pragma unroll
  for (int c = 1; c <= 5; ++c) buf[6 * e + c - 1] = S.v(F_Q, c, a.n);
  buf[6 * e + 5] = with_nut ? S.s(F_NUT, a.n) : 0.0;
}

// average2: q = (q + q_neighbour)*0.5, applied once per subface that holds the
// node, in the reference's block/subface order.
__global__ void k_avg_apply(const BlockView* __restrict__ blocks, const AvgDst* __restrict__ dst,
                            long ndst, const double* __restrict__ buf, int with_nut) {
  long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= ndst) return;
  AvgDst a = dst[e];
  const BlockView& D = blocks[a.blk];
  double q[6];
#pragma unroll
  for (int c = 1; c <= 5; ++c) q[c - 1] = D.v(F_Q, c, a.n);
  q[5] = with_nut ? D.s(F_NUT, a.n) : 0.0;
  for (int x = a.first; x < a.first + a.count; ++x) {
#pragma unroll
    for (int c = 0; c < 5; ++c) q[c] = (q[c] + buf[6 * x + c]) * 0.5;
    if (with_nut) q[5] = (q[5] + buf[6 * x + 5]) * 0.5;
  }
#pragma unroll
  for (int c = 1; c <= 5; ++c) D.v(F_Q, c, a.n) = q[c - 1];
  if (with_nut) D.s(F_NUT, a.n) = q[5];
}

// Retirement (aero_set_retirement): a block whose status word holds any bit
// stops advancing; its live flag is set once per step, before any kernel of
// the step reads it.
__global__ void k_retire(const unsigned* __restrict__ bstat, int* __restrict__ live, int nb) {
  int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < nb) live[m] = bstat[m] == 0u ? 1 : 0;
}

// Residual norm, pass 1: per-CTA partial sums of (rhs*dt/inv_j)^2 (5 values)
// and (sa_rhs*dt)^2 over the updated nodes (sub_output_residual.f90:32-44).
__global__ void k_residual_partial(const BlockView* __restrict__ blocks, double* __restrict__ part,
                                   int with_sa) {
  const BlockView& B = blocks[blockIdx.y];
  const Box& b1 = B.b1;
  long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  // a retired block contributes zeros (its partial slots are still written)
  if (t < b1.size() && !B.retired()) {
    int i = b1.is + (int)(t % b1.nx());
    long r = t / b1.nx();
    int j = b1.js + (int)(r % b1.ny());
    int k = b1.ks + (int)(r / b1.ny());
    long n = B.at(i, j, k);
    double dt = B.s(F_DT, n), ij = B.s(F_INVJ, n);
#pragma unroll
    for (int c = 0; c < 5; ++c) v[c] = p2(B.v(F_RHS, c + 1, n) * dt / ij);
    if (with_sa) v[5] = p2(B.s(F_SARHS, n) * dt);
  }
  __shared__ double sm[6][32];
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    double x = v[c];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sm[c][threadIdx.x >> 5] = x;
  }
  __syncthreads();
  if (threadIdx.x < 32) {
    int nw = blockDim.x >> 5;
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      double x = threadIdx.x < nw ? sm[c][threadIdx.x] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      if (threadIdx.x == 0) {
        part[6 * ((long)blockIdx.y * gridDim.x + blockIdx.x) + c] = x;
        if (!isfinite(x)) B.raise(ST_NONFINITE_RESIDUAL);  // this block's own bit
      }
    }
  }
}

// Residual norm, pass 2: one CTA adds the partials in a fixed order and forms
// sqrt(sum/totalnodes) (sub_output_residual.f90:55-56).
__global__ void k_residual_final(const double* __restrict__ part, long npart, double totalnodes,
                                 double* __restrict__ out7, unsigned* status) {
  __shared__ double sm[6][256];
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (long p = threadIdx.x; p < npart; p += blockDim.x)
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
    bool bad = false;
    for (int c = 0; c < 6; ++c) {
      out7[c] = sqrt(sm[c][0] / totalnodes);
      if (!isfinite(out7[c])) bad = true;
    }
    out7[6] = 0.0;
    if (bad && status) atomicOr(status, (unsigned)ST_NONFINITE_RESIDUAL);
  }
}

// The norms of each block on its own (the residual a one-block case prints):
// CTA m adds block m's partials in a fixed order and divides by that block's
// physical node count.  out7 holds 7 values per block.
__global__ void k_residual_final_blocks(const BlockView* __restrict__ blocks, const double* __restrict__ part,
                                        int ctas, double* __restrict__ out7, unsigned* status) {
  __shared__ double sm[6][256];
  const int m = blockIdx.x;
  double v[6] = {0, 0, 0, 0, 0, 0};
  for (int p = threadIdx.x; p < ctas; p += blockDim.x)
#pragma unroll
    for (int c = 0; c < 6; ++c) v[c] += part[6 * ((long)m * ctas + p) + c];
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
    double nodes = (double)blocks[m].b0.size();
    bool bad = false;
    for (int c = 0; c < 6; ++c) {
      out7[7 * m + c] = sqrt(sm[c][0] / nodes);
      if (!isfinite(out7[7 * m + c])) bad = true;
    }
    out7[7 * m + 6] = 0.0;
    if (bad && status) atomicOr(status, (unsigned)ST_NONFINITE_RESIDUAL);
  }
}

}  // namespace aero
