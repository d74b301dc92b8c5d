// Kernel declarations and the device tables built by the host runtime.
#pragma once
#include "aero_device.cuh"

namespace aero {

// Physical boundary operation on one subface; types resolved on the host from
// blk_t and the solver (sub_bc.f90:39-60).
enum BcType { BCT_INFLOW = 0, BCT_OUTFLOW, BCT_MIRROR, BCT_NOSLIP, BCT_FARFIELD };
struct BcOp {
  int type;
  int face;
  Box sb;  // subface box exactly as the BC routine receives it
};
// One op of a physical-BC launch: the op and its block.
struct BcEntry {
  int op, blk;
};

// One ghost node of the halo and the interior node it copies.
struct HaloEntry {
  int dst_blk, src_blk;
  long dst_n, src_n;
};
enum HaloMode { HALO_Q = 0, HALO_Q_NUT = 1, HALO_COORD = 2 };

// average1 source (the neighbour's interface node) and average2 destination
// (own interface node with its contributions buf[first .. first+count)).
struct AvgSrc {
  int blk;
  long n;
};
struct AvgDst {
  int blk;
  int first, count;
  long n;
};

// One wall subface (blk_t = -20) of clcd_output: quads (t1, t2) with t1 in
// [lo1, lo1+n1) along the inner tangential direction, t2 in [lo2, lo2+n2)
// along the outer one; w0 the wall layer; qoff the first quad's global index.
struct WallFace {
  int block, face;
  int lo1, n1, lo2, n2, w0;
  long qoff;
};

// One wall subface of surface_output: its node box and the offset of its
// first node in the output.
struct SurfZone {
  int block, face;
  int is, js, ks, nx, ny, nz;
  long off;
};

__global__ void k_surface_cp(const BlockView* __restrict__ blocks, const SurfZone* __restrict__ zones, int nzone,
                             long nnode, CaseConsts cc_launch, double* __restrict__ out);
__global__ void k_getpri(const BlockView* __restrict__ blocks, CaseConsts cc, unsigned* status);
__global__ void k_forces(const BlockView* __restrict__ blocks, const WallFace* __restrict__ walls, int nwall,
                         long nquad, CaseConsts cc, double* __restrict__ part);
__global__ void k_residual_final_blocks(const BlockView* __restrict__ blocks, const double* __restrict__ part,
                                        int ctas, double* __restrict__ out7, unsigned* status);
__global__ void k_crank_rhs(const BlockView* __restrict__ blocks);
__global__ void k_crank_sweep(const BlockView* __restrict__ blocks, int d, double gamma);
__global__ void k_crank_update(const BlockView* __restrict__ blocks);
__global__ void k_update_q0(const BlockView* __restrict__ blocks);
__global__ void k_forces_final(const double* __restrict__ part, int npart, CaseConsts cc, double sref,
                               double* __restrict__ out8);
__global__ void k_fill(const BlockView* __restrict__ blocks, int fid, int nc, double val);
// inviscid flux, FP64 and mixed, for CTA tiles of 32, 64 and 128 nodes (x 3 directions)
__global__ void k_inviscid_32(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_64(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_128(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_mixed_32(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_mixed_64(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_mixed_128(const BlockView* __restrict__ blocks, CaseConsts cc);
// face-based variant: face fluxes into FVH planes, then the node combine
__global__ void k_inviscid_faces(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_faces_o6(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_faces_o8(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_faces_staged(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_faces_mixed_o10(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_faces_mixed(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_inviscid_combine(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_faces_sw_weno5(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_faces_wcns5(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_faces_sw_weno5_mixed(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_faces_wcns5_mixed(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_viscous_a(const BlockView* __restrict__ blocks, CaseConsts cc, int store_dudx_tao);
__global__ void k_viscous_a_bound(const BlockView* __restrict__ blocks, CaseConsts cc, int store_dudx_tao);
__global__ void k_viscous_a_mixed(const BlockView* __restrict__ blocks, CaseConsts cc, int store_dudx_tao);
__global__ void k_viscous_b(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_find_dt(const BlockView* __restrict__ blocks, CaseConsts cc, double* cta_max);
__global__ void k_dt_minmax(const BlockView* __restrict__ blocks, int m, const double* cta_max,
                            int ncta, int cta_size, double* out2);
__global__ void k_weno3_states(const BlockView* __restrict__ blocks, int coord, int direction, Box r0);
__global__ void k_roe_states(const BlockView* __restrict__ blocks, int coord, Box r0, double gamma);
__global__ void k_retire(const unsigned* __restrict__ bstat, int* __restrict__ live, int nb);
__global__ void k_lusgs_radii(const BlockView* __restrict__ blocks);
__global__ void k_lusgs_prep(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_lusgs_sca(const BlockView* __restrict__ blocks);
__global__ void k_lusgs_sca_f32(const BlockView* __restrict__ blocks);
__global__ void k_plane_index(const BlockView* __restrict__ blocks);
__global__ void k_lusgs_mats(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_lusgs_mats_f32(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_sa_length(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_sa_a(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_sa_b(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_sa_b_mixed(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_sa_recs(const BlockView* __restrict__ blocks, CaseConsts cc);
__global__ void k_sa_sweep(const BlockView* __restrict__ blocks);
__global__ void k_sa_sweep_768(const BlockView* __restrict__ blocks);
__global__ void k_sa_sweep_slab(const BlockView* __restrict__ blocks, unsigned* status, int So, int L, int D);
__global__ void k_lusgs_sweep_staged(const BlockView* __restrict__ blocks, int nst, unsigned* status,
                                     long spin_limit, int stall_plane);
__global__ void k_lusgs_sweep_global(const BlockView* __restrict__ blocks, int nst, unsigned* status);
__global__ void k_lusgs_sweep_cluster(const BlockView* __restrict__ blocks);
// the same with the off-diagonal blocks stored in FP32 (mixed precision)
__global__ void k_lusgs_sweep_staged_f32(const BlockView* __restrict__ blocks, int nst, unsigned* status,
                                         long spin_limit, int stall_plane);
__global__ void k_lusgs_sweep_global_f32(const BlockView* __restrict__ blocks, int nst, unsigned* status);
__global__ void k_lusgs_sweep_cluster_f32(const BlockView* __restrict__ blocks);
// cluster sweeps exchanging plane values by bulk copies between shared memories
__global__ void k_lusgs_sweep_bulk(const BlockView* __restrict__ blocks, unsigned* status, int pf);
__global__ void k_lusgs_sweep_bulk_f32(const BlockView* __restrict__ blocks, unsigned* status, int pf);
// the same for CTAs of at most 384 threads, two resident per SM
__global__ void k_lusgs_sweep_bulk_o2(const BlockView* __restrict__ blocks, unsigned* status, int pf);
__global__ void k_lusgs_sweep_bulk_o2_f32(const BlockView* __restrict__ blocks, unsigned* status, int pf);
// the same for CTAs of at most 256 threads, records loaded two planes ahead
__global__ void k_lusgs_sweep_bulk2(const BlockView* __restrict__ blocks, unsigned* status, int pf);
__global__ void k_lusgs_sweep_bulk2_f32(const BlockView* __restrict__ blocks, unsigned* status, int pf);
// cluster sweeps pipelined by k-slabs (D slots: rings of 5 x So values, edge
// inboxes and staging areas of 5 x L values)
__global__ void k_lusgs_sweep_slab(const BlockView* __restrict__ blocks, unsigned* status, int So, int L, int D);
__global__ void k_lusgs_sweep_slab_f32(const BlockView* __restrict__ blocks, unsigned* status, int So, int L, int D);
// the same for slab planes of at most 256 rows, record loads two steps ahead
__global__ void k_lusgs_sweep_slab2(const BlockView* __restrict__ blocks, unsigned* status, int So, int L, int D);
__global__ void k_lusgs_sweep_slab2_f32(const BlockView* __restrict__ blocks, unsigned* status, int So, int L, int D);
__global__ void k_lusgs_update(const BlockView* __restrict__ blocks);
__global__ void k_physical_bc(const BlockView* __restrict__ blocks, const BcOp* __restrict__ ops,
                              const BcEntry* __restrict__ list, int first, CaseConsts cc);
__global__ void k_sa_clip(const BlockView* __restrict__ blocks);
__global__ void k_halo(const BlockView* __restrict__ blocks, const HaloEntry* __restrict__ map,
                       long nmap, int mode);
__global__ void k_avg_gather(const BlockView* __restrict__ blocks, const AvgSrc* __restrict__ src,
                             long nsrc, double* __restrict__ buf, int with_nut);
__global__ void k_avg_apply(const BlockView* __restrict__ blocks, const AvgDst* __restrict__ dst,
                            long ndst, const double* __restrict__ buf, int with_nut);
__global__ void k_residual_partial(const BlockView* __restrict__ blocks, double* __restrict__ part,
                                   int with_sa);
__global__ void k_residual_final(const double* __restrict__ part, long npart, double totalnodes,
                                 double* __restrict__ out7, unsigned* status);
// Host (Fortran column-major, component fastest) <-> device (component planes).
__global__ void k_aos_to_soa(const double* __restrict__ src, double* __restrict__ dst, long n,
                             int nc, long plane);
__global__ void k_soa_to_aos(const double* __restrict__ src, double* __restrict__ dst, long n,
                             int nc, long plane);
__global__ void k_fill_plane(double* __restrict__ p, long n, double val);
// one-time geometry
__global__ void k_metric_pass1(const BlockView* __restrict__ blocks);
__global__ void k_metric_pass2(const BlockView* __restrict__ blocks);
__global__ void k_spacing(const BlockView* __restrict__ blocks);
__global__ void k_wall_points(const BlockView* __restrict__ blocks, const AvgSrc* __restrict__ wall,
                              long nwall, double* __restrict__ xyz);
__global__ void k_walldist(const BlockView* __restrict__ blocks, const double* __restrict__ xyz,
                           const long* __restrict__ range);

}  // namespace aero
