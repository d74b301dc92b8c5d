/*
 * aerocfd_gpu.h - C ABI of the B200 (sm_100a) residual-and-update path of the
 * aerocfd multi-block structured compressible-flow solver.
 *
 * The reference's hot-path routines are external Fortran subroutines with
 * implicit interfaces: every argument by reference, arrays explicit-shape and
 * column-major with caller-supplied bounds, e.g. q(5,is:ie,js:je,ks:ke).  The
 * drop-in entry points below take exactly those arguments, in the same order
 * and with the same meaning, so a Fortran `interface ... bind(C)` block can
 * route the existing call sites of main.f90:357-447 here unchanged
 * (fortran/aerocfd_gpu.f90).  The Fortran routines return nothing and print or
 * stop on errors; these return a status (0 = AERO_OK) that the Fortran shim
 * turns into the reference's print + stop.
 *
 * Two modes:
 *  - transient: called with arrays that were never registered, an entry point
 *    copies its inputs to the GPU, runs, and copies its outputs back;
 *  - resident: after aero_register_block/aero_bind_field/aero_finish_setup and
 *    aero_sync_to_device, calls whose array arguments are registered host
 *    arrays run purely on the device copies; host arrays are refreshed only by
 *    aero_sync_to_host.  The no-argument routines (physical_bc, halo, average,
 *    residual) work on the registered blocks, the way the reference works on
 *    its module state.
 *
 * One host thread drives the library; calls run in order on the library's
 * CUDA stream.  3-D cases (iflag_dimension = 3) and 2-D cases
 * (iflag_dimension = 2: every block the single plane k = 1, faces 1-4 only,
 * interface orientation codes 2 and 3 as UpdateBuffer2d reads them) are
 * supported, with the steady 1st-order implicit (LU-SGS) or the unsteady
 * 2nd-order Crank-Nicolson time advance; other flags are rejected.  Transient
 * calls take boxes of one k-plane in a 2-D configuration and of at least three
 * in a 3-D one.
 */
#ifndef AEROCFD_GPU_H
#define AEROCFD_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define AERO_OK 0
#define AERO_ERR_ARG 1      /* bad argument: size, field id, unsupported flag   */
#define AERO_ERR_STATE 2    /* call out of order (no aero_init / no setup)      */
#define AERO_ERR_CUDA 3     /* CUDA runtime error (text in aero_last_error)     */
#define AERO_ERR_NOMEM 4    /* device allocation failed                         */
#define AERO_ERR_DEVICE 5   /* device status word set (see aero_get_status)     */

/* device status word bits (aero_get_status) */
#define AERO_ST_NEG_DENSITY 1u        /* sub_getpri_v.f90:54-56 would print  */
#define AERO_ST_NONFINITE_RESIDUAL 2u /* NaN/Inf in the residual norm        */
#define AERO_ST_TIMEOUT 8u            /* an LU-SGS sweep wait ran out of polls
                                         (that iteration's update is incomplete) */

/* ---- field ids (module_block.f90:20-91 arrays) ------------------------- */
enum {
  AERO_F_Q = 0,     /* q(5,...)       conservative variables                */
  AERO_F_PRI_V,     /* pri_v(7,...)   d,u,v,w,p,t,c                        */
  AERO_F_RHSI,      /* rhsi(5,...)                                          */
  AERO_F_RHSV,      /* rhsv(5,...)                                          */
  AERO_F_RHS,       /* rhs(5,...)                                           */
  AERO_F_DT,        /* dt(...)                                              */
  AERO_F_DXIDX,     /* dxidx(9,...)   metric terms                          */
  AERO_F_INV_J,     /* inv_j(...)     1/J                                   */
  AERO_F_AMU,       /* amu(3,...)     laminar, eddy, total viscosity        */
  AERO_F_NUT,       /* nut(...)       SA working variable                   */
  AERO_F_SA_RHS,    /* sa_rhs(...)                                          */
  AERO_F_X, AERO_F_Y, AERO_F_Z,
  AERO_F_DIST,      /* dist(...)      wall distance                         */
  AERO_F_ALPHA, AERO_F_BETA, AERO_F_GGAMMA, /* aalpha/bbeta/ggamma(3,...)   */
  AERO_F_DUDX,      /* dudx(9,...)                                          */
  AERO_F_TAO,       /* tao(6,...)                                           */
  AERO_F_VOR,       /* vor(...)                                             */
  AERO_F_LENGTH,    /* length(...)    SA length scale                       */
  AERO_F_SPACING,   /* spacing(...)                                         */
  AERO_F_Q0,        /* q0(-1:0,5,...) the two earlier time levels (Crank-Nicolson) */
  AERO_NUM_FIELDS
};
#define AERO_MASK(f) (1ull << (f))
#define AERO_MASK_ALL ((1ull << AERO_NUM_FIELDS) - 1ull)

/* ---- runtime ----------------------------------------------------------- */
int aero_init(int device);
/* Releases everything; the execution options (aero_set_precision,
 * aero_use_graphs, launch shapes) return to their defaults. */
int aero_finalize(void);
/* Text of the last error (valid until the next call). */
const char* aero_last_error(void);
/* OR of the device status bits raised since the last call; clears them. */
int aero_get_status(unsigned* status);
/* Where the first cluster-sweep wait that gave up (AERO_ST_TIMEOUT) was, since
 * the last call: out5 = sweep (1: mean-flow bulk exchange, 2: mean-flow slab,
 * 3: SA slab, 4: the one-CTA staged sweep, whose waits have the poll budget
 * of aero_set_poll_budget), block (0-based), the CTA's rank in its cluster, the step
 * (plane step of the forward then backward pass) and the wait (1: a plane's
 * values, 2: the downstream slab's progress, 3: the last plane's values);
 * all -1 when none gave up.  Clears the record.  The cluster sweeps bound
 * every wait by one second of the GPU's global timer. */
int aero_timeout_site(int* out5);

/* Per-block status and retirement (batches of independent cases, where a
 * case is one block; no counterpart in the reference, which stops the run).
 * Every registered block has its own status word, raised with the same
 * AERO_ST_* bits as the global one by that block's kernels (negative density
 * in get_primitivevariables, a non-finite partial sum of its residual, a
 * sweep wait that ran out).  aero_get_block_status copies the nblocks words
 * (block m at out[m-1]) without clearing them; aero_clear_block_status clears
 * them.  With aero_set_retirement(1) every step begins by retiring each block
 * whose word is non-zero: no kernel of the step touches it, so its state stays
 * as it was after the step that raised the bit, its residual norms count as 0
 * (aero_residual, aero_residual_blocks) and the other blocks advance as if it
 * were not there (their kernels never read another block, halos aside: retire
 * a multi-block case as a whole).  Clearing a block's word brings it back at
 * the next step; aero_set_retirement(0) (the default) brings every block back. */
int aero_get_block_status(unsigned* out);
int aero_clear_block_status(void);
int aero_set_retirement(int on);

/* ---- case set-up (replaces init_readcontrolfile / init_readbcinfo /
 *      init_allocatememory module state, main.f90:80-140) ---------------- */
/* iflags[8]: iflag_dimension, iflag_solver, iflag_time, iflag_timeadvance,
 *            iflag_turbulence, iflag_des, bufferLength, iflag_inviscid
 *            (sub_init_readcontrolfile.f90:30-47, main.f90:636-653)
 * params[7]: ma, re, tinf, aoa (degrees), cfl, dt, nutinf               */
int aero_configure(const int* iflags, const double* params);
/* Arithmetic of the flux kernels (no counterpart in the reference, which is
 * FP64 throughout).  mode 0 (default): FP64 in the reference's operation order.
 * mode 1 (mixed): the WENO3 corrections, the Roe dissipation and the viscous
 * stresses and fluxes in FP32, each formed from FP64 differences around FP64
 * base states, and the off-diagonal 5x5 blocks of the LU-SGS sweeps stored in
 * FP32 (their products and sums are FP64); metrics, the grid Jacobian, rhs,
 * the implicit diagonal, dq, the time step, the viscosity and the residual
 * stay FP64.  Applies to later calls. */
int aero_set_precision(int mode);
/* Batches (no counterpart in the reference, which runs one case per job):
 * gives block m its own Control.in values (params[7] as aero_configure) so
 * that independent cases, e.g. a Mach sweep, run together as the blocks of one
 * registered set; the flags of aero_configure apply to all.  Call after
 * aero_register_block(m) and before aero_finish_setup.  aero_residual_blocks
 * then returns each block's own residual norms (7 per block, normalised by its
 * own node count). */
int aero_set_block_params(int m, const double* params);
int aero_residual_blocks(double* out7_per_block);
/* box18: is,ie,js,je,ks,ke, is0..ke0, is1..ke1 of block m (1-based)
 *        (sub_init_allocatememory.f90:73-144)
 * subfaces: num_subface rows of f_no,face,is,ie,js,je,ks,ke,blk_t,
 *           subface_t,ori (sub_init_readbcinfo.f90:96-98)               */
int aero_register_block(int m, const int* box18, int num_subface, const int* subfaces);
/* Associates host array `host` (the reference's blk(m)%<field>) with field
 * `field` of block m.  The array is page-locked for fast transfers. */
int aero_bind_field(int m, int field, double* host);
/* Allocates the device arena, builds the halo/average/BC tables. */
int aero_finish_setup(void);
/* Copies the bound host arrays of the fields in `mask` to / from the GPU. */
int aero_sync_to_device(unsigned long long mask);
int aero_sync_to_host(unsigned long long mask);

/* ---- drop-in mirrors of the hot-path routines ------------------------- */
/* sub_getpri_v.f90:19 */
int aero_get_primitivevariables(const int* mm, double* pri_v, const double* q, const double* gamma,
                                const double* cv, const int* is, const int* ie, const int* js,
                                const int* je, const int* ks, const int* ke);
/* sub_inviscid1.f90:8-11 (Roe flux on WENO3 states, all directions) */
int aero_inviscid_flux_1(double* rhsi, const double* q, const double* dxidx, const double* inv_j,
                         const int* is, const int* ie, const int* js, const int* je,
                         const int* ks, const int* ke, const int* is0, const int* ie0,
                         const int* js0, const int* je0, const int* ks0, const int* ke0,
                         const int* is1, const int* ie1, const int* js1, const int* je1,
                         const int* ks1, const int* ke1, const double* gamma);

/* thirdorder_weno(df,f,is..ke,is0..ke0,coord,direction)
 * sub_inviscid_upwind.f90:1 -- the WENO3 states of inviscid_flux_1 as a
 * routine of its own (for unit tests, as the reference's internal entry
 * point): at every face i+1/2 of is0..ke0 grown by one node down along coord,
 * df = the right state (direction 1) or the left state (direction -1; any
 * other value writes nothing, as in the reference); df keeps its values at
 * the other nodes.  Unregistered arrays only. */
int aero_thirdorder_weno(double* df, const double* f, const int* is, const int* ie, const int* js, const int* je,
                         const int* ks, const int* ke, const int* is0, const int* ie0, const int* js0,
                         const int* je0, const int* ks0, const int* ke0, const int* coord, const int* direction);
/* roe_3d(ql,qr,flux,dxidx,inv_j,gamma,is..ke,is0..ke0,coord)
 * sub_inviscid_splitting.f90:1 -- the Roe flux with Harten's fix at the same
 * faces from primitive states ql, qr (d, u, v, w, p); flux keeps its values
 * at the other nodes.  Unregistered arrays only. */
int aero_roe_3d(const double* ql, const double* qr, double* flux, const double* dxidx, const double* inv_j,
                const double* gamma, const int* is, const int* ie, const int* js, const int* je, const int* ks,
                const int* ke, const int* is0, const int* ie0, const int* js0, const int* je0, const int* ks0,
                const int* ke0, const int* coord);
/* Extension schemes with inviscid_flux_1's argument list (no counterpart in
 * the reference, which defines iflag_inviscid = 5 and 8 in module_flags.f90:68,
 * 71 but stops on them in GetBufferLength, main.f90:636-653): Steger-Warming
 * flux-vector splitting with WENO5 reconstruction, and WCNS5 interpolation with
 * the Roe flux and a 4th-order hybrid face/node difference.  Both need three
 * ghost layers at block interfaces (bufferLength = 3); near physical
 * boundaries they fall back to lower-order stencils.  aero_configure with
 * iflag_inviscid = 5 or 8 and bufferLength = 3 makes aero_step use them. */
int aero_inviscid_flux_weno5(double* rhsi, const double* q, const double* dxidx, const double* inv_j,
                             const int* is, const int* ie, const int* js, const int* je,
                             const int* ks, const int* ke, const int* is0, const int* ie0,
                             const int* js0, const int* je0, const int* ks0, const int* ke0,
                             const int* is1, const int* ie1, const int* js1, const int* je1,
                             const int* ks1, const int* ke1, const double* gamma);
int aero_inviscid_flux_wcns5(double* rhsi, const double* q, const double* dxidx, const double* inv_j,
                             const int* is, const int* ie, const int* js, const int* je,
                             const int* ks, const int* ke, const int* is0, const int* ie0,
                             const int* js0, const int* je0, const int* ks0, const int* ke0,
                             const int* is1, const int* ie1, const int* js1, const int* je1,
                             const int* ks1, const int* ke1, const double* gamma);
/* sub_viscous.f90:9-12 */
int aero_viscous_flux(double* rhsv, const double* pri_v, double* amu, double* vor, double* dudx,
                      double* tao, const double* dxidx, const double* inv_j, const double* tinf,
                      const double* prl, const double* prt, const double* gamma, const double* cv,
                      const double* re, const int* is, const int* ie, const int* js,
                      const int* je, const int* ks, const int* ke, const int* is0,
                      const int* ie0, const int* js0, const int* je0, const int* ks0,
                      const int* ke0, const int* is1, const int* ie1, const int* js1,
                      const int* je1, const int* ks1, const int* ke1, const int* mm);
/* sub_timeadvancement_finddt.f90:24-25 (steady branch) */
int aero_find_dt(double* dt, double* dtmax, double* dtmin, double* cflmax, double* cflmin,
                 const double* pri_v, const double* amu, const double* dxidx, const double* re,
                 double* cfl, const int* is, const int* ie, const int* js, const int* je,
                 const int* ks, const int* ke, const int* iflag_time, const int* iflag_steady,
                 const int* iflag_unsteady);
/* sub_timeadvancement_1stimplicit.f90:7-11 (xx,yy,zz are debug-only, unused) */
int aero_implicit1st(double* q, const double* dt, const double* pri_v, double* rhs,
                     const double* rhsi, const double* rhsv, const double* dxidx,
                     const double* inv_j, const int* is, const int* ie, const int* js,
                     const int* je, const int* ks, const int* ke, const int* is0,
                     const int* ie0, const int* js0, const int* je0, const int* ks0,
                     const int* ke0, const int* is1, const int* ie1, const int* js1,
                     const int* je1, const int* ks1, const int* ke1, const double* gamma,
                     const double* cfl, const double* xx, const double* yy, const double* zz);

/* sub_tur_sa.f90:7-11, with the DES97 (iflag_des = 1) and DDES (2) length
 * scales of :51-97; spac is read by both, dudx by DDES (through the
 * reference's (3, ..., 3) view of the (9, ...) array). */
int aero_sa_model(double* nut, double* sa_rhs, const double* dt, const double* pri_v, const double* amu,
                  const double* dudx, const double* vor, const double* dxidx, const double* inv_j,
                  const double* alpha, const double* beta, const double* gamma, double* length,
                  const double* dist, const double* spac, const double* re, const double* cfl,
                  const int* is, const int* ie, const int* js, const int* je, const int* ks,
                  const int* ke, const int* is0, const int* ie0, const int* js0, const int* je0,
                  const int* ks0, const int* ke0, const int* is1, const int* ie1, const int* js1,
                  const int* je1, const int* ks1, const int* ke1);
/* sub_init_gridtransformation.f90:27-29 (3-D and 2-D branches): metrics,
 * 1/J, alpha/beta/gamma.
 * Ghost-corner nodes (two or more indices in overlap layers) are left as the
 * caller stored them, as in the reference. */
int aero_gridtransformation(double* dxidx, double* inv_j, double* alpha, double* beta, double* gamma,
                            const double* x, const double* y, const double* z, const int* is,
                            const int* ie, const int* js, const int* je, const int* ks,
                            const int* ke, const int* is0, const int* ie0, const int* js0,
                            const int* je0, const int* ks0, const int* ke0, const int* m0);

/* sub_timeadvancement_2ndcrank.f90:1-11 (crank2nd; 2-D: no k lines): the dual-time
 * Crank-Nicolson sub-iteration update of q (alph = 1/2) with the factorised
 * point-implicit i, j, k line recurrences; q0 is q0(-1:0,5,is:ie,js:je,ks:ke).
 * mm and ssub are accepted for the reference's argument list. */
int aero_crank2nd(double* q, const double* q0, const double* dt, const double* pri_v, double* rhs,
                  const double* rhsi, const double* rhsv, const double* dxidx, const double* inv_j,
                  const int* is, const int* ie, const int* js, const int* je, const int* ks, const int* ke,
                  const int* is0, const int* ie0, const int* js0, const int* je0, const int* ks0,
                  const int* ke0, const int* is1, const int* ie1, const int* js1, const int* je1,
                  const int* ks1, const int* ke1, const double* gamma, const int* mm, const int* ssub);
/* main.f90:692-711 (update_q0): q0(-1) = q0(0), q0(0) = q on the physical nodes */
int aero_update_q0(double* q0, const double* q, const int* is, const int* ie, const int* js, const int* je,
                   const int* ks, const int* ke, const int* is0, const int* ie0, const int* js0,
                   const int* je0, const int* ks0, const int* ke0);

/* ---- module-state routines (no arguments in the reference) ------------ */
int aero_physical_bc(void);          /* sub_bc.f90:9                        */
/* In a 2-D configuration these four are UpdateBuffer2d
 * (sub_bc_updatebuffer2d.f90:10), average2d1 / average2d2
 * (sub_bc_updatebufferaverage2d.f90:10, :317) and UpdateBufferCoordinate2d
 * (sub_bc_updatebuffercoordinate2d.f90:10). */
int aero_updatebuffer(void);         /* sub_bc_updatebuffer.f90:10          */
int aero_average1(void);             /* sub_bc_updatebufferaverage.f90:10   */
int aero_average2(void);             /* sub_bc_updatebufferaverage.f90:442  */
int aero_updatebuffercoordinate(void); /* sub_bc_updatebuffercoordinate.f90:10 */
/* The same under the reference's 2-D names, for the iflag_dimension = 2 arms
 * of main.f90:142-146, :310-318, :424-432; AERO_ERR_STATE in a 3-D case. */
int aero_updatebuffer2d(void);       /* sub_bc_updatebuffer2d.f90:10        */
int aero_average2d1(void);           /* sub_bc_updatebufferaverage2d.f90:10 */
int aero_average2d2(void);           /* sub_bc_updatebufferaverage2d.f90:317 */
int aero_updatebuffercoordinate2d(void); /* sub_bc_updatebuffercoordinate2d.f90:10 */
/* sub_output_residual.f90:8: out7 = rms of rho,rho*u,rho*v,rho*w,rho*E,
 * nut, (unused) over the updated nodes / totalnodes; the reference prints
 * these and appends them to resi_history.dat. */
int aero_residual(double* out7);
/* sub_output_forceintegration.f90:8-479 (clcd_output, 3-D quads and 2-D
 * wall edges): pressure and
 * viscous forces over every wall subface (blk_t = -20) of the registered
 * blocks from their current pri_v, dxidx, amu and x, y, z, then the lift and
 * drag coefficients.  out8 = fpx, fpy, fpz, fvx, fvy, fvz, cl, cd (what the
 * reference prints and appends to clcd_history.dat); sref is Control.in's
 * reference area.  The per-element arithmetic is the reference's; the sums
 * over elements run in a fixed parallel order. */
int aero_clcd_output(double sref, double* out8);
/* sub_output_surface.f90:8-118 (surface_output): the rows the reference writes
 * to result/surfcp_<timestep>_<rank>.dat.  aero_surface_count gives the number
 * of wall-subface nodes and of wall subfaces (zones); aero_surface_output fills
 * xyzcp (4 doubles per node: x, y, z, cp = (p - p0) / qinf, block by block,
 * subface by subface in bcinfo order, then k, j, i) and zones (5 ints per
 * zone: block (1-based), face, idim, jdim, kdim of the zone header) from the
 * device's current pri_v and coordinates. */
int aero_surface_count(long long* n_nodes, int* n_zones);
int aero_surface_output(double* xyzcp, int* zones);
/* sub_init_flowfield.f90:29-111 (freestream start) on all registered blocks */
int aero_init_flowfield(void);
/* sub_init_walldist.f90:9 (wall distance of every physical node) */
int aero_init_walldist(void);
/* main.f90:142-208 for every registered block on the device: coordinate halo,
 * metrics, spacing (sub_init_spacing.f90) and, if with_walldist, wall distance */
int aero_compute_geometry(int with_walldist);
/* primitives of all registered blocks (main.f90:434-447) */
int aero_getpri_all(void);

/* ---- whole iterations (main.f90:343-447, or :450-573 for Crank-Nicolson,
 *      for every block, plus the residual
 *      of main.f90:603 each step); resid_hist receives nsteps x 7 values
 *      when not NULL.  dt_minmax (may be NULL) receives dtmax, dtmin of the
 *      last block's find_dt of the last step (steady runs; the unsteady
 *      find_dt leaves dt unchanged and dt_minmax is not written).  Every step
 *      ends with the primitives of all blocks, as main.f90:434-447. ------- */
int aero_step(int nsteps, double* resid_hist, double* dt_minmax);

/* Benchmark form of aero_step: nsteps iterations, each with its residual
 * norm, timed on the device with CUDA events (device_ms = total); with
 * flush_l2 != 0 the L2 cache is overwritten before every step, outside the
 * timed interval. */
int aero_step_timed(int nsteps, int flush_l2, double* device_ms);

/* ---- execution options (no counterpart in the reference) ---------------
 * aero_use_graphs(1): aero_step and aero_step_timed replay each time step
 * (iteration, closing primitives, residual) from a CUDA graph captured on its
 * first use; results are those of the launches it replays.
 * aero_autotune(iters): times iters steps for each candidate launch shape
 * (inviscid-flux CTA tile, element-wise / viscous / block-record thread
 * counts, sweep stages, CTAs per block of the LU-SGS sweep), keeps the fastest
 * of each in turn, and restores the
 * solution state (q, nut, q0, dt, amu) it started from; the arithmetic is the
 * same for every shape.  aero_tuning() describes the shapes in use. */
int aero_use_graphs(int on);
int aero_autotune(int iters);
const char* aero_tuning(void);
/* Sets the launch shapes directly (e.g. to apply a saved tuning): inviscid
 * tile 0 (face-based kernels; -6 / -8: the FP64 face kernel under a register
 * bound for 6 / 8 CTAs per SM, -10: the FP64 face kernel reading its WENO
 * stencils from shared memory, and in mixed precision for any of the three
 * the mixed face kernel bounded for 10), 32, 64 or 128; element-wise threads 128, 256,
 * 512; viscous and block-record threads 64, 128, 256; sweep stages 2..4. */
int aero_set_tuning(int inv_tile, int ew, int visc, int mats, int nst_max);
/* CTAs that share each block's LU-SGS sweep: 1 (one CTA per block, the
 * records staged in shared memory when its planes fit) or a thread-block
 * cluster of 2, 4 or 8 CTAs, or 16 CTAs (a non-portable cluster size, with
 * the bulk-copy or the slab exchange only; accepted after aero_finish_setup
 * when the device can hold such a cluster).  The arithmetic is the same for
 * every choice. */
int aero_set_sweep_cluster(int ctas);
/* How a cluster's CTAs share a block's sweep: 0 (default) every CTA a part
 * of each hyperplane, the values passed through L2 with a cluster barrier
 * per plane; 1 the same with bulk copies between the CTAs' shared memories
 * counted on mbarriers (used when every row of the largest plane has its own
 * thread: 5 x plane nodes <= 512 x CTAs); 2 every CTA one range of k
 * (a k-slab), the CTAs pipelined plane by plane, each passing only its edge
 * k-segment's values to the next CTA (used when each slab's part of a plane
 * has at most 102 nodes; else 1); 3 as 1 with CTAs of at most 384 threads
 * built for two resident per SM (for batches whose sweep CTAs outnumber the
 * SMs; larger CTAs take 1).  The arithmetic is the same for every choice. */
int aero_set_sweep_exchange(int mode);
/* CTAs that share each block's SA sweep: 1 (default; one CTA per block) or a
 * cluster of 2, 4 or 8 CTAs pipelined by k-slabs as exchange 2 above (used
 * when each slab's part of a plane has at most 512 nodes), or 16 (accepted
 * after aero_finish_setup when the device can hold such a cluster).  The
 * arithmetic is the same for every choice. */
int aero_set_sa_sweep_cluster(int ctas);
/* 1: the FP64 viscous part a kernel under a register bound of 64 per thread
 * (more resident warps, a few spills); 0 (default): without.  The arithmetic
 * is the same either way; aero_autotune chooses it too. */
int aero_set_register_bound(int on);
/* Planes ahead (2, the default, 3 or 4) at which the bulk-exchange sweep's
 * CTAs prefetch their shares of the plane records into L2.  Results are the
 * same for every choice; aero_autotune chooses it too. */
int aero_set_sweep_prefetch(int planes);
/* Polls each bounded wait of the staged LU-SGS sweep (one CTA per block)
 * makes before it gives up, 0..1048576 (the default); each poll may suspend
 * the waiting thread for a short, system-dependent time.  A wait that gives
 * up ends the sweep with AERO_ST_TIMEOUT in the status word and leaves the
 * context usable. */
int aero_set_poll_budget(long long polls);
/* Fault injection for tests: in every staged LU-SGS sweep the copies of
 * forward hyperplane `plane` (0-based) are never issued, so the waits for
 * them run out and the sweep ends with AERO_ST_TIMEOUT; -1 (default) turns it
 * off.  The iteration's update is then incomplete. */
int aero_inject_sweep_stall(int plane);

/* ---- warm-start network (no counterpart in the reference) --------------
 * aero_mlp_gemm: c[M x N] = a[M x K] * b[N x K]^T on the tcgen05 tensor cores,
 * a and b BF16 bit patterns (row-major), c FP32, host arrays; M and N
 * multiples of 128, K a multiple of 64; splits > 1 splits K over CTAs and
 * adds the partial tiles in a fixed order. */
int aero_mlp_gemm(const unsigned short* a, const unsigned short* b, float* c, int M, int N, int K, int splits);
/* The same GEMM on device operands of its own (constant values), reps times
 * back to back after one warm-up; ms_per_gemm receives the mean device time
 * of one, CUDA events on the default stream (benchmarking). */
int aero_mlp_gemm_timed(int M, int N, int K, int reps, double* ms_per_gemm);
/* The network: n_in inputs (<= 128), depth hidden SiLU layers of `width`
 * (a multiple of 128), n_out outputs (<= 128); BF16 weights and activations,
 * FP32 accumulation, FP32 master weights trained with Adam on the mean
 * squared error over mini-batches of `batch` rows (a multiple of 512).
 * Parameters are laid out layer by layer as W [nout x nin] (row-major, with
 * the padded sizes 128 for the input and output layers) then b [nout].
 * x, t, y are host arrays, row-major (n x n_in, n x n_out). */
int aero_mlp_create(int n_in, int n_out, int width, int depth, int batch, unsigned long long seed);
int aero_mlp_destroy(void);
int aero_mlp_param_count(long long* count);
int aero_mlp_get_params(float* out);
/* loss and gradients of one batch (n <= batch rows), parameters unchanged */
int aero_mlp_gradients(const float* x, const float* t, int n, float* loss, float* grad);
/* steps Adam steps on shuffled mini-batches; loss_hist (may be NULL) gets the
 * batch loss of every step */
int aero_mlp_train(const float* x, const float* t, long long n, int steps, float lr, unsigned long long seed,
                   float* loss_hist);
int aero_mlp_predict(const float* x, long long n, float* y);

/* ---- instrumentation ---------------------------------------------------
 * aero_profile(1) starts timing every kernel launch with CUDA events on the
 * library's stream (and zeroes the totals); aero_profile(0) stops.
 * aero_profile_read fills ms[i] (total milliseconds) and counts[i] (launches)
 * for kernel class i < n and returns the number of classes;
 * aero_profile_name(i) names class i.  aero_launch_count returns how many
 * kernels the library has launched since it was loaded. */
int aero_profile(int enable);
int aero_profile_read(double* ms, long long* counts, int n);
const char* aero_profile_name(int id);
/* The launches timed since the previous read (in launch order): their class
 * ids[i], and start_ms[i] / end_ms[i], the times of the events recorded on
 * their own streams before and after them, in milliseconds after the first
 * launch's start; ids[i] = class + 100 x the stream (0 the library's first
 * stream, 1 and 2 its others).  Fills at most n entries and returns how many launches
 * there were.  Kernels on the library's other streams overlap those on its
 * first, so this is the time line of a step, not a sum of durations. */
int aero_profile_timeline(int* ids, double* start_ms, double* end_ms, int n);
int aero_launch_count(unsigned long long* count);

/* ---- test hook: the device's exact elementary functions ----------------
 * The FP64 kernels evaluate the reference's x**y and exp(x) with correctly
 * rounded double-double implementations that give the same bits on the host
 * (the CPU oracle uses them too).  aero_math_eval runs them on the device for
 * n host values: fn 0 = pow(x[i], y[i]), fn 1 = exp(x[i]) (y unused), results
 * in out (host).  It needs no aero_init; it allocates device memory for the
 * call and synchronises.  No counterpart in the reference (a test hook). */
int aero_math_eval(int fn, const double* x, const double* y, double* out, long long n);

/* ---- residual of caller-owned device arrays, without allocation --------
 * No counterpart in the reference: it is the computation of
 * sub_output_residual.f90:8-67 (what aero_residual returns) for a caller that
 * keeps its block arrays on the device itself, e.g. a CUDA Fortran or OpenACC
 * port of the solver, and cannot let a library allocate: cudaMalloc and
 * cudaFree synchronise the device, are not allowed while a stream is being
 * captured, and draw on memory such a caller budgets itself.  The call needs
 * neither aero_init nor a registered case, allocates no device memory and
 * calls no allocating CUDA or library routine; on a rejected argument it only
 * records the message that aero_last_error returns.
 *
 * Block m (0-based, m < nblocks) is given by device pointers to arrays in the
 * reference layout over its full box: rhs[m] -> rhs(5,is:ie,js:je,ks:ke),
 * dt[m], inv_j[m] and, when sa_rhs is not NULL, sa_rhs[m] -> (is:ie,...);
 * rhs, dt, inv_j and sa_rhs are host arrays of nblocks pointers.
 * boxes holds 12 ints per block: is,ie,js,je,ks,ke, is1,ie1,js1,je1,ks1,ke1.
 * out7 is a DEVICE pointer to 7 doubles, written as aero_residual's out7
 * (component 6 is 0 when sa_rhs is NULL).  Both kernels are enqueued on
 * `stream` (a cudaStream_t; NULL = the legacy default stream) and the call
 * returns without waiting for them.
 *
 * Limits: 1 <= nblocks <= AERO_NOALLOC_MAX_BLOCKS, and nblocks x
 * ceil(largest updated box / 256) <= AERO_NOALLOC_MAX_PARTS (about 4.2 million
 * updated nodes in equal blocks); larger calls return AERO_ERR_ARG before any
 * device work.  The partial sums live in one fixed device array per device;
 * the first call in each CUDA context of a device looks its address up (make
 * that first call outside any stream capture; a context re-created after a
 * device reset gets a fresh lookup, and a failed lookup is retried by the
 * next call), and nothing in it has to start at zero.  Calls
 * whose kernels can overlap on one device (other streams, other host threads)
 * share that array and race: order them on one stream. */
#define AERO_NOALLOC_MAX_BLOCKS 32
#define AERO_NOALLOC_MAX_PARTS 16384
int aero_residual_device_noalloc(int nblocks, const double* const* rhs, const double* const* dt,
                                 const double* const* inv_j, const double* const* sa_rhs,
                                 const int* boxes, double totalnodes, double* out7, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* AEROCFD_GPU_H */
