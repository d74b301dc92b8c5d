// Host runtime and C-ABI of libaerocfd_gpu.so (declared in include/aerocfd_gpu.h).
//
// State mirrors the reference's module variables: the flag and constant values
// of Control.in (flag_var, ns_const, sa_var), the per-block index boxes and
// subfaces (blk_var, glbindex_var), and, once registered, the per-block arrays,
// which live on the device in one arena and are copied to or from the caller's
// host arrays only on request.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/aerocfd_gpu.h"
#include "aero_device.cuh"
#include "aero_kernels.h"
#include "aero_topology.h"

using namespace aero;

namespace {

struct HostBlock {
  bool used = false;
  Box b{}, b0{}, b1{};
  std::vector<SubRow> subs;
  double* host[kNumPublicFields] = {};
  bool pinned[kNumPublicFields] = {};
  long plane = 0;
  size_t arena_off = 0;  // doubles
  void* ws = nullptr;    // LU-SGS workspace (one allocation)
  bool own_params = false;  // aero_set_block_params: this block's case constants
  double params[7] = {};
  CaseConsts cc{};
};

// Hyperplane offsets of an nx1 x ny1 x nz1 updated box (planes h = a+b+c).
std::vector<long> plane_offsets(const Box& b1, int& pmax) {
  int nx1 = b1.nx(), ny1 = b1.ny(), nz1 = b1.nz();
  int H = nx1 + ny1 + nz1 - 2;
  std::vector<long> off(H + 1, 0);
  pmax = 0;
  for (int h = 0; h < H; ++h) {
    long n = 0;
    for (int c = 0; c < nz1; ++c) {
      int r = h - c;
      if (r < 0) break;
      int bmin = std::max(0, r - (nx1 - 1)), bmax = std::min(ny1 - 1, r);
      if (bmax >= bmin) n += bmax - bmin + 1;
    }
    off[h + 1] = off[h] + n;
    pmax = std::max<long>(pmax, n);
  }
  return off;
}

// k-segment starts of every plane of an nx1 x ny1 x nz1 updated box
// (BlockView::seg): entry h*(nz1+2) + c+1 = nodes of plane h with k-offset
// below c, for c = -1 .. nz1.
std::vector<int> plane_segments(const Box& b1) {
  const int nx1 = b1.nx(), ny1 = b1.ny(), nz1 = b1.nz();
  const int H = nx1 + ny1 + nz1 - 2, SW = nz1 + 2;
  std::vector<int> seg((size_t)std::max(H, 0) * SW, 0);
  for (int h = 0; h < H; ++h) {
    int n = 0;
    for (int c = 0; c < nz1; ++c) {
      seg[(size_t)h * SW + c + 1] = n;
      const int r = h - c;
      const int bmin = std::max(0, r - (nx1 - 1)), bmax = std::min(ny1 - 1, r);
      if (r >= 0 && bmax >= bmin) n += bmax - bmin + 1;
    }
    seg[(size_t)h * SW + nz1 + 1] = n;
  }
  return seg;
}

// Shape of the slab sweeps of one block over clusters of `ncta` CTAs: the
// block's k-offsets 0..nz1-1 split into ce = min(ncta, nz1) slabs, slab r
// holding [r*nz1/ce, (r+1)*nz1/ce).  own: the most nodes of one plane inside
// a slab; edge: the most nodes of one k-segment of one plane (a slab's edge
// segment, the values it passes to the next slab).
void slab_shape(const Box& b1, int ncta, int& own, int& edge) {
  const int nz1 = b1.nz(), H = b1.nx() + b1.ny() + nz1 - 2, SW = nz1 + 2;
  const std::vector<int> seg = plane_segments(b1);
  const int ce = std::max(1, std::min(ncta, nz1));
  own = edge = 0;
  for (int h = 0; h < H; ++h) {
    const int* s = seg.data() + (size_t)h * SW + 1;  // s[c] for c = -1 .. nz1
    for (int c = 0; c < nz1; ++c) edge = std::max(edge, s[c + 1] - s[c]);
    for (int r = 0; r < ce; ++r) own = std::max(own, s[(r + 1) * nz1 / ce] - s[r * nz1 / ce]);
  }
}

// Launch shape of a slab sweep (k_lusgs_sweep_slab: `rows` = 5 rows per node;
// k_sa_sweep_slab: 1) over clusters of ncta CTAs for a set of blocks: So
// values per row of a ring slot, L per row of an edge slot (even, so every
// copied slot is a multiple of 16 bytes), threads T (one per row of a slab's
// plane) and slots D (up to kSlabSlots in 200 KB of shared memory).  ok is
// false when a slab's plane needs more than 512 threads or fewer than two
// slots fit.
struct SlabFit {
  bool ok = false;
  int So = 0, L = 0, T = 0, D = 0;
};
SlabFit slab_fit(const BlockView* hv, int nblk, int ncta, int rows) {
  SlabFit f;
  int own = 0, edge = 0;
  for (int m = 0; m < nblk; ++m) {
    int o = 0, e = 0;
    slab_shape(hv[m].b1, ncta, o, e);
    own = std::max(own, o);
    edge = std::max(edge, e);
  }
  if (rows * own > 512 || own <= 0) return f;
  f.So = own;
  f.L = (edge + 1) & ~1;
  f.T = std::max(64, (rows * own + 31) / 32 * 32);
  const size_t slot = (size_t)rows * (f.So + 2 * f.L) * sizeof(double);
  f.D = (int)std::min<size_t>(kSlabSlots, (size_t)(200 * 1024) / slot);
  f.ok = f.D >= 2;
  return f;
}
size_t slab_smem(const SlabFit& f, int rows) { return (size_t)f.D * rows * (f.So + 2 * f.L) * sizeof(double); }

// slab_fit of the registered blocks (hv null; cached per setup) or of the
// nblk host views hv.
SlabFit slab_fit_for(const BlockView* hv, int nblk, int ncta, int rows);

// Largest (and default) number of polls of each wait of the staged LU-SGS
// sweep, the kernel's own bound.
constexpr long kPollBudgetMax = 1L << 20;

struct State {
  bool inited = false;
  int device = 0;
  cudaStream_t stream = nullptr;
  // second stream of a steady iteration: inviscid_flux_1 runs on it beside
  // viscous_flux and find_dt, and sa_model beside implicit1st (in each pair
  // neither reads what the other writes); each is forked and joined with events
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_fork2 = nullptr, ev_join2 = nullptr;  // inviscid beside viscous + find_dt
  cudaEvent_t ev_prep = nullptr, ev_resid = nullptr;   // residual norm beside the LU-SGS sweeps
  // third stream: the LU-SGS radii and off-diagonal blocks beside the flux and
  // time-step kernels (they read q, the primitives and the metrics only)
  cudaStream_t stream3 = nullptr;
  cudaEvent_t ev_join3 = nullptr;
  cudaEvent_t ev_dt = nullptr;  // find_dt done: the SA records may start
  // fourth stream: sa_model, forked after find_dt, beside the rest of the
  // mean-flow iteration
  cudaStream_t stream4 = nullptr;
  std::vector<cudaEvent_t> xfer_ev;  // host transfers: one per array of a batch, plus one
  // dynamic shared memory limits already raised on this device (cudaFuncSetAttribute
  // is per device), per sweep kernel [FP64 records, FP32 records]
  // bulk sweep (index: 0 / 1 FP64 / FP32 records, 2 / 3 the variants with
  // loads two planes ahead, 4 / 5 the ones with two CTAs per SM): dynamic
  // shared memory set so far, clusters of 16 CTAs allowed on this device
  size_t smem_staged[2] = {0, 0}, smem_bulk[6] = {0, 0, 0, 0, 0, 0};
  bool np_cluster[6] = {false, false, false, false, false, false};
  // slab sweeps (mean flow FP64 / FP32 records, SA): dynamic shared memory
  // set so far, clusters of 16 allowed, and the launch shapes of the
  // registered blocks per (cluster size, rows per node)
  // (index: 0 / 1 mean flow FP64 / FP32 records, 2 SA, 3 / 4 the mean-flow
  // variants with loads two steps ahead)
  size_t smem_slab[5] = {0, 0, 0, 0, 0};
  bool np_slab[5] = {false, false, false, false, false};
  std::map<int, SlabFit> slab_fits;
  long spin_limit = kPollBudgetMax;  // polls of each staged-sweep wait (aero_set_poll_budget)
  int stall_plane = -1;              // forward plane whose copies are withheld (aero_inject_sweep_stall)
  bool configured = false;
  int iflags[8] = {};
  double params[7] = {};
  CaseConsts cc{};
  std::vector<HostBlock> blocks;
  bool setup = false;
  // device
  double* arena = nullptr;
  size_t arena_doubles = 0;
  BlockView* d_blocks = nullptr;
  BlockView* d_blocks_chain = nullptr;  // the views, longest sweep chain first
  std::vector<BlockView> views;
  BcOp* d_bc_ops = nullptr;
  // physical-BC launches: the entries of dependency level L are
  // d_bc_list[bc_lstart[L] .. bc_lstart[L+1]), the largest face bc_lface[L]
  BcEntry* d_bc_list = nullptr;
  std::vector<int> bc_lstart;
  std::vector<long> bc_lface;
  HaloEntry* d_halo = nullptr;
  long nhalo = 0;
  AvgSrc* d_avg_src = nullptr;
  AvgDst* d_avg_dst = nullptr;
  long navg_src = 0, navg_dst = 0;
  double* d_avg_buf = nullptr;
  double* d_part = nullptr;
  int resid_ctas = 0;
  WallFace* d_walls = nullptr;  // clcd_output: wall subfaces and per-CTA force partials
  int nwall = 0;
  long nquad = 0;
  double* d_fpart = nullptr;
  std::vector<SurfZone> surf;     // surface_output: wall subfaces (all nodes) and the x, y, z, cp rows
  SurfZone* d_surf = nullptr;
  long nsurf = 0;
  int nsurf_live = 0;
  double* d_surf_out = nullptr;
  CaseConsts* d_ccb = nullptr;   // per-block case constants (batches)
  double* d_resid_blocks = nullptr;  // 7 per block (aero_residual_blocks)
  unsigned* d_bstat = nullptr;       // per-block status words (aero_get_block_status)
  int* d_live = nullptr;             // per-block live flags (aero_set_retirement)
  bool retire = false;               // refresh the live flags from the status words every step
  double* d_out = nullptr;   // residual (7) + dt min/max (2)
  double* h_out = nullptr;   // pinned
  unsigned* d_status = nullptr;
  double* d_staging = nullptr;
  size_t staging_doubles = 0;
  double totalnodes = 0;
  long max_box = 0, max_b0 = 0, max_b1 = 0, max_ext = 0;
  Box max_b1_box{1, 0, 1, 0, 1, 0};  // largest updated extent per direction over the blocks
  long max_b1_face = 0;               // largest face of an updated box (nodes)
  std::map<const double*, std::pair<int, int>> registry;  // host array -> (block, field)
  // transient mode pool
  double* t_arena = nullptr;
  size_t t_doubles = 0;
  BlockView* d_tview = nullptr;
  void* t_ws = nullptr;
  size_t t_ws_bytes = 0;
  int pmax_all = 0;
  int hmax_all = 0;
  bool mixed = false;  // aero_set_precision(1): FP32 increments in the flux kernels
  // rhsi holds 0 on every node outside the updated boxes of the registered
  // blocks (set by init_flowfield and by every full fill; cleared when the
  // caller uploads rhsi).  The inviscid kernels write only updated nodes and
  // nothing else writes rhsi, so while it holds the whole-iteration path skips
  // inviscid_flux_1's full-box zeroing.
  bool rhsi_ghosts_zero = false;
  // launch shapes (aero_autotune); none of them changes the arithmetic
  struct Tune {
    int inv_tile = 64;  // nodes per CTA of the inviscid flux; 0: face-based kernels (-6, -8: FP64 faces for 6, 8 CTAs/SM;
                        // -10: FP64 faces with shared-memory stencils)
    int ew = 256;       // threads per CTA of the element-wise kernels
    int visc = 128;     // threads per CTA of k_viscous_a
    int bound = 0;      // 1: the register-bounded FP64 k_viscous_a
    int mats = 128;     // threads per CTA of k_lusgs_mats
    int nst_max = 4;    // most shared-memory stages of the staged sweep
    int sweep_cl = 0;   // CTAs per block of the global-memory sweep (0, 1: one CTA; 2..8: a cluster)
    int sweep_x = 0;    // cluster exchange: 0 through L2, 1 bulk copies between shared memories (when it fits),
                        // 2 pipelined k-slabs (when it fits; else 1)
    int sa_cl = 0;      // CTAs per block of the SA sweep (0, 1: one CTA; 2..16: a cluster pipelined by k-slabs)
    int sweep_pf = 2;   // L2 prefetch distance of the bulk-exchange sweep, in planes (2..4)
  } tune;
  // CUDA graph of one time step (aero_use_graphs)
  bool graph_want = false;
  cudaGraphExec_t graph_exec = nullptr;
  unsigned long long graph_kernels = 0;
  double* d_tmax = nullptr;
  size_t t_tmax = 0;
  std::string err;
  std::string tuning = "inviscid_tile=64 elementwise_threads=256 viscous_threads=128 mats_threads=128 sweep_stages<=4 "
                       "sweep_cluster=1 sweep_exchange=l2";
};

State g;

SlabFit slab_fit_for(const BlockView* hv, int nblk, int ncta, int rows) {
  if (hv) return slab_fit(hv, nblk, ncta, rows);
  const int key = ncta * 8 + rows;
  auto it = g.slab_fits.find(key);
  if (it != g.slab_fits.end()) return it->second;
  SlabFit f = slab_fit(g.views.data(), (int)g.views.size(), ncta, rows);
  g.slab_fits[key] = f;
  return f;
}

// ---------------------------------------------------------------- profiling
// Per-kernel CUDA-event timing on the library's stream (aero_profile_*), and a
// count of every kernel this library launches (aero_launch_count).
enum ProfId {
  P_GETPRI, P_FILL, P_INVISCID, P_VISC_A, P_VISC_B, P_FIND_DT, P_DT_MINMAX, P_LUSGS_PREP,
  P_LUSGS_MATS, P_LUSGS_SWEEP, P_LUSGS_UPDATE, P_SA_A, P_SA_B, P_SA_RECS, P_SA_SWEEP, P_INDEX, P_BC, P_SA_CLIP, P_HALO, P_AVG_GATHER, P_AVG_APPLY, P_RESID_PART, P_RESID_FINAL,
  P_TRANSFER, P_GEOMETRY, P_FORCES, P_CRANK, P_LUSGS_RADII, P_LUSGS_SCA, P_NUM
};
const char* kProfName[P_NUM] = {
    "k_getpri", "k_fill", "k_inviscid", "k_viscous_a", "k_viscous_b", "k_find_dt", "k_dt_minmax",
    "k_lusgs_prep", "k_lusgs_mats", "k_lusgs_sweep", "k_lusgs_update", "k_sa_a", "k_sa_b", "k_sa_recs", "k_sa_sweep",
    "k_plane_index", "k_physical_bc", "k_sa_clip", "k_halo", "k_avg_gather",
    "k_avg_apply", "k_residual_partial", "k_residual_final", "k_transfer", "k_geometry", "k_forces", "k_crank",
    "k_lusgs_radii", "k_lusgs_sca"};
struct Prof {
  bool on = false;
  std::vector<cudaEvent_t> pool;
  size_t used = 0;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> marks;
  double ms[P_NUM] = {};
  long count[P_NUM] = {};
  unsigned long long launches = 0;
  // the launches of the last collected batch of marks: class, start and end in
  // ms after the first of them (aero_profile_timeline)
  std::vector<int> tl_id;
  std::vector<double> tl_start, tl_end;
} gp;

cudaEvent_t prof_event() {
  if (gp.used == gp.pool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    gp.pool.push_back(e);
  }
  return gp.pool[gp.used++];
}
int stream_index(cudaStream_t s);
struct ProfScope {
  int id;
  cudaEvent_t a{}, b{};
  ProfScope(int id_, cudaStream_t s) : id(id_ + 100 * stream_index(s)) {
    ++gp.launches;
    if (gp.on) {
      a = prof_event();
      cudaEventRecord(a, s);
    }
  }
  void end(cudaStream_t s) {
    if (gp.on) {
      b = prof_event();
      cudaEventRecord(b, s);
      gp.marks.push_back({id, {a, b}});
    }
  }
};
#define PROF_ON(id, st, launch)          \
  do {                                   \
    ProfScope ps_(id, st);               \
    launch;                              \
    ps_.end(st);                         \
  } while (0)
#define PROF(id, launch) PROF_ON(id, g.stream, launch)

// 0 for the library's first stream, 1, 2 and 3 for its others
int stream_index(cudaStream_t s) { return s == g.stream2 ? 1 : (s == g.stream3 ? 2 : (s == g.stream4 ? 3 : 0)); }

void prof_collect() {
  if (gp.marks.empty()) return;
  cudaStreamSynchronize(g.stream);
  cudaDeviceSynchronize();  // marks on the other streams too
  gp.tl_id.clear();
  gp.tl_start.clear();
  gp.tl_end.clear();
  const cudaEvent_t t0 = gp.marks.front().second.first;
  for (auto& m : gp.marks) {
    float t = 0.f, a = 0.f, b = 0.f;
    cudaEventElapsedTime(&t, m.second.first, m.second.second);
    gp.ms[m.first % 100] += t;
    gp.count[m.first % 100] += 1;
    cudaEventElapsedTime(&a, t0, m.second.first);
    cudaEventElapsedTime(&b, t0, m.second.second);
    gp.tl_id.push_back(m.first);
    gp.tl_start.push_back(a);
    gp.tl_end.push_back(b);
  }
  gp.marks.clear();
  gp.used = 0;
}

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g.err = buf;
  return code;
}

#define CK(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return fail(e_ == cudaErrorMemoryAllocation ? AERO_ERR_NOMEM : AERO_ERR_CUDA,       \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)
#define CKL() CK(cudaGetLastError())

long round32(long n) { return (n + 31) / 32 * 32; }
unsigned cdiv(long a, long b) { return (unsigned)((a + b - 1) / b); }

Box box_of(const int* is, const int* ie, const int* js, const int* je, const int* ks, const int* ke) {
  return Box{*is, *ie, *js, *je, *ks, *ke};
}
bool same(const Box& a, const Box& b) {
  return a.is == b.is && a.ie == b.ie && a.js == b.js && a.je == b.je && a.ks == b.ks && a.ke == b.ke;
}

int need_init() {
  if (!g.inited) return fail(AERO_ERR_STATE, "aero_init has not been called");
  return AERO_OK;
}
int need_setup() {
  if (!g.inited || !g.setup) return fail(AERO_ERR_STATE, "case set-up is not finished (aero_finish_setup)");
  return AERO_OK;
}

// Every field of a view gets `plane`-strided component planes.
size_t view_doubles(long plane) {
  size_t s = 0;
  for (int f = 0; f < F_NUM; ++f) s += (size_t)field_nc(f) * plane;
  return s;
}
void fill_view(BlockView& v, const Box& b, const Box& b0, const Box& b1, long plane, double* base) {
  v.b = b; v.b0 = b0; v.b1 = b1;
  v.ccb = nullptr;
  v.bstat = nullptr;
  v.live = nullptr;
  v.nx = b.nx(); v.ny = b.ny();
  v.plane = plane;
  size_t off = 0;
  for (int f = 0; f < F_NUM; ++f) {
    v.f[f] = base + off;
    off += (size_t)field_nc(f) * plane;
  }
}

// LU-SGS workspace of one view (see BlockView): one device allocation holding
// poff, rec_f, rec_b, sca, dqs, dq, sa_rec, sa_dq, nat, nbr, pidx, seg, each array
// starting on a 256-byte boundary (the sweeps' bulk copies and L2 prefetches
// of plane chunks need 16-byte aligned starts).
constexpr size_t kWsAlign = 256;
constexpr int kWsArrays = 12;
size_t ws_round(size_t bytes) { return (bytes + kWsAlign - 1) / kWsAlign * kWsAlign; }
size_t workspace_bytes(const Box& b1, int H) {
  size_t N1 = (size_t)b1.size();
  return (size_t)(H + 1) * sizeof(long) + N1 * (2 * kRec + kSca + 8 + 5 + kSaRec + 1) * sizeof(double) +
         N1 * sizeof(long) + N1 * 7 * sizeof(int) + (size_t)H * (b1.nz() + 2) * sizeof(int) +
         (kWsArrays + 1) * kWsAlign;
}
int attach_workspace(BlockView& v, void* ws, const std::vector<long>& poff, int pmax) {
  size_t N1 = (size_t)v.b1.size();
  char* p = (char*)ws;
  auto take = [&](size_t bytes) {
    char* at = p;
    p += ws_round(bytes);
    return at;
  };
  v.nplanes = (int)poff.size() - 1;
  v.pmax = pmax;
  v.rec_f = (double*)take(N1 * kRec * sizeof(double));
  v.rec_b = (double*)take(N1 * kRec * sizeof(double));
  v.sca = (double*)take(N1 * kSca * sizeof(double));
  v.dqs = (double*)take(N1 * 8 * sizeof(double));
  v.dq = (double*)take(N1 * 5 * sizeof(double));
  v.sa_rec = (double*)take(N1 * kSaRec * sizeof(double));
  v.sa_dq = (double*)take(N1 * sizeof(double));
  v.nat = (long*)take(N1 * sizeof(long));
  v.poff = (long*)take(poff.size() * sizeof(long));
  v.nbr = (int*)take(N1 * 7 * sizeof(int));
  v.pidx = v.nbr + 6 * N1;
  const std::vector<int> seg = plane_segments(v.b1);
  v.seg = (int*)take(seg.size() * sizeof(int));
  CK(cudaMemcpyAsync(v.poff, poff.data(), poff.size() * sizeof(long), cudaMemcpyHostToDevice, g.stream));
  if (!seg.empty())
    CK(cudaMemcpyAsync(v.seg, seg.data(), seg.size() * sizeof(int), cudaMemcpyHostToDevice, g.stream));
  return AERO_OK;
}

int ensure_staging(size_t doubles) {
  if (doubles <= g.staging_doubles) return AERO_OK;
  if (g.d_staging) CK(cudaFree(g.d_staging));
  g.d_staging = nullptr;
  CK(cudaMalloc(&g.d_staging, doubles * sizeof(double)));
  g.staging_doubles = doubles;
  return AERO_OK;
}

// host (c, i, j, k) column-major <-> one field of a view
int upload(const double* host, double* dev_field, long n, int nc, long plane) {
  int rc = ensure_staging((size_t)n * nc);
  if (rc) return rc;
  CK(cudaMemcpyAsync(g.d_staging, host, (size_t)n * nc * sizeof(double), cudaMemcpyHostToDevice, g.stream));
  PROF(P_TRANSFER, (k_aos_to_soa<<<cdiv(n, 256), 256, 0, g.stream>>>(g.d_staging, dev_field, n, nc, plane)));
  CKL();
  return AERO_OK;
}
int download(double* host, const double* dev_field, long n, int nc, long plane) {
  int rc = ensure_staging((size_t)n * nc);
  if (rc) return rc;
  PROF(P_TRANSFER, (k_soa_to_aos<<<cdiv(n, 256), 256, 0, g.stream>>>(dev_field, g.d_staging, n, nc, plane)));
  CKL();
  CK(cudaMemcpyAsync(host, g.d_staging, (size_t)n * nc * sizeof(double), cudaMemcpyDeviceToHost, g.stream));
  return AERO_OK;
}

// ------------------------------------------------------------ block operations
// A drop-in call names its arrays; it runs resident (registered arrays of one
// block, device copies) or transient (unregistered arrays, copied in and out).
struct Arg {
  int fid;
  const double* host;
  bool out;
};

struct BlockTarget {
  const BlockView* d_view;  // device pointer to one view
  BlockView view;           // host copy
  bool resident;
  int m;
};

int resolve(const Box& b, const Box& b0, const Box& b1, const std::vector<Arg>& args, BlockTarget& t) {
  int nreg = 0, m = -1;
  for (const Arg& a : args) {
    auto it = g.registry.find(a.host);
    if (it != g.registry.end()) {
      ++nreg;
      if (it->second.second != a.fid)
        return fail(AERO_ERR_ARG, "array for field %d is registered as field %d", a.fid, it->second.second);
      if (m >= 0 && it->second.first != m)
        return fail(AERO_ERR_ARG, "arrays of blocks %d and %d in one call", m + 1, it->second.first + 1);
      m = it->second.first;
    }
  }
  if (nreg != 0 && nreg != (int)args.size())
    return fail(AERO_ERR_ARG, "call mixes registered and unregistered arrays");
  if (nreg > 0) {
    const HostBlock& H = g.blocks[m];
    if (!same(H.b, b) || !same(H.b0, b0) || !same(H.b1, b1))
      return fail(AERO_ERR_ARG, "index bounds differ from block %d's registered boxes", m + 1);
    t.resident = true;
    t.m = m;
    t.view = g.views[m];
    t.d_view = g.d_blocks + m;
    return AERO_OK;
  }
  // transient: a 2-D configuration works on one-plane boxes, a 3-D one on
  // boxes of at least three planes (the kernels reach k-1 and k+1 there)
  const int dim = g.configured ? g.cc.dimension : IFLAG_3D;
  if (dim == IFLAG_2D ? (b.nz() != 1) : (b.nz() < 3))
    return fail(AERO_ERR_ARG, "index box with %d k-planes in a %d-D configuration", b.nz(), dim);
  long plane = round32(b.size());
  size_t need = view_doubles(plane);
  if (need > g.t_doubles) {
    if (g.t_arena) CK(cudaFree(g.t_arena));
    g.t_arena = nullptr;
    CK(cudaMalloc(&g.t_arena, need * sizeof(double)));
    g.t_doubles = need;
  }
  if (!g.d_tview) CK(cudaMalloc(&g.d_tview, sizeof(BlockView)));
  CK(cudaMemsetAsync(g.t_arena, 0, need * sizeof(double), g.stream));
  fill_view(t.view, b, b0, b1, plane, g.t_arena);
  if (b1.nx() > 0 && b1.ny() > 0 && b1.nz() > 0) {
    int pmax = 0;
    std::vector<long> poff = plane_offsets(b1, pmax);
    size_t wsb = workspace_bytes(b1, (int)poff.size() - 1);
    if (wsb > g.t_ws_bytes) {
      if (g.t_ws) CK(cudaFree(g.t_ws));
      g.t_ws = nullptr;
      CK(cudaMalloc(&g.t_ws, wsb));
      g.t_ws_bytes = wsb;
    }
    int rc2 = attach_workspace(t.view, g.t_ws, poff, pmax);
    if (rc2) return rc2;
  }
  CK(cudaMemcpyAsync(g.d_tview, &t.view, sizeof(BlockView), cudaMemcpyHostToDevice, g.stream));
  t.d_view = g.d_tview;
  t.resident = false;
  t.m = -1;
  for (const Arg& a : args) {
    int rc = upload(a.host, t.view.f[a.fid], b.size(), field_nc(a.fid), plane);
    if (rc) return rc;
  }
  return AERO_OK;
}

// Routines that take only the full box (get_primitivevariables, find_dt):
// resident calls use the registered block's inner boxes.
int resolve_full(const Box& b, const std::vector<Arg>& args, BlockTarget& t) {
  auto it = g.registry.find(args[0].host);
  if (it != g.registry.end()) {
    const HostBlock& H = g.blocks[it->second.first];
    if (!same(H.b, b)) return fail(AERO_ERR_ARG, "index bounds differ from block %d's box", it->second.first + 1);
    return resolve(H.b, H.b0, H.b1, args, t);
  }
  return resolve(b, b, b, args, t);
}

int finish(const BlockTarget& t, const std::vector<Arg>& args) {
  if (!t.resident) {
    for (const Arg& a : args)
      if (a.out) {
        int rc = download(const_cast<double*>(a.host), t.view.f[a.fid], t.view.b.size(),
                          field_nc(a.fid), t.view.plane);
        if (rc) return rc;
      }
    CK(cudaStreamSynchronize(g.stream));
  }
  CKL();
  return AERO_OK;
}

CaseConsts consts_with(double gamma, double cv, double re) {
  CaseConsts c = g.cc;
  if (!g.configured) c.dimension = IFLAG_3D;  // drop-in calls before aero_configure: 3-D
  c.gamma = gamma;
  c.cv = cv;
  c.re = re;
  return c;
}

// --------------------------------------------------------- launch helpers
int launch_getpri(const BlockView* views, int nblk, long maxN, const CaseConsts& cc) {
  const int ew = g.tune.ew;
  PROF(P_GETPRI, (k_getpri<<<dim3(cdiv(maxN, ew), nblk), ew, 0, g.stream>>>(views, cc, g.d_status)));
  CKL();
  return AERO_OK;
}
// inviscid_flux_1 on nblk views, on stream st (the library's stream when null).
// fill = false skips the full-box zeroing of rhsi (sub_inviscid1.f90:32-48),
// for registered blocks whose rhsi is already 0 outside the updated boxes.
int launch_inviscid(const BlockView* views, int nblk, long maxN, long maxN1, long maxFace, const CaseConsts& cc,
                    cudaStream_t st = nullptr, bool fill = true) {
  if (!st) st = g.stream;
  if (fill) {
    PROF_ON(P_FILL, st, (k_fill<<<dim3(cdiv(maxN, g.tune.ew), nblk), g.tune.ew, 0, st>>>(views, F_RHSI, 5, 0.0)));
    CKL();
  }
  const int tile = g.tune.inv_tile;
  if (cc.inviscid == IFLAG_5THWENO || cc.inviscid == IFLAG_5THWCNS) {
    // extension schemes: faces, then the combine
    long maxF = maxN1 + maxFace;
    auto faces = cc.inviscid == IFLAG_5THWENO ? (g.mixed ? k_faces_sw_weno5_mixed : k_faces_sw_weno5)
                                              : (g.mixed ? k_faces_wcns5_mixed : k_faces_wcns5);
    PROF_ON(P_INVISCID, st, (faces<<<dim3(cdiv(maxF, 128), nblk, 3), 128, 0, st>>>(views, cc)));
    CKL();
    PROF_ON(P_INVISCID, st, (k_inviscid_combine<<<dim3(cdiv(maxN1, g.tune.ew), nblk), g.tune.ew, 0, st>>>(views, cc)));
  } else if (tile <= 0) {  // face-based: each face once, then the combine
    // faces per direction <= updated box grown by one node in that direction
    // (tile -6 / -8: the FP64 kernel under a register bound for 6 / 8 CTAs per
    // SM; in mixed precision both take the mixed kernel bounded for 10)
    long maxF = maxN1 + maxFace;
    auto faces = g.mixed ? (tile < 0 ? k_inviscid_faces_mixed_o10 : k_inviscid_faces_mixed)
                         : (tile == -6    ? k_inviscid_faces_o6
                            : tile == -8  ? k_inviscid_faces_o8
                            : tile == -10 ? k_inviscid_faces_staged
                                          : k_inviscid_faces);
    PROF_ON(P_INVISCID, st, (faces<<<dim3(cdiv(maxF, 128), nblk, 3), 128, 0, st>>>(views, cc)));
    CKL();
    PROF_ON(P_INVISCID, st, (k_inviscid_combine<<<dim3(cdiv(maxN1, g.tune.ew), nblk), g.tune.ew, 0, st>>>(views, cc)));
  } else {
    auto kern = g.mixed ? (tile == 32 ? k_inviscid_mixed_32 : tile == 128 ? k_inviscid_mixed_128 : k_inviscid_mixed_64)
                        : (tile == 32 ? k_inviscid_32 : tile == 128 ? k_inviscid_128 : k_inviscid_64);
    PROF_ON(P_INVISCID, st, (kern<<<dim3(cdiv(maxN1, tile), nblk), dim3(tile, 3), 0, st>>>(views, cc)));
  }
  CKL();
  return AERO_OK;
}
// viscous_flux in two parts: part a (gradients, viscosity, vorticity, the
// contravariant fluxes; everything find_dt and sa_model read) and part b (the
// divergence of the fluxes into rhsv).
int launch_viscous_a(const BlockView* views, int nblk, long maxN0, const CaseConsts& cc, int store) {
  const int vt = g.tune.visc;
  if (g.mixed)
    PROF(P_VISC_A, (k_viscous_a_mixed<<<dim3(cdiv(maxN0, vt), nblk), vt, 0, g.stream>>>(views, cc, store)));
  else
    PROF(P_VISC_A, ((g.tune.bound ? k_viscous_a_bound : k_viscous_a)<<<dim3(cdiv(maxN0, vt), nblk), vt, 0, g.stream>>>(
                       views, cc, store)));
  CKL();
  return AERO_OK;
}
int launch_viscous_b(const BlockView* views, int nblk, long maxN0, const CaseConsts& cc) {
  const int ew = g.tune.ew;
  PROF(P_VISC_B, (k_viscous_b<<<dim3(cdiv(maxN0, ew), nblk), ew, 0, g.stream>>>(views, cc)));
  CKL();
  return AERO_OK;
}
int launch_viscous(const BlockView* views, int nblk, long maxN0, const CaseConsts& cc, int store) {
  int rc = launch_viscous_a(views, nblk, maxN0, cc, store);
  return rc ? rc : launch_viscous_b(views, nblk, maxN0, cc);
}
int launch_find_dt(const BlockView* views, int nblk, long maxN, const CaseConsts& cc) {
  PROF(P_FIND_DT, (k_find_dt<<<dim3(cdiv(maxN, g.tune.ew), nblk), g.tune.ew, 0, g.stream>>>(views, cc, nullptr)));
  CKL();
  return AERO_OK;
}
int launch_dt_minmax(const BlockView* views, int m, double* d_out2) {
  PROF(P_DT_MINMAX, (k_dt_minmax<<<1, 1024, 0, g.stream>>>(views, m, nullptr, 0, 0, d_out2)));
  CKL();
  return AERO_OK;
}
// The part of implicit1st that needs only q, the primitives and the metrics:
// the spectral radii and the off-diagonal blocks of the sweeps, on stream st
// (the library's stream when null).  A steady iteration runs it on its own
// stream beside the flux and time-step kernels.
int launch_implicit_blocks(const BlockView* views, int nblk, long maxExt, long maxN1, const CaseConsts& cc,
                           cudaStream_t st = nullptr) {
  if (!st) st = g.stream;
  const int f = g.mixed ? 1 : 0;
  PROF_ON(P_LUSGS_RADII, st, (k_lusgs_radii<<<dim3(cdiv(maxExt, g.tune.ew), nblk), g.tune.ew, 0, st>>>(views)));
  CKL();
  PROF_ON(P_LUSGS_MATS, st, ((f ? k_lusgs_mats_f32 : k_lusgs_mats)<<<dim3(cdiv(3 * maxN1, g.tune.mats), nblk),
                                                                    g.tune.mats, 0, st>>>(views, cc)));
  CKL();
  return AERO_OK;
}

// The rest of implicit1st after launch_implicit_blocks: rhs and the diagonal,
// the per-node sweep scalars, the forward and backward sweeps and q += dq.
// with_blocks also runs launch_implicit_blocks first, on the same stream.
// sweep_views (null: views) is the view array the sweep kernels index: the
// same blocks, possibly in another order.
// Launches kern over nblk clusters of cl CTAs (grid x = nblk * cl) of
// `threads` threads with `smem` bytes of dynamic shared memory on stream st.
template <typename K, typename... A>
cudaError_t launch_clusters(K kern, int nblk, int cl, int threads, size_t smem, cudaStream_t st, A... args) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = dim3((unsigned)(nblk * cl));
  lc.blockDim = dim3((unsigned)threads);
  lc.dynamicSmemBytes = smem;
  lc.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = (unsigned)cl;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  lc.attrs = at;
  lc.numAttrs = 1;
  return cudaLaunchKernelEx(&lc, kern, args...);
}
// The attributes a slab sweep kernel (index k of State::smem_slab) needs for
// smem bytes of dynamic shared memory and clusters of cl CTAs.
template <typename K>
int prepare_slab(K kern, int k, size_t smem, int cl) {
  if (smem > 48 * 1024 && smem > g.smem_slab[k]) {
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    g.smem_slab[k] = smem;
  }
  if (cl > 8 && !g.np_slab[k]) {  // 16 CTAs: a non-portable cluster size
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    g.np_slab[k] = true;
  }
  return AERO_OK;
}

int launch_implicit(const BlockView* views, int nblk, long maxExt, long maxN1, int pmax, int hmax,
                    const CaseConsts& cc, cudaEvent_t after_prep = nullptr, bool with_blocks = true,
                    const BlockView* sweep_views = nullptr, const BlockView* host_views = nullptr) {
  const BlockView* sv = sweep_views ? sweep_views : views;
  // mixed precision stores the off-diagonal blocks in FP32 (products and sums
  // stay FP64); f selects that variant of every kernel that touches them
  const int f = g.mixed ? 1 : 0;
  int rc;
  if (with_blocks && (rc = launch_implicit_blocks(views, nblk, maxExt, maxN1, cc))) return rc;
  PROF(P_LUSGS_PREP, (k_lusgs_prep<<<dim3(cdiv(maxExt, g.tune.ew), nblk), g.tune.ew, 0, g.stream>>>(views, cc)));
  CKL();
  if (after_prep) CK(cudaEventRecord(after_prep, g.stream));
  PROF(P_LUSGS_SCA, ((f ? k_lusgs_sca_f32 : k_lusgs_sca)<<<dim3(cdiv(maxN1, g.tune.ew), nblk), g.tune.ew, 0,
                                                           g.stream>>>(views)));
  CKL();
  // Staged sweep: plane offsets + ring of two planes + nst staged planes
  // (records, scalars, dq*) + 2*nst+1 mbarriers, as many stages as fit
  // (2..4); one consumer thread per row of every node of the largest plane
  // plus one producer warp.
  if (pmax >= (1 << 21) - 1) return fail(AERO_ERR_ARG, "hyperplane of %d nodes exceeds the LU-SGS index range", pmax);
  const size_t kSmemMax = 227 * 1024;
  const size_t rec_words = f ? 40 : kRec;  // record words per node, in doubles
  size_t offs = (size_t)((hmax + 2) & ~1) * sizeof(long);
  size_t ring = (size_t)2 * 5 * std::max(pmax, 1) * sizeof(double);
  size_t stage = (size_t)std::max(pmax, 1) * (rec_words + kSca + 8) * sizeof(double);
  int nst = g.tune.nst_max;
  while (nst >= 2 && offs + ring + nst * stage + (2 * nst + 1) * 8 > kSmemMax) --nst;
  auto staged = f ? k_lusgs_sweep_staged_f32 : k_lusgs_sweep_staged;
  static int staged_max_threads[2] = {0, 0};  // limited by the kernel's registers
  if (!staged_max_threads[f]) {
    cudaFuncAttributes fa;
    CK(cudaFuncGetAttributes(&fa, staged));
    staged_max_threads[f] = fa.maxThreadsPerBlock;
  }
  // consumer threads: one per row of every node of the largest plane
  auto consumers_for = [](int p) { return (5 * std::max(p, 1) + 31) / 32 * 32; };
  if (nst >= 2 && consumers_for(pmax) + 32 > staged_max_threads[f]) nst = 0;
  // slab sweep when every block's slab rows fit one CTA; else the bulk
  // exchange when the planes fit the cluster
  SlabFit sf;
  const bool slabbed = g.tune.sweep_cl >= 2 && g.tune.sweep_x == 2 &&
                       (sf = slab_fit_for(host_views, nblk, g.tune.sweep_cl, 5)).ok;
  const bool bulk = !slabbed && g.tune.sweep_cl >= 2 && g.tune.sweep_x >= 1 && 5L * pmax <= 512L * g.tune.sweep_cl;
  if (slabbed) {
    // one cluster per block, each CTA one k-slab, pipelined plane by plane
    const int cl = g.tune.sweep_cl;
    const size_t smem = slab_smem(sf, 5);
    // slab planes of at most 256 rows take the variant with loads two steps ahead
    const bool deep = sf.T <= 256;
    auto kern = deep ? (f ? k_lusgs_sweep_slab2_f32 : k_lusgs_sweep_slab2) : (f ? k_lusgs_sweep_slab_f32 : k_lusgs_sweep_slab);
    if ((rc = prepare_slab(kern, f + (deep ? 3 : 0), smem, cl))) return rc;
    cudaError_t le = cudaSuccess;
    PROF(P_LUSGS_SWEEP,
         (le = launch_clusters(kern, nblk, cl, sf.T, smem, g.stream, sv, g.d_status, sf.So, sf.L, sf.D)));
    CK(le);
  } else if (bulk) {
    // one cluster per block, one thread per row of every node of the largest
    // plane; the plane values travel between the CTAs' shared memories
    const int cl = g.tune.sweep_cl;
    int threads = (int)std::max<long>(64, ((5L * pmax + cl - 1) / cl + 31) / 32 * 32);
    const size_t smem = (size_t)2 * ((size_t)cl * threads + 2) * sizeof(double);
    // clusters of 16 CTAs (at most 256 threads each on planes that fit them)
    // take the variant with loads two planes ahead; smaller clusters keep the
    // leaner one, which leaves room for two CTAs per SM when a batch has more
    // CTAs than SMs
    const bool deep = cl >= 16 && threads <= 256;
    // exchange 3: two CTAs per SM (80 registers) where the rows fit 384 threads
    const bool two = !deep && g.tune.sweep_x == 3 && threads <= 384;
    const int k = f + (deep ? 2 : two ? 4 : 0);
    auto kern = deep  ? (f ? k_lusgs_sweep_bulk2_f32 : k_lusgs_sweep_bulk2)
                : two ? (f ? k_lusgs_sweep_bulk_o2_f32 : k_lusgs_sweep_bulk_o2)
                      : (f ? k_lusgs_sweep_bulk_f32 : k_lusgs_sweep_bulk);
    if (smem > 48 * 1024 && smem > g.smem_bulk[k]) {
      CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      g.smem_bulk[k] = smem;
    }
    if (cl > 8 && !g.np_cluster[k]) {  // 16 CTAs: a non-portable cluster size
      CK(cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
      g.np_cluster[k] = true;
    }
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)(nblk * cl));
    lc.blockDim = dim3((unsigned)threads);
    lc.dynamicSmemBytes = smem;
    lc.stream = g.stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    cudaError_t le = cudaSuccess;
    PROF(P_LUSGS_SWEEP, (le = cudaLaunchKernelEx(&lc, kern, sv, g.d_status, g.tune.sweep_pf)));
    CK(le);
  } else if (g.tune.sweep_cl >= 2) {
    // one cluster of sweep_cl CTAs per block, one thread per row of every
    // node of the largest plane (at most 512 per CTA; more rows loop); the
    // exchange through L2 takes portable cluster sizes only (8 for 16)
    const int cl = std::min(8, g.tune.sweep_cl);
    int threads = (int)std::min<long>(512, std::max<long>(64, ((5L * pmax + cl - 1) / cl + 31) / 32 * 32));
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)(nblk * cl));
    lc.blockDim = dim3((unsigned)threads);
    lc.dynamicSmemBytes = 0;
    lc.stream = g.stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    cudaError_t le = cudaSuccess;
    PROF(P_LUSGS_SWEEP, (le = cudaLaunchKernelEx(&lc, f ? k_lusgs_sweep_cluster_f32 : k_lusgs_sweep_cluster, sv)));
    CK(le);
  } else if (nst >= 2) {
    int consumers = consumers_for(pmax);
    size_t smem = offs + ring + nst * stage + (2 * nst + 1) * 8;
    if (smem > 48 * 1024 && smem > g.smem_staged[f]) {
      CK(cudaFuncSetAttribute(staged, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      g.smem_staged[f] = smem;
    }
    PROF(P_LUSGS_SWEEP, (staged<<<nblk, consumers + 32, smem, g.stream>>>(sv, nst, g.d_status, g.spin_limit,
                                                                       g.stall_plane)));
  } else {
    auto global = f ? k_lusgs_sweep_global_f32 : k_lusgs_sweep_global;
    static int global_max_threads[2] = {0, 0};  // limited by the kernel's registers
    if (!global_max_threads[f]) {
      cudaFuncAttributes fa;
      CK(cudaFuncGetAttributes(&fa, global));
      global_max_threads[f] = fa.maxThreadsPerBlock / 32 * 32;
    }
    int threads = (int)std::min<long>(global_max_threads[f], std::max<long>(64, (2L * pmax + 31) / 32 * 32));
    PROF(P_LUSGS_SWEEP, (global<<<nblk, threads, 0, g.stream>>>(sv, 1, g.d_status)));
  }
  CKL();
  PROF(P_LUSGS_UPDATE, (k_lusgs_update<<<dim3(cdiv(maxN1, g.tune.ew), nblk), g.tune.ew, 0, g.stream>>>(views)));
  CKL();
  return AERO_OK;
}

int launch_index(const BlockView* views, int nblk, long maxN1) {
  PROF(P_INDEX, (k_plane_index<<<dim3(cdiv(maxN1, 256), nblk), 256, 0, g.stream>>>(views)));
  CKL();
  return AERO_OK;
}

// sa_model (sub_tur_sa.f90:7-122) on nblk views, on stream st (the library's
// stream when null); needs the hyperplane index.
// parts: 1 the length scale and the right-hand side (sa_rhs1/2/3; they read
// pri_v, amu, vor, dudx and the metrics), 2 the records and the sweeps (the
// records also read dt); 3 both.
int launch_sa(const BlockView* views, int nblk, long maxN, long maxN1, int pmax, const CaseConsts& cc,
              cudaStream_t st = nullptr, const BlockView* host_views = nullptr, int parts = 3) {
  if (!st) st = g.stream;
  if (parts & 1) {
    PROF_ON(P_FILL, st, (k_sa_length<<<dim3(cdiv(maxN, 256), nblk), 256, 0, st>>>(views, cc)));
    CKL();
    PROF_ON(P_SA_A, st, (k_sa_a<<<dim3(cdiv(maxN1, 256), nblk), 256, 0, st>>>(views, cc)));
    CKL();
    PROF_ON(P_SA_B, st,
            ((g.mixed ? k_sa_b_mixed : k_sa_b)<<<dim3(cdiv(maxN1, 128), nblk), 128, 0, st>>>(views, cc)));
    CKL();
  }
  if (!(parts & 2)) return AERO_OK;
  PROF_ON(P_SA_RECS, st, (k_sa_recs<<<dim3(cdiv(maxN1, 256), nblk), 256, 0, st>>>(views, cc)));
  CKL();
  SlabFit sf;
  if (g.tune.sa_cl >= 2 && (sf = slab_fit_for(host_views, nblk, g.tune.sa_cl, 1)).ok) {
    // one cluster per block, each CTA one k-slab, pipelined plane by plane
    const int cl = g.tune.sa_cl;
    const size_t smem = slab_smem(sf, 1);
    int rc = prepare_slab(k_sa_sweep_slab, 2, smem, cl);
    if (rc) return rc;
    cudaError_t le = cudaSuccess;
    PROF_ON(P_SA_SWEEP, st, (le = launch_clusters(k_sa_sweep_slab, nblk, cl, sf.T, smem, st, views, g.d_status,
                                                  sf.So, sf.L, sf.D)));
    CK(le);
    return AERO_OK;
  }
  size_t smem = (size_t)2 * std::max(pmax, 1) * sizeof(double);
  int threads = (int)std::min<long>(1024, std::max<long>(64, (pmax + 31) / 32 * 32));
  PROF_ON(P_SA_SWEEP, st, ((threads <= 768 ? k_sa_sweep_768 : k_sa_sweep)<<<nblk, threads, smem, st>>>(views)));
  CKL();
  return AERO_OK;
}

bool viscous_on() { return g.cc.solver == IFLAG_NSSOLVER; }
// DDES reads dudx, which the viscous kernel then stores
int ddes_on() { return g.cc.turbulence == IFLAG_SA && g.cc.des == IFLAG_DDES ? 1 : 0; }
bool sa_on() { return g.cc.turbulence == IFLAG_SA && g.cc.solver == IFLAG_NSSOLVER; }

int do_physical_bc() {
  int nb = (int)g.blocks.size();
  for (size_t L = 0; L + 1 < g.bc_lstart.size(); ++L) {
    const int first = g.bc_lstart[L], count = g.bc_lstart[L + 1] - first;
    PROF(P_BC, (k_physical_bc<<<dim3(cdiv(g.bc_lface[L], 128), count), 128, 0, g.stream>>>(
                    g.d_blocks, g.d_bc_ops, g.d_bc_list, first, g.cc)));
    CKL();
  }
  if (sa_on()) {
    PROF(P_SA_CLIP, (k_sa_clip<<<dim3(cdiv(g.max_box, 256), nb), 256, 0, g.stream>>>(g.d_blocks)));
    CKL();
  }
  return AERO_OK;
}
int do_halo() {
  if (g.nhalo == 0) return AERO_OK;
  int mode = g.cc.turbulence == IFLAG_SA ? HALO_Q_NUT : HALO_Q;
  PROF(P_HALO, (k_halo<<<cdiv(g.nhalo, 256), 256, 0, g.stream>>>(g.d_blocks, g.d_halo, g.nhalo, mode)));
  CKL();
  return AERO_OK;
}
int do_average1() {
  if (g.navg_src == 0) return AERO_OK;
  PROF(P_AVG_GATHER, (k_avg_gather<<<cdiv(g.navg_src, 256), 256, 0, g.stream>>>(
                         g.d_blocks, g.d_avg_src, g.navg_src, g.d_avg_buf, g.cc.turbulence == IFLAG_SA)));
  CKL();
  return AERO_OK;
}
int do_average2() {
  if (g.navg_dst == 0) return AERO_OK;
  PROF(P_AVG_APPLY, (k_avg_apply<<<cdiv(g.navg_dst, 256), 256, 0, g.stream>>>(
                        g.d_blocks, g.d_avg_dst, g.navg_dst, g.d_avg_buf, g.cc.turbulence == IFLAG_SA)));
  CKL();
  return AERO_OK;
}
int do_residual(double* d_out7, cudaStream_t st = nullptr) {
  if (!st) st = g.stream;
  int nb = (int)g.blocks.size();
  PROF_ON(P_RESID_PART, st, (k_residual_partial<<<dim3(g.resid_ctas, nb), 256, 0, st>>>(g.d_blocks, g.d_part, sa_on())));
  CKL();
  PROF_ON(P_RESID_FINAL, st, (k_residual_final<<<1, 256, 0, st>>>(g.d_part, (long)g.resid_ctas * nb,
                                                                    g.totalnodes, d_out7, g.d_status)));
  CKL();
  return AERO_OK;
}
int do_getpri_all() {
  return launch_getpri(g.d_blocks, (int)g.blocks.size(), g.max_box, g.cc);
}

// One iteration of main.f90:343-447 over every block.  main.f90:446 recomputes
// the primitives at the end of an iteration from the same q that :357 uses at
// the start of the next one, so the device computes them once, at the start;
// aero_step recomputes them after its last iteration so the state it leaves
// matches the reference's.
// crank2nd on nblk views (sub_timeadvancement_2ndcrank.f90): dual-time rhs,
// dq = 0, the i, j, k line recurrences, q += dq/inv_j.
int launch_crank(const BlockView* views, int nblk, long maxN, long maxN1, const Box* lines, const CaseConsts& cc) {
  PROF(P_CRANK, (k_crank_rhs<<<dim3(cdiv(maxN1, 256), nblk), 256, 0, g.stream>>>(views)));
  CKL();
  PROF(P_CRANK, (k_fill<<<dim3(cdiv(maxN, 256), nblk), 256, 0, g.stream>>>(views, F_FVH, 5, 0.0)));
  CKL();
  const long nl[3] = {(long)lines->ny() * lines->nz(), (long)lines->nx() * lines->nz(), (long)lines->nx() * lines->ny()};
  // 2-D (sub_timeadvancement_2ndcrank.f90:335): no k lines
  for (int d = 0; d < (cc.dimension == IFLAG_2D ? 2 : 3); ++d) {
    PROF(P_CRANK, (k_crank_sweep<<<dim3(cdiv(nl[d], 64), nblk), 64, 0, g.stream>>>(views, d, cc.gamma)));
    CKL();
  }
  PROF(P_CRANK, (k_crank_update<<<dim3(cdiv(maxN1, 256), nblk), 256, 0, g.stream>>>(views)));
  CKL();
  return AERO_OK;
}

bool crank_on() { return g.cc.time == IFLAG_UNSTEADY; }

// main.f90:450-573: three dual-time sub-iterations, then update_q0, SA and
// the closing BCs / halo / averaging (the primitives are recomputed by the
// caller, as after the implicit path).  find_dt's unsteady branch leaves dt
// unchanged, so it launches nothing here.
int do_iteration_crank() {
  int nb = (int)g.blocks.size();
  int rc;
  for (int sub = 1; sub <= 3; ++sub) {
    if ((rc = do_physical_bc())) return rc;
    if ((rc = do_halo())) return rc;
    if ((rc = do_average1())) return rc;
    if ((rc = do_average2())) return rc;
    if ((rc = do_getpri_all())) return rc;
    if ((rc = launch_inviscid(g.d_blocks, nb, g.max_box, g.max_b1, g.max_b1_face, g.cc, nullptr,
                              !g.rhsi_ghosts_zero)))
      return rc;
    g.rhsi_ghosts_zero = true;
    if (viscous_on() && (rc = launch_viscous(g.d_blocks, nb, g.max_b0, g.cc, ddes_on()))) return rc;
    if ((rc = launch_crank(g.d_blocks, nb, g.max_box, g.max_b1, &g.max_b1_box, g.cc))) return rc;
  }
  PROF(P_CRANK, (k_update_q0<<<dim3(cdiv(g.max_b0, 256), nb), 256, 0, g.stream>>>(g.d_blocks)));
  CKL();
  if (sa_on() && (rc = launch_sa(g.d_blocks, nb, g.max_box, g.max_b1, g.pmax_all, g.cc))) return rc;
  if ((rc = do_physical_bc())) return rc;
  if ((rc = do_halo())) return rc;
  if ((rc = do_average1())) return rc;
  if ((rc = do_average2())) return rc;
  return AERO_OK;
}

// With resid_beside, the residual norm of the iteration (rhs, dt, inv_j and
// sa_rhs, none of which is written after k_lusgs_prep and sa_model's rhs) is
// computed on the second stream beside the LU-SGS sweeps, into g.d_out, and
// g.ev_resid marks its end.
// With retirement on: every block whose status word is non-zero stops (its
// live flag drops to 0 for the whole step).
int do_retire() {
  if (!g.retire) return AERO_OK;
  const int nb = (int)g.blocks.size();
  PROF(P_BC, (k_retire<<<cdiv(nb, 128), 128, 0, g.stream>>>(g.d_bstat, g.d_live, nb)));
  CKL();
  return AERO_OK;
}

int do_iteration(bool want_dt_minmax, bool resid_beside = false) {
  int rc;
  if ((rc = do_retire())) return rc;
  if (crank_on()) return do_iteration_crank();
  int nb = (int)g.blocks.size();
  if ((rc = do_getpri_all())) return rc;
  // inviscid_flux_1 (rhsi and its face scratch) beside viscous_flux and
  // find_dt (rhsv, amu, vor, dudx, tao, their scratch, dt): neither side reads
  // what the other writes
  CK(cudaEventRecord(g.ev_fork2, g.stream));
  CK(cudaStreamWaitEvent(g.stream2, g.ev_fork2, 0));
  if ((rc = launch_inviscid(g.d_blocks, nb, g.max_box, g.max_b1, g.max_b1_face, g.cc, g.stream2,
                            !g.rhsi_ghosts_zero)))
    return rc;
  g.rhsi_ghosts_zero = true;
  CK(cudaEventRecord(g.ev_join2, g.stream2));
  // the LU-SGS radii and off-diagonal blocks (q, primitives, metrics) beside
  // both: nothing before the sweeps writes what they read or reads what they
  // write
  CK(cudaStreamWaitEvent(g.stream3, g.ev_fork2, 0));
  if ((rc = launch_implicit_blocks(g.d_blocks, nb, g.max_ext, g.max_b1, g.cc, g.stream3))) return rc;
  CK(cudaEventRecord(g.ev_join3, g.stream3));
  // viscous part a, then find_dt (it reads the viscosity part a forms);
  // sa_model runs on a fourth stream: it reads pri_v, amu, dudx, vor, dt and
  // the metrics and writes nut, sa_rhs and its own scratch, none of which the
  // rest of the mean-flow iteration (find_dt, viscous part b, implicit1st)
  // reads or writes, so it runs beside all of them, its right-hand side from
  // viscous part a on and its records (which read dt) from find_dt on
  if (viscous_on() && (rc = launch_viscous_a(g.d_blocks, nb, g.max_b0, g.cc, ddes_on()))) return rc;
  const bool sa = sa_on();
  if (sa) {
    CK(cudaEventRecord(g.ev_fork, g.stream));
    CK(cudaStreamWaitEvent(g.stream4, g.ev_fork, 0));
    if ((rc = launch_sa(g.d_blocks, nb, g.max_box, g.max_b1, g.pmax_all, g.cc, g.stream4, nullptr, 1))) return rc;
  }
  if ((rc = launch_find_dt(g.d_blocks, nb, g.max_box, g.cc))) return rc;
  if (want_dt_minmax && (rc = launch_dt_minmax(g.d_blocks, nb - 1, g.d_out + 7))) return rc;
  if (sa) {
    CK(cudaEventRecord(g.ev_dt, g.stream));
    CK(cudaStreamWaitEvent(g.stream4, g.ev_dt, 0));
    if ((rc = launch_sa(g.d_blocks, nb, g.max_box, g.max_b1, g.pmax_all, g.cc, g.stream4, nullptr, 2))) return rc;
    CK(cudaEventRecord(g.ev_join, g.stream4));
  }
  if (viscous_on() && (rc = launch_viscous_b(g.d_blocks, nb, g.max_b0, g.cc))) return rc;
  CK(cudaStreamWaitEvent(g.stream, g.ev_join2, 0));
  CK(cudaStreamWaitEvent(g.stream, g.ev_join3, 0));
  if ((rc = launch_implicit(g.d_blocks, nb, g.max_ext, g.max_b1, g.pmax_all, g.hmax_all, g.cc,
                            resid_beside ? g.ev_prep : nullptr, false, g.d_blocks_chain)))
    return rc;
  if (resid_beside) {
    // the residual norm reads rhs (k_lusgs_prep), dt, inv_j and sa_rhs: with
    // SA on the SA stream after its kernels, otherwise on the second stream
    cudaStream_t rs = sa ? g.stream4 : g.stream2;
    CK(cudaStreamWaitEvent(rs, g.ev_prep, 0));
    if ((rc = do_residual(g.d_out, rs))) return rc;
    CK(cudaEventRecord(g.ev_resid, rs));
  }
  if (sa) CK(cudaStreamWaitEvent(g.stream, g.ev_join, 0));
  if ((rc = do_physical_bc())) return rc;
  if ((rc = do_halo())) return rc;
  if ((rc = do_average1())) return rc;
  if ((rc = do_average2())) return rc;
  return AERO_OK;
}

// Case constants from Control.in's flags and values; the nondimensional
// freestream of sub_init_flowfield.f90:30-39.
CaseConsts consts_from(const int* iflags, const double* params) {
  CaseConsts c{};
  const double pi = 3.1415926535897932;
  c.gamma = 1.4; c.prl = 0.72; c.prt = 0.90;
  double ma = params[0];
  c.re = params[1]; c.tinf = params[2]; c.cfl = params[4]; c.nutinf = params[6];
  c.d_0 = 1.0; c.u_0 = 1.0;
  double t_0 = 1.0;
  c.p_0 = c.d_0 * t_0 / c.gamma / ma / ma;
  c.c_0 = std::sqrt(t_0) / ma;
  c.cv = 1.0 / c.gamma / (c.gamma - 1.0) / ma / ma;
  c.aoa = params[3] * pi / 180.0;
  c.cos_aoa = std::cos(c.aoa);
  c.sin_aoa = std::sin(c.aoa);
  c.dimension = iflags[0]; c.solver = iflags[1]; c.time = iflags[2];
  c.turbulence = iflags[4]; c.des = iflags[5]; c.bufferLength = iflags[6];
  c.inviscid = iflags[7];
  return c;
}

// One time step as aero_step runs it: the iteration, the closing primitives
// and the residual norm (into g.d_out; beside the sweeps for the implicit
// update, after the step for the dual-time one).
int step_once() {
  int rc;
  const bool beside = !crank_on();
  if ((rc = do_iteration(false, beside))) return rc;
  if ((rc = do_getpri_all())) return rc;
  if (!beside) return do_residual(g.d_out);
  CK(cudaStreamWaitEvent(g.stream, g.ev_resid, 0));
  return AERO_OK;
}

void graph_release() {
  if (g.graph_exec) cudaGraphExecDestroy(g.graph_exec);
  g.graph_exec = nullptr;
  g.graph_kernels = 0;
}

// step_once, replayed from a CUDA graph captured on first use when graphs are
// on (and profiling is off); the graph is captured again after any change of
// precision mode or launch shapes.
int run_step() {
  if (!g.graph_want || gp.on) return step_once();
  if (!g.graph_exec) {
    unsigned long long before = gp.launches;
    CK(cudaStreamBeginCapture(g.stream, cudaStreamCaptureModeRelaxed));
    int rc = step_once();
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(g.stream, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (e != cudaSuccess) return fail(AERO_ERR_CUDA, "stream capture failed: %s", cudaGetErrorString(e));
    // each kernel node keeps the priority of the stream it was captured from
    e = cudaGraphInstantiate(&g.graph_exec, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      g.graph_exec = nullptr;
      return fail(AERO_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(e));
    }
    g.graph_kernels = gp.launches - before;
    gp.launches = before;
  }
  CK(cudaGraphLaunch(g.graph_exec, g.stream));
  gp.launches += g.graph_kernels;
  return AERO_OK;
}

}  // namespace

namespace aero {
// Error reporting for the C-ABI entries defined in other files of the library.
int set_last_error(int code, const char* msg) { return fail(code, "%s", msg); }
}  // namespace aero

// =================================================================== C ABI
extern "C" {

const char* aero_last_error(void) { return g.err.c_str(); }

int aero_init(int device) {
  if (g.inited) return AERO_OK;
  CK(cudaSetDevice(device));
  for (int f = 0; f < 2; ++f) g.smem_staged[f] = 0;
  for (int f = 0; f < 6; ++f) {
    g.smem_bulk[f] = 0;
    g.np_cluster[f] = false;
  }
  // The mean-flow chain (the library's stream, fed by the inviscid and the
  // block-record streams) is the iteration's critical path; the SA stream,
  // which has slack beside it, takes the lowest priority, so where both have
  // CTAs waiting for an SM the block scheduler serves the mean flow first.
  int prio_low = 0, prio_high = 0;
  CK(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
  CK(cudaStreamCreateWithPriority(&g.stream, cudaStreamNonBlocking, prio_high));
  CK(cudaStreamCreateWithPriority(&g.stream2, cudaStreamNonBlocking, prio_high));
  CK(cudaStreamCreateWithPriority(&g.stream3, cudaStreamNonBlocking, prio_high));
  CK(cudaStreamCreateWithPriority(&g.stream4, cudaStreamNonBlocking, prio_low));
  CK(cudaEventCreateWithFlags(&g.ev_join3, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&g.ev_dt, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&g.ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&g.ev_join, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&g.ev_fork2, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&g.ev_join2, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&g.ev_prep, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&g.ev_resid, cudaEventDisableTiming));
  // word 0: the status word; words 1..6: the first cluster-sweep wait that
  // gave up (note_timeout, aero_timeout_site)
  CK(cudaMalloc(&g.d_status, 8 * sizeof(unsigned)));
  CK(cudaMemset(g.d_status, 0, 8 * sizeof(unsigned)));
  CK(cudaMalloc(&g.d_out, 16 * sizeof(double)));
  CK(cudaMallocHost(&g.h_out, 16 * sizeof(double)));
  g.device = device;
  g.inited = true;
  return AERO_OK;
}

static void release_case() {
  for (auto& H : g.blocks) {
    for (int f = 0; f < kNumPublicFields; ++f)
      if (H.pinned[f]) cudaHostUnregister(H.host[f]);
    if (H.ws) cudaFree(H.ws);
    H.ws = nullptr;
  }
  g.blocks.clear();
  g.registry.clear();
  g.rhsi_ghosts_zero = false;
  cudaFree(g.arena); g.arena = nullptr;
  cudaFree(g.d_blocks); g.d_blocks = nullptr;
  cudaFree(g.d_blocks_chain); g.d_blocks_chain = nullptr;
  cudaFree(g.d_bc_ops); g.d_bc_ops = nullptr;
  cudaFree(g.d_bc_list); g.d_bc_list = nullptr;
  g.bc_lstart.clear();
  g.bc_lface.clear();
  cudaFree(g.d_halo); g.d_halo = nullptr;
  cudaFree(g.d_avg_src); g.d_avg_src = nullptr;
  cudaFree(g.d_avg_dst); g.d_avg_dst = nullptr;
  cudaFree(g.d_avg_buf); g.d_avg_buf = nullptr;
  cudaFree(g.d_part); g.d_part = nullptr;
  cudaFree(g.d_walls); g.d_walls = nullptr;
  cudaFree(g.d_fpart); g.d_fpart = nullptr;
  cudaFree(g.d_surf); g.d_surf = nullptr;
  cudaFree(g.d_surf_out); g.d_surf_out = nullptr;
  g.surf.clear();
  g.nsurf = 0;
  cudaFree(g.d_ccb); g.d_ccb = nullptr;
  graph_release();
  cudaFree(g.d_resid_blocks); g.d_resid_blocks = nullptr;
  cudaFree(g.d_bstat); g.d_bstat = nullptr;
  cudaFree(g.d_live); g.d_live = nullptr;
  g.retire = false;
  g.nwall = 0;
  g.nquad = 0;
  g.views.clear();
  g.setup = false;
}

int aero_finalize(void) {
  if (!g.inited) return AERO_OK;
  cudaStreamSynchronize(g.stream);
  release_case();
  cudaFree(g.d_staging); g.d_staging = nullptr; g.staging_doubles = 0;
  cudaFree(g.t_arena); g.t_arena = nullptr; g.t_doubles = 0;
  cudaFree(g.d_tview); g.d_tview = nullptr;
  cudaFree(g.t_ws); g.t_ws = nullptr; g.t_ws_bytes = 0;
  cudaFree(g.d_status); g.d_status = nullptr;
  cudaFree(g.d_out); g.d_out = nullptr;
  cudaFreeHost(g.h_out); g.h_out = nullptr;
  cudaStreamDestroy(g.stream); g.stream = nullptr;
  cudaStreamDestroy(g.stream2); g.stream2 = nullptr;
  cudaStreamDestroy(g.stream3); g.stream3 = nullptr;
  cudaStreamDestroy(g.stream4); g.stream4 = nullptr;
  cudaEventDestroy(g.ev_join3); g.ev_join3 = nullptr;
  cudaEventDestroy(g.ev_fork); g.ev_fork = nullptr;
  cudaEventDestroy(g.ev_dt); g.ev_dt = nullptr;
  cudaEventDestroy(g.ev_join); g.ev_join = nullptr;
  cudaEventDestroy(g.ev_fork2); g.ev_fork2 = nullptr;
  cudaEventDestroy(g.ev_join2); g.ev_join2 = nullptr;
  cudaEventDestroy(g.ev_prep); g.ev_prep = nullptr;
  cudaEventDestroy(g.ev_resid); g.ev_resid = nullptr;
  for (cudaEvent_t e : g.xfer_ev) cudaEventDestroy(e);
  g.xfer_ev.clear();
  g.inited = false;
  g.configured = false;
  // execution options of the finished run
  g.mixed = false;
  g.spin_limit = kPollBudgetMax;
  g.stall_plane = -1;
  g.tune = State::Tune{};
  g.graph_want = false;
  g.tuning = State{}.tuning;
  return AERO_OK;
}

int aero_set_block_params(int m, const double* params) {
  int rc = need_init();
  if (rc) return rc;
  if (!g.configured) return fail(AERO_ERR_STATE, "aero_configure has not been called");
  if (g.setup) return fail(AERO_ERR_STATE, "block parameters must be set before aero_finish_setup");
  if (m < 1 || m > (int)g.blocks.size() || !g.blocks[m - 1].used)
    return fail(AERO_ERR_ARG, "block %d is not registered", m);
  if (!(params[0] > 0.0) || !(params[1] > 0.0) || !(params[4] > 0.0))
    return fail(AERO_ERR_ARG, "block %d: ma, re and cfl must be positive", m);
  HostBlock& H = g.blocks[m - 1];
  std::memcpy(H.params, params, sizeof H.params);
  H.cc = consts_from(g.iflags, params);
  H.own_params = true;
  return AERO_OK;
}

int aero_residual_blocks(double* out7) {
  int rc = need_setup();
  if (rc) return rc;
  int nb = (int)g.blocks.size();
  PROF(P_RESID_PART, (k_residual_partial<<<dim3(g.resid_ctas, nb), 256, 0, g.stream>>>(g.d_blocks, g.d_part, sa_on())));
  CKL();
  PROF(P_RESID_FINAL, (k_residual_final_blocks<<<nb, 256, 0, g.stream>>>(g.d_blocks, g.d_part, g.resid_ctas,
                                                                         g.d_resid_blocks, g.d_status)));
  CKL();
  CK(cudaMemcpyAsync(out7, g.d_resid_blocks, (size_t)7 * nb * sizeof(double), cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  return AERO_OK;
}

int aero_use_graphs(int on) {
  int rc = need_init();
  if (rc) return rc;
  g.graph_want = on != 0;
  if (!g.graph_want) graph_release();
  return AERO_OK;
}

// Whether the bulk-exchange sweep can run as clusters of 16 CTAs: the
// largest plane's rows fit 16 CTAs of at most 512 threads, and the device can
// hold at least one such cluster (a non-portable cluster size).
bool bulk_cluster16_fits() {
  if (!g.setup || 5L * g.pmax_all > 512L * 16) return false;
  const int cl = 16;
  const int threads = (int)std::max<long>(64, ((5L * g.pmax_all + cl - 1) / cl + 31) / 32 * 32);
  const size_t smem = (size_t)2 * ((size_t)cl * threads + 2) * sizeof(double);
  for (int f = 0; f < 2; ++f) {
    const int k = f + (threads <= 256 ? 2 : 0);
    auto kern = threads <= 256 ? (f ? k_lusgs_sweep_bulk2_f32 : k_lusgs_sweep_bulk2)
                               : (f ? k_lusgs_sweep_bulk_f32 : k_lusgs_sweep_bulk);
    if (cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) break;
    g.np_cluster[k] = true;
    if (smem > 48 * 1024 && smem > g.smem_bulk[k]) {
      if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) break;
      g.smem_bulk[k] = smem;
    }
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)cl);
    lc.blockDim = dim3((unsigned)threads);
    lc.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = (unsigned)cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &lc) != cudaSuccess || n < 1) {
      cudaGetLastError();
      return false;
    }
    if (f == 1) return true;
  }
  cudaGetLastError();
  return false;
}

// Whether a slab sweep can run as clusters of 16 CTAs on this device for the
// registered blocks (rows = 5: the mean-flow sweep; 1: the SA sweep).
bool slab_cluster16_fits(int rows) {
  if (!g.setup) return false;
  const SlabFit sf = slab_fit_for(nullptr, 0, 16, rows);
  if (!sf.ok) return false;
  const size_t smem = slab_smem(sf, rows);
  const int nk = rows == 5 ? 2 : 1;
  const bool deep = rows == 5 && sf.T <= 256;
  for (int k = 0; k < nk; ++k) {
    const int idx = rows == 5 ? k + (deep ? 3 : 0) : 2;
    void (*kern)(const BlockView*, unsigned*, int, int, int) =
        rows == 5 ? (deep ? (k ? k_lusgs_sweep_slab2_f32 : k_lusgs_sweep_slab2)
                          : (k ? k_lusgs_sweep_slab_f32 : k_lusgs_sweep_slab))
                  : k_sa_sweep_slab;
    if (prepare_slab(kern, idx, smem, 16) != AERO_OK) {
      cudaGetLastError();
      return false;
    }
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(16u);
    lc.blockDim = dim3((unsigned)sf.T);
    lc.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 16;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    lc.attrs = at;
    lc.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, kern, &lc) != cudaSuccess || n < 1) {
      cudaGetLastError();
      return false;
    }
  }
  return true;
}

const char* exchange_name(int x) { return x == 3 ? "shared2" : x == 2 ? "slab" : x == 1 ? "shared" : "l2"; }

void set_tuning_text() {
  char buf[280];
  std::snprintf(buf, sizeof buf,
                "inviscid_tile=%d elementwise_threads=%d viscous_threads=%d mats_threads=%d sweep_stages<=%d "
                "sweep_cluster=%d sweep_exchange=%s sa_sweep_cluster=%d register_bound=%d sweep_prefetch=%d",
                g.tune.inv_tile, g.tune.ew, g.tune.visc, g.tune.mats, g.tune.nst_max, std::max(1, g.tune.sweep_cl),
                exchange_name(g.tune.sweep_x), std::max(1, g.tune.sa_cl), g.tune.bound, g.tune.sweep_pf);
  g.tuning = buf;
}

int aero_autotune(int iters) {
  int rc = need_setup();
  if (rc) return rc;
  if (iters < 1) return fail(AERO_ERR_ARG, "iters = %d", iters);
  // the solution state that carries over between steps
  const int kState[] = {F_Q, F_NUT, F_Q0, F_DT, F_AMU};
  size_t per_block = 0;
  for (int f : kState) per_block += (size_t)field_nc(f);
  int nb = (int)g.blocks.size();
  size_t total = 0;
  for (int m = 0; m < nb; ++m) total += per_block * g.views[m].plane;
  double* snap = nullptr;
  CK(cudaMalloc(&snap, total * sizeof(double)));
  auto copy_state = [&](bool save) -> int {
    size_t off = 0;
    for (int m = 0; m < nb; ++m)
      for (int f : kState) {
        size_t n = (size_t)field_nc(f) * g.views[m].plane;
        double* dev = g.views[m].f[f];
        CK(cudaMemcpyAsync(save ? snap + off : dev, save ? dev : snap + off, n * sizeof(double),
                           cudaMemcpyDeviceToDevice, g.stream));
        off += n;
      }
    return AERO_OK;
  };
  if ((rc = copy_state(true))) { cudaFree(snap); return rc; }
  bool graphs = g.graph_want;
  g.graph_want = false;
  graph_release();
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  auto time_steps = [&](double& ms) -> int {
    int r;
    if ((r = step_once())) return r;  // warm
    CK(cudaEventRecord(a, g.stream));
    for (int x = 0; x < iters; ++x)
      if ((r = step_once())) return r;
    CK(cudaEventRecord(b, g.stream));
    CK(cudaEventSynchronize(b));
    float f = 0.f;
    CK(cudaEventElapsedTime(&f, a, b));
    ms = f;
    return AERO_OK;
  };
  // the sweep's cluster size and exchange are one knob (value 4 * ctas +
  // exchange), since the exchanges are only eligible for some sizes
  int sweep_mode = 4 * g.tune.sweep_cl + g.tune.sweep_x;
  struct Knob { int* v; std::vector<int> cand; };
  std::vector<Knob> knobs = {{&g.tune.inv_tile, {0, -6, -8, -10, 32, 64, 128}}, {&g.tune.ew, {128, 256, 512}},
                             {&g.tune.visc, {64, 128, 256}}, {&g.tune.mats, {64, 128, 256}},
                             {&g.tune.nst_max, {2, 3, 4}},
                             {&sweep_mode, {0, 8, 16, 32, 9, 17, 33, 10, 18, 34, 11, 19, 35}},
                             {&g.tune.bound, {0, 1}}, {&g.tune.sweep_pf, {2, 3, 4}}};
  for (Knob& k : knobs)
    if (k.v == &sweep_mode) {
      if (bulk_cluster16_fits()) k.cand.push_back(65);   // 16 CTAs, bulk exchange
      if (slab_cluster16_fits(5)) k.cand.push_back(66);  // 16 CTAs, slabs
    }
  if (sa_on()) {
    knobs.push_back({&g.tune.sa_cl, {0, 2, 4, 8}});
    if (slab_cluster16_fits(1)) knobs.back().cand.push_back(16);
  }
  for (Knob& k : knobs) {
    int best = *k.v;
    double best_ms = 1e300;
    for (int c : k.cand) {
      *k.v = c;
      g.tune.sweep_cl = sweep_mode / 4;
      g.tune.sweep_x = sweep_mode % 4;
      double ms = 0;
      if ((rc = time_steps(ms))) break;
      if (ms < best_ms) { best_ms = ms; best = c; }
    }
    *k.v = best;
    g.tune.sweep_cl = sweep_mode / 4;
    g.tune.sweep_x = sweep_mode % 4;
    if (rc) break;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  int rc2 = copy_state(false);
  CK(cudaStreamSynchronize(g.stream));
  cudaFree(snap);
  g.graph_want = graphs;
  if (rc) return rc;
  if (rc2) return rc2;
  set_tuning_text();
  return AERO_OK;
}

const char* aero_tuning(void) { return g.tuning.c_str(); }

int aero_set_tuning(int inv_tile, int ew, int visc, int mats, int nst_max) {
  int rc = need_init();
  if (rc) return rc;
  auto in = [](int v, std::initializer_list<int> ok) { return std::find(ok.begin(), ok.end(), v) != ok.end(); };
  if (!in(inv_tile, {-10, -8, -6, 0, 32, 64, 128}) || !in(ew, {128, 256, 512}) || !in(visc, {64, 128, 256}) ||
      !in(mats, {64, 128, 256}) || !in(nst_max, {2, 3, 4}))
    return fail(AERO_ERR_ARG, "launch shape %d/%d/%d/%d/%d is not one the autotuner offers", inv_tile, ew, visc, mats,
                nst_max);
  g.tune.inv_tile = inv_tile;
  g.tune.ew = ew;
  g.tune.visc = visc;
  g.tune.mats = mats;
  g.tune.nst_max = nst_max;
  graph_release();
  set_tuning_text();
  return AERO_OK;
}

int aero_set_poll_budget(long long polls) {
  int rc = need_init();
  if (rc) return rc;
  if (polls < 0 || polls > kPollBudgetMax)
    return fail(AERO_ERR_ARG, "poll budget %lld is outside 0..%ld", polls, kPollBudgetMax);
  g.spin_limit = (long)polls;
  graph_release();
  return AERO_OK;
}

int aero_inject_sweep_stall(int plane) {
  int rc = need_init();
  if (rc) return rc;
  if (plane < -1) return fail(AERO_ERR_ARG, "stall plane %d is neither -1 nor a plane index", plane);
  g.stall_plane = plane;
  graph_release();
  return AERO_OK;
}

int aero_set_sweep_exchange(int mode) {
  int rc = need_init();
  if (rc) return rc;
  if (mode < 0 || mode > 3)
    return fail(AERO_ERR_ARG,
                "sweep exchange %d is not 0 (L2), 1 (shared memory), 2 (pipelined k-slabs) or 3 (shared memory, "
                "two CTAs per SM)", mode);
  g.tune.sweep_x = mode;
  graph_release();
  set_tuning_text();
  return AERO_OK;
}

int aero_set_sweep_cluster(int ctas) {
  int rc = need_init();
  if (rc) return rc;
  if (ctas != 1 && ctas != 2 && ctas != 4 && ctas != 8 && ctas != 16)
    return fail(AERO_ERR_ARG, "sweep cluster of %d CTAs is not 1, 2, 4, 8 or 16", ctas);
  if (ctas == 16 && !bulk_cluster16_fits() && !slab_cluster16_fits(5))
    return fail(AERO_ERR_ARG, "a cluster of 16 sweep CTAs does not fit this device or these blocks "
                              "(16 CTAs take the bulk or the slab exchange only)");
  g.tune.sweep_cl = ctas == 1 ? 0 : ctas;
  graph_release();
  set_tuning_text();
  return AERO_OK;
}

int aero_set_sweep_prefetch(int planes) {
  int rc = need_init();
  if (rc) return rc;
  if (planes < 2 || planes > 4) return fail(AERO_ERR_ARG, "sweep prefetch distance %d is outside 2..4", planes);
  g.tune.sweep_pf = planes;
  graph_release();
  set_tuning_text();
  return AERO_OK;
}

int aero_set_register_bound(int on) {
  int rc = need_init();
  if (rc) return rc;
  if (on != 0 && on != 1) return fail(AERO_ERR_ARG, "register bound %d is not 0 or 1", on);
  g.tune.bound = on;
  graph_release();
  set_tuning_text();
  return AERO_OK;
}

int aero_set_sa_sweep_cluster(int ctas) {
  int rc = need_init();
  if (rc) return rc;
  if (ctas != 1 && ctas != 2 && ctas != 4 && ctas != 8 && ctas != 16)
    return fail(AERO_ERR_ARG, "SA sweep cluster of %d CTAs is not 1, 2, 4, 8 or 16", ctas);
  if (ctas == 16 && !slab_cluster16_fits(1))
    return fail(AERO_ERR_ARG, "a cluster of 16 SA sweep CTAs does not fit this device or these blocks");
  g.tune.sa_cl = ctas == 1 ? 0 : ctas;
  graph_release();
  set_tuning_text();
  return AERO_OK;
}

int aero_set_precision(int mode) {
  if (mode != 0 && mode != 1) return fail(AERO_ERR_ARG, "precision mode %d is not 0 (FP64) or 1 (mixed)", mode);
  if (g.mixed != (mode == 1)) graph_release();
  g.mixed = mode == 1;
  return AERO_OK;
}

int aero_get_status(unsigned* status) {
  int rc = need_init();
  if (rc) return rc;
  unsigned h = 0;
  CK(cudaMemcpyAsync(&h, g.d_status, sizeof(unsigned), cudaMemcpyDeviceToHost, g.stream));
  CK(cudaMemsetAsync(g.d_status, 0, sizeof(unsigned), g.stream));
  CK(cudaStreamSynchronize(g.stream));
  *status = h;
  return AERO_OK;
}

int aero_timeout_site(int* out5) {
  int rc = need_init();
  if (rc) return rc;
  unsigned h[7] = {0, 0, 0, 0, 0, 0, 0};
  CK(cudaMemcpyAsync(h, g.d_status, 7 * sizeof(unsigned), cudaMemcpyDeviceToHost, g.stream));
  CK(cudaMemsetAsync(g.d_status + 1, 0, 6 * sizeof(unsigned), g.stream));
  CK(cudaStreamSynchronize(g.stream));
  for (int x = 0; x < 5; ++x) out5[x] = h[1] ? (int)h[2 + x] : -1;
  return AERO_OK;
}

int aero_get_block_status(unsigned* out) {
  int rc = need_setup();
  if (rc) return rc;
  const int nb = (int)g.blocks.size();
  CK(cudaMemcpyAsync(out, g.d_bstat, nb * sizeof(unsigned), cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  return AERO_OK;
}

int aero_clear_block_status(void) {
  int rc = need_setup();
  if (rc) return rc;
  const int nb = (int)g.blocks.size();
  std::vector<int> ones(nb, 1);
  CK(cudaMemsetAsync(g.d_bstat, 0, nb * sizeof(unsigned), g.stream));
  CK(cudaMemcpyAsync(g.d_live, ones.data(), nb * sizeof(int), cudaMemcpyHostToDevice, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  return AERO_OK;
}

int aero_set_retirement(int on) {
  int rc = need_setup();
  if (rc) return rc;
  if ((on != 0) == g.retire) return AERO_OK;
  g.retire = on != 0;
  graph_release();  // the captured step gains or loses the refresh
  if (!g.retire) {
    const int nb = (int)g.blocks.size();
    std::vector<int> ones(nb, 1);
    CK(cudaMemcpyAsync(g.d_live, ones.data(), nb * sizeof(int), cudaMemcpyHostToDevice, g.stream));
    CK(cudaStreamSynchronize(g.stream));
  }
  return AERO_OK;
}

int aero_configure(const int* iflags, const double* params) {
  int rc = need_init();
  if (rc) return rc;
  if (iflags[0] != IFLAG_3D && iflags[0] != IFLAG_2D)
    return fail(AERO_ERR_ARG, "iflag_dimension=%d is not 2 or 3", iflags[0]);
  if (iflags[1] != IFLAG_NSSOLVER && iflags[1] != IFLAG_EULERSOLVER)
    return fail(AERO_ERR_ARG, "iflag_solver=%d is not 0 (NS) or 1 (Euler)", iflags[1]);
  bool steady_lusgs = iflags[2] == IFLAG_STEADY && iflags[3] == IFLAG_1STIMPLICIT;
  bool unsteady_crank = iflags[2] == IFLAG_UNSTEADY && iflags[3] == IFLAG_2NDCRANK;
  if (!steady_lusgs && !unsteady_crank)
    return fail(AERO_ERR_ARG,
                "iflag_time=%d/iflag_timeadvance=%d: supported are steady 1st-order implicit (0/2) and "
                "unsteady 2nd-order Crank-Nicolson (1/3)", iflags[2], iflags[3]);
  if (iflags[4] != IFLAG_LAMINAR && iflags[4] != IFLAG_SA)
    return fail(AERO_ERR_ARG, "Wrong turbulence model type is input!!! (%d)", iflags[4]);
  const bool scheme_ok = (iflags[7] == IFLAG_3RDWENO && iflags[6] == 2) ||
                         ((iflags[7] == IFLAG_5THWENO || iflags[7] == IFLAG_5THWCNS) && iflags[6] == 3);
  if (!scheme_ok)
    return fail(AERO_ERR_ARG,
                "bufferLength=%d/iflag_inviscid=%d: supported are the 3rd-order WENO with 2 layers and "
                "WENO5 (5) or WCNS5 (8) with 3", iflags[6], iflags[7]);
  if (iflags[5] != 0 && iflags[5] != IFLAG_DES97 && iflags[5] != IFLAG_DDES)
    return fail(AERO_ERR_ARG, "iflag_des=%d is not 0, 1 (DES97) or 2 (DDES)", iflags[5]);
  std::memcpy(g.iflags, iflags, sizeof g.iflags);
  std::memcpy(g.params, params, sizeof g.params);
  g.cc = consts_from(iflags, params);
  g.configured = true;
  return AERO_OK;
}

int aero_register_block(int m, const int* box18, int num_subface, const int* subfaces) {
  int rc = need_init();
  if (rc) return rc;
  if (g.setup) release_case();
  if (m < 1 || num_subface < 0) return fail(AERO_ERR_ARG, "bad block number %d", m);
  if ((int)g.blocks.size() < m) g.blocks.resize(m);
  HostBlock& H = g.blocks[m - 1];
  H = HostBlock();
  H.used = true;
  H.b = Box{box18[0], box18[1], box18[2], box18[3], box18[4], box18[5]};
  H.b0 = Box{box18[6], box18[7], box18[8], box18[9], box18[10], box18[11]};
  H.b1 = Box{box18[12], box18[13], box18[14], box18[15], box18[16], box18[17]};
  // Stencils reach two nodes along each direction and the updated box sits
  // inside the physical one; require at least 3 nodes per direction and
  // consistent nested boxes.  A 2-D block (iflag_dimension = 2) is the single
  // plane k = 1 in all three boxes (sub_init_allocatememory.f90:66-68,
  // :134-144).
  const Box &b = H.b, &b0 = H.b0, &b1 = H.b1;
  const bool plane = b0.nz() == 1;
  if (b0.nx() < 3 || b0.ny() < 3 || (!plane && b0.nz() < 3))
    return fail(AERO_ERR_ARG, "block %d: need at least 3 nodes per direction (one k-plane in 2-D)", m);
  if (plane && (b.ks != b0.ks || b.ke != b0.ke || b1.ks != b0.ks || b1.ke != b0.ke))
    return fail(AERO_ERR_ARG, "block %d: a 2-D block has the one plane k = %d in every index box", m, b0.ks);
  const int kg = plane ? 0 : 1;
  if (b.is > b0.is || b.ie < b0.ie || b.js > b0.js || b.je < b0.je || b.ks > b0.ks || b.ke < b0.ke ||
      b1.is < b.is + 1 || b1.ie > b.ie - 1 || b1.js < b.js + 1 || b1.je > b.je - 1 ||
      b1.ks < b.ks + kg || b1.ke > b.ke - kg || b1.is < b0.is - 0 || b1.ie > b0.ie)
    return fail(AERO_ERR_ARG, "block %d: index boxes are not nested as is <= is0 <= is1", m);
  for (int s = 0; s < num_subface; ++s) {
    const int* r = subfaces + 11 * s;
    H.subs.push_back(SubRow{r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9], r[10]});
  }
  return AERO_OK;
}

int aero_bind_field(int m, int field, double* host) {
  int rc = need_init();
  if (rc) return rc;
  if (m < 1 || m > (int)g.blocks.size() || !g.blocks[m - 1].used) return fail(AERO_ERR_ARG, "block %d not registered", m);
  if (field < 0 || field >= kNumPublicFields) return fail(AERO_ERR_ARG, "unknown field %d", field);
  HostBlock& H = g.blocks[m - 1];
  if (H.pinned[field]) cudaHostUnregister(H.host[field]);
  H.host[field] = host;
  H.pinned[field] = false;
  size_t bytes = (size_t)H.b.size() * field_nc(field) * sizeof(double);
  if (host && cudaHostRegister(host, bytes, cudaHostRegisterDefault) == cudaSuccess) H.pinned[field] = true;
  cudaGetLastError();  // an unpinnable array is still usable (pageable copies)
  if (host) g.registry[host] = std::make_pair(m - 1, field);
  return AERO_OK;
}

int aero_finish_setup(void) {
  int rc = need_init();
  if (rc) return rc;
  if (!g.configured) return fail(AERO_ERR_STATE, "aero_configure has not been called");
  int nb = (int)g.blocks.size();
  if (nb == 0) return fail(AERO_ERR_STATE, "no blocks registered");
  for (int m = 0; m < nb; ++m) {
    if (!g.blocks[m].used) return fail(AERO_ERR_ARG, "block %d missing (blocks must be 1..n)", m + 1);
    if ((g.blocks[m].b0.nz() == 1) != (g.cc.dimension == IFLAG_2D))
      return fail(AERO_ERR_ARG, "block %d: %s block in a %d-D case", m + 1,
                  g.blocks[m].b0.nz() == 1 ? "a one-plane" : "a 3-D", g.cc.dimension);
  }
  // topology tables
  std::vector<TopoBlock> tb(nb);
  for (int m = 0; m < nb; ++m) {
    tb[m].b = g.blocks[m].b; tb[m].b0 = g.blocks[m].b0; tb[m].b1 = g.blocks[m].b1;
    tb[m].subs = g.blocks[m].subs;
  }
  Topology topo;
  std::string why = build_topology(tb, g.cc.bufferLength, g.cc.solver, g.cc.dimension, topo);
  if (!why.empty()) return fail(AERO_ERR_ARG, "%s", why.c_str());
  // arena
  size_t total = 0;
  g.max_box = g.max_b0 = g.max_b1 = g.max_ext = 0;
  g.max_b1_box = Box{1, 0, 1, 0, 1, 0};
  g.max_b1_face = 0;
  g.totalnodes = 0;
  long max_b1 = 0;
  for (auto& H : g.blocks) {
    H.plane = round32(H.b.size());
    H.arena_off = total;
    total += view_doubles(H.plane);
    g.max_box = std::max(g.max_box, H.b.size());
    g.max_b0 = std::max(g.max_b0, H.b0.size());
    max_b1 = std::max(max_b1, H.b1.size());
    g.max_ext = std::max(g.max_ext, grown_box(H.b, H.b1).size());
    g.totalnodes += (double)H.b0.size();
    g.max_b1_face = std::max({g.max_b1_face, (long)H.b1.ny() * H.b1.nz(), (long)H.b1.nx() * H.b1.nz(),
                              (long)H.b1.nx() * H.b1.ny()});
    g.max_b1_box.ie = std::max(g.max_b1_box.ie, H.b1.nx());
    g.max_b1_box.je = std::max(g.max_b1_box.je, H.b1.ny());
    g.max_b1_box.ke = std::max(g.max_b1_box.ke, H.b1.nz());
  }
  g.max_b1 = max_b1;
  CK(cudaMalloc(&g.arena, total * sizeof(double)));
  CK(cudaMemsetAsync(g.arena, 0, total * sizeof(double), g.stream));
  g.arena_doubles = total;
  g.views.resize(nb);
  g.pmax_all = 0;
  g.slab_fits.clear();
  g.hmax_all = 0;
  for (int m = 0; m < nb; ++m) {
    HostBlock& H = g.blocks[m];
    fill_view(g.views[m], H.b, H.b0, H.b1, H.plane, g.arena + H.arena_off);
    int pmax = 0;
    std::vector<long> poff = plane_offsets(H.b1, pmax);
    CK(cudaMalloc(&H.ws, workspace_bytes(H.b1, (int)poff.size() - 1)));
    if ((rc = attach_workspace(g.views[m], H.ws, poff, pmax))) return rc;
    g.pmax_all = std::max(g.pmax_all, pmax);
    g.hmax_all = std::max(g.hmax_all, (int)poff.size() - 1);
  }
  // per-block case constants of a batch (aero_set_block_params)
  bool any_own = false;
  for (auto& H : g.blocks) any_own = any_own || H.own_params;
  if (any_own) {
    std::vector<CaseConsts> ccs(nb);
    for (int m = 0; m < nb; ++m) ccs[m] = g.blocks[m].own_params ? g.blocks[m].cc : g.cc;
    CK(cudaMalloc(&g.d_ccb, nb * sizeof(CaseConsts)));
    CK(cudaMemcpyAsync(g.d_ccb, ccs.data(), nb * sizeof(CaseConsts), cudaMemcpyHostToDevice, g.stream));
    for (int m = 0; m < nb; ++m)
      if (g.blocks[m].own_params) g.views[m].ccb = g.d_ccb + m;
  }
  // per-block status words (zero) and live flags (one)
  CK(cudaMalloc(&g.d_bstat, nb * sizeof(unsigned)));
  CK(cudaMalloc(&g.d_live, nb * sizeof(int)));
  CK(cudaMemsetAsync(g.d_bstat, 0, nb * sizeof(unsigned), g.stream));
  {
    std::vector<int> ones(nb, 1);
    CK(cudaMemcpyAsync(g.d_live, ones.data(), nb * sizeof(int), cudaMemcpyHostToDevice, g.stream));
    CK(cudaStreamSynchronize(g.stream));
  }
  for (int m = 0; m < nb; ++m) {
    g.views[m].bstat = g.d_bstat + m;
    g.views[m].live = g.d_live + m;
  }
  CK(cudaMalloc(&g.d_blocks, nb * sizeof(BlockView)));
  CK(cudaMemcpyAsync(g.d_blocks, g.views.data(), nb * sizeof(BlockView), cudaMemcpyHostToDevice, g.stream));
  // the same views with the longest hyperplane chains first, for the LU-SGS
  // sweeps: when a batch's sweep CTAs outnumber the SMs, the blocks whose
  // sweeps take longest are the first to be given SMs
  {
    std::vector<BlockView> chain(g.views);
    std::stable_sort(chain.begin(), chain.end(),
                     [](const BlockView& a, const BlockView& b) { return a.nplanes > b.nplanes; });
    CK(cudaMalloc(&g.d_blocks_chain, nb * sizeof(BlockView)));
    CK(cudaMemcpyAsync(g.d_blocks_chain, chain.data(), nb * sizeof(BlockView), cudaMemcpyHostToDevice, g.stream));
  }
  // tables
  CK(cudaMalloc(&g.d_bc_ops, std::max<size_t>(1, topo.bc_ops.size()) * sizeof(BcOp)));
  if (!topo.bc_ops.empty())
    CK(cudaMemcpyAsync(g.d_bc_ops, topo.bc_ops.data(), topo.bc_ops.size() * sizeof(BcOp), cudaMemcpyHostToDevice, g.stream));
  {
    // launch lists by dependency level
    auto face_nodes = [](const BcOp& op) {
      int dir = (op.face - 1) / 2;
      return dir == 0 ? (long)op.sb.ny() * op.sb.nz() : dir == 1 ? (long)op.sb.nx() * op.sb.nz()
                                                                  : (long)op.sb.nx() * op.sb.ny();
    };
    int nlev = 0;
    for (int l : topo.bc_level) nlev = std::max(nlev, l + 1);
    std::vector<BcEntry> list;
    g.bc_lstart.assign(1, 0);
    g.bc_lface.clear();
    for (int L = 0; L < nlev; ++L) {
      long face = 1;
      for (int m = 0; m < nb; ++m)
        for (int idx = topo.bc_start[m]; idx < topo.bc_start[m + 1]; ++idx)
          if (topo.bc_level[idx] == L) {
            list.push_back({idx, m});
            face = std::max(face, face_nodes(topo.bc_ops[idx]));
          }
      g.bc_lstart.push_back((int)list.size());
      g.bc_lface.push_back(face);
    }
    CK(cudaMalloc(&g.d_bc_list, std::max<size_t>(1, list.size()) * sizeof(BcEntry)));
    if (!list.empty())
      CK(cudaMemcpyAsync(g.d_bc_list, list.data(), list.size() * sizeof(BcEntry), cudaMemcpyHostToDevice, g.stream));
  }
  g.nhalo = (long)topo.halo.size();
  g.navg_src = (long)topo.avg_src.size();
  g.navg_dst = (long)topo.avg_dst.size();
  CK(cudaMalloc(&g.d_halo, std::max<size_t>(1, topo.halo.size()) * sizeof(HaloEntry)));
  CK(cudaMalloc(&g.d_avg_src, std::max<size_t>(1, topo.avg_src.size()) * sizeof(AvgSrc)));
  CK(cudaMalloc(&g.d_avg_dst, std::max<size_t>(1, topo.avg_dst.size()) * sizeof(AvgDst)));
  CK(cudaMalloc(&g.d_avg_buf, std::max<size_t>(1, topo.avg_src.size()) * 6 * sizeof(double)));
  if (g.nhalo) CK(cudaMemcpyAsync(g.d_halo, topo.halo.data(), g.nhalo * sizeof(HaloEntry), cudaMemcpyHostToDevice, g.stream));
  if (g.navg_src) CK(cudaMemcpyAsync(g.d_avg_src, topo.avg_src.data(), g.navg_src * sizeof(AvgSrc), cudaMemcpyHostToDevice, g.stream));
  if (g.navg_dst) CK(cudaMemcpyAsync(g.d_avg_dst, topo.avg_dst.data(), g.navg_dst * sizeof(AvgDst), cudaMemcpyHostToDevice, g.stream));
  if ((rc = launch_index(g.d_blocks, nb, g.max_b1))) return rc;
  g.resid_ctas = (int)cdiv(g.max_b1, 256);
  CK(cudaMalloc(&g.d_part, (size_t)g.resid_ctas * nb * 6 * sizeof(double)));
  CK(cudaMalloc(&g.d_resid_blocks, (size_t)nb * 7 * sizeof(double)));
  // wall subfaces of clcd_output, in block and bcinfo order
  {
    std::vector<WallFace> walls;
    long q = 0;
    for (int m = 0; m < nb; ++m)
      for (const SubRow& r : g.blocks[m].subs) {
        if (r.blk_t != BC_WALL) continue;
        int D = (r.face - 1) / 2;
        int T1 = D == 0 ? 1 : 0, T2 = D == 2 ? 1 : 2;
        const int lo[3] = {r.is, r.js, r.ks}, hi[3] = {r.ie, r.je, r.ke};
        WallFace w{m, r.face, lo[T1], hi[T1] - lo[T1], lo[T2], hi[T2] - lo[T2], r.face % 2 ? lo[D] : hi[D], q};
        if (g.cc.dimension == IFLAG_2D) w.n2 = 1;  // 2-D: one row of wall edges along T1
        if (w.n1 <= 0 || w.n2 <= 0) continue;  // a wall line has no quads
        walls.push_back(w);
        q += (long)w.n1 * w.n2;
      }
    g.nwall = (int)walls.size();
    g.nquad = q;
    if (g.nwall) {
      CK(cudaMalloc(&g.d_walls, walls.size() * sizeof(WallFace)));
      CK(cudaMemcpyAsync(g.d_walls, walls.data(), walls.size() * sizeof(WallFace), cudaMemcpyHostToDevice,
                         g.stream));
      CK(cudaMalloc(&g.d_fpart, (size_t)cdiv(q, 256) * 6 * sizeof(double)));
    }
  }
  // wall subfaces of surface_output: every node of the subface, lines included;
  // zones without nodes keep their header but own no node index
  {
    g.surf.clear();
    std::vector<SurfZone> live;
    long q = 0;
    for (int m = 0; m < nb; ++m)
      for (const SubRow& r : g.blocks[m].subs) {
        if (r.blk_t != BC_WALL) continue;
        SurfZone z{m, r.face, r.is, r.js, r.ks, r.ie - r.is + 1, r.je - r.js + 1, r.ke - r.ks + 1, q};
        g.surf.push_back(z);
        if (z.nx > 0 && z.ny > 0 && z.nz > 0) {
          live.push_back(z);
          q += (long)z.nx * z.ny * z.nz;
        }
      }
    g.nsurf = q;
    g.nsurf_live = (int)live.size();
    if (!live.empty()) {
      CK(cudaMalloc(&g.d_surf, live.size() * sizeof(SurfZone)));
      CK(cudaMemcpyAsync(g.d_surf, live.data(), live.size() * sizeof(SurfZone), cudaMemcpyHostToDevice, g.stream));
      CK(cudaMalloc(&g.d_surf_out, (size_t)q * 4 * sizeof(double)));
    }
  }
  CK(cudaStreamSynchronize(g.stream));
  g.setup = true;
  return AERO_OK;
}

// Every registered array of the mask, in batches that share the staging
// buffer (up to 64 MiB, or one array if larger).  The copies of a batch run
// back to back on the main stream and the transposes on the second stream,
// each array's transpose chained to its own copy by an event: an upload
// transposes array k while array k+1 is still crossing the bus, a download
// copies array k while array k+1 is transposed.
static int sync_fields(unsigned long long mask, bool to_device) {
  int rc = need_setup();
  if (rc) return rc;
  if (to_device && (mask & (1ull << F_RHSI)) && g.rhsi_ghosts_zero) {
    // the uploaded rhsi may be non-zero outside the updated boxes: the next
    // iteration zeroes it again (a captured step without that fill is stale)
    g.rhsi_ghosts_zero = false;
    graph_release();
  }
  struct Item {
    double* host;
    double* dev;
    long n;
    int nc;
    long plane;
    size_t off;
  };
  std::vector<Item> items;
  for (int m = 0; m < (int)g.blocks.size(); ++m) {
    HostBlock& H = g.blocks[m];
    for (int f = 0; f < kNumPublicFields; ++f)
      if ((mask & (1ull << f)) && H.host[f]) items.push_back({H.host[f], g.views[m].f[f], H.b.size(), field_nc(f), H.plane, 0});
  }
  const size_t cap = (size_t)8 << 20;  // doubles per batch
  for (size_t i = 0; i < items.size();) {
    size_t j = i, total = 0;
    while (j < items.size()) {
      size_t len = ((size_t)items[j].n * items[j].nc + 31) / 32 * 32;  // 256-byte aligned slots
      if (j > i && total + len > cap) break;
      items[j].off = total;
      total += len;
      ++j;
    }
    if ((rc = ensure_staging(total))) return rc;
    while (g.xfer_ev.size() < j - i + 1) {
      cudaEvent_t e = nullptr;
      CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      g.xfer_ev.push_back(e);
    }
    cudaEvent_t* ev = g.xfer_ev.data();
    const size_t last = j - i;  // the event joining the two streams
    if (!to_device) {
      // the transposes wait for everything before them on the main stream
      CK(cudaEventRecord(ev[last], g.stream));
      CK(cudaStreamWaitEvent(g.stream2, ev[last], 0));
    }
    for (size_t k = i; k < j; ++k) {
      const Item& it = items[k];
      double* st = g.d_staging + it.off;
      const size_t bytes = (size_t)it.n * it.nc * sizeof(double);
      if (to_device) {
        CK(cudaMemcpyAsync(st, it.host, bytes, cudaMemcpyHostToDevice, g.stream));
        CK(cudaEventRecord(ev[k - i], g.stream));
        CK(cudaStreamWaitEvent(g.stream2, ev[k - i], 0));
        PROF_ON(P_TRANSFER, g.stream2,
                (k_aos_to_soa<<<cdiv(it.n, 256), 256, 0, g.stream2>>>(st, it.dev, it.n, it.nc, it.plane)));
        CKL();
      } else {
        PROF_ON(P_TRANSFER, g.stream2,
                (k_soa_to_aos<<<cdiv(it.n, 256), 256, 0, g.stream2>>>(it.dev, st, it.n, it.nc, it.plane)));
        CKL();
        CK(cudaEventRecord(ev[k - i], g.stream2));
        CK(cudaStreamWaitEvent(g.stream, ev[k - i], 0));
        CK(cudaMemcpyAsync(it.host, st, bytes, cudaMemcpyDeviceToHost, g.stream));
      }
    }
    if (to_device) {
      // later work on the main stream (and the next batch's copies into the
      // staging buffer) waits for the transposes
      CK(cudaEventRecord(ev[last], g.stream2));
      CK(cudaStreamWaitEvent(g.stream, ev[last], 0));
    }
    i = j;
  }
  CK(cudaStreamSynchronize(g.stream));
  return AERO_OK;
}
int aero_sync_to_device(unsigned long long mask) { return sync_fields(mask, true); }
int aero_sync_to_host(unsigned long long mask) { return sync_fields(mask, false); }

// ------------------------------------------------------------ drop-in mirrors
int aero_get_primitivevariables(const int* mm, double* pri_v, const double* q, const double* gamma,
                                const double* cv, const int* is, const int* ie, const int* js,
                                const int* je, const int* ks, const int* ke) {
  (void)mm;
  int rc = need_init();
  if (rc) return rc;
  Box b = box_of(is, ie, js, je, ks, ke);
  std::vector<Arg> args = {{F_Q, q, false}, {F_PRI, pri_v, true}};
  BlockTarget t;
  if ((rc = resolve_full(b, args, t))) return rc;
  CaseConsts cc = consts_with(*gamma, *cv, g.cc.re);
  if ((rc = launch_getpri(t.d_view, 1, b.size(), cc))) return rc;
  return finish(t, args);
}

int aero_inviscid_flux_1(double* rhsi, const double* q, const double* dxidx, const double* inv_j,
                         const int* is, const int* ie, const int* js, const int* je, const int* ks,
                         const int* ke, const int* is0, const int* ie0, const int* js0,
                         const int* je0, const int* ks0, const int* ke0, const int* is1,
                         const int* ie1, const int* js1, const int* je1, const int* ks1,
                         const int* ke1, const double* gamma) {
  int rc = need_init();
  if (rc) return rc;
  Box b = box_of(is, ie, js, je, ks, ke), b0 = box_of(is0, ie0, js0, je0, ks0, ke0),
      b1 = box_of(is1, ie1, js1, je1, ks1, ke1);
  std::vector<Arg> args = {{F_Q, q, false}, {F_DXIDX, dxidx, false}, {F_INVJ, inv_j, false}, {F_RHSI, rhsi, true}};
  BlockTarget t;
  if ((rc = resolve(b, b0, b1, args, t))) return rc;
  CaseConsts cc = consts_with(*gamma, g.cc.cv, g.cc.re);
  cc.inviscid = IFLAG_3RDWENO;  // this routine is the reference's Roe + WENO3 flux
  long maxFace = std::max({(long)b1.ny() * b1.nz(), (long)b1.nx() * b1.nz(), (long)b1.nx() * b1.ny()});
  if ((rc = launch_inviscid(t.d_view, 1, b.size(), b1.size(), maxFace, cc))) return rc;
  return finish(t, args);
}

// The faces of is0..ke0 grown by one node down along coord, and the node up
// along coord each face also reads, lie inside the box is..ke (the drop-in
// face routines below read nothing outside it; a one-plane 2-D box has no
// faces along k).
bool faces_inside(const Box& b, const Box& e, int coord) {
  if (e.is < b.is || e.ie > b.ie || e.js < b.js || e.je > b.je || e.ks < b.ks || e.ke > b.ke) return false;
  const int hi = coord == 1 ? e.ie : (coord == 2 ? e.je : e.ke);
  const int bh = coord == 1 ? b.ie : (coord == 2 ? b.je : b.ke);
  return hi <= bh - 1;
}

// thirdorder_weno (sub_inviscid_upwind.f90:1): the WENO3 state at every face
// of the caller's box is0..ke0 grown by one node down along coord, right
// (direction 1) or left (direction -1) of the face; df keeps the caller's
// values elsewhere.  Always transient (the reference calls it on scratch
// arrays of inviscid_flux_1).
int aero_thirdorder_weno(double* df, const double* f, const int* is, const int* ie, const int* js, const int* je,
                         const int* ks, const int* ke, const int* is0, const int* ie0, const int* js0,
                         const int* je0, const int* ks0, const int* ke0, const int* coord, const int* direction) {
  int rc = need_init();
  if (rc) return rc;
  if (*coord < 1 || *coord > 3) return fail(AERO_ERR_ARG, "thirdorder_weno: coord %d is not 1, 2 or 3", *coord);
  Box b = box_of(is, ie, js, je, ks, ke), r0 = box_of(is0, ie0, js0, je0, ks0, ke0);
  std::vector<Arg> args = {{F_Q, f, false}, {F_RHSI, df, true}};
  BlockTarget t;
  if ((rc = resolve(b, r0, r0, args, t))) return rc;
  if (t.resident) return fail(AERO_ERR_ARG, "thirdorder_weno works on unregistered arrays");
  Box e = r0;
  if (*coord == 1) e.is -= 1; else if (*coord == 2) e.js -= 1; else e.ks -= 1;
  if (e.size() > 0 && !faces_inside(b, e, *coord))
    return fail(AERO_ERR_ARG, "thirdorder_weno: faces along coord %d reach outside the array", *coord);
  // direction 1: right states, -1: left states, anything else: nothing (the
  // reference's if / else if)
  if (e.size() > 0 && (*direction == 1 || *direction == -1)) {
    k_weno3_states<<<cdiv(e.size(), 128), 128, 0, g.stream>>>(t.d_view, *coord, *direction, r0);
    CKL();
  }
  return finish(t, args);
}

// roe_3d (sub_inviscid_splitting.f90:1): the Roe flux at every face of
// is0..ke0 grown by one down along coord from primitive states ql, qr
// (d, u, v, w, p); flux keeps the caller's values elsewhere.  Always transient.
int aero_roe_3d(const double* ql, const double* qr, double* flux, const double* dxidx, const double* inv_j,
                const double* gamma, const int* is, const int* ie, const int* js, const int* je, const int* ks,
                const int* ke, const int* is0, const int* ie0, const int* js0, const int* je0, const int* ks0,
                const int* ke0, const int* coord) {
  int rc = need_init();
  if (rc) return rc;
  if (*coord < 1 || *coord > 3) return fail(AERO_ERR_ARG, "roe_3d: coord %d is not 1, 2 or 3", *coord);
  Box b = box_of(is, ie, js, je, ks, ke), r0 = box_of(is0, ie0, js0, je0, ks0, ke0);
  std::vector<Arg> args = {{F_Q, ql, false}, {F_RHSI, qr, false}, {F_RHSV, flux, true},
                           {F_DXIDX, dxidx, false}, {F_INVJ, inv_j, false}};
  BlockTarget t;
  if ((rc = resolve(b, r0, r0, args, t))) return rc;
  if (t.resident) return fail(AERO_ERR_ARG, "roe_3d works on unregistered arrays");
  Box e = r0;
  if (*coord == 1) e.is -= 1; else if (*coord == 2) e.js -= 1; else e.ks -= 1;
  if (e.size() > 0 && !faces_inside(b, e, *coord))
    return fail(AERO_ERR_ARG, "roe_3d: faces along coord %d reach outside the array", *coord);
  if (e.size() > 0) {
    k_roe_states<<<cdiv(e.size(), 128), 128, 0, g.stream>>>(t.d_view, *coord, r0, *gamma);
    CKL();
  }
  return finish(t, args);
}

// The extension schemes with inviscid_flux_1's argument list (no counterpart
// in the reference): scheme IFLAG_5THWENO or IFLAG_5THWCNS.
static int inviscid_ext(int scheme, double* rhsi, const double* q, const double* dxidx, const double* inv_j,
                        const int* is, const int* ie, const int* js, const int* je, const int* ks, const int* ke,
                        const int* is0, const int* ie0, const int* js0, const int* je0, const int* ks0,
                        const int* ke0, const int* is1, const int* ie1, const int* js1, const int* je1,
                        const int* ks1, const int* ke1, const double* gamma) {
  int rc = need_init();
  if (rc) return rc;
  Box b = box_of(is, ie, js, je, ks, ke), b0 = box_of(is0, ie0, js0, je0, ks0, ke0),
      b1 = box_of(is1, ie1, js1, je1, ks1, ke1);
  std::vector<Arg> args = {{F_Q, q, false}, {F_DXIDX, dxidx, false}, {F_INVJ, inv_j, false}, {F_RHSI, rhsi, true}};
  BlockTarget t;
  if ((rc = resolve(b, b0, b1, args, t))) return rc;
  CaseConsts cc = consts_with(*gamma, g.cc.cv, g.cc.re);
  cc.inviscid = scheme;
  long maxFace = std::max({(long)b1.ny() * b1.nz(), (long)b1.nx() * b1.nz(), (long)b1.nx() * b1.ny()});
  if ((rc = launch_inviscid(t.d_view, 1, b.size(), b1.size(), maxFace, cc))) return rc;
  return finish(t, args);
}
int aero_inviscid_flux_weno5(double* rhsi, const double* q, const double* dxidx, const double* inv_j,
                             const int* is, const int* ie, const int* js, const int* je, const int* ks,
                             const int* ke, const int* is0, const int* ie0, const int* js0, const int* je0,
                             const int* ks0, const int* ke0, const int* is1, const int* ie1, const int* js1,
                             const int* je1, const int* ks1, const int* ke1, const double* gamma) {
  return inviscid_ext(IFLAG_5THWENO, rhsi, q, dxidx, inv_j, is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0,
                      ke0, is1, ie1, js1, je1, ks1, ke1, gamma);
}
int aero_inviscid_flux_wcns5(double* rhsi, const double* q, const double* dxidx, const double* inv_j,
                             const int* is, const int* ie, const int* js, const int* je, const int* ks,
                             const int* ke, const int* is0, const int* ie0, const int* js0, const int* je0,
                             const int* ks0, const int* ke0, const int* is1, const int* ie1, const int* js1,
                             const int* je1, const int* ks1, const int* ke1, const double* gamma) {
  return inviscid_ext(IFLAG_5THWCNS, rhsi, q, dxidx, inv_j, is, ie, js, je, ks, ke, is0, ie0, js0, je0, ks0,
                      ke0, is1, ie1, js1, je1, ks1, ke1, gamma);
}

int aero_viscous_flux(double* rhsv, const double* pri_v, double* amu, double* vor, double* dudx,
                      double* tao, const double* dxidx, const double* inv_j, const double* tinf,
                      const double* prl, const double* prt, const double* gamma, const double* cv,
                      const double* re, const int* is, const int* ie, const int* js,
                      const int* je, const int* ks, const int* ke, const int* is0,
                      const int* ie0, const int* js0, const int* je0, const int* ks0,
                      const int* ke0, const int* is1, const int* ie1, const int* js1,
                      const int* je1, const int* ks1, const int* ke1, const int* mm) {
  (void)mm;
  int rc = need_init();
  if (rc) return rc;
  Box b = box_of(is, ie, js, je, ks, ke), b0 = box_of(is0, ie0, js0, je0, ks0, ke0),
      b1 = box_of(is1, ie1, js1, je1, ks1, ke1);
  std::vector<Arg> args = {{F_PRI, pri_v, false}, {F_AMU, amu, true},  {F_VOR, vor, true},
                           {F_DUDX, dudx, true},  {F_TAO, tao, true},  {F_DXIDX, dxidx, false},
                           {F_INVJ, inv_j, false}, {F_RHSV, rhsv, true}};
  BlockTarget t;
  if ((rc = resolve(b, b0, b1, args, t))) return rc;
  CaseConsts cc = consts_with(*gamma, *cv, *re);
  cc.tinf = *tinf; cc.prl = *prl; cc.prt = *prt;
  if ((rc = launch_viscous(t.d_view, 1, b0.size(), cc, 1))) return rc;
  return finish(t, args);
}

int aero_find_dt(double* dt, double* dtmax, double* dtmin, double* cflmax, double* cflmin,
                 const double* pri_v, const double* amu, const double* dxidx, const double* re,
                 double* cfl, const int* is, const int* ie, const int* js, const int* je,
                 const int* ks, const int* ke, const int* iflag_time, const int* iflag_steady,
                 const int* iflag_unsteady) {
  (void)iflag_steady; (void)iflag_unsteady;
  int rc = need_init();
  if (rc) return rc;
  if (*iflag_time != IFLAG_STEADY) return fail(AERO_ERR_ARG, "find_dt: only the steady branch is supported");
  Box b = box_of(is, ie, js, je, ks, ke);
  std::vector<Arg> args = {{F_PRI, pri_v, false}, {F_AMU, amu, false}, {F_DXIDX, dxidx, false}, {F_DT, dt, true}};
  BlockTarget t;
  if ((rc = resolve_full(b, args, t))) return rc;
  CaseConsts cc = consts_with(g.cc.gamma, g.cc.cv, *re);
  cc.cfl = *cfl;
  if ((rc = launch_find_dt(t.d_view, 1, b.size(), cc))) return rc;
  if ((rc = launch_dt_minmax(t.d_view, 0, g.d_out + 7))) return rc;
  CK(cudaMemcpyAsync(g.h_out + 7, g.d_out + 7, 2 * sizeof(double), cudaMemcpyDeviceToHost, g.stream));
  if ((rc = finish(t, args))) return rc;
  CK(cudaStreamSynchronize(g.stream));
  *dtmax = g.h_out[7];
  *dtmin = g.h_out[8];
  *cflmax = 0.0;
  *cflmin = 1.0e10;
  return AERO_OK;
}

int aero_implicit1st(double* q, const double* dt, const double* pri_v, double* rhs,
                     const double* rhsi, const double* rhsv, const double* dxidx,
                     const double* inv_j, const int* is, const int* ie, const int* js,
                     const int* je, const int* ks, const int* ke, const int* is0,
                     const int* ie0, const int* js0, const int* je0, const int* ks0,
                     const int* ke0, const int* is1, const int* ie1, const int* js1,
                     const int* je1, const int* ks1, const int* ke1, const double* gamma,
                     const double* cfl, const double* xx, const double* yy, const double* zz) {
  (void)xx; (void)yy; (void)zz;
  int rc = need_init();
  if (rc) return rc;
  Box b = box_of(is, ie, js, je, ks, ke), b0 = box_of(is0, ie0, js0, je0, ks0, ke0),
      b1 = box_of(is1, ie1, js1, je1, ks1, ke1);
  std::vector<Arg> args = {{F_Q, q, true},        {F_DT, dt, false},       {F_PRI, pri_v, false},
                           {F_RHS, rhs, true},    {F_RHSI, rhsi, false},   {F_RHSV, rhsv, false},
                           {F_DXIDX, dxidx, false}, {F_INVJ, inv_j, false}};
  BlockTarget t;
  if ((rc = resolve(b, b0, b1, args, t))) return rc;
  CaseConsts cc = consts_with(*gamma, g.cc.cv, g.cc.re);
  cc.cfl = *cfl;
  Box e = grown_box(b, b1);
  if (!t.resident && (rc = launch_index(t.d_view, 1, b1.size()))) return rc;
  if ((rc = launch_implicit(t.d_view, 1, e.size(), b1.size(), t.view.pmax, t.view.nplanes, cc, nullptr, true,
                            nullptr, &t.view)))
    return rc;
  return finish(t, args);
}

int aero_crank2nd(double* q, const double* q0, const double* dt, const double* pri_v, double* rhs,
                  const double* rhsi, const double* rhsv, const double* dxidx, const double* inv_j,
                  const int* is, const int* ie, const int* js, const int* je, const int* ks, const int* ke,
                  const int* is0, const int* ie0, const int* js0, const int* je0, const int* ks0,
                  const int* ke0, const int* is1, const int* ie1, const int* js1, const int* je1,
                  const int* ks1, const int* ke1, const double* gamma, const int* mm, const int* ssub) {
  (void)mm; (void)ssub;
  int rc = need_init();
  if (rc) return rc;
  Box b = box_of(is, ie, js, je, ks, ke), b0 = box_of(is0, ie0, js0, je0, ks0, ke0),
      b1 = box_of(is1, ie1, js1, je1, ks1, ke1);
  std::vector<Arg> args = {{F_Q, q, true},         {F_Q0, q0, false},     {F_DT, dt, false},
                           {F_PRI, pri_v, false},  {F_RHS, rhs, true},    {F_RHSI, rhsi, false},
                           {F_RHSV, rhsv, false},  {F_DXIDX, dxidx, false}, {F_INVJ, inv_j, false}};
  BlockTarget t;
  if ((rc = resolve(b, b0, b1, args, t))) return rc;
  CaseConsts cc = consts_with(*gamma, g.cc.cv, g.cc.re);
  Box lines{1, b1.nx(), 1, b1.ny(), 1, b1.nz()};
  if ((rc = launch_crank(t.d_view, 1, b.size(), b1.size(), &lines, cc))) return rc;
  return finish(t, args);
}

int aero_update_q0(double* q0, const double* q, const int* is, const int* ie, const int* js, const int* je,
                   const int* ks, const int* ke, const int* is0, const int* ie0, const int* js0,
                   const int* je0, const int* ks0, const int* ke0) {
  int rc = need_init();
  if (rc) return rc;
  Box b = box_of(is, ie, js, je, ks, ke), b0 = box_of(is0, ie0, js0, je0, ks0, ke0);
  std::vector<Arg> args = {{F_Q0, q0, true}, {F_Q, q, false}};
  BlockTarget t;
  if ((rc = resolve(b, b0, b0, args, t))) return rc;
  PROF(P_CRANK, (k_update_q0<<<cdiv(b0.size(), 256), 256, 0, g.stream>>>(t.d_view)));
  CKL();
  return finish(t, args);
}

// ------------------------------------------------------ module-state routines
int aero_physical_bc(void) {
  int rc = need_setup();
  return rc ? rc : do_physical_bc();
}
int aero_updatebuffer(void) {
  int rc = need_setup();
  return rc ? rc : do_halo();
}
int aero_average1(void) {
  int rc = need_setup();
  return rc ? rc : do_average1();
}
int aero_average2(void) {
  int rc = need_setup();
  return rc ? rc : do_average2();
}
int aero_updatebuffercoordinate(void) {
  int rc = need_setup();
  if (rc) return rc;
  if (g.nhalo == 0) return AERO_OK;
  PROF(P_HALO, (k_halo<<<cdiv(g.nhalo, 256), 256, 0, g.stream>>>(g.d_blocks, g.d_halo, g.nhalo, HALO_COORD)));
  CKL();
  return AERO_OK;
}
int aero_getpri_all(void) {
  int rc = need_setup();
  return rc ? rc : do_getpri_all();
}
// The reference's 2-D names (sub_bc_updatebuffer2d.f90:10,
// sub_bc_updatebufferaverage2d.f90:10, :317, sub_bc_updatebuffercoordinate2d.f90:10):
// the same tables, which a 2-D configuration builds with the 2-D index maps;
// in a 3-D configuration they are an error, as calling them there would be a
// mistake in the caller.
static int need_2d(const char* name) {
  int rc = need_setup();
  if (rc) return rc;
  if (g.cc.dimension != IFLAG_2D) return fail(AERO_ERR_STATE, "%s: the case is not 2-D (iflag_dimension = %d)", name,
                                               g.cc.dimension);
  return AERO_OK;
}
int aero_updatebuffer2d(void) {
  int rc = need_2d("UpdateBuffer2d");
  return rc ? rc : do_halo();
}
int aero_average2d1(void) {
  int rc = need_2d("average2d1");
  return rc ? rc : do_average1();
}
int aero_average2d2(void) {
  int rc = need_2d("average2d2");
  return rc ? rc : do_average2();
}
int aero_updatebuffercoordinate2d(void) {
  int rc = need_2d("UpdateBufferCoordinate2d");
  return rc ? rc : aero_updatebuffercoordinate();
}

int aero_residual(double* out7) {
  int rc = need_setup();
  if (rc) return rc;
  if ((rc = do_residual(g.d_out))) return rc;
  CK(cudaMemcpyAsync(g.h_out, g.d_out, 7 * sizeof(double), cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  std::memcpy(out7, g.h_out, 7 * sizeof(double));
  return AERO_OK;
}

int aero_clcd_output(double sref, double* out8) {
  int rc = need_setup();
  if (rc) return rc;
  if (!(sref > 0.0)) return fail(AERO_ERR_ARG, "sref = %g is not positive", sref);
  if (!g.nwall) {
    for (int x = 0; x < 8; ++x) out8[x] = 0.0;
    return AERO_OK;
  }
  unsigned ctas = cdiv(g.nquad, 256);
  PROF(P_FORCES, (k_forces<<<ctas, 256, 0, g.stream>>>(g.d_blocks, g.d_walls, g.nwall, g.nquad, g.cc, g.d_fpart)));
  CKL();
  PROF(P_FORCES, (k_forces_final<<<1, 256, 0, g.stream>>>(g.d_fpart, (int)ctas, g.cc, sref, g.d_out)));
  CKL();
  CK(cudaMemcpyAsync(g.h_out, g.d_out, 8 * sizeof(double), cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  std::memcpy(out8, g.h_out, 8 * sizeof(double));
  return AERO_OK;
}

int aero_surface_count(long long* n_nodes, int* n_zones) {
  int rc = need_setup();
  if (rc) return rc;
  if (!n_nodes || !n_zones) return fail(AERO_ERR_ARG, "null output pointer");
  *n_nodes = g.nsurf;
  *n_zones = (int)g.surf.size();
  return AERO_OK;
}

int aero_surface_output(double* xyzcp, int* zones) {
  int rc = need_setup();
  if (rc) return rc;
  if ((g.nsurf && !xyzcp) || (!g.surf.empty() && !zones)) return fail(AERO_ERR_ARG, "null output pointer");
  for (size_t z = 0; z < g.surf.size(); ++z) {
    const SurfZone& Z = g.surf[z];
    int* o = zones + 5 * z;
    o[0] = Z.block + 1;
    o[1] = Z.face;
    o[2] = Z.nx;
    o[3] = Z.ny;
    o[4] = Z.nz;
  }
  if (!g.nsurf) return AERO_OK;
  PROF(P_FORCES, (k_surface_cp<<<cdiv(g.nsurf, 256), 256, 0, g.stream>>>(g.d_blocks, g.d_surf, g.nsurf_live,
                                                                         g.nsurf, g.cc, g.d_surf_out)));
  CKL();
  CK(cudaMemcpyAsync(xyzcp, g.d_surf_out, (size_t)g.nsurf * 4 * sizeof(double), cudaMemcpyDeviceToHost, g.stream));
  CK(cudaStreamSynchronize(g.stream));
  return AERO_OK;
}

int aero_init_flowfield(void) {
  int rc = need_setup();
  if (rc) return rc;
  // Fill on the host arrays' device copies: q, pri_v, dt, amu, nut, sa_rhs and
  // the zeroed work arrays (sub_init_flowfield.f90:55-111).
  int nb = (int)g.blocks.size();
  double t_0 = 1.0;
  bool sa = g.cc.turbulence == IFLAG_SA;
  double amu2 = sa ? 0.009 : 0.0;
  double av[3] = {1.0, amu2, 1.0 + amu2};
  for (int m = 0; m < nb; ++m) {
    const CaseConsts& c = g.blocks[m].own_params ? g.blocks[m].cc : g.cc;
    const double dt0 = g.blocks[m].own_params ? g.blocks[m].params[5] : g.params[5];
    double qv[5] = {c.d_0, c.d_0 * c.u_0 * std::cos(c.aoa), c.d_0 * c.u_0 * std::sin(c.aoa), 0.0,
                    c.d_0 * t_0 * c.cv + 0.5 * c.d_0 * c.u_0 * c.u_0};
    double pv[7] = {c.d_0, c.u_0 * std::cos(c.aoa), c.u_0 * std::sin(c.aoa), 0.0, c.p_0, t_0, c.c_0};
    const BlockView& v = g.views[m];
    long N = g.blocks[m].b.size();
    auto put = [&](double* dst, double val) -> int {
      PROF(P_FILL, (k_fill_plane<<<cdiv(N, 256), 256, 0, g.stream>>>(dst, N, val)));
      CKL();
      return AERO_OK;
    };
    for (int x = 0; x < 5; ++x) if ((rc = put(v.f[F_Q] + x * v.plane, qv[x]))) return rc;
    for (int x = 0; x < 7; ++x) if ((rc = put(v.f[F_PRI] + x * v.plane, pv[x]))) return rc;
    for (int x = 0; x < 3; ++x) if ((rc = put(v.f[F_AMU] + x * v.plane, av[x]))) return rc;
    if ((rc = put(v.f[F_DT], dt0))) return rc;
    for (int x = 0; x < 10; ++x)  // q0(l, c) = q(c) at both time levels (sub_init_flowfield.f90:78-82)
      if ((rc = put(v.f[F_Q0] + x * v.plane, qv[x / 2]))) return rc;
    if (sa) {
      if ((rc = put(v.f[F_NUT], c.nutinf))) return rc;
      if ((rc = put(v.f[F_SARHS], 0.0))) return rc;
    }
    for (int fid : {F_DUDX, F_VOR, F_TAO, F_RHSV, F_RHSI, F_RHS})
      for (int x = 0; x < field_nc(fid); ++x)
        if ((rc = put(v.f[fid] + x * v.plane, 0.0))) return rc;
  }
  g.rhsi_ghosts_zero = true;
  CK(cudaStreamSynchronize(g.stream));
  return AERO_OK;
}

int aero_sa_model(double* nut, double* sa_rhs, const double* dt, const double* pri_v, const double* amu,
                  const double* dudx, const double* vor, const double* dxidx, const double* inv_j,
                  const double* alpha, const double* beta, const double* gamma, double* length,
                  const double* dist, const double* spac, const double* re, const double* cfl,
                  const int* is, const int* ie, const int* js, const int* je, const int* ks,
                  const int* ke, const int* is0, const int* ie0, const int* js0, const int* je0,
                  const int* ks0, const int* ke0, const int* is1, const int* ie1, const int* js1,
                  const int* je1, const int* ks1, const int* ke1) {
  int rc = need_init();
  if (rc) return rc;
  Box b = box_of(is, ie, js, je, ks, ke), b0 = box_of(is0, ie0, js0, je0, ks0, ke0),
      b1 = box_of(is1, ie1, js1, je1, ks1, ke1);
  std::vector<Arg> args = {{F_NUT, nut, true},     {F_SARHS, sa_rhs, true}, {F_DT, dt, false},
                           {F_PRI, pri_v, false},  {F_AMU, amu, false},     {F_VOR, vor, false},
                           {F_DXIDX, dxidx, false}, {F_INVJ, inv_j, false}, {F_ALPHA, alpha, false},
                           {F_BETA, beta, false},  {F_GAMMA, gamma, false}, {F_LENGTH, length, true},
                           {F_DIST, dist, false}};
  if (g.cc.des == IFLAG_DES97 || g.cc.des == IFLAG_DDES) args.push_back({F_SPACING, spac, false});
  if (g.cc.des == IFLAG_DDES) args.push_back({F_DUDX, dudx, false});
  BlockTarget t;
  if ((rc = resolve(b, b0, b1, args, t))) return rc;
  CaseConsts cc = consts_with(g.cc.gamma, g.cc.cv, *re);
  cc.cfl = *cfl;
  if (!t.resident && (rc = launch_index(t.d_view, 1, b1.size()))) return rc;
  if ((rc = launch_sa(t.d_view, 1, b.size(), b1.size(), t.view.pmax, cc, nullptr, &t.view))) return rc;
  return finish(t, args);
}

int aero_gridtransformation(double* dxidx, double* inv_j, double* alpha, double* beta, double* gamma,
                            const double* x, const double* y, const double* z, const int* is,
                            const int* ie, const int* js, const int* je, const int* ks,
                            const int* ke, const int* is0, const int* ie0, const int* js0,
                            const int* je0, const int* ks0, const int* ke0, const int* m0) {
  (void)m0;
  int rc = need_init();
  if (rc) return rc;
  Box b = box_of(is, ie, js, je, ks, ke), b0 = box_of(is0, ie0, js0, je0, ks0, ke0);
  std::vector<Arg> args = {{F_X, x, false},        {F_Y, y, false},        {F_Z, z, false},
                           {F_DXIDX, dxidx, true}, {F_INVJ, inv_j, true},  {F_ALPHA, alpha, true},
                           {F_BETA, beta, true},   {F_GAMMA, gamma, true}};
  BlockTarget t;
  auto it = g.registry.find(x);
  if (it != g.registry.end()) {
    const HostBlock& H = g.blocks[it->second.first];
    if (!same(H.b, b) || !same(H.b0, b0)) return fail(AERO_ERR_ARG, "gridtransformation: bounds differ from the registered block");
    rc = resolve(H.b, H.b0, H.b1, args, t);
  } else {
    rc = resolve(b, b0, b0, args, t);
  }
  if (rc) return rc;
  PROF(P_GEOMETRY, (k_metric_pass1<<<dim3(cdiv(b.size(), 256), 1), 256, 0, g.stream>>>(t.d_view)));
  CKL();
  PROF(P_GEOMETRY, (k_metric_pass2<<<dim3(cdiv(b.size(), 128), 1), 128, 0, g.stream>>>(t.d_view)));
  CKL();
  return finish(t, args);
}

int aero_init_walldist(void) {
  int rc = need_setup();
  if (rc) return rc;
  // Independent cases registered together (a batch) are the connected
  // components of the block-interface graph; every node's distance is to the
  // walls of its own case, as when that case runs alone (one case: all
  // walls, as the reference).
  const int nb = (int)g.blocks.size();
  std::vector<int> root(nb);
  for (int m = 0; m < nb; ++m) root[m] = m;
  auto find = [&](int m) {
    while (root[m] != m) m = root[m] = root[root[m]];
    return m;
  };
  for (int m = 0; m < nb; ++m)
    for (const SubRow& s : g.blocks[m].subs)
      if (s.blk_t > 0 && s.blk_t <= nb) {
        const int a = find(m), b = find(s.blk_t - 1);
        if (a != b) root[std::max(a, b)] = std::min(a, b);
      }
  // wall-subface nodes of every block (sub_init_readbcinfo.f90:286-388),
  // grouped by case; range[2m], range[2m+1]: first and count of block m's case
  std::vector<AvgSrc> wall;
  std::vector<long> range(2 * (size_t)nb, 0);
  for (int c = 0; c < nb; ++c) {
    if (find(c) != c) continue;
    const long first = (long)wall.size();
    for (int m = 0; m < nb; ++m) {
      if (find(m) != c) continue;
      const HostBlock& H = g.blocks[m];
      for (const SubRow& s : H.subs) {
        if (s.blk_t != BC_WALL) continue;
        for (int k = s.ks; k <= s.ke; ++k)
          for (int j = s.js; j <= s.je; ++j)
            for (int i = s.is; i <= s.ie; ++i) {
              int ii = s.face == 1 ? H.b0.is : s.face == 2 ? H.b0.ie : i;
              int jj = s.face == 3 ? H.b0.js : s.face == 4 ? H.b0.je : j;
              int kk = s.face == 5 ? H.b0.ks : s.face == 6 ? H.b0.ke : k;
              long n = (long)(ii - H.b.is) + (long)H.b.nx() * ((long)(jj - H.b.js) + (long)H.b.ny() * (long)(kk - H.b.ks));
              wall.push_back(AvgSrc{m, n});
            }
      }
    }
    for (int m = 0; m < nb; ++m)
      if (find(m) == c) {
        range[2 * m] = first;
        range[2 * m + 1] = (long)wall.size() - first;
      }
  }
  long nw = (long)wall.size();
  AvgSrc* d_wall = nullptr;
  double* d_xyz = nullptr;
  if (nw > 0) {
    CK(cudaMalloc(&d_wall, nw * sizeof(AvgSrc)));
    CK(cudaMalloc(&d_xyz, nw * 3 * sizeof(double)));
    CK(cudaMemcpyAsync(d_wall, wall.data(), nw * sizeof(AvgSrc), cudaMemcpyHostToDevice, g.stream));
    PROF(P_GEOMETRY, (k_wall_points<<<cdiv(nw, 256), 256, 0, g.stream>>>(g.d_blocks, d_wall, nw, d_xyz)));
    CKL();
  }
  long* d_range = nullptr;
  CK(cudaMalloc(&d_range, range.size() * sizeof(long)));
  CK(cudaMemcpyAsync(d_range, range.data(), range.size() * sizeof(long), cudaMemcpyHostToDevice, g.stream));
  PROF(P_GEOMETRY, (k_walldist<<<dim3(cdiv(g.max_b0, 256), (unsigned)nb), 256, 256 * 3 * sizeof(double), g.stream>>>(
                       g.d_blocks, d_xyz, d_range)));
  CKL();
  CK(cudaStreamSynchronize(g.stream));
  if (d_wall) CK(cudaFree(d_wall));
  if (d_xyz) CK(cudaFree(d_xyz));
  CK(cudaFree(d_range));
  return AERO_OK;
}

// Coordinate halo, metrics, spacing and (optionally) wall distance for every
// registered block: main.f90:142-208 on the device.
int aero_compute_geometry(int with_walldist) {
  int rc = need_setup();
  if (rc) return rc;
  if ((rc = aero_updatebuffercoordinate())) return rc;
  int nb = (int)g.blocks.size();
  PROF(P_GEOMETRY, (k_metric_pass1<<<dim3(cdiv(g.max_box, 256), nb), 256, 0, g.stream>>>(g.d_blocks)));
  CKL();
  PROF(P_GEOMETRY, (k_metric_pass2<<<dim3(cdiv(g.max_box, 128), nb), 128, 0, g.stream>>>(g.d_blocks)));
  CKL();
  PROF(P_GEOMETRY, (k_spacing<<<dim3(cdiv(g.max_b0, 256), nb), 256, 0, g.stream>>>(g.d_blocks)));
  CKL();
  if (with_walldist && (rc = aero_init_walldist())) return rc;
  CK(cudaStreamSynchronize(g.stream));
  return AERO_OK;
}

// Device-timed iterations for benchmarking: each step is one iteration plus the
// residual norm (the reference computes it every iteration, outinterval = 1).
// With flush_l2 a 256 MiB buffer is overwritten (cudaMemsetAsync, outside the
// timed interval) before every step so each step starts with a cold L2.
int aero_step_timed(int nsteps, int flush_l2, double* device_ms) {
  int rc = need_setup();
  if (rc) return rc;
  static void* flush = nullptr;
  const size_t fbytes = 256ull << 20;
  if (flush_l2 && !flush) CK(cudaMalloc(&flush, fbytes));
  cudaEvent_t a, b;
  CK(cudaEventCreate(&a));
  CK(cudaEventCreate(&b));
  double total = 0.0;
  for (int s = 0; s < nsteps; ++s) {
    if (flush_l2) CK(cudaMemsetAsync(flush, s & 0xff, fbytes, g.stream));
    CK(cudaEventRecord(a, g.stream));
    if ((rc = run_step())) return rc;  // iteration, closing primitives, residual
    CK(cudaEventRecord(b, g.stream));
    CK(cudaEventSynchronize(b));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, a, b));
    total += ms;
  }
  CK(cudaStreamSynchronize(g.stream));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *device_ms = total;
  return AERO_OK;
}

int aero_profile(int enable) {
  int rc = need_init();
  if (rc) return rc;
  prof_collect();
  gp.on = enable != 0;
  if (enable) {
    for (int i = 0; i < P_NUM; ++i) { gp.ms[i] = 0.0; gp.count[i] = 0; }
  }
  return AERO_OK;
}

int aero_profile_read(double* ms, long long* counts, int n) {
  int rc = need_init();
  if (rc) return rc;
  prof_collect();
  for (int i = 0; i < n && i < P_NUM; ++i) {
    ms[i] = gp.ms[i];
    counts[i] = gp.count[i];
  }
  return P_NUM;
}

const char* aero_profile_name(int id) { return (id >= 0 && id < P_NUM) ? kProfName[id] : ""; }

int aero_profile_timeline(int* ids, double* start_ms, double* end_ms, int n) {
  int rc = need_init();
  if (rc) return rc;
  prof_collect();
  const int m = (int)gp.tl_id.size();
  for (int i = 0; i < n && i < m; ++i) {
    ids[i] = gp.tl_id[i];
    start_ms[i] = gp.tl_start[i];
    end_ms[i] = gp.tl_end[i];
  }
  return m;
}

int aero_launch_count(unsigned long long* count) {
  *count = gp.launches;
  return AERO_OK;
}

int aero_step(int nsteps, double* resid_hist, double* dt_minmax) {
  int rc = need_setup();
  if (rc) return rc;
  for (int s = 0; s < nsteps; ++s) {
    bool last = (s == nsteps - 1);
    if (last && dt_minmax != nullptr) {
      if ((rc = do_iteration(true))) return rc;
      if ((rc = do_getpri_all())) return rc;  // end of the time step (main.f90:434-447)
      if ((rc = do_residual(g.d_out))) return rc;
    } else if ((rc = run_step())) {
      return rc;
    }
    if (resid_hist) {
      CK(cudaMemcpyAsync(g.h_out, g.d_out, 7 * sizeof(double), cudaMemcpyDeviceToHost, g.stream));
      CK(cudaStreamSynchronize(g.stream));
      std::memcpy(resid_hist + 7 * s, g.h_out, 7 * sizeof(double));
    }
  }
  if (dt_minmax) {
    CK(cudaMemcpyAsync(g.h_out + 7, g.d_out + 7, 2 * sizeof(double), cudaMemcpyDeviceToHost, g.stream));
    CK(cudaStreamSynchronize(g.stream));
    dt_minmax[0] = g.h_out[7];
    dt_minmax[1] = g.h_out[8];
  }
  CK(cudaStreamSynchronize(g.stream));
  return AERO_OK;
}

}  // extern "C"
