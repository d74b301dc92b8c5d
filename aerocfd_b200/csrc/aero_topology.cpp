// Host-side construction of the halo, averaging and boundary tables.
//
// The reference moves interface data in three steps per subface: pack the
// donor's layers into buffer_send (indexed by the donor's own face indices),
// re-index the received buffer into a 2-D array ua(l,m) with a per-face (l,m)
// convention (sub_bc_updatebuffer.f90:265-354), reorient it by `ori`
// (:358-395) and write it into the receiver's ghost layers with the
// receiver's per-face convention (:398-540).  Composing those three index
// maps once gives, for every ghost node, the donor node it receives; the GPU
// then does a single gather per iteration.  The same composition with layer 0
// gives the shared interface nodes of average1 (sub_bc_updatebufferaverage.f90).
#include "aero_topology.h"

#include <algorithm>
#include <cstdio>
#include <map>
#include <tuple>

namespace aero {

namespace {

// Node layers one physical-BC op writes (its face layer) and reads (up to
// three layers inward along the face normal: no-slip extrapolates from
// three, outflow, symmetry and farfield read one, inflow none), as index
// boxes; the metrics it reads are never written by a BC.
struct Layers {
  int w[2][3], r[2][3];
  bool reads;
};
Layers bc_layers(const BcOp& op) {
  const int dir = (op.face - 1) / 2;
  const int s = op.face % 2 == 1 ? 1 : -1;
  const int lo[3] = {op.sb.is, op.sb.js, op.sb.ks}, hi[3] = {op.sb.ie, op.sb.je, op.sb.ke};
  Layers L;
  for (int d = 0; d < 3; ++d) {
    L.w[0][d] = L.r[0][d] = lo[d];
    L.w[1][d] = L.r[1][d] = hi[d];
  }
  const int f = s > 0 ? lo[dir] : hi[dir];
  const int depth = op.type == BCT_NOSLIP ? 3 : (op.type == BCT_INFLOW ? 0 : 1);
  L.w[0][dir] = L.w[1][dir] = f;
  L.reads = depth > 0;
  L.r[0][dir] = std::min(f + s, f + s * depth);
  L.r[1][dir] = std::max(f + s, f + s * depth);
  return L;
}
bool meet(const int a[2][3], const int b[2][3]) {
  for (int d = 0; d < 3; ++d)
    if (a[1][d] < b[0][d] || b[1][d] < a[0][d]) return false;
  return true;
}

}  // namespace

// Dependency levels of each block's physical-BC ops.  The reference applies a
// block's subfaces one after another; an op must follow an earlier op of its
// block when their written layers meet or one reads what the other writes.
// Its level is one more than the highest level of such earlier ops, so the
// ops of one level touch disjoint nodes, read nothing another writes, and can
// run in one launch with the serial result.
void bc_levels(Topology& out) {
  out.bc_level.assign(out.bc_ops.size(), 0);
  for (size_t m = 0; m + 1 < out.bc_start.size(); ++m) {
    for (int i = out.bc_start[m]; i < out.bc_start[m + 1]; ++i) {
      const Layers Li = bc_layers(out.bc_ops[i]);
      for (int j = out.bc_start[m]; j < i; ++j) {
        const Layers Lj = bc_layers(out.bc_ops[j]);
        bool dep = meet(Lj.w, Li.w) || (Li.reads && meet(Lj.w, Li.r)) || (Lj.reads && meet(Lj.r, Li.w));
        if (dep) out.bc_level[i] = std::max(out.bc_level[i], out.bc_level[j] + 1);
      }
    }
  }
}

namespace {

// 2-D mode (sub_bc_updatebuffer2d.f90, sub_bc_updatebuffercoordinate2d.f90,
// sub_bc_updatebufferaverage2d.f90): a face is a line and ua(ll) runs along
// it (j on faces 1/2, i on faces 3/4), nn = max(n11, n12) of the donor
// subface (:218-222); ori 2 keeps the order, ori 3 reverses it (:284-293).
// The maps below take (l, m) = (ll, 1) when `two` is set.

// (l,m) extents of a donor subface as ua is shaped for its face.
void donor_extent(bool two, const SubRow& d, int& l1, int& m1) {
  if (two) {
    l1 = std::max(d.ie - d.is + 1, d.je - d.js + 1);
    m1 = 1;
    return;
  }
  int n1 = d.ie - d.is + 1, n2 = d.je - d.js + 1, n3 = d.ke - d.ks + 1;
  static const int L[6] = {3, 2, 1, 3, 2, 1};  // extent used for l on faces 1..6
  static const int M[6] = {2, 3, 3, 1, 1, 2};  // extent used for m
  int ext[4] = {0, n1, n2, n3};
  l1 = ext[L[d.face - 1]];
  m1 = ext[M[d.face - 1]];
}

// Donor face node feeding ua(l,m).
void donor_face_node(bool two, const SubRow& d, int l, int m, int& i, int& j, int& k) {
  if (two) {
    k = d.ks;
    i = d.face <= 2 ? (d.face == 1 ? d.is : d.ie) : d.is + l - 1;
    j = d.face <= 2 ? d.js + l - 1 : (d.face == 3 ? d.js : d.je);
    return;
  }
  switch (d.face) {
    case 1: i = d.is; j = d.js + m - 1; k = d.ks + l - 1; break;
    case 2: i = d.ie; j = d.js + l - 1; k = d.ks + m - 1; break;
    case 3: i = d.is + l - 1; j = d.js; k = d.ks + m - 1; break;
    case 4: i = d.is + m - 1; j = d.je; k = d.ks + l - 1; break;
    case 5: i = d.is + m - 1; j = d.js + l - 1; k = d.ks; break;
    default: i = d.is + l - 1; j = d.js + m - 1; k = d.ke; break;
  }
}

// Reoriented array ua2(l2,m2) takes ua(l,m) with (l,m) from (l2,m2) by ori.
void ori_extent(bool two, int ori, int l1, int m1, int& l2, int& m2) {
  bool swap = !two && (ori == 2 || ori == 4);
  l2 = swap ? m1 : l1;
  m2 = swap ? l1 : m1;
}
void ori_source(bool two, int ori, int l1, int m1, int l2i, int m2i, int& l, int& m) {
  if (two) {
    l = ori == 2 ? l2i : l1 - l2i + 1;
    m = m2i;
    return;
  }
  if (ori == 1) { l = l2i; m = m1 - m2i + 1; }
  else if (ori == 2) { l = m2i; m = l2i; }
  else if (ori == 3) { l = l1 - l2i + 1; m = m2i; }
  else { l = l1 - m2i + 1; m = m1 - l2i + 1; }
}

// Receiver face node written by ua2(a,b), and the outward unit step.
void own_face_node(bool two, const SubRow& s, int a, int b, int& i, int& j, int& k, int& di, int& dj, int& dk) {
  di = dj = dk = 0;
  if (two) {
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
    case 1: i = s.is; j = s.js + b - 1; k = s.ks + a - 1; di = -1; break;
    case 2: i = s.ie; j = s.js + a - 1; k = s.ks + b - 1; di = 1; break;
    case 3: i = s.is + a - 1; j = s.js; k = s.ks + b - 1; dj = -1; break;
    case 4: i = s.is + b - 1; j = s.je; k = s.ks + a - 1; dj = 1; break;
    case 5: i = s.is + b - 1; j = s.js + a - 1; k = s.ks; dk = -1; break;
    default: i = s.is + a - 1; j = s.js + b - 1; k = s.ke; dk = 1; break;
  }
}

// Interior step of a donor face (pack reads plane + step*layer).
void inward_step(int face, int& di, int& dj, int& dk) {
  di = dj = dk = 0;
  int s = (face % 2 == 1) ? 1 : -1;
  int dir = (face - 1) / 2;
  if (dir == 0) di = s; else if (dir == 1) dj = s; else dk = s;
}

bool planar(const SubRow& s) {
  int dir = (s.face - 1) / 2;
  return dir == 0 ? s.is == s.ie : dir == 1 ? s.js == s.je : s.ks == s.ke;
}

}  // namespace

std::string build_topology(const std::vector<TopoBlock>& blocks, int buffer_length, int solver,
                           int dimension, Topology& out) {
  char msg[256];
  int nb = (int)blocks.size();
  out = Topology{};
  const bool two = dimension == IFLAG_2D;
  // ---------------------------------------------------------------- validate
  for (int m = 0; m < nb; ++m) {
    for (size_t s = 0; s < blocks[m].subs.size(); ++s) {
      const SubRow& r = blocks[m].subs[s];
      if (r.face < 1 || r.face > (two ? 4 : 6) || !planar(r)) {
        std::snprintf(msg, sizeof msg, "block %d subface %zu: bad face or non-planar range", m + 1, s + 1);
        return msg;
      }
      const Box& b0 = blocks[m].b0;
      if (!b0.contains(r.is, r.js, r.ks) || !b0.contains(r.ie, r.je, r.ke)) {
        std::snprintf(msg, sizeof msg, "block %d subface %zu: range outside the block's nodes", m + 1, s + 1);
        return msg;
      }
      // the no-slip wall reads three nodes inward, the other routines one
      int dir = (r.face - 1) / 2;
      int n0[3] = {b0.nx(), b0.ny(), b0.nz()};
      int need = (r.blk_t == BC_WALL && solver == IFLAG_NSSOLVER) ? 4 : 2;
      if (r.blk_t < 0 && n0[dir] < need) {
        std::snprintf(msg, sizeof msg, "block %d: fewer than %d nodes normal to boundary face %d", m + 1,
                      need, r.face);
        return msg;
      }
      if (r.blk_t > 0) {
        if (r.blk_t > nb || r.subface_t < 1 || r.subface_t > (int)blocks[r.blk_t - 1].subs.size() ||
            (two ? (r.ori != 2 && r.ori != 3) : (r.ori < 1 || r.ori > 4))) {
          std::snprintf(msg, sizeof msg, "block %d subface %zu: bad neighbour/orientation", m + 1, s + 1);
          return msg;
        }
      }
    }
  }
  // ------------------------------------------------------------- halo gather
  // key: (dst block, dst node) -> index into out.halo; a later writer replaces
  // the source, as the later unpack overwrites the earlier one.
  std::map<std::pair<int, long>, size_t> where;
  std::map<std::pair<int, long>, int> srcset;
  for (int m = 0; m < nb; ++m) {
    const TopoBlock& B = blocks[m];
    for (const SubRow& s : B.subs) {
      if (s.blk_t <= 0) continue;
      const TopoBlock& D = blocks[s.blk_t - 1];
      const SubRow& d = D.subs[s.subface_t - 1];
      int l1, m1, l2, m2;
      donor_extent(two, d, l1, m1);
      ori_extent(two, s.ori, l1, m1, l2, m2);
      int own_n = (s.ie - s.is + 1) * (s.je - s.js + 1) * (s.ke - s.ks + 1);
      if (l2 * m2 != own_n) {
        std::snprintf(msg, sizeof msg, "block %d subface %d: neighbour face has %d nodes, own %d",
                      m + 1, s.f_no, l2 * m2, own_n);
        return msg;
      }
      int sdi, sdj, sdk;
      inward_step(d.face, sdi, sdj, sdk);
      for (int b2 = 1; b2 <= m2; ++b2)
        for (int a2 = 1; a2 <= l2; ++a2) {
          int l, mm;
          ori_source(two, s.ori, l1, m1, a2, b2, l, mm);
          int si, sj, sk, oi, oj, ok, di, dj, dk;
          donor_face_node(two, d, l, mm, si, sj, sk);
          own_face_node(two, s, a2, b2, oi, oj, ok, di, dj, dk);
          for (int layer = 1; layer <= buffer_length; ++layer) {
            int gi = oi + di * layer, gj = oj + dj * layer, gk = ok + dk * layer;
            int xi = si + sdi * layer, xj = sj + sdj * layer, xk = sk + sdk * layer;
            if (!B.b.contains(gi, gj, gk) || !D.b0.contains(xi, xj, xk)) {
              std::snprintf(msg, sizeof msg, "block %d subface %d: halo node outside the boxes", m + 1, s.f_no);
              return msg;
            }
            HaloEntry e{m, s.blk_t - 1, B.at(gi, gj, gk), D.at(xi, xj, xk)};
            auto key = std::make_pair(m, e.dst_n);
            auto it = where.find(key);
            if (it == where.end()) {
              where[key] = out.halo.size();
              out.halo.push_back(e);
            } else {
              out.halo[it->second] = e;
            }
          }
        }
    }
  }
  for (const HaloEntry& e : out.halo) srcset[std::make_pair(e.src_blk, e.src_n)] = 1;
  for (const HaloEntry& e : out.halo)
    if (srcset.count(std::make_pair(e.dst_blk, e.dst_n)))
      return "halo: a ghost node is also a donor node (needs a two-phase exchange)";

  // ------------------------------------------------------------ averaging
  // own interface node <- neighbour's node, per subface in reference order.
  std::map<std::pair<int, long>, std::vector<AvgSrc>> contrib;
  std::vector<std::pair<int, long>> order;  // first-appearance order of destinations
  for (int m = 0; m < nb; ++m) {
    const TopoBlock& B = blocks[m];
    for (const SubRow& s : B.subs) {
      if (s.blk_t <= 0) continue;
      const TopoBlock& D = blocks[s.blk_t - 1];
      const SubRow& d = D.subs[s.subface_t - 1];
      int l1, m1, l2, m2;
      donor_extent(two, d, l1, m1);
      ori_extent(two, s.ori, l1, m1, l2, m2);
      // buffer(own node) <- donor face node (average1); then average2 walks the
      // own subface box in k, j, i order.
      std::map<long, AvgSrc> buffer;
      for (int b2 = 1; b2 <= m2; ++b2)
        for (int a2 = 1; a2 <= l2; ++a2) {
          int l, mm;
          ori_source(two, s.ori, l1, m1, a2, b2, l, mm);
          int si, sj, sk, oi, oj, ok, di, dj, dk;
          donor_face_node(two, d, l, mm, si, sj, sk);
          own_face_node(two, s, a2, b2, oi, oj, ok, di, dj, dk);
          buffer[B.at(oi, oj, ok)] = AvgSrc{s.blk_t - 1, D.at(si, sj, sk)};
        }
      for (int k = s.ks; k <= s.ke; ++k)
        for (int j = s.js; j <= s.je; ++j)
          for (int i = s.is; i <= s.ie; ++i) {
            long n = B.at(i, j, k);
            auto it = buffer.find(n);
            if (it == buffer.end()) return "average: interface node without a neighbour value";
            auto key = std::make_pair(m, n);
            if (!contrib.count(key)) order.push_back(key);
            contrib[key].push_back(it->second);
          }
    }
  }
  for (const auto& key : order) {
    const auto& v = contrib[key];
    AvgDst a{key.first, (int)out.avg_src.size(), (int)v.size(), key.second};
    out.avg_dst.push_back(a);
    for (const AvgSrc& x : v) out.avg_src.push_back(x);
  }

  // ------------------------------------------------------- physical BC ops
  out.bc_start.push_back(0);
  for (int m = 0; m < nb; ++m) {
    const TopoBlock& B = blocks[m];
    for (const SubRow& s : B.subs) {
      BcOp op;
      op.face = s.face;
      op.sb = s.box();
      switch (s.blk_t) {
        case BC_INFLOW: op.type = BCT_INFLOW; break;
        case BC_OUTFLOW: op.type = BCT_OUTFLOW; break;
        case BC_SYMM: op.type = BCT_MIRROR; break;
        case BC_WALL:
          if (solver == IFLAG_NSSOLVER) op.type = BCT_NOSLIP;
          else if (solver == IFLAG_EULERSOLVER) op.type = BCT_MIRROR;
          else continue;
          break;
        case BC_FARFIELD:
          op.type = BCT_FARFIELD;
          op.sb.js = B.b.js;  // the reference passes the block's js (sub_bc.f90:59)
          break;
        default:
          continue;  // interfaces; user (-90) and periodic (-60) do nothing here
      }
      out.bc_ops.push_back(op);
    }
    out.bc_start.push_back((int)out.bc_ops.size());
  }
  bc_levels(out);
  return std::string();
}

}  // namespace aero
