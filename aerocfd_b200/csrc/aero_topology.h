// Host-side builders of the device tables that replace the reference's
// per-iteration MPI exchange bookkeeping: the ghost-node gather map of
// UpdateBuffer / UpdateBufferCoordinate, the source/destination lists of
// average1 / average2, and the ordered physical-BC operations of physical_bc.
#pragma once
#include <string>
#include <vector>

#include "aero_kernels.h"

namespace aero {

struct SubRow {
  int f_no, face, is, ie, js, je, ks, ke, blk_t, subface_t, ori;
  Box box() const { return Box{is, ie, js, je, ks, ke}; }
};

struct TopoBlock {
  Box b, b0, b1;
  std::vector<SubRow> subs;
  long at(int i, int j, int k) const {
    return (long)(i - b.is) + (long)b.nx() * ((long)(j - b.js) + (long)b.ny() * (long)(k - b.ks));
  }
};

struct Topology {
  std::vector<HaloEntry> halo;     // ghost <- donor interior, all layers
  std::vector<AvgSrc> avg_src;     // grouped by destination, in reference order
  std::vector<AvgDst> avg_dst;
  std::vector<BcOp> bc_ops;        // per block, bcinfo order
  std::vector<int> bc_start;       // nblock+1 offsets into bc_ops
  std::vector<int> bc_level;       // per op: dependency level within its block (see bc_levels)
};

// Builds all tables (dimension: iflag_dimension, 2 or 3); returns an empty
// string on success or the reason the block/subface description is
// inconsistent.
std::string build_topology(const std::vector<TopoBlock>& blocks, int buffer_length, int solver,
                           int dimension, Topology& out);

// Fills out.bc_level from out.bc_ops and out.bc_start: each op's dependency
// level within its block (build_topology calls it).
void bc_levels(Topology& out);

}  // namespace aero
