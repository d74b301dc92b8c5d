"""Dependency levels of the physical-BC operations (aero_topology.cpp,
bc_levels), checked on the host: the topology source compiled as plain C++
and run on hand-made subface lists.  Ops of one level must touch disjoint
nodes and read nothing another writes; an op that overlaps an earlier one
must come after it, as the reference applies a block's subfaces in order
(sub_bc.f90:26-62)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SRC = r"""
#include <cmath>
using std::fabs; using std::fma;
#define __host__
#define __device__
#define __global__
#define __forceinline__ inline
#define __noinline__
#include "aero_topology.cpp"
#include <cstdio>
using namespace aero;

static BcOp op(int type, int face, int is, int ie, int js, int je, int ks, int ke) {
  BcOp o;
  o.type = type;
  o.face = face;
  o.sb = Box{is, ie, js, je, ks, ke};
  return o;
}
static int fails = 0;
static void expect(const char* what, const Topology& t, std::vector<int> want) {
  bool ok = t.bc_level == want;
  if (!ok) {
    ++fails;
    std::printf("%s: got", what);
    for (int l : t.bc_level) std::printf(" %d", l);
    std::printf("\n");
  }
}
int main() {
  {  // aerofoil O-grid block 129 x 65 x 3: wall, farfield, two symmetry planes
    Topology t;
    t.bc_ops = {op(BCT_NOSLIP, 3, 1, 129, 1, 1, 1, 3), op(BCT_FARFIELD, 4, 1, 129, 1, 65, 1, 3),
                op(BCT_MIRROR, 5, 1, 129, 1, 65, 1, 1), op(BCT_MIRROR, 6, 1, 129, 1, 65, 3, 3)};
    t.bc_start = {0, 4};
    bc_levels(t);
    expect("aerofoil block", t, {0, 0, 1, 1});
  }
  {  // the same subfaces, symmetry planes first: the j faces meet both
    Topology t;
    t.bc_ops = {op(BCT_MIRROR, 5, 1, 129, 1, 65, 1, 1), op(BCT_MIRROR, 6, 1, 129, 1, 65, 3, 3),
                op(BCT_NOSLIP, 3, 1, 129, 1, 1, 1, 3), op(BCT_FARFIELD, 4, 1, 129, 1, 65, 1, 3)};
    t.bc_start = {0, 4};
    bc_levels(t);
    expect("symmetry first", t, {0, 0, 1, 1});
  }
  {  // thin block (4 nodes in j): the no-slip wall reads j = 2..4, which the
     // farfield writes (j = 4), so the farfield must follow it
    Topology t;
    t.bc_ops = {op(BCT_NOSLIP, 3, 1, 9, 1, 1, 1, 5), op(BCT_FARFIELD, 4, 1, 9, 1, 4, 1, 5)};
    t.bc_start = {0, 2};
    bc_levels(t);
    expect("thin block", t, {0, 1});
  }
  {  // the same with 5 nodes in j: no overlap, one level
    Topology t;
    t.bc_ops = {op(BCT_NOSLIP, 3, 1, 9, 1, 1, 1, 5), op(BCT_FARFIELD, 4, 1, 9, 1, 5, 1, 5)};
    t.bc_start = {0, 2};
    bc_levels(t);
    expect("5 nodes in j", t, {0, 0});
  }
  {  // inflow reads nothing, outflow one layer: opposite i faces of a 3-node
     // block are independent (outflow reads i = 2, inflow writes i = 1)
    Topology t;
    t.bc_ops = {op(BCT_INFLOW, 1, 1, 1, 1, 9, 1, 9), op(BCT_OUTFLOW, 2, 3, 3, 1, 9, 1, 9)};
    t.bc_start = {0, 2};
    bc_levels(t);
    expect("inflow / outflow", t, {0, 0});
  }
  {  // two subfaces side by side on one face, then a third across both edges:
     // a chain only where layers meet
    Topology t;
    t.bc_ops = {op(BCT_MIRROR, 5, 1, 10, 1, 5, 1, 1), op(BCT_NOSLIP, 5, 11, 20, 1, 5, 1, 1),
                op(BCT_OUTFLOW, 2, 20, 20, 1, 5, 1, 7), op(BCT_OUTFLOW, 1, 1, 1, 1, 5, 1, 7)};
    t.bc_start = {0, 4};
    bc_levels(t);
    expect("split face", t, {0, 0, 1, 1});
  }
  {  // levels are per block: the second block starts again at 0
    Topology t;
    t.bc_ops = {op(BCT_MIRROR, 5, 1, 9, 1, 9, 1, 1), op(BCT_MIRROR, 1, 1, 1, 1, 9, 1, 9),
                op(BCT_MIRROR, 5, 1, 9, 1, 9, 1, 1), op(BCT_MIRROR, 6, 1, 9, 1, 9, 9, 9)};
    t.bc_start = {0, 2, 4};
    bc_levels(t);
    expect("two blocks", t, {0, 1, 0, 0});
  }
  std::printf("fails=%d\n", fails);
  return fails != 0;
}
"""


def test_bc_levels(tmp_path):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("g++ not available")
    src = tmp_path / "t.cpp"
    src.write_text(SRC)
    exe = tmp_path / "t"
    subprocess.run([cxx, "-O1", "-std=c++17", "-I", os.path.join(ROOT, "aerocfd_b200", "csrc"),
                    "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
