"""2-D interface exchange (UpdateBuffer2d, UpdateBufferCoordinate2d,
average2d1/2d2): the gather and averaging tables the device applies
(aero_topology.cpp, compiled here as plain C++) give, applied with numpy, the
same bits as the oracle's restatement of the reference's pack / reorient /
unpack on random fields.  Two 2-D cases: the four-block aerofoil O-grid
(shared faces in the same direction, orientation code 2) and the two-block
bump channel whose second block is turned by 180 degrees (opposite
directions, code 3)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from aerocfd_b200 import grids
from aerocfd_b200.case import IFLAG_2D, IFLAG_NSSOLVER, IFLAG_SA, Config

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
#include <cstdlib>
using namespace aero;

// stdin: dimension bufferLength solver nblock, then per block its 18 box
// indices, its subface count and 11 integers per subface.  stdout: the halo
// gather (H dst_blk dst_n src_blk src_n), the averaging destinations in
// order (A blk n count) each followed by its sources (S blk n).
int main() {
  int dim, bl, solver, nb;
  auto get = [](int& v) { if (std::scanf("%d", &v) != 1) std::exit(2); };
  get(dim); get(bl); get(solver); get(nb);
  std::vector<TopoBlock> tb(nb);
  for (int m = 0; m < nb; ++m) {
    int v[18], ns;
    for (int x = 0; x < 18; ++x) get(v[x]);
    tb[m].b = Box{v[0], v[1], v[2], v[3], v[4], v[5]};
    tb[m].b0 = Box{v[6], v[7], v[8], v[9], v[10], v[11]};
    tb[m].b1 = Box{v[12], v[13], v[14], v[15], v[16], v[17]};
    get(ns);
    for (int s = 0; s < ns; ++s) {
      int r[11];
      for (int x = 0; x < 11; ++x) get(r[x]);
      tb[m].subs.push_back(SubRow{r[0], r[1], r[2], r[3], r[4], r[5], r[6], r[7], r[8], r[9], r[10]});
    }
  }
  Topology t;
  std::string why = build_topology(tb, bl, solver, dim, t);
  if (!why.empty()) {
    std::printf("E %s\n", why.c_str());
    return 1;
  }
  for (const HaloEntry& e : t.halo) std::printf("H %d %ld %d %ld\n", e.dst_blk, e.dst_n, e.src_blk, e.src_n);
  for (const AvgDst& a : t.avg_dst) {
    std::printf("A %d %ld %d\n", a.blk, a.n, a.count);
    for (int x = 0; x < a.count; ++x) {
      const AvgSrc& s = t.avg_src[a.first + x];
      std::printf("S %d %ld\n", s.blk, s.n);
    }
  }
  return 0;
}
"""


@pytest.fixture(scope="module")
def tables_exe(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no host C++ compiler")
    d = tmp_path_factory.mktemp("halo2d")
    src = d / "halo2d.cpp"
    src.write_text(SRC)
    exe = d / "halo2d"
    subprocess.run([cxx, "-std=c++17", "-O1", "-I", os.path.join(ROOT, "aerocfd_b200", "csrc"), str(src),
                    "-o", str(exe)], check=True)
    return str(exe)


def tables(exe, case):
    cfg = case.cfg
    lines = [f"{cfg.dimension} {cfg.buffer_length} {cfg.solver} {len(case.blocks)}"]
    for b in case.blocks:
        lines.append(" ".join(map(str, b.box18())))
        lines.append(str(len(b.subfaces)))
        for s in b.subfaces:
            lines.append(" ".join(map(str, s.row())))
    out = subprocess.run([exe], input="\n".join(lines) + "\n", capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    halo, avg = [], []
    for ln in out.stdout.splitlines():
        p = ln.split()
        if p[0] == "H":
            halo.append(tuple(int(x) for x in p[1:]))
        elif p[0] == "A":
            avg.append([int(p[1]), int(p[2]), int(p[3]), []])
        elif p[0] == "S":
            avg[-1][3].append((int(p[1]), int(p[2])))
    return halo, avg


def naca2d():
    cfg = Config(solver=IFLAG_NSSOLVER, ma=0.5, re=5000.0, aoa_deg=2.0, cfl=2.0, dimension=IFLAG_2D,
                 turbulence=IFLAG_SA)
    return grids.naca_ogrid(nblk=4, ni=17, nj=9, cfg=cfg)


def bump2d():
    return grids.bump_channel_2d(ni=33, nj=13)


def randomise(case, seed):
    rng = np.random.default_rng(seed)
    for b in case.blocks:
        for name in ("q", "nut", "x", "y", "z"):
            b.fields[name][...] = rng.standard_normal(b.fields[name].shape)


def flat(b, name):
    a = b.fields[name]
    return a.reshape(-1, a.shape[-1]) if a.ndim == 4 else a.reshape(-1, 1)


@pytest.mark.parametrize("make", [naca2d, bump2d], ids=["ogrid_ori2", "rotated_ori3"])
def test_2d_halo_and_average_tables_match_the_oracle(oracle_mod, tables_exe, make):
    case = make()
    assert {s.ori for b in case.blocks for s in b.subfaces if s.blk_t > 0} <= {2, 3}
    halo, avg = tables(tables_exe, case)
    assert halo and avg
    oc = oracle_mod.OracleCase(case)
    names = ("q", "nut") if case.cfg.turbulence else ("q",)
    # UpdateBuffer2d
    randomise(case, 1)
    want = {(b.m, n): flat(b, n).copy() for b in case.blocks for n in names}
    for dst_b, dst_n, src_b, src_n in halo:
        for n in names:
            want[(dst_b + 1, n)][dst_n] = flat(case.blocks[src_b], n)[src_n]
    oc.updatebuffer()
    for b in case.blocks:
        for n in names:
            assert np.array_equal(flat(b, n), want[(b.m, n)]), (b.m, n)
    # UpdateBufferCoordinate2d: the same gather on x, y, z
    randomise(case, 2)
    want = {(b.m, n): flat(b, n).copy() for b in case.blocks for n in ("x", "y", "z")}
    for dst_b, dst_n, src_b, src_n in halo:
        for n in ("x", "y", "z"):
            want[(dst_b + 1, n)][dst_n] = flat(case.blocks[src_b], n)[src_n]
    oc.L.oracle_updatebuffercoordinate()
    for b in case.blocks:
        for n in ("x", "y", "z"):
            assert np.array_equal(flat(b, n), want[(b.m, n)]), (b.m, n)
    # average2d1 + average2d2: the neighbour values are taken before any
    # node is averaged, then each subface averages in turn
    randomise(case, 3)
    orig = {(b.m, n): flat(b, n).copy() for b in case.blocks for n in names}
    want = {k: v.copy() for k, v in orig.items()}
    for blk, node, _cnt, srcs in avg:
        for n in names:
            v = orig[(blk + 1, n)][node].copy()
            for sb, sn in srcs:
                v = (v + orig[(sb + 1, n)][sn]) * 0.5
            want[(blk + 1, n)][node] = v
    oc.average1()
    oc.average2()
    for b in case.blocks:
        for n in names:
            assert np.array_equal(flat(b, n), want[(b.m, n)]), (b.m, n)


def test_2d_tables_reject_k_faces_and_3d_orientations(tables_exe):
    from aerocfd_b200.case import BC_SYMM, Subface
    case = bump2d()
    case.blocks[0].subfaces[1].ori = 1      # a 3-D code on a 2-D interface
    with pytest.raises(AssertionError, match="orientation"):
        tables(tables_exe, case)
    case = bump2d()
    b = case.blocks[0]
    b.subfaces.append(Subface(5, 5, 1, b.ni, 1, b.nj, 1, 1, BC_SYMM))   # a k face in 2-D
    with pytest.raises(AssertionError, match="bad face"):
        tables(tables_exe, case)
