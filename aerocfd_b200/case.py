"""Host-side data model of a multi-block case, laid out exactly as the
reference's per-block arrays (module_block.f90:20-91) so the same host buffers
can be handed to the C-ABI drop-in routines.

Every field is a numpy array whose memory is the Fortran column-major array
``a(nc, is:ie, js:je, ks:ke)``; numpy sees it as C-order shape ``(nz, ny, nx, nc)``
(or ``(nz, ny, nx)`` for scalars).  ``Block.at(field, c, i, j, k)`` indexes it
with the reference's 1-based indices.
"""
from __future__ import annotations

import dataclasses
from typing import Dict, List, Sequence, Tuple

import numpy as np

# module_flags.f90:30-87
IFLAG_2D, IFLAG_3D = 2, 3
IFLAG_NSSOLVER, IFLAG_EULERSOLVER = 0, 1
IFLAG_STEADY, IFLAG_UNSTEADY = 0, 1
IFLAG_1STIMPLICIT, IFLAG_2NDCRANK = 2, 3
IFLAG_LAMINAR, IFLAG_SA = 0, 2
IFLAG_3RDWENO = 4
# Extension schemes: the reference defines these flag values (module_flags.f90:
# 68, 71) but stops on them (main.f90:636-653); here iflag_inviscid = 5 is
# Steger-Warming splitting with WENO5 and 8 is WCNS5 with the Roe flux.
IFLAG_5THWENO, IFLAG_5THWCNS = 5, 8
SCHEME_NAMES = {IFLAG_3RDWENO: "roe_weno3", IFLAG_5THWENO: "sw_weno5", IFLAG_5THWCNS: "wcns5_roe"}


def buffer_length_for(inviscid: int) -> int:
    """Ghost layers of a block interface for the inviscid scheme: 2 for the
    3rd-order WENO (GetBufferLength, main.f90:636-653), 3 for the 5th-order
    extension schemes (their stencils reach three nodes past a face)."""
    if inviscid == IFLAG_3RDWENO:
        return 2
    if inviscid in (IFLAG_5THWENO, IFLAG_5THWCNS):
        return 3
    raise ValueError("Buffer length is not correct, please check the iflag_inviscid!")
BC_INFLOW, BC_OUTFLOW, BC_SYMM, BC_WALL, BC_FARFIELD = -50, -40, -30, -20, -10

# Field table shared with include/aerocfd_gpu.h (AERO_F_*): name, components.
FIELDS: List[Tuple[str, int]] = [
    ("q", 5), ("pri_v", 7), ("rhsi", 5), ("rhsv", 5), ("rhs", 5), ("dt", 1),
    ("dxidx", 9), ("inv_j", 1), ("amu", 3), ("nut", 1), ("sa_rhs", 1),
    ("x", 1), ("y", 1), ("z", 1), ("dist", 1), ("alpha", 3), ("beta", 3),
    ("ggamma", 3), ("dudx", 9), ("tao", 6), ("vor", 1), ("length", 1),
    ("spacing", 1), ("q0", 10),
]
FIELD_ID = {name: n for n, (name, _) in enumerate(FIELDS)}
FIELD_NC = dict(FIELDS)


@dataclasses.dataclass
class Subface:
    """One line of the bcinfo file (sub_init_readbcinfo.f90:96-98)."""
    f_no: int
    face: int
    is_: int
    ie: int
    js: int
    je: int
    ks: int
    ke: int
    blk_t: int          # > 0: neighbour block; < 0: physical BC type
    subface_t: int = 0  # neighbour's subface number
    ori: int = 0        # orientation code of the neighbour's face indexing
    fwh: int = 0

    def row(self) -> List[int]:
        return [self.f_no, self.face, self.is_, self.ie, self.js, self.je, self.ks,
                self.ke, self.blk_t, self.subface_t, self.ori]


def index_boxes(ni: int, nj: int, nk: int, subfaces: Sequence[Subface],
                buffer_length: int = 2, dimension: int = IFLAG_3D):
    """The three nested index boxes of a block (sub_init_allocatememory.f90:73-144):
    is..ie includes ``buffer_length`` overlap ghosts on every face that carries a
    block interface; is0..ie0 are the physical nodes 1..ni; is1..ie1 the nodes
    the implicit update touches (physical faces keep their boundary node)."""
    b0 = [1, ni, 1, nj, 1, nk]
    b = list(b0)
    for s in subfaces:
        if s.blk_t > 0:
            d = (s.face - 1) // 2
            if s.face % 2 == 1:
                b[2 * d] = b0[2 * d] - buffer_length
            else:
                b[2 * d + 1] = b0[2 * d + 1] + buffer_length
    b1 = list(b0)
    for d in range(3):
        allow = d < 2 or dimension == IFLAG_3D
        b1[2 * d] = b0[2 * d] + 1 if (b0[2 * d] == b[2 * d] and allow) else b0[2 * d]
        b1[2 * d + 1] = b0[2 * d + 1] - 1 if (b0[2 * d + 1] == b[2 * d + 1] and allow) else b0[2 * d + 1]
    return b, b0, b1


class Block:
    def __init__(self, m: int, ni: int, nj: int, nk: int, subfaces: Sequence[Subface],
                 buffer_length: int = 2, dimension: int = IFLAG_3D):
        self.m = m
        self.ni, self.nj, self.nk = ni, nj, nk
        self.subfaces = list(subfaces)
        self.box, self.box0, self.box1 = index_boxes(ni, nj, nk, self.subfaces, buffer_length, dimension)
        is_, ie, js, je, ks, ke = self.box
        self.shape = (ke - ks + 1, je - js + 1, ie - is_ + 1)
        self.fields: Dict[str, np.ndarray] = {}
        for name, nc in FIELDS:
            shp = self.shape + ((nc,) if nc > 1 else ())
            self.fields[name] = np.zeros(shp, dtype=np.float64)

    @property
    def nodes(self) -> int:
        return self.ni * self.nj * self.nk

    def box18(self) -> np.ndarray:
        return np.array(self.box + self.box0 + self.box1, dtype=np.int32)

    def sub_table(self) -> np.ndarray:
        return np.array([s.row() for s in self.subfaces], dtype=np.int32).reshape(-1, 11)

    def sl(self, box=None):
        """numpy slices (k, j, i) selecting a Fortran index box."""
        is_, ie, js, je, ks, ke = self.box
        b = box if box is not None else self.box
        return (slice(b[4] - ks, b[5] - ks + 1), slice(b[2] - js, b[3] - js + 1),
                slice(b[0] - is_, b[1] - is_ + 1))

    def at(self, name: str, c: int, i: int, j: int, k: int) -> float:
        is_, _, js, _, ks, _ = self.box
        a = self.fields[name]
        if a.ndim == 4:
            return a[k - ks, j - js, i - is_, c - 1]
        return a[k - ks, j - js, i - is_]

    def ptr(self, name: str) -> int:
        return self.fields[name].ctypes.data


@dataclasses.dataclass
class Config:
    """Control.in values on the path (sub_init_readcontrolfile.f90:30-47)."""
    dimension: int = IFLAG_3D
    solver: int = IFLAG_EULERSOLVER
    time: int = IFLAG_STEADY
    timeadvance: int = IFLAG_1STIMPLICIT
    turbulence: int = IFLAG_LAMINAR
    des: int = 0
    inviscid: int = IFLAG_3RDWENO
    ma: float = 0.5
    re: float = 1.0e6
    tinf: float = 288.15
    aoa_deg: float = 0.0
    cfl: float = 5.0
    dt: float = 1.0
    nutinf: float = 1.341946   # module_tursa.f90:11

    @property
    def buffer_length(self) -> int:
        """bufferLength, derived from iflag_inviscid as main.f90:81 does."""
        return buffer_length_for(self.inviscid)

    def iflags(self) -> np.ndarray:
        return np.array([self.dimension, self.solver, self.time, self.timeadvance,
                         self.turbulence, self.des, self.buffer_length, self.inviscid],
                        dtype=np.int32)

    def params(self) -> np.ndarray:
        return np.array([self.ma, self.re, self.tinf, self.aoa_deg, self.cfl, self.dt,
                         self.nutinf], dtype=np.float64)


class Case:
    """A set of blocks plus the Control.in values (one reference run)."""

    def __init__(self, name: str, cfg: Config, blocks: List[Block]):
        self.name = name
        self.cfg = cfg
        self.blocks = blocks
        self.check_topology()

    @property
    def nodes(self) -> int:
        return sum(b.nodes for b in self.blocks)

    def check_topology(self) -> None:
        """Rejects what the reference would reject or corrupt: a face that is both
        physical and an interface (main.f90:655-690, CheckBoundary), non-planar
        subfaces, and interface pairs that do not point back at each other."""
        for b in self.blocks:
            phys, itf = set(), set()
            for s in b.subfaces:
                d = (s.face - 1) // 2
                lo, hi = [(s.is_, s.ie), (s.js, s.je), (s.ks, s.ke)][d]
                if lo != hi:
                    raise ValueError(f"block {b.m} subface {s.f_no}: face {s.face} is not planar")
                (itf if s.blk_t > 0 else phys).add(s.face)
            if phys & itf:
                raise ValueError(f"block {b.m}: face(s) {sorted(phys & itf)} both physical and interface")
            for n, s in enumerate(b.subfaces, start=1):
                if s.blk_t > 0:
                    t = self.blocks[s.blk_t - 1].subfaces[s.subface_t - 1]
                    if t.blk_t != b.m or t.subface_t != n:
                        raise ValueError(f"block {b.m} subface {n}: partner does not point back")
