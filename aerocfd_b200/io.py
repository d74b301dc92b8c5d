"""Reference file formats: Control.in, the grid and bcinfo files, and the
flow-field output that also serves as the restart file.

The reference reads all three with Fortran list-directed input on rank 0:

* Control.in — sub_init_readcontrolfile.f90:30-47: seven value lines, each
  after two comment lines;
* grid — sub_init_allocatememory.f90:36-71 and :380-410: ``nblock``; one
  ``ni nj [nk]`` line per block; then per block one list of x, y[, z] over
  the physical nodes, i fastest, scaled by ``scale_*/lref``;
* bcinfo — sub_init_readbcinfo.f90:45-104: three header lines; per block two
  lines, ``num_subface``, one line, one row per subface
  ``f_no face is ie js je [ks ke] blk_t subface_t ori fwh`` and one line.

``read_*`` accept what a list-directed read accepts (blanks or commas as
separators, ``d`` exponents, quoted strings, ``r*value`` repeats); ``write_*``
produce files the reference can read.  ``load_case`` builds a
:class:`~aerocfd_b200.case.Case` from a Control.in and the grid and bcinfo it
names; ``save_case`` writes the three files for a case.  ``write_flowfield``
and ``read_restart`` follow sub_output_flowfield.f90 and the restart branch of
sub_init_flowfield.f90.
"""
from __future__ import annotations

import os
import re
from dataclasses import dataclass, field
from typing import Iterator, List, Sequence, Tuple

import numpy as np

from .case import Block, Case, Config, Subface, IFLAG_2D, IFLAG_3D, buffer_length_for

_TOKEN = re.compile(r"'[^']*'|\"[^\"]*\"|[^\s,]+")


def _tokens(line: str) -> List[str]:
    """Values of one list-directed record (a '/' ends the record)."""
    out: List[str] = []
    for t in _TOKEN.findall(line):
        if t == "/":
            break
        if t[0] in "'\"":
            out.append(t[1:-1])
            continue
        m = re.fullmatch(r"(\d+)\*(.*)", t)
        if m and m.group(2):
            out.extend([m.group(2)] * int(m.group(1)))
        else:
            out.append(t)
    return out


def _num(t: str) -> float:
    return float(t.replace("d", "e").replace("D", "e"))


class _Reader:
    """Sequential list-directed reads over the lines of a file.  Like Fortran,
    a read takes values from as many records as it needs and drops the rest of
    the last one."""

    def __init__(self, path: str):
        with open(path) as f:
            self.lines = f.read().splitlines()
        self.pos = 0
        self.path = path

    def skip(self, n: int = 1) -> None:
        self.pos += n

    def read(self, n: int) -> List[str]:
        vals: List[str] = []
        while len(vals) < n:
            if self.pos >= len(self.lines):
                raise ValueError(f"{self.path}: end of file after {len(vals)} of {n} values")
            vals.extend(_tokens(self.lines[self.pos]))
            self.pos += 1
        return vals[:n]

    def read_records(self, n: int, m: int) -> np.ndarray:
        """n read statements of m values each: every read starts on a new
        record and drops what is left of its last one."""
        out = np.empty((n, m))
        for r in range(n):
            out[r] = [_num(t) for t in self.read(m)]
        return out

    def read_array(self, n: int) -> np.ndarray:
        out = np.empty(n)
        k = 0
        while k < n:
            if self.pos >= len(self.lines):
                raise ValueError(f"{self.path}: end of file after {k} of {n} values")
            toks = _tokens(self.lines[self.pos])
            self.pos += 1
            take = toks[: n - k]
            out[k:k + len(take)] = [_num(t) for t in take]
            k += len(take)
        return out


# ----------------------------------------------------------------- Control.in
@dataclass
class Control:
    """The values of Control.in (sub_init_readcontrolfile.f90:30-47)."""
    iflag_dimension: int = IFLAG_3D
    iflag_solver: int = 1
    iflag_time: int = 0
    cfl: float = 5.0
    dt: float = 1.0
    ma: float = 0.5
    re: float = 1.0e6
    tinf: float = 288.15
    aoa: float = 0.0
    scale_x: float = 1.0
    scale_y: float = 1.0
    scale_z: float = 1.0
    lref: float = 1.0
    sref: float = 1.0
    fltr: float = 0.0
    iflag_splittingtype: int = 3
    iflag_inviscid: int = 4
    iflag_filter: int = 0
    iflag_timeadvance: int = 2
    iflag_turbulence: int = 0
    iflag_des: int = 0
    writeinterval: int = 1000
    ntstep: int = 1000
    grid: str = "grid.dat"
    bcinfo: str = "bcinfo.dat"
    iflag_init: int = 0
    restartfile: str = "restart.dat"
    nfile: int = 0
    restart_timestep: int = 0
    acoustic: List[float] = field(default_factory=lambda: [0, 0.0, 0.0, 0, 0, 0, 0, 0, 0, 0])

    LINES = (
        ("iflag_dimension", int), ("iflag_solver", int), ("iflag_time", int), ("cfl", float), ("dt", float)), (
        ("ma", float), ("re", float), ("tinf", float), ("aoa", float)), (
        ("scale_x", float), ("scale_y", float), ("scale_z", float), ("lref", float), ("sref", float),
        ("fltr", float)), (
        ("iflag_splittingtype", int), ("iflag_inviscid", int), ("iflag_filter", int),
        ("iflag_timeadvance", int), ("iflag_turbulence", int), ("iflag_des", int)), (
        ("writeinterval", int), ("ntstep", int), ("grid", str), ("bcinfo", str), ("iflag_init", int),
        ("restartfile", str), ("nfile", int), ("restart_timestep", int))

    def config(self, nutinf: float = 1.341946) -> Config:
        """The library's Config (bufferLength from iflag_inviscid, as GetBufferLength,
        main.f90:636-653, does for the 3rd-order WENO)."""
        buffer_length_for(self.iflag_inviscid)  # rejects what the reference rejects
        return Config(dimension=self.iflag_dimension, solver=self.iflag_solver, time=self.iflag_time,
                      timeadvance=self.iflag_timeadvance, turbulence=self.iflag_turbulence, des=self.iflag_des,
                      inviscid=self.iflag_inviscid, ma=self.ma, re=self.re, tinf=self.tinf,
                      aoa_deg=self.aoa, cfl=self.cfl, dt=self.dt, nutinf=nutinf)


def read_control(path: str) -> Control:
    r = _Reader(path)
    c = Control()
    for names in Control.LINES:
        r.skip(2)
        vals = r.read(len(names))
        for (name, typ), v in zip(names, vals):
            setattr(c, name, int(_num(v)) if typ is int else (_num(v) if typ is float else v))
    r.skip(2)
    c.acoustic = [_num(v) for v in r.read(10)]
    return c


def _fmt(v) -> str:
    if isinstance(v, str):
        return f"'{v}'"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    return repr(float(v))


def write_control(path: str, c: Control) -> None:
    heads = ("dimension solver time cfl dt", "ma re tinf aoa", "scale_x scale_y scale_z lref sref fltr",
             "splitting inviscid filter timeadvance turbulence des",
             "writeinterval ntstep grid bcinfo init restartfile nfile restart_timestep")
    out = []
    for head, names in zip(heads, Control.LINES):
        out += ["!" + "-" * 60, "! " + head, " ".join(_fmt(getattr(c, n)) for n, _ in names)]
    out += ["!" + "-" * 60, "! acoustic / averaging", " ".join(_fmt(v) for v in c.acoustic)]
    with open(path, "w") as f:
        f.write("\n".join(out) + "\n")


# ----------------------------------------------------------------------- grid
def read_grid(path: str, dimension: int = IFLAG_3D, scale: Sequence[float] = (1.0, 1.0, 1.0),
              lref: float = 1.0) -> List[Tuple[int, int, int, np.ndarray, np.ndarray, np.ndarray]]:
    """Blocks as (ni, nj, nk, X, Y, Z) with X etc. of shape (nk, nj, ni),
    scaled by scale_*/lref as the reference does."""
    r = _Reader(path)
    nblock = int(_num(r.read(1)[0]))
    dims = []
    for _ in range(nblock):
        if dimension == IFLAG_3D:
            ni, nj, nk = (int(_num(v)) for v in r.read(3))
        else:
            ni, nj = (int(_num(v)) for v in r.read(2))
            nk = 1
        dims.append((ni, nj, nk))
    out = []
    for ni, nj, nk in dims:
        n = ni * nj * nk
        ncomp = 3 if dimension == IFLAG_3D else 2
        vals = r.read_array(ncomp * n)
        xyz = [vals[c * n:(c + 1) * n].reshape(nk, nj, ni) for c in range(ncomp)]
        if ncomp == 2:
            xyz.append(np.zeros((nk, nj, ni)))
        out.append((ni, nj, nk, xyz[0] * scale[0] / lref, xyz[1] * scale[1] / lref, xyz[2] * scale[2] / lref))
    return out


def write_grid(path: str, blocks: Sequence[Tuple[np.ndarray, np.ndarray, np.ndarray]]) -> None:
    """blocks: (X, Y, Z) arrays of shape (nk, nj, ni); values written with 17
    significant digits (exact round trip), five per line."""
    with open(path, "w") as f:
        f.write(f"{len(blocks)}\n")
        for X, _, _ in blocks:
            nk, nj, ni = X.shape
            f.write(f"{ni} {nj} {nk}\n")
        for X, Y, Z in blocks:
            vals = np.concatenate([X.ravel(), Y.ravel(), Z.ravel()])
            for s in range(0, len(vals), 5):
                f.write(" ".join(f"{v:.17e}" for v in vals[s:s + 5]) + "\n")


# --------------------------------------------------------------------- bcinfo
def read_bcinfo(path: str, nblock: int, dimension: int = IFLAG_3D) -> List[List[Subface]]:
    r = _Reader(path)
    r.skip(3)
    out = []
    for _ in range(nblock):
        r.skip(2)
        nsub = int(_num(r.read(1)[0]))
        r.skip(1)
        subs = []
        for _ in range(nsub):
            if dimension == IFLAG_3D:
                v = [int(_num(x)) for x in r.read(12)]
                f_no, face, is_, ie, js, je, ks, ke, blk_t, sub_t, ori = v[:11]
            else:
                v = [int(_num(x)) for x in r.read(10)]
                f_no, face, is_, ie, js, je, blk_t, sub_t, ori = v[:9]
                ks = ke = 1
            subs.append(Subface(f_no, face, is_, ie, js, je, ks, ke, blk_t, sub_t, ori))
        r.skip(1)
        out.append(subs)
    return out


def write_bcinfo(path: str, blocks: Sequence[Sequence[Subface]]) -> None:
    lines = ["! bcinfo", "! f_no face is ie js je ks ke blk_t subface_t ori fwh", "!"]
    for m, subs in enumerate(blocks, start=1):
        lines += [f"! block {m}", "! num_subface", str(len(subs)), "!"]
        for s in subs:
            lines.append(" ".join(str(int(v)) for v in (s.f_no, s.face, s.is_, s.ie, s.js, s.je, s.ks, s.ke,
                                                        s.blk_t, s.subface_t, s.ori, 0)))
        lines.append("!")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


# ---------------------------------------------------------------------- cases
def load_case(control_path: str, name: str = "case") -> Tuple[Case, Control]:
    """Control.in plus the grid and bcinfo files it names (relative to its
    directory) as a Case with the physical-node coordinates set."""
    c = read_control(control_path)
    base = os.path.dirname(os.path.abspath(control_path))
    grid = read_grid(os.path.join(base, c.grid), c.iflag_dimension, (c.scale_x, c.scale_y, c.scale_z), c.lref)
    subs = read_bcinfo(os.path.join(base, c.bcinfo), len(grid), c.iflag_dimension)
    cfg = c.config()
    blocks = []
    for m, ((ni, nj, nk, X, Y, Z), sb) in enumerate(zip(grid, subs), start=1):
        blk = Block(m, ni, nj, nk, sb, cfg.buffer_length, cfg.dimension)
        s = blk.sl(blk.box0)
        blk.fields["x"][s] = X
        blk.fields["y"][s] = Y
        blk.fields["z"][s] = Z
        blocks.append(blk)
    return Case(name, cfg, blocks), c


def save_case(case: Case, directory: str, control: Control = None) -> str:
    """Writes Control.in, grid.dat and bcinfo.dat for `case`; returns the
    Control.in path."""
    os.makedirs(directory, exist_ok=True)
    cfg = case.cfg
    c = control or Control()
    c.iflag_dimension, c.iflag_solver, c.iflag_time = cfg.dimension, cfg.solver, cfg.time
    c.cfl, c.dt, c.ma, c.re, c.tinf, c.aoa = cfg.cfl, cfg.dt, cfg.ma, cfg.re, cfg.tinf, cfg.aoa_deg
    c.iflag_inviscid, c.iflag_timeadvance = cfg.inviscid, cfg.timeadvance
    c.iflag_turbulence, c.iflag_des = cfg.turbulence, cfg.des
    c.scale_x = c.scale_y = c.scale_z = c.lref = 1.0
    write_grid(os.path.join(directory, c.grid),
               [tuple(b.fields[n][b.sl(b.box0)] for n in ("x", "y", "z")) for b in case.blocks])
    write_bcinfo(os.path.join(directory, c.bcinfo), [b.subfaces for b in case.blocks])
    path = os.path.join(directory, "Control.in")
    write_control(path, c)
    return path


# ------------------------------------------------- flow field output / restart
def write_flowfield(path: str, case: Case) -> None:
    """flowfield_output (sub_output_flowfield.f90:15-90): per block a
    Tecplot point-format zone of x, y, z, d, u, v, w, p, nut over the physical
    nodes, i fastest (2-D, :36-57: x, y, d, u, v, w, p, nut and no k
    extent), from the case's host arrays (sync them from the device first).
    Values carry 17 significant digits, so the file restarts a run exactly as
    the reference's list-directed output does."""
    two = case.cfg.dimension == IFLAG_2D
    with open(path, "w") as f:
        for b in case.blocks:
            s = b.sl(b.box0)
            pri = b.fields["pri_v"][s]
            xyz = [b.fields["x"][s], b.fields["y"][s]] + ([] if two else [b.fields["z"][s]])
            cols = xyz + [pri[..., c] for c in range(5)] + [b.fields["nut"][s]]
            if two:
                f.write(" variables = x,y,d,u,v,w,p,nut\n")
                f.write(f" zone i= {b.ni} j= {b.nj} datapacking=point\n")
            else:
                f.write(" variables = x,y,z,d,u,v,w,p,nut\n")
                f.write(f" zone i= {b.ni} j= {b.nj} k= {b.nk} datapacking=point\n")
            table = np.stack([c.ravel() for c in cols], axis=1)
            for row in table:
                f.write(" ".join(f"{v:.17e}" for v in row) + "\n")


def surface_path(timestep: int, rank: int = 0, directory: str = "result") -> str:
    """The reference's surface file name (sub_output_surface.f90:30)."""
    return os.path.join(directory, f"surfcp_{timestep:06d}_{rank:04d}.dat")


def write_surface(path: str, zones: np.ndarray, rows: np.ndarray) -> None:
    """surface_output's file (sub_output_surface.f90:32-113): per wall subface
    a Tecplot point-format zone header and its x, y, z, cp rows, in the order
    ``GpuCase.surface_output`` returns them; 17 significant digits."""
    off = 0
    with open(path, "w") as f:
        for _, _, idim, jdim, kdim in np.asarray(zones).tolist():
            f.write(" variables = x,y,z,cp\n")
            f.write(f" zone i= {idim} j= {jdim} k= {kdim} datapacking=point\n")
            n = idim * jdim * kdim if min(idim, jdim, kdim) > 0 else 0
            for row in rows[off:off + n]:
                f.write(" ".join(f"{v:.17e}" for v in row) + "\n")
            off += n


def read_surface(path: str) -> List[Tuple[Tuple[int, int, int], np.ndarray]]:
    """Zones of a surface file: ((idim, jdim, kdim), rows x 4) each."""
    out = []
    r = _Reader(path)
    while r.pos < len(r.lines) and r.lines[r.pos].strip():
        r.skip(1)
        head = r.read(7)
        dims = (int(head[2]), int(head[4]), int(head[6]))
        n = dims[0] * dims[1] * dims[2] if min(dims) > 0 else 0
        out.append((dims, r.read_array(4 * n).reshape(n, 4)))
    return out


def read_restart(path: str, case: Case) -> None:
    """The restart branch of sub_init_flowfield.f90:117-268 (iflag_init = 1):
    reads a flowfield file written by flowfield_output and sets, on the
    physical nodes of every block, q from (d, u, v, w, p), the primitive
    variables the reference derives there, rhs = rhsi = rhsv = 0, dt = the
    Control.in dt, amu(1) = 1 and, with SA, nut.  The derived primitives keep
    the reference's expressions, including q2 = d**2 + u**2 + v**2 and
    c = sqrt(p)/ma; the iteration's start-up recomputes them from q.

    2-D (:163-210): each record holds seven values, x, y, d, u, v, p, nut (the
    reference reads no w there; its w array is never set on that branch and
    is taken as 0 here).  A 2-D file of flowfield_output has eight columns
    (w before p), which this record layout reads as the reference does: the
    first seven values of each line."""
    cfg = case.cfg
    gamma = 1.4
    ma = cfg.ma
    cv = 1.0 / gamma / (gamma - 1.0) / ma / ma
    two = cfg.dimension == IFLAG_2D
    r = _Reader(path)
    for b in case.blocks:
        r.skip(2)
        n = b.ni * b.nj * b.nk
        if two:
            rows = r.read_records(n, 7)
            col = lambda c: rows[:, c].reshape(b.nk, b.nj, b.ni)
            d, u, v, p, tur = col(2), col(3), col(4), col(5), col(6)
            w = np.zeros_like(d)
        else:
            vals = r.read_array(9 * n).reshape(n, 9)
            col = lambda c: vals[:, c].reshape(b.nk, b.nj, b.ni)
            d, u, v, w, p, tur = col(3), col(4), col(5), col(6), col(7), col(8)
        s = b.sl(b.box0)
        t = p / d * gamma * ma * ma
        q = b.fields["q"][s]
        q[..., 0] = d
        q[..., 1] = d * u
        q[..., 2] = d * v
        q[..., 3] = d * w
        q[..., 4] = d * t * cv + 0.5 * d * (u * u + v * v + w * w)
        pri = b.fields["pri_v"][s]
        pri[..., 0] = q[..., 0]
        pri[..., 1] = q[..., 1] / pri[..., 0]
        pri[..., 2] = q[..., 2] / pri[..., 0]
        pri[..., 3] = q[..., 3] / pri[..., 0]
        q2 = pri[..., 0] ** 2 + pri[..., 1] ** 2 + pri[..., 2] ** 2
        pri[..., 5] = (q[..., 4] / pri[..., 0] - 0.5 * q2) / cv
        pri[..., 4] = pri[..., 0] * pri[..., 5] / gamma / ma / ma
        pri[..., 6] = np.sqrt(pri[..., 4]) / ma
        for name in ("rhs", "rhsi", "rhsv"):
            b.fields[name][s] = 0.0
        b.fields["dt"][s] = cfg.dt
        b.fields["amu"][s][..., 0] = 1.0
        if cfg.turbulence == 2:
            b.fields["nut"][s] = tur
