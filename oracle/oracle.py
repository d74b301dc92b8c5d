"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, as the checker or the timed CPU baseline.  Parity against the
reference's own outputs is UNPINNED (no Fortran compiler in this image, no
reference fixtures); see oracle_common.h.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}


def build() -> None:
    """Compiles the three oracle builds (make, in this directory)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib(fast: bool = False, libm: bool = False) -> ctypes.CDLL:
    """The bounds-checked build (default), the -O3 build (fast) or the -O3
    build with the platform libm's pow and exp (libm: the timed CPU
    baseline; the others use the correctly rounded pow and exp the GPU uses)."""
    name = "liboracle_libm.so" if libm else ("liboracle_fast.so" if fast else "liboracle.so")
    if name not in _LIBS:
        path = os.path.join(HERE, "_build", name)
        if not os.path.exists(path):
            build()
        _LIBS[name] = ctypes.CDLL(path)
    return _LIBS[name]


def _d(x: float):
    return ctypes.byref(ctypes.c_double(x))


def _i(x: int):
    return ctypes.byref(ctypes.c_int(x))


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return ctypes.c_void_p(a.ctypes.data)


def box_args(box):
    return [_i(v) for v in box]


class OracleCase:
    """Registers a Case's host arrays with the oracle (the oracle works on them
    in place) and exposes the module-level routines."""

    def __init__(self, case, fast: bool = False, libm: bool = False):
        self.case = case
        self.L = lib(fast, libm)
        L = self.L
        L.oracle_reset()
        L.oracle_configure(case.cfg.iflags().ctypes.data_as(ctypes.c_void_p),
                           case.cfg.params().ctypes.data_as(ctypes.c_void_p))
        from aerocfd_b200.case import FIELDS
        self._keep = []
        for b in case.blocks:
            box = b.box18()
            sub = b.sub_table()
            self._keep += [box, sub]
            L.oracle_register_block(b.m, box.ctypes.data_as(ctypes.c_void_p), len(b.subfaces),
                                    sub.ctypes.data_as(ctypes.c_void_p))
            for fid, (name, _) in enumerate(FIELDS):
                L.oracle_bind_field(b.m, fid, ctypes.c_void_p(b.ptr(name)))
        L.oracle_finish_setup()

    # --- one-time setup: coordinate halo, metrics, spacing, wall distance
    def geometry(self, walldist: Optional[bool] = None) -> None:
        L = self.L
        L.oracle_updatebuffercoordinate()
        for b in self.case.blocks:
            f = b.fields
            L.oracle_gridtransformation(_p(f["dxidx"]), _p(f["inv_j"]), _p(f["alpha"]), _p(f["beta"]),
                                        _p(f["ggamma"]), _p(f["x"]), _p(f["y"]), _p(f["z"]),
                                        *box_args(b.box), *box_args(b.box0), _i(b.m))
            scratch = [np.zeros(b.shape) for _ in range(4)]
            L.oracle_init_spacing(_p(scratch[0]), _p(scratch[1]), _p(scratch[2]), _p(f["spacing"]),
                                  _p(scratch[3]), _p(f["x"]), _p(f["y"]), _p(f["z"]),
                                  *box_args(b.box), *box_args(b.box0))
        if walldist is None:
            walldist = self.case.cfg.turbulence > 0
        if walldist:
            L.oracle_init_walldist()

    def init_flowfield(self) -> None:
        c = self.case.cfg
        self.L.oracle_init_flowfield(_d(c.ma), _d(c.aoa_deg), _d(c.dt))

    def consts(self) -> np.ndarray:
        out = np.zeros(10)
        self.L.oracle_get_consts(_p(out))
        return out

    def physical_bc(self):
        self.L.oracle_physical_bc()

    def updatebuffer(self):
        self.L.oracle_updatebuffer()

    def average1(self):
        self.L.oracle_average1()

    def average2(self):
        self.L.oracle_average2()

    def getpri_all(self):
        c = self.consts()
        for b in self.case.blocks:
            self.L.oracle_get_primitivevariables(_i(b.m), _p(b.fields["pri_v"]), _p(b.fields["q"]),
                                                 _d(c[8]), _d(c[5]), *box_args(b.box))

    def start(self) -> None:
        """The pre-loop sequence of main.f90:249-318: BCs, primitives, BCs, halo."""
        self.physical_bc()
        self.getpri_all()
        self.physical_bc()
        self.updatebuffer()
        self.average1()
        self.average2()

    def iterate(self, nsteps: int, nthreads: int = 1) -> np.ndarray:
        hist = np.zeros((nsteps, 7))
        self.L.oracle_iterate(ctypes.c_int(nsteps), ctypes.c_int(nthreads), _p(hist))
        return hist

    def residual(self) -> np.ndarray:
        out = np.zeros(7)
        self.L.oracle_residual(_p(out))
        return out

    def clcd_output(self, sref: float = 1.0) -> np.ndarray:
        """fp(3), fv(3), cl, cd, then the sums of |f_prs| and |f_vis| per component."""
        out = np.zeros(14)
        self.L.oracle_clcd_output(ctypes.c_double(sref), _p(out))
        return out

    def surface_output(self):
        """surface_output (sub_output_surface.f90:24-113) over the case's host
        arrays: zones (block 1-based, face, idim, jdim, kdim) of every wall
        subface in block and bcinfo order, and its rows x, y, z,
        cp = (p - p0)/qinf in k, j, i order, p0 = d_0 t_0/gamma/ma/ma and
        qinf = 0.5 d_0 u_0**2 (:25-26)."""
        gamma, d_0, u_0, t_0 = 1.4, 1.0, 1.0, 1.0
        ma = self.case.cfg.ma
        p0 = d_0 * t_0 / gamma / ma / ma
        qinf = 0.5 * d_0 * u_0 ** 2
        zones, rows = [], []
        for m, b in enumerate(self.case.blocks):
            for sf in b.subfaces:
                if sf.blk_t != -20:
                    continue
                box = (sf.is_, sf.ie, sf.js, sf.je, sf.ks, sf.ke)
                dims = (sf.ie - sf.is_ + 1, sf.je - sf.js + 1, sf.ke - sf.ks + 1)
                zones.append((m + 1, sf.face) + dims)
                if min(dims) <= 0:
                    continue
                s = b.sl(box)
                p = b.fields["pri_v"][s][..., 4]
                cp = (p - p0) / qinf
                cols = [b.fields["x"][s], b.fields["y"][s], b.fields["z"][s], cp]
                rows.append(np.stack([c.ravel() for c in cols], axis=1))
        out = np.concatenate(rows) if rows else np.zeros((0, 4))
        return np.array(zones, dtype=np.int64).reshape(-1, 5), out

    def last_dt_minmax(self) -> np.ndarray:
        out = np.zeros(4)
        self.L.oracle_last_dt_minmax(_p(out))
        return out
