"""Host driver: replays the reference's main loop (main.f90:249-447) through the
C-ABI, the way the Fortran program would once its call sites are routed to
libaerocfd_gpu.so.

``GpuCase`` registers a :class:`~aerocfd_b200.case.Case`'s host arrays with the
library (resident mode).  Each drop-in method takes the same arguments the
Fortran call site passes; ``step`` runs whole iterations on the device.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from .case import FIELD_ID, FIELDS, Case

ALL = (1 << len(FIELDS)) - 1


def mask(*names: str) -> int:
    m = 0
    for n in names:
        m |= 1 << FIELD_ID[n]
    return m


def _i(v: int):
    return ctypes.byref(ctypes.c_int(int(v)))


def _d(v: float):
    return ctypes.byref(ctypes.c_double(float(v)))


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return ctypes.c_void_p(a.ctypes.data)


def boxargs(box):
    return [_i(v) for v in box]


GAMMA, PRL, PRT = 1.4, 0.72, 0.90


class GpuCase:
    def __init__(self, case: Case, device: int = 0, block_params=None):
        """block_params: optional {m: Config} giving blocks their own Control.in
        values (a batch of independent cases, aero_set_block_params)."""
        self.case = case
        L = self.L = _lib.load()
        _lib.check(L.aero_init(ctypes.c_int(device)), "aero_init")
        iflags = case.cfg.iflags()
        params = case.cfg.params()
        _lib.check(L.aero_configure(_p_int(iflags), _p(params)), "aero_configure")
        self._keep = [iflags, params]
        for b in case.blocks:
            box = b.box18()
            sub = b.sub_table()
            self._keep += [box, sub]
            _lib.check(L.aero_register_block(ctypes.c_int(b.m), _p_int(box), ctypes.c_int(len(b.subfaces)),
                                             _p_int(sub)), "aero_register_block")
            for fid, (name, _) in enumerate(FIELDS):
                _lib.check(L.aero_bind_field(ctypes.c_int(b.m), ctypes.c_int(fid),
                                             ctypes.c_void_p(b.ptr(name))), "aero_bind_field")
        for m, cfg in (block_params or {}).items():
            prm = cfg.params()
            self._keep.append(prm)
            _lib.check(L.aero_set_block_params(ctypes.c_int(m), _p(prm)), "aero_set_block_params")
        _lib.check(L.aero_finish_setup(), "aero_finish_setup")
        ma = case.cfg.ma
        self.cv = 1.0 / GAMMA / (GAMMA - 1.0) / ma / ma

    # ------------------------------------------------------------- transfers
    def sync_to_device(self, m: int = ALL) -> None:
        _lib.check(self.L.aero_sync_to_device(ctypes.c_ulonglong(m)), "aero_sync_to_device")

    def sync_to_host(self, m: int = ALL) -> None:
        _lib.check(self.L.aero_sync_to_host(ctypes.c_ulonglong(m)), "aero_sync_to_host")

    # ------------------------------------------------- module-state routines
    def compute_geometry(self, walldist: Optional[bool] = None) -> None:
        """main.f90:142-208 on the device: uploads the grid coordinates, then the
        coordinate halo, metrics, spacing and (SA cases) the wall distance."""
        if walldist is None:
            walldist = self.case.cfg.turbulence > 0
        self.sync_to_device(mask("x", "y", "z"))
        _lib.check(self.L.aero_compute_geometry(ctypes.c_int(1 if walldist else 0)), "aero_compute_geometry")

    def init_flowfield(self) -> None:
        _lib.check(self.L.aero_init_flowfield(), "aero_init_flowfield")

    def physical_bc(self) -> None:
        _lib.check(self.L.aero_physical_bc(), "aero_physical_bc")

    def updatebuffer(self) -> None:
        _lib.check(self.L.aero_updatebuffer(), "aero_updatebuffer")

    def updatebuffercoordinate(self) -> None:
        _lib.check(self.L.aero_updatebuffercoordinate(), "aero_updatebuffercoordinate")

    def average1(self) -> None:
        _lib.check(self.L.aero_average1(), "aero_average1")

    def average2(self) -> None:
        _lib.check(self.L.aero_average2(), "aero_average2")

    def getpri_all(self) -> None:
        _lib.check(self.L.aero_getpri_all(), "aero_getpri_all")

    def residual(self) -> np.ndarray:
        out = np.zeros(7)
        _lib.check(self.L.aero_residual(_p(out)), "aero_residual")
        return out

    def residual_blocks(self) -> np.ndarray:
        """Each block's own residual norms (nblocks x 7)."""
        out = np.zeros((len(self.case.blocks), 7))
        _lib.check(self.L.aero_residual_blocks(_p(out)), "aero_residual_blocks")
        return out

    def use_graphs(self, on: bool = True) -> None:
        _lib.check(self.L.aero_use_graphs(ctypes.c_int(1 if on else 0)), "aero_use_graphs")

    def autotune(self, iters: int = 3) -> str:
        _lib.check(self.L.aero_autotune(ctypes.c_int(iters)), "aero_autotune")
        self.L.aero_tuning.restype = ctypes.c_char_p
        return self.L.aero_tuning().decode()

    def set_tuning(self, inv_tile: int = 64, ew: int = 256, visc: int = 128, mats: int = 128, nst_max: int = 4) -> None:
        _lib.check(self.L.aero_set_tuning(ctypes.c_int(inv_tile), ctypes.c_int(ew), ctypes.c_int(visc),
                                          ctypes.c_int(mats), ctypes.c_int(nst_max)), "aero_set_tuning")

    def set_sweep_cluster(self, ctas: int) -> None:
        """aero_set_sweep_cluster: CTAs per block of the LU-SGS sweep (1, 2, 4, 8, 16)."""
        _lib.check(self.L.aero_set_sweep_cluster(ctypes.c_int(ctas)), "aero_set_sweep_cluster")

    def set_sweep_exchange(self, mode) -> None:
        """aero_set_sweep_exchange: how a cluster shares a sweep: "l2" (or
        False), "shared" (or True: bulk copies between shared memories),
        "slab" (CTAs pipelined by k-slabs) or "shared2" (bulk copies, two CTAs
        per SM)."""
        code = {"l2": 0, "shared": 1, "slab": 2, "shared2": 3}[mode] if isinstance(mode, str) else (1 if mode else 0)
        _lib.check(self.L.aero_set_sweep_exchange(ctypes.c_int(code)), "aero_set_sweep_exchange")

    def set_sweep_prefetch(self, planes: int) -> None:
        """aero_set_sweep_prefetch: L2 prefetch distance of the bulk-exchange
        sweep (2..4 planes)."""
        _lib.check(self.L.aero_set_sweep_prefetch(ctypes.c_int(planes)), "aero_set_sweep_prefetch")

    def set_register_bound(self, on: bool) -> None:
        """aero_set_register_bound: the register-bounded FP64 viscous part a
        kernel."""
        _lib.check(self.L.aero_set_register_bound(ctypes.c_int(1 if on else 0)), "aero_set_register_bound")

    def set_sa_sweep_cluster(self, ctas: int) -> None:
        """aero_set_sa_sweep_cluster: CTAs per block of the SA sweep (1, 2, 4,
        8, 16), pipelined by k-slabs."""
        _lib.check(self.L.aero_set_sa_sweep_cluster(ctypes.c_int(ctas)), "aero_set_sa_sweep_cluster")

    def set_poll_budget(self, polls: int) -> None:
        """aero_set_poll_budget: polls of each bounded wait of the staged LU-SGS
        sweep (0..2**20, the default); a wait that gives up raises
        AERO_ST_TIMEOUT in the status word."""
        _lib.check(self.L.aero_set_poll_budget(ctypes.c_longlong(polls)), "aero_set_poll_budget")

    def inject_sweep_stall(self, plane: int) -> None:
        """aero_inject_sweep_stall: test hook; the staged LU-SGS sweep never
        issues the copies of forward hyperplane `plane` (-1: off), so its
        waits run out and the status word gets AERO_ST_TIMEOUT."""
        _lib.check(self.L.aero_inject_sweep_stall(ctypes.c_int(plane)), "aero_inject_sweep_stall")

    def set_precision(self, mixed: bool) -> None:
        """aero_set_precision: 0 = FP64 reference arithmetic, 1 = mixed."""
        _lib.check(self.L.aero_set_precision(ctypes.c_int(1 if mixed else 0)), "aero_set_precision")

    def clcd_output(self, sref: float = 1.0) -> np.ndarray:
        """clcd_output on the device: fpx, fpy, fpz, fvx, fvy, fvz, cl, cd."""
        out = np.zeros(8)
        _lib.check(self.L.aero_clcd_output(ctypes.c_double(sref), _p(out)), "aero_clcd_output")
        return out

    def surface_output(self):
        """surface_output on the device: zones (n x 5: block 1-based, face,
        idim, jdim, kdim) and rows (m x 4: x, y, z, cp) of every wall subface."""
        nn, nz = ctypes.c_longlong(0), ctypes.c_int(0)
        _lib.check(self.L.aero_surface_count(ctypes.byref(nn), ctypes.byref(nz)), "aero_surface_count")
        rows = np.zeros((nn.value, 4))
        zones = np.zeros((nz.value, 5), dtype=np.int32)
        _lib.check(self.L.aero_surface_output(_p(rows), ctypes.c_void_p(zones.ctypes.data)), "aero_surface_output")
        return zones, rows

    def status(self) -> int:
        s = ctypes.c_uint(0)
        _lib.check(self.L.aero_get_status(ctypes.byref(s)), "aero_get_status")
        return s.value

    def block_status(self) -> np.ndarray:
        """aero_get_block_status: every block's status word (not cleared)."""
        out = np.zeros(len(self.case.blocks), dtype=np.uint32)
        _lib.check(self.L.aero_get_block_status(ctypes.c_void_p(out.ctypes.data)), "aero_get_block_status")
        return out

    def clear_block_status(self) -> None:
        _lib.check(self.L.aero_clear_block_status(), "aero_clear_block_status")

    def set_retirement(self, on: bool = True) -> None:
        """aero_set_retirement: blocks with a non-zero status word stop
        advancing from the next step on."""
        _lib.check(self.L.aero_set_retirement(ctypes.c_int(1 if on else 0)), "aero_set_retirement")

    def start(self) -> None:
        """main.f90:249-318 on the device: BCs, primitives, BCs, halo, averaging."""
        self.physical_bc()
        self.getpri_all()
        self.physical_bc()
        self.updatebuffer()
        self.average1()
        self.average2()

    def step(self, nsteps: int, history: bool = True, dt_minmax: bool = False):
        hist = np.zeros((nsteps, 7)) if history else None
        dtm = np.zeros(2) if dt_minmax else None
        _lib.check(self.L.aero_step(ctypes.c_int(nsteps), _p(hist) if history else None,
                                    _p(dtm) if dt_minmax else None), "aero_step")
        return (hist, dtm) if dt_minmax else hist

    # ------------------------------------------- drop-in calls (one block)
    def get_primitivevariables(self, b) -> None:
        f = b.fields
        _lib.check(self.L.aero_get_primitivevariables(_i(b.m), _p(f["pri_v"]), _p(f["q"]), _d(GAMMA),
                                                      _d(self.cv), *boxargs(b.box)), "get_primitivevariables")

    def inviscid_flux_1(self, b) -> None:
        f = b.fields
        _lib.check(self.L.aero_inviscid_flux_1(_p(f["rhsi"]), _p(f["q"]), _p(f["dxidx"]), _p(f["inv_j"]),
                                               *boxargs(b.box), *boxargs(b.box0), *boxargs(b.box1),
                                               _d(GAMMA)), "inviscid_flux_1")

    def viscous_flux(self, b) -> None:
        f = b.fields
        c = self.case.cfg
        _lib.check(self.L.aero_viscous_flux(_p(f["rhsv"]), _p(f["pri_v"]), _p(f["amu"]), _p(f["vor"]),
                                            _p(f["dudx"]), _p(f["tao"]), _p(f["dxidx"]), _p(f["inv_j"]),
                                            _d(c.tinf), _d(PRL), _d(PRT), _d(GAMMA), _d(self.cv), _d(c.re),
                                            *boxargs(b.box), *boxargs(b.box0), *boxargs(b.box1), _i(b.m)),
                   "viscous_flux")

    def find_dt(self, b):
        f = b.fields
        c = self.case.cfg
        out = [ctypes.c_double(0) for _ in range(4)]
        cfl = ctypes.c_double(c.cfl)
        _lib.check(self.L.aero_find_dt(_p(f["dt"]), *[ctypes.byref(x) for x in out], _p(f["pri_v"]),
                                       _p(f["amu"]), _p(f["dxidx"]), _d(c.re), ctypes.byref(cfl),
                                       *boxargs(b.box), _i(c.time), _i(0), _i(1)), "find_dt")
        return [x.value for x in out]

    def implicit1st(self, b) -> None:
        f = b.fields
        c = self.case.cfg
        _lib.check(self.L.aero_implicit1st(_p(f["q"]), _p(f["dt"]), _p(f["pri_v"]), _p(f["rhs"]),
                                           _p(f["rhsi"]), _p(f["rhsv"]), _p(f["dxidx"]), _p(f["inv_j"]),
                                           *boxargs(b.box), *boxargs(b.box0), *boxargs(b.box1), _d(GAMMA),
                                           _d(c.cfl), _p(f["x"]), _p(f["y"]), _p(f["z"])), "implicit1st")

    def close(self) -> None:
        _lib.check(self.L.aero_finalize(), "aero_finalize")


def _p_int(a: np.ndarray):
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return ctypes.c_void_p(a.ctypes.data)
