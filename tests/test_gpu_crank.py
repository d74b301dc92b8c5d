"""Unsteady 2nd-order Crank-Nicolson dual-time path (crank2nd, update_q0,
main.f90:450-573) on the GPU against the oracle, FP64: the drop-in crank2nd in
transient mode, and whole physical time steps (three sub-iterations each) in
resident mode.  Tolerances as for the steady path: 1e-12 of each field's
maximum per step, residual histories within 1e-10 (each row against its
largest component)."""
import ctypes

import numpy as np
import pytest

from aerocfd_b200 import grids
from aerocfd_b200.case import FIELDS, IFLAG_2NDCRANK, IFLAG_NSSOLVER, IFLAG_UNSTEADY, Config
from conftest import perturb, relerr

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _p(a):
    return ctypes.c_void_p(a.ctypes.data)


def _i(x):
    return ctypes.byref(ctypes.c_int(x))


def _d(x):
    return ctypes.byref(ctypes.c_double(x))


@pytest.fixture(scope="module")
def gpu():
    from aerocfd_b200 import build, solver
    build.build()
    return solver


def bump_cn():
    cfg = Config(solver=IFLAG_NSSOLVER, time=IFLAG_UNSTEADY, timeadvance=IFLAG_2NDCRANK, ma=0.5, re=1.0e4, dt=2e-3)
    return grids.bump_channel(ni=33, nj=17, nk=7, cfg=cfg)


def plate_cn():
    cfg = Config(solver=IFLAG_NSSOLVER, turbulence=2, time=IFLAG_UNSTEADY, timeadvance=IFLAG_2NDCRANK, ma=0.2,
                 re=1.0e5, dt=1e-3, nutinf=3.0)
    return grids.flat_plate(ni=17, nj=13, nk=7, dy_wall=1e-3, cfg=cfg)


def prepared(make, oracle_mod, seed=0):
    co, cg = make(), make()
    oc = oracle_mod.OracleCase(co)
    oc.geometry()
    oc.init_flowfield()
    perturb(co, seed=seed)
    oc.start()
    for bo, bg in zip(co.blocks, cg.blocks):
        for name, _ in FIELDS:
            bg.fields[name][...] = bo.fields[name]
    return oc, co, cg


def test_crank2nd_transient(gpu, oracle_mod):
    oc, co, cg = prepared(bump_cn, oracle_mod, seed=2)
    gc = gpu.GpuCase(cg)
    try:
        b = co.blocks[0]
        F = b.fields
        rng = np.random.default_rng(4)
        q0 = F["q0"]
        for l in range(2):   # two distinct earlier time levels
            q0[..., l::2] = F["q"] * (1.0 + 0.01 * (l - 0.5) * rng.standard_normal(F["q"].shape))
        rhsi = rng.standard_normal(F["rhsi"].shape) * 1e-2
        rhsv = rng.standard_normal(F["rhsv"].shape) * 1e-3
        F["rhsi"][...] = rhsi
        F["rhsv"][...] = rhsv
        f = {k: v.copy() for k, v in F.items()}
        names = ("q", "q0", "dt", "pri_v", "rhs", "rhsi", "rhsv", "dxidx", "inv_j")
        assert gc.L.aero_crank2nd(*[_p(f[k]) for k in names], *[_i(v) for v in b.box + b.box0 + b.box1],
                                  _d(1.4), _i(1), _i(1)) == 0, gc.L.aero_last_error()
        box18 = np.array(b.box + b.box0 + b.box1, dtype=np.int32)
        oc.L.oracle_crank2nd(*[_p(F[k]) for k in names], box18.ctypes.data_as(ctypes.c_void_p),
                             ctypes.c_double(1.4))
        for k in ("q", "rhs"):
            assert relerr(f[k], F[k]) <= TOL, (k, relerr(f[k], F[k]))
        assert gc.L.aero_update_q0(_p(f["q0"]), _p(f["q"]), *[_i(v) for v in b.box + b.box0]) == 0
        oc.L.oracle_update_q0(_p(F["q0"]), _p(F["q"]), box18.ctypes.data_as(ctypes.c_void_p))
        assert relerr(f["q0"], F["q0"]) == 0.0
    finally:
        gc.close()


@pytest.mark.parametrize("make,nsteps", [(bump_cn, 4), (plate_cn, 2)])
def test_crank_time_steps_match_oracle(gpu, oracle_mod, make, nsteps):
    oc, co, cg = prepared(make, oracle_mod, seed=1)
    gc = gpu.GpuCase(cg)
    try:
        gc.sync_to_device(gpu.ALL)
        ho = oc.iterate(nsteps)
        hg = gc.step(nsteps)
        assert np.all(np.isfinite(ho))
        scale = np.maximum(np.abs(ho[:, :6]), 1e-6 * np.max(np.abs(ho[:, :5]), axis=1, keepdims=True))
        assert np.max(np.abs(hg[:, :6] - ho[:, :6]) / scale) <= 1e-10
        gc.sync_to_host(gpu.ALL)
        fields = ["q", "q0", "pri_v", "rhs"] + (["nut"] if co.cfg.turbulence else [])
        for bo, bg in zip(co.blocks, cg.blocks):
            for k in fields:
                assert relerr(bg.fields[k], bo.fields[k]) <= TOL, (k, relerr(bg.fields[k], bo.fields[k]))
        assert gc.status() == 0
    finally:
        gc.close()
