"""2-D mode (iflag_dimension = 2) on the GPU against the oracle, FP64, through
the C-ABI: geometry (sub_init_gridtransformation.f90:270-273, :543-557),
whole steady iterations (the in-plane fluxes, LU-SGS without the zeta radius
and neighbour, SA, the 2-D interface exchange of sub_bc_updatebuffer2d.f90 and
sub_bc_updatebufferaverage2d.f90), the set-up flow the runner uses, the 2-D
wall force integration (sub_output_forceintegration.f90:48-180) and
Crank-Nicolson time steps without k lines (sub_timeadvancement_2ndcrank.f90:
84-99, :335).  Tolerances as for the 3-D path: 1e-12 of each field's maximum,
residual histories within 1e-10."""
import ctypes

import numpy as np
import pytest

from aerocfd_b200 import grids
from aerocfd_b200.case import (FIELDS, IFLAG_2D, IFLAG_2NDCRANK, IFLAG_EULERSOLVER, IFLAG_NSSOLVER, IFLAG_SA,
                               IFLAG_UNSTEADY, Config)
from conftest import perturb, relerr
from test_gpu_parity import run_parity

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def gpu():
    from aerocfd_b200 import build, solver
    build.build()
    return solver


def bump2d_euler():
    return grids.bump_channel_2d(ni=49, nj=17)


def bump2d_ns():
    cfg = Config(solver=IFLAG_NSSOLVER, ma=0.5, re=2000.0, cfl=3.0, dimension=IFLAG_2D)
    return grids.bump_channel_2d(ni=49, nj=17, cfg=cfg)


def naca2d(turb=0):
    cfg = Config(solver=IFLAG_NSSOLVER, ma=0.5, re=5000.0, aoa_deg=2.0, cfl=2.0, dimension=IFLAG_2D,
                 turbulence=turb)
    return grids.naca_ogrid(nblk=4, ni=33, nj=17, first=1e-3, cfg=cfg)


def naca2d_sa():
    return naca2d(IFLAG_SA)


@pytest.mark.parametrize("make", [bump2d_euler, naca2d], ids=["bump_ori3", "ogrid_ori2"])
def test_2d_geometry_matches_oracle(gpu, oracle_mod, make):
    co, cg = make(), make()
    oc = oracle_mod.OracleCase(co)
    oc.geometry(walldist=True)
    gc = gpu.GpuCase(cg)
    try:
        gc.sync_to_device(gpu.mask("x", "y", "z"))
        from aerocfd_b200 import _lib
        _lib.check(gc.L.aero_compute_geometry(ctypes.c_int(1)), "aero_compute_geometry")
        names = ("x", "y", "z", "dxidx", "inv_j", "alpha", "beta", "ggamma", "spacing", "dist")
        gc.sync_to_host(gpu.mask(*names))
        for bo, bg in zip(co.blocks, cg.blocks):
            for k in names:
                a, b = bg.fields[k], bo.fields[k]
                if k in ("spacing", "dist"):
                    a, b = a[bg.sl(bg.box0)], b[bo.sl(bo.box0)]
                assert relerr(a, b) <= TOL, (bo.m, k, relerr(a, b))
    finally:
        gc.close()


@pytest.mark.parametrize("make,nsteps", [(bump2d_euler, 20), (bump2d_ns, 12), (naca2d, 12), (naca2d_sa, 8)],
                         ids=["bump_euler", "bump_ns", "ogrid_ns", "ogrid_sa"])
def test_2d_iterations(gpu, oracle_mod, make, nsteps):
    run_parity(make, oracle_mod, gpu, nsteps=nsteps)


def test_2d_device_setup_flow(gpu, oracle_mod):
    co, cg = naca2d_sa(), naca2d_sa()
    oc = oracle_mod.OracleCase(co)
    oc.geometry()
    oc.init_flowfield()
    oc.start()
    ho = oc.iterate(10)
    gc = gpu.GpuCase(cg)
    try:
        gc.compute_geometry()
        gc.init_flowfield()
        gc.start()
        hg = gc.step(10)
        assert np.all(np.isfinite(hg))
        scale = np.maximum(np.abs(ho[:, :6]), 1e-6 * np.max(np.abs(ho[:, :5]), axis=1, keepdims=True))
        assert np.max(np.abs(hg[:, :6] - ho[:, :6]) / scale) <= 1e-10
        gc.sync_to_host(gpu.mask("q", "nut"))
        for bo, bg in zip(co.blocks, cg.blocks):
            assert relerr(bg.fields["q"], bo.fields["q"]) <= TOL
            assert relerr(bg.fields["nut"], bo.fields["nut"]) <= TOL
        assert gc.status() == 0
    finally:
        gc.close()


@pytest.mark.parametrize("make", [bump2d_ns, naca2d], ids=["walls_on_faces_3_and_4", "ogrid"])
def test_2d_forces_match_oracle(gpu, oracle_mod, make):
    co, cg = make(), make()
    oc = oracle_mod.OracleCase(co)
    oc.geometry()
    oc.init_flowfield()
    perturb(co, seed=3, amp=0.02)
    oc.start()
    rng = np.random.default_rng(5)
    for b in co.blocks:
        b.fields["amu"][..., 2] = 1.0 + 0.3 * rng.random(b.fields["amu"].shape[:-1])
    for bo, bg in zip(co.blocks, cg.blocks):
        for name, _ in FIELDS:
            bg.fields[name][...] = bo.fields[name]
    ref = oc.clcd_output(1.0)
    gc = gpu.GpuCase(cg)
    try:
        gc.sync_to_device(gpu.ALL)
        got = gc.clcd_output(1.0)
    finally:
        gc.close()
    # x and y components (z is exactly zero in 2-D)
    scale = np.array([ref[8], ref[9], ref[11], ref[12]])
    assert np.all(scale > 0)
    assert got[2] == 0.0 and got[5] == 0.0
    err = np.abs(got[[0, 1, 3, 4]] - ref[[0, 1, 3, 4]]) / scale
    assert err.max() <= TOL, (got[:6], ref[:6])
    sc = 2.0 * scale.sum()
    assert np.all(np.abs(got[6:8] - ref[6:8]) <= TOL * sc), (got[6:8], ref[6:8])


def test_2d_crank_time_steps(gpu, oracle_mod):
    def make():
        cfg = Config(solver=IFLAG_NSSOLVER, time=IFLAG_UNSTEADY, timeadvance=IFLAG_2NDCRANK, ma=0.5, re=1.0e4,
                     dt=2e-3, dimension=IFLAG_2D)
        return grids.bump_channel_2d(ni=33, nj=13, cfg=cfg)
    co, cg = make(), make()
    oc = oracle_mod.OracleCase(co)
    oc.geometry()
    oc.init_flowfield()
    perturb(co, seed=1)
    oc.start()
    for bo, bg in zip(co.blocks, cg.blocks):
        for name, _ in FIELDS:
            bg.fields[name][...] = bo.fields[name]
    gc = gpu.GpuCase(cg)
    try:
        gc.sync_to_device(gpu.ALL)
        ho = oc.iterate(3)
        hg = gc.step(3)
        assert np.all(np.isfinite(ho))
        scale = np.maximum(np.abs(ho[:, :6]), 1e-6 * np.max(np.abs(ho[:, :5]), axis=1, keepdims=True))
        assert np.max(np.abs(hg[:, :6] - ho[:, :6]) / scale) <= 1e-10
        gc.sync_to_host(gpu.ALL)
        for bo, bg in zip(co.blocks, cg.blocks):
            for k in ("q", "q0", "pri_v", "rhs"):
                assert relerr(bg.fields[k], bo.fields[k]) <= TOL, k
        assert gc.status() == 0
    finally:
        gc.close()


def test_2d_named_halo_entries(gpu, oracle_mod):
    """aero_updatebuffer2d, aero_average2d1 and aero_average2d2 (the
    reference's 2-D names) on random q and nut match the oracle's
    UpdateBuffer2d / average2d1 / average2d2 bit for bit; in a 3-D case they
    refuse with AERO_ERR_STATE."""
    co, cg = naca2d_sa(), naca2d_sa()
    rng = np.random.default_rng(7)
    for bo, bg in zip(co.blocks, cg.blocks):
        for name in ("q", "nut"):
            bo.fields[name][...] = 1.0 + rng.random(bo.fields[name].shape)
            bg.fields[name][...] = bo.fields[name]
    oc = oracle_mod.OracleCase(co)
    gc = gpu.GpuCase(cg)
    try:
        gc.sync_to_device(gpu.mask("q", "nut"))
        for f in ("aero_updatebuffer2d", "aero_average2d1", "aero_average2d2"):
            assert getattr(gc.L, f)() == 0, f
        gc.sync_to_host(gpu.mask("q", "nut"))
        oc.updatebuffer()
        oc.average1()
        oc.average2()
        for bo, bg in zip(co.blocks, cg.blocks):
            for name in ("q", "nut"):
                assert np.array_equal(bg.fields[name], bo.fields[name]), (bo.m, name)
    finally:
        gc.close()
    g3 = gpu.GpuCase(grids.naca_ogrid(nblk=4, ni=17, nj=9, nk=3))
    try:
        for f in ("aero_updatebuffer2d", "aero_average2d1", "aero_average2d2", "aero_updatebuffercoordinate2d"):
            assert getattr(g3.L, f)() == 2, f   # AERO_ERR_STATE
    finally:
        g3.close()
