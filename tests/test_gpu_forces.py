"""clcd_output (sub_output_forceintegration.f90) on the GPU against the oracle.

Same state on both sides (oracle geometry, freestream start with a seeded
perturbation, a perturbed total viscosity).  The per-element arithmetic is the
reference's and only the order of the sums over wall elements differs, so each
force component must agree to 1e-12 of the sum of the magnitudes of its
terms, and cl / cd to 1e-12 of the corresponding scale.  The cavity case has a
no-slip wall on all six faces, so every face branch of the reference routine
(with its own metric-component mix in the normal) is exercised.
"""
import numpy as np
import pytest

from aerocfd_b200 import grids
from aerocfd_b200.case import BC_WALL, FIELDS, IFLAG_NSSOLVER, Block, Case, Config, Subface
from conftest import perturb

pytestmark = pytest.mark.gpu
TOL = 1e-12


@pytest.fixture(scope="module")
def gpu():
    from aerocfd_b200 import build, solver
    build.build()
    return solver


def cavity(ni=13, nj=11, nk=9):
    subs = [Subface(1, 1, 1, 1, 1, nj, 1, nk, BC_WALL), Subface(2, 2, ni, ni, 1, nj, 1, nk, BC_WALL),
            Subface(3, 3, 1, ni, 1, 1, 1, nk, BC_WALL), Subface(4, 4, 1, ni, nj, nj, 1, nk, BC_WALL),
            Subface(5, 5, 1, ni, 1, nj, 1, 1, BC_WALL), Subface(6, 6, 1, ni, 1, nj, nk, nk, BC_WALL)]
    cfg = Config(solver=IFLAG_NSSOLVER, ma=0.3, re=1000.0, cfl=1.0, aoa_deg=3.0)
    blk = Block(1, ni, nj, nk, subs, cfg.buffer_length, cfg.dimension)
    k, j, i = np.meshgrid(np.linspace(0, 1, nk), np.linspace(0, 1, nj), np.linspace(0, 1, ni), indexing="ij")
    X = 1.2 * i + 0.05 * np.sin(np.pi * j) * np.sin(np.pi * k)
    Y = 0.9 * j + 0.04 * np.sin(np.pi * i) * np.cos(0.5 * np.pi * k) + 0.1 * i * i
    Z = 0.7 * k + 0.03 * np.sin(np.pi * i) * np.sin(np.pi * j)
    grids._set_coords(blk, X, Y, Z)
    return Case("cavity", cfg, [blk])


def naca_small():
    return grids.naca_ogrid(nblk=4, ni=33, nj=17, nk=3)


@pytest.mark.parametrize("make", [cavity, naca_small])
def test_clcd_output_matches_oracle(gpu, oracle_mod, make):
    co, cg = make(), make()
    oc = oracle_mod.OracleCase(co)
    oc.geometry()
    oc.init_flowfield()
    perturb(co, seed=3, amp=0.02)
    oc.start()
    rng = np.random.default_rng(5)
    for b in co.blocks:
        amu = b.fields["amu"]
        amu[..., 2] = 1.0 + 0.3 * rng.random(amu.shape[:-1])
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
    scale = np.concatenate([ref[8:11], ref[11:14]])
    assert np.all(scale > 0)
    err = np.abs(got[:6] - ref[:6]) / scale
    print("forces:", got[:6], "cl, cd:", got[6:8], "max rel err", err.max())
    assert err.max() <= TOL, (got[:6], ref[:6])
    div = 2.0  # 1 / (0.5 * rho * u^2 * sref) with rho = u = sref = 1
    sc = div * (scale[0] + scale[1] + scale[3] + scale[4])
    assert np.all(np.abs(got[6:8] - ref[6:8]) <= TOL * sc), (got[6:8], ref[6:8])


@pytest.mark.parametrize("make", [cavity, naca_small])
def test_surface_output_matches_oracle(gpu, oracle_mod, make):
    """surface_output: zone headers equal and every x, y, z, cp bit-identical
    (cp is one subtraction and one division per node)."""
    co, cg = make(), make()
    oc = oracle_mod.OracleCase(co)
    oc.geometry()
    oc.init_flowfield()
    perturb(co, seed=4, amp=0.02)
    oc.start()
    oc.iterate(2)
    for bo, bg in zip(co.blocks, cg.blocks):
        for name, _ in FIELDS:
            bg.fields[name][...] = bo.fields[name]
    zref, rref = oc.surface_output()
    gc = gpu.GpuCase(cg)
    try:
        gc.sync_to_device(gpu.ALL)
        zgot, rgot = gc.surface_output()
    finally:
        gc.close()
    assert np.array_equal(zgot, zref)
    assert rgot.shape == rref.shape and len(rgot) > 0
    assert np.array_equal(rgot, rref), np.abs(rgot - rref).max()
