"""The oracle's 2-D mode (iflag_dimension = 2) on the CPU: the in-plane metrics
against their closed form on a uniform grid (sub_init_gridtransformation.f90:
270-273, :543-557), and whole iterations of the 2-D cases in the
bounds-checked build (every index the 2-D branches touch stays inside the
one-plane blocks), converging where the 3-D twins converge."""
import numpy as np

from aerocfd_b200 import grids
from aerocfd_b200.case import (BC_INFLOW, BC_OUTFLOW, BC_SYMM, IFLAG_2D, IFLAG_EULERSOLVER, IFLAG_NSSOLVER,
                               IFLAG_SA, Block, Case, Config, Subface)


def rectangle(ni=9, nj=7, dx=0.3, dy=0.2):
    cfg = Config(solver=IFLAG_EULERSOLVER, dimension=IFLAG_2D)
    subs = [Subface(1, 1, 1, 1, 1, nj, 1, 1, BC_INFLOW), Subface(2, 2, ni, ni, 1, nj, 1, 1, BC_OUTFLOW),
            Subface(3, 3, 1, ni, 1, 1, 1, 1, BC_SYMM), Subface(4, 4, 1, ni, nj, nj, 1, 1, BC_SYMM)]
    b = Block(1, ni, nj, 1, subs, cfg.buffer_length, cfg.dimension)
    X, Y = np.meshgrid(dx * np.arange(ni), dy * np.arange(nj))
    grids._set_coords(b, X[None], Y[None], np.zeros((1, nj, ni)))
    return Case("rect2d", cfg, [b])


def test_2d_metrics_closed_form(oracle_mod):
    dx, dy = 0.3, 0.2
    case = rectangle(dx=dx, dy=dy)
    oracle_mod.OracleCase(case).geometry(walldist=False)
    b = case.blocks[0]
    s = b.sl(b.box0)
    m = b.fields["dxidx"][s]
    ij = b.fields["inv_j"][s]
    assert np.allclose(ij, dx * dy, rtol=1e-14)
    want = np.array([1 / dx, 0, 0, 0, 1 / dy, 0, 0, 0, 1])
    assert np.allclose(m, want, rtol=1e-14, atol=1e-15)
    assert np.all(m[..., 8] == 1.0) and np.all(m[..., [2, 5, 6, 7]] == 0.0)
    # alpha, beta, gamma = metric products times 1/J
    assert np.allclose(b.fields["alpha"][s][..., 0], dy / dx, rtol=1e-14)
    assert np.allclose(b.fields["beta"][s][..., 1], dx / dy, rtol=1e-14)
    assert np.allclose(b.fields["ggamma"][s][..., 2], dx * dy, rtol=1e-14)


def run(case, oracle_mod, nsteps):
    oc = oracle_mod.OracleCase(case)
    oc.geometry()
    oc.init_flowfield()
    oc.start()
    return oc.iterate(nsteps)


def test_2d_bump_euler_converges(oracle_mod):
    h = run(grids.bump_channel_2d(ni=33, nj=13), oracle_mod, 200)
    assert np.all(np.isfinite(h))
    assert h[-1, 0] < 1e-2 * h[0, 0]


def test_2d_aerofoil_navier_stokes_and_sa_run(oracle_mod):
    for turb in (0, IFLAG_SA):
        cfg = Config(solver=IFLAG_NSSOLVER, ma=0.5, re=5000.0, aoa_deg=2.0, cfl=2.0, dimension=IFLAG_2D,
                     turbulence=turb)
        h = run(grids.naca_ogrid(nblk=4, ni=17, nj=13, first=1e-3, cfg=cfg), oracle_mod, 40)
        assert np.all(np.isfinite(h))
        assert h[-1, 0] < h[0, 0]
