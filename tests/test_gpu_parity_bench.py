"""FP64 parity at the sizes and set-ups the benchmark runs, for 50 iterations.

Protocol: the oracle computes the geometry, the freestream start and the
start-up boundary pass (main.f90:142-318) on its copy of the case; the GPU
case receives the same arrays, and then both advance one iteration at a time
(main.f90:343-447).  After every iteration the residual history must agree to
1e-10 relative (a component that is round-off, the z-momentum of a quasi-2-D
case, is scaled by the row's largest component), and q, pri_v, dt, rhs (plus
nut, sa_rhs, amu with SA) to 1e-12 relative to each field's largest
magnitude, on every node of every block, ghosts included.

Cases (each the exact grid, flow and scheme of a benchmark workload):
* the Euler bump channel 97 x 49 x 5, M 0.5, CFL 5, with the reference's
  Roe + WENO3 and with Steger-Warming + WENO5;
* the laminar NACA0012 O-grid 4 x 129 x 65 x 3 (blunt trailing edge), M 0.5,
  Re 5000, AoA 2, CFL 2, with Roe + WENO3 and with WCNS5;
* the SA flat plate 193 x 129 x 33 as 8 blocks of 25 x 129 x 33, wall spacing
  5e-6, ratio 1.1, M 0.2, Re_L 5e6, nu_t,inf = 3 nu_inf, CFL 5;
* the 64-case uneven bump batch (seed 0) run as one batch in FP64: its
  smallest, median and largest members against the oracle's run of each
  member alone (per-block residuals every iteration, fields every 5).
The oracle runs its -O3 build (same arithmetic as the bounds-checked build:
no contraction, no fast-math) on one host thread per block.
"""
import os

import numpy as np
import pytest

from aerocfd_b200 import grids
from aerocfd_b200.case import FIELDS, Config, IFLAG_EULERSOLVER, IFLAG_NSSOLVER
from conftest import relerr

pytestmark = pytest.mark.gpu
NSTEPS = 50
TOL = 1e-12
HTOL = 1e-10


@pytest.fixture(scope="module")
def gpu():
    from aerocfd_b200 import build, solver
    build.build()
    return solver


def _threads(nblk):
    return max(1, min(nblk, os.cpu_count() or 1))


def _started(make, oracle_mod):
    """Oracle set-up on one copy of the case, the same arrays in the other."""
    co, cg = make(), make()
    oc = oracle_mod.OracleCase(co, fast=True)
    oc.geometry()
    oc.init_flowfield()
    oc.start()
    for bo, bg in zip(co.blocks, cg.blocks):
        for name, _ in FIELDS:
            bg.fields[name][...] = bo.fields[name]
    return oc, co, cg


def _hist_err(hg, ho):
    """Largest relative difference of one residual row (components 1-5, and
    the nu_t norm when it is non-zero), each against max(|component|, 1e-6 x
    the row's largest mean-flow component)."""
    ncomp = 6 if ho[5] != 0.0 else 5
    scale = np.maximum(np.abs(ho[:ncomp]), 1e-6 * np.max(np.abs(ho[:5])))
    return float(np.max(np.abs(hg[:ncomp] - ho[:ncomp]) / scale))


def _run(make, oracle_mod, gpu, nsteps=NSTEPS):
    oc, co, cg = _started(make, oracle_mod)
    thr = _threads(len(co.blocks))
    names = ("q", "pri_v", "dt", "rhs") + (("nut", "sa_rhs", "amu") if co.cfg.turbulence else ())
    gc = gpu.GpuCase(cg)
    worst_f, worst_h = 0.0, 0.0
    try:
        gc.sync_to_device()
        for s in range(nsteps):
            ho = oc.iterate(1, thr)[0]
            hg = gc.step(1)[0]
            assert np.all(np.isfinite(hg)), s
            e = _hist_err(hg, ho)
            worst_h = max(worst_h, e)
            assert e <= HTOL, f"step {s + 1}: residual history differs by {e}"
            gc.sync_to_host(gpu.mask(*names))
            for bo, bg in zip(co.blocks, cg.blocks):
                for k in names:
                    e = relerr(bg.fields[k], bo.fields[k])
                    worst_f = max(worst_f, e)
                    assert e <= TOL, f"step {s + 1}, block {bo.m}, {k}: {e}"
        assert gc.status() == 0
    finally:
        gc.close()
    return worst_f, worst_h


def bump(inviscid):
    return lambda: grids.bump_channel(cfg=Config(solver=IFLAG_EULERSOLVER, ma=0.5, re=1.0e6, cfl=5.0,
                                                 inviscid=inviscid))


def naca(inviscid):
    return lambda: grids.naca_ogrid(cfg=Config(solver=IFLAG_NSSOLVER, ma=0.5, re=5000.0, aoa_deg=2.0, cfl=2.0,
                                               inviscid=inviscid))


def sa_plate():
    cfg = Config(solver=IFLAG_NSSOLVER, turbulence=2, ma=0.2, re=5.0e6, cfl=5.0, nutinf=3.0)
    return grids.flat_plate(nbi=8, nbj=1, nbk=1, cfg=cfg)


@pytest.mark.parametrize("inviscid", [4, 5], ids=["roe_weno3", "sw_weno5"])
def test_bump_97x49x5_50_iterations(gpu, oracle_mod, inviscid):
    _run(bump(inviscid), oracle_mod, gpu)


@pytest.mark.parametrize("inviscid", [4, 8], ids=["roe_weno3", "wcns5"])
def test_naca_4x129x65x3_50_iterations(gpu, oracle_mod, inviscid):
    _run(naca(inviscid), oracle_mod, gpu)


def test_sa_plate_193x129x33_8_blocks_50_iterations(gpu, oracle_mod):
    case = sa_plate()
    assert case.nodes == 851400 and len(case.blocks) == 8
    _run(sa_plate, oracle_mod, gpu)


def test_batch_of_64_members_50_iterations(gpu, oracle_mod):
    """The benchmark's 64-case batch in FP64: every member is set up by the
    oracle, the batch runs as one registered set with per-block case
    constants; three members (fewest, median and most nodes) follow the
    oracle's run of that member alone."""
    cases = grids.bump_batch(64, seed=0)
    order = sorted(range(len(cases)), key=lambda c: cases[c].nodes)
    picks = [order[0], order[len(order) // 2], order[-1]]
    oracles = {}
    for c, case in enumerate(cases):
        oc = oracle_mod.OracleCase(case, fast=True)
        oc.geometry()
        oc.init_flowfield()
        oc.start()
        if c in picks:
            # an OracleCase binds the library's module state: keep the picked
            # members' start states and replay each alone below
            oracles[c] = {k: v.copy() for k, v in case.blocks[0].fields.items()}
    batch, params = grids.batch_case(cases)
    gc = gpu.GpuCase(batch, block_params=params)
    try:
        gc.sync_to_device()
        hist_g = np.zeros((NSTEPS, len(cases), 7))
        q_g = {c: [] for c in picks}
        for s in range(NSTEPS):
            gc.step(1, history=False)
            hist_g[s] = gc.residual_blocks()
            if (s + 1) % 5 == 0:
                gc.sync_to_host(gpu.mask("q", "pri_v", "dt", "rhs"))
                for c in picks:
                    q_g[c].append({k: batch.blocks[c].fields[k].copy() for k in ("q", "pri_v", "dt", "rhs")})
        assert gc.status() == 0
    finally:
        gc.close()
    for c in picks:
        case = grids.bump_batch(64, seed=0)[c]
        oc = oracle_mod.OracleCase(case, fast=True)
        # init_flowfield sets the member's freestream constants in the oracle
        # (the inflow boundary uses them); then its start state is put back
        oc.init_flowfield()
        for k, v in oracles[c].items():
            case.blocks[0].fields[k][...] = v
        snap = iter(q_g[c])
        for s in range(NSTEPS):
            ho = oc.iterate(1)[0]
            e = _hist_err(hist_g[s, c], ho)
            assert e <= HTOL, f"member {c}, step {s + 1}: residual differs by {e}"
            if (s + 1) % 5 == 0:
                got = next(snap)
                for k, a in got.items():
                    e = relerr(a, case.blocks[0].fields[k])
                    assert e <= TOL, f"member {c}, step {s + 1}, {k}: {e}"
