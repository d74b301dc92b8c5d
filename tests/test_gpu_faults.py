"""Failure detection through the device status word (aero_get_status), with
every fault made on the host side, none on the GPU: a negative density and a
NaN planted in q between iterations, and a staged LU-SGS sweep whose producer
never issues one plane's copies (aero_inject_sweep_stall), so that the
consumers' bounded waits run out.  Each raises its status bit, the call itself
returns normally, and the same context runs clean iterations afterwards."""
import ctypes
import time

import numpy as np
import pytest

from aerocfd_b200 import grids

pytestmark = pytest.mark.gpu

ST_NEG_DENSITY, ST_NONFINITE_RESIDUAL, ST_TIMEOUT = 1, 2, 8


@pytest.fixture(scope="module")
def gpu():
    from aerocfd_b200 import build, solver
    build.build()
    return solver


def started(gpu):
    """A 4-block aerofoil case after a few clean iterations, its host copy in step."""
    case = grids.naca_ogrid(nblk=4, ni=33, nj=17, nk=3)
    gc = gpu.GpuCase(case)
    gc.compute_geometry()
    gc.init_flowfield()
    gc.start()
    gc.step(5)
    assert gc.status() == 0
    gc.sync_to_host(gpu.ALL)
    return case, gc


def interior(q):
    return tuple(s // 2 for s in q.shape[:3])


def clean_run_after(gpu, case, gc, snapshot):
    """Put the saved state back and check that iterations run clean again."""
    for b, q in zip(case.blocks, snapshot):
        b.fields["q"][...] = q
    gc.sync_to_device(gpu.mask("q"))
    gc.getpri_all()
    hist = gc.step(3)
    assert np.all(np.isfinite(hist))
    assert gc.status() == 0


def test_negative_density_raises_its_bit(gpu):
    case, gc = started(gpu)
    snap = [b.fields["q"].copy() for b in case.blocks]
    q = case.blocks[1].fields["q"]
    q[interior(q) + (0,)] *= -1.0
    gc.sync_to_device(gpu.mask("q"))
    gc.step(1)
    assert gc.status() & ST_NEG_DENSITY
    clean_run_after(gpu, case, gc, snap)
    gc.close()


def test_nan_raises_nonfinite_residual(gpu):
    case, gc = started(gpu)
    snap = [b.fields["q"].copy() for b in case.blocks]
    q = case.blocks[2].fields["q"]
    q[interior(q) + (4,)] = np.nan
    gc.sync_to_device(gpu.mask("q"))
    gc.step(1)
    assert gc.status() & ST_NONFINITE_RESIDUAL
    clean_run_after(gpu, case, gc, snap)
    gc.close()


@pytest.mark.parametrize("graphs", [False, True])
@pytest.mark.parametrize("plane", [0, 5])
def test_withheld_plane_times_out_and_recovers(gpu, graphs, plane):
    case, gc = started(gpu)
    snap = [b.fields["q"].copy() for b in case.blocks]
    gc.use_graphs(graphs)
    gc.set_poll_budget(4096)
    gc.inject_sweep_stall(plane)
    t0 = time.perf_counter()
    gc.step(1)
    waited = time.perf_counter() - t0
    site = (ctypes.c_int * 5)()
    assert gc.L.aero_timeout_site(site) == 0
    assert gc.status() & ST_TIMEOUT
    assert waited < 30.0
    # the staged sweep (4), one of the case's blocks, its only CTA, the
    # withheld plane's step, a plane's values (1)
    assert site[0] == 4 and 0 <= site[1] < len(case.blocks) and site[2] == 0, list(site)
    assert site[3] == plane and site[4] == 1, list(site)
    gc.L.aero_timeout_site(site)
    assert list(site) == [-1] * 5
    gc.inject_sweep_stall(-1)
    gc.set_poll_budget(1 << 20)
    clean_run_after(gpu, case, gc, snap)
    gc.close()


def test_hook_arguments_are_checked(gpu):
    from aerocfd_b200 import _lib
    case, gc = started(gpu)
    for bad in (-1, (1 << 20) + 1):
        with pytest.raises(_lib.AeroError):
            gc.set_poll_budget(bad)
    with pytest.raises(_lib.AeroError):
        gc.inject_sweep_stall(-2)
    gc.close()
