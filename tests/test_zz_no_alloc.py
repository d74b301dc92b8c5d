"""aero_residual_device_noalloc: the residual norms of caller-owned device
arrays, computed with the library's fixed device scratch instead of an
allocation.  Its result is compared with aero_residual on the same state
(same partition of the sums, so the two agree to rounding; bound 1e-13
relative per component), on two calls in a row.  The argument checks run on
the CPU: they return before any device work.
"""
import ctypes

import numpy as np
import pytest

from aerocfd_b200 import _lib, grids
from aerocfd_b200.case import Config, IFLAG_NSSOLVER

TOL = 1e-13
NAMES = ("rhs", "dt", "inv_j", "sa_rhs")


def _ptrs(vals):
    return (ctypes.c_void_p * len(vals))(*vals)


def _call(L, nblocks, rhs, dt, invj, sa, boxes, totalnodes, out, stream):
    L.aero_residual_device_noalloc.restype = ctypes.c_int
    return L.aero_residual_device_noalloc(
        ctypes.c_int(nblocks), _ptrs(rhs), _ptrs(dt), _ptrs(invj), _ptrs(sa) if sa is not None else None,
        boxes.ctypes.data_as(ctypes.c_void_p), ctypes.c_double(totalnodes), ctypes.c_void_p(out),
        ctypes.c_void_p(stream))


def _boxes(case):
    return np.array([v for b in case.blocks for v in list(b.box) + list(b.box1)], dtype=np.int32)


def naca_small():
    return grids.naca_ogrid(nblk=4, ni=33, nj=17, nk=3)


def plate_small():
    return grids.flat_plate(ni=33, nj=25, nk=9, dy_wall=1e-4, cfg=Config(
        solver=IFLAG_NSSOLVER, turbulence=2, ma=0.2, re=1.0e5, cfl=2.0, nutinf=3.0))


@pytest.mark.gpu
@pytest.mark.parametrize("make", [naca_small, plate_small])
def test_noalloc_residual_matches_aero_residual(make):
    torch = pytest.importorskip("torch")
    from aerocfd_b200 import build, solver
    build.build()
    case = make()
    gc = solver.GpuCase(case)
    try:
        gc.compute_geometry()
        gc.init_flowfield()
        gc.start()
        gc.step(3, history=False)
        ref = gc.residual()
        gc.sync_to_host(solver.mask(*NAMES))
        dev = {n: [torch.from_numpy(b.fields[n]).to("cuda:0") for b in case.blocks] for n in NAMES}
        sa = [t.data_ptr() for t in dev["sa_rhs"]] if case.cfg.turbulence else None
        boxes = _boxes(case)
        totalnodes = float(sum(np.prod([b.box0[2 * d + 1] - b.box0[2 * d] + 1 for d in range(3)])
                               for b in case.blocks))
        out = torch.empty(7, dtype=torch.float64, device="cuda:0")
        stream = torch.cuda.current_stream().cuda_stream
        for _ in range(2):
            out.fill_(float("nan"))
            rc = _call(gc.L, len(case.blocks), [t.data_ptr() for t in dev["rhs"]],
                       [t.data_ptr() for t in dev["dt"]], [t.data_ptr() for t in dev["inv_j"]], sa, boxes,
                       totalnodes, out.data_ptr(), stream)
            assert rc == 0, gc.L.aero_last_error()
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.isfinite(got))
            err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
            assert np.all((err <= TOL) | (got == ref)), (got, ref)
    finally:
        gc.close()


def test_noalloc_rejects_out_of_range_calls():
    L = _lib.load()
    L.aero_last_error.restype = ctypes.c_char_p
    one = [1]
    box = np.array([1, 9, 1, 9, 1, 9, 2, 8, 2, 8, 2, 8], dtype=np.int32)
    assert _call(L, 0, one, one, one, None, box, 1.0, 1, 0) == 1
    assert b"limit" in L.aero_last_error()
    many = 33
    boxes = np.tile(box, many)
    assert _call(L, many, one * many, one * many, one * many, None, boxes, 1.0, 1, 0) == 1
    assert b"limit" in L.aero_last_error()
    # 2 blocks of 8192 x 512 x 1 updated nodes: 2 x 16384 partial sums > 16384 slots
    big = np.array([1, 8192, 1, 512, 1, 1, 1, 8192, 1, 512, 1, 1] * 2, dtype=np.int32)
    assert _call(L, 2, one * 2, one * 2, one * 2, None, big, 1.0, 1, 0) == 1
    assert b"scratch" in L.aero_last_error()
    # updated box outside the full box
    bad = np.array([1, 9, 1, 9, 1, 9, 0, 8, 2, 8, 2, 8], dtype=np.int32)
    assert _call(L, 1, one, one, one, None, bad, 1.0, 1, 0) == 1
    assert b"bad box" in L.aero_last_error()
