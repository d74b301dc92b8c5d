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


def _reference_norms(blocks, totalnodes):
    """sub_output_residual.f90:27-56 in exact arithmetic (math.fsum) over the
    updated box of every block: sqrt(sum((rhs_n dt / inv_j)^2) / totalnodes)
    and, with sa_rhs, sqrt(sum((sa_rhs dt)^2) / totalnodes)."""
    import math
    out = np.zeros(7)
    for c in range(6):
        terms = []
        for rhs, dt, invj, sa, bx in blocks:
            i0, j0, k0 = bx[6] - bx[0], bx[8] - bx[2], bx[10] - bx[4]
            i1, j1, k1 = bx[7] - bx[0] + 1, bx[9] - bx[2] + 1, bx[11] - bx[4] + 1
            d = dt[k0:k1, j0:j1, i0:i1]
            if c < 5:
                terms.append(((rhs[k0:k1, j0:j1, i0:i1, c] * d / invj[k0:k1, j0:j1, i0:i1]) ** 2).ravel())
            elif sa is not None:
                terms.append(((sa[k0:k1, j0:j1, i0:i1] * d) ** 2).ravel())
        out[c] = math.sqrt(math.fsum(np.concatenate(terms)) / totalnodes) if terms else 0.0
    return out


@pytest.mark.gpu
def test_noalloc_residual_uneven_blocks_large_then_small_call():
    """Blocks of different sizes (so the partial-sum grid has CTAs past the
    end of the smaller blocks), one large call followed by a smaller one
    (which leaves stale partial sums of the first call in the shared
    scratch): each result equals the exact norm of its own arrays to 1e-13."""
    torch = pytest.importorskip("torch")
    from aerocfd_b200 import build
    build.build()
    L = _lib.load()
    rng = np.random.default_rng(7)

    def make_block(ni, nj, nk, with_sa):
        # full box 1..n with one ghost layer outside the updated box 2..n-1
        bx = [1, ni, 1, nj, 1, nk, 2, ni - 1, 2, nj - 1, 2, nk - 1]
        rhs = rng.standard_normal((nk, nj, ni, 5))
        dt = rng.uniform(0.1, 2.0, (nk, nj, ni))
        invj = rng.uniform(0.5, 3.0, (nk, nj, ni))
        sa = rng.standard_normal((nk, nj, ni)) if with_sa else None
        return rhs, dt, invj, sa, bx

    calls = [[make_block(70, 45, 22, True), make_block(17, 9, 5, True), make_block(33, 65, 3, True)],
             [make_block(12, 7, 4, True), make_block(9, 30, 6, True)]]
    stream = torch.cuda.current_stream().cuda_stream
    for blocks in calls:
        dev = [[torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0") for a in blk[:4]] for blk in blocks]
        boxes = np.array([v for blk in blocks for v in blk[4]], dtype=np.int32)
        totalnodes = float(sum((b[4][1] - b[4][0] - 1) * (b[4][3] - b[4][2] - 1) * (b[4][5] - b[4][4] - 1)
                               for b in blocks))
        ref = _reference_norms(blocks, totalnodes)
        out = torch.empty(7, dtype=torch.float64, device="cuda:0")
        out.fill_(float("nan"))
        rc = _call(L, len(blocks), [d[0].data_ptr() for d in dev], [d[1].data_ptr() for d in dev],
                   [d[2].data_ptr() for d in dev], [d[3].data_ptr() for d in dev], boxes, totalnodes,
                   out.data_ptr(), stream)
        assert rc == 0, L.aero_last_error()
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert got[6] == 0.0
        err = np.abs(got[:6] - ref[:6]) / np.abs(ref[:6])
        assert np.all(err <= TOL), (got, ref)
