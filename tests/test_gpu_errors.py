"""Error behaviour of the C-ABI: flags the library does not support, launch
options outside their sets and calls before set-up return their status
(AERO_ERR_ARG = 1, AERO_ERR_STATE = 2) with a message, and change nothing."""
import ctypes

import numpy as np
import pytest

from aerocfd_b200 import _lib

pytestmark = pytest.mark.gpu
ERR_ARG, ERR_STATE = 1, 2


@pytest.fixture()
def lib():
    L = _lib.load()
    L.aero_finalize()
    assert L.aero_init(ctypes.c_int(0)) == 0
    yield L
    L.aero_finalize()


def _configure(L, **over):
    # dimension, solver, time, timeadvance, turbulence, des, bufferLength, inviscid
    f = dict(dimension=3, solver=0, time=0, timeadvance=2, turbulence=0, des=0, buffer=2, inviscid=4)
    f.update(over)
    iflags = np.array([f["dimension"], f["solver"], f["time"], f["timeadvance"], f["turbulence"], f["des"],
                       f["buffer"], f["inviscid"]], dtype=np.int32)
    params = np.array([0.5, 5000.0, 288.15, 2.0, 2.0, 1.0, 1.341946])
    return L.aero_configure(ctypes.c_void_p(iflags.ctypes.data), ctypes.c_void_p(params.ctypes.data))


@pytest.mark.parametrize("over, text", [
    (dict(dimension=1), b"iflag_dimension"),
    (dict(solver=5), b"iflag_solver"),
    (dict(time=0, timeadvance=3), b"iflag_time"),
    (dict(time=1, timeadvance=2), b"iflag_time"),
    (dict(turbulence=1), b"turbulence"),
    (dict(des=3), b"iflag_des"),
    (dict(inviscid=5, buffer=2), b"bufferLength"),
    (dict(inviscid=4, buffer=3), b"bufferLength"),
    (dict(inviscid=6, buffer=3), b"bufferLength"),
])
def test_unsupported_flags_are_rejected(lib, over, text):
    assert _configure(lib) == 0  # the supported set is accepted
    assert _configure(lib, **over) == ERR_ARG
    assert text in lib.aero_last_error()


def test_supported_extensions_are_accepted(lib):
    for over in (dict(inviscid=5, buffer=3), dict(inviscid=8, buffer=3), dict(turbulence=2, des=1),
                 dict(turbulence=2, des=2), dict(time=1, timeadvance=3), dict(dimension=2)):
        assert _configure(lib, **over) == 0, over


def test_launch_options_outside_their_sets(lib):
    assert lib.aero_set_sweep_cluster(ctypes.c_int(3)) == ERR_ARG
    assert lib.aero_set_sweep_exchange(ctypes.c_int(4)) == ERR_ARG
    assert lib.aero_set_sa_sweep_cluster(ctypes.c_int(3)) == ERR_ARG
    assert lib.aero_set_precision(ctypes.c_int(2)) == ERR_ARG
    assert lib.aero_set_tuning(ctypes.c_int(48), ctypes.c_int(256), ctypes.c_int(128), ctypes.c_int(128),
                               ctypes.c_int(4)) == ERR_ARG
    for call in (lambda: lib.aero_set_sweep_cluster(ctypes.c_int(8)), lambda: lib.aero_set_sweep_exchange(ctypes.c_int(1)),
                 lambda: lib.aero_set_sweep_exchange(ctypes.c_int(2)), lambda: lib.aero_set_sa_sweep_cluster(ctypes.c_int(8)),
                 lambda: lib.aero_set_precision(ctypes.c_int(1))):
        assert call() == 0


def test_calls_before_setup_are_state_errors(lib):
    assert _configure(lib) == 0
    out = np.zeros(7)
    assert lib.aero_step(ctypes.c_int(1), ctypes.c_void_p(out.ctypes.data), None) == ERR_STATE
    assert lib.aero_residual(ctypes.c_void_p(out.ctypes.data)) == ERR_STATE
    assert lib.aero_last_error()
