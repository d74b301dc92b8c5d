"""The C-ABI library loads, exports every entry point its header declares,
and refuses to run without a GPU instead of falling back to the CPU."""
import ctypes
import glob
import os
import subprocess

import pytest

from aerocfd_b200 import _lib


@pytest.fixture(scope="module")
def lib():
    from aerocfd_b200 import build
    build.build()
    return _lib.load()


def test_header_declares_drop_in_and_module_routines():
    syms = _lib.header_symbols()
    for name in ["aero_get_primitivevariables", "aero_inviscid_flux_1", "aero_viscous_flux",
                 "aero_find_dt", "aero_implicit1st", "aero_physical_bc", "aero_updatebuffer",
                 "aero_average1", "aero_average2", "aero_updatebuffercoordinate", "aero_residual",
                 "aero_step", "aero_register_block", "aero_bind_field", "aero_finish_setup"]:
        assert name in syms


def test_fortran_module_binds_every_header_symbol():
    """fortran/aerocfd_gpu.f90 (source only here: no Fortran compiler) gives
    every C entry point a bind(C) interface under its own name, and keeps to
    free-form source's 132-column lines."""
    import re
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "fortran", "aerocfd_gpu.f90")
    text = open(path).read()
    bound = set(re.findall(r'bind\(C,\s*name="(aero_[a-z0-9_]+)"\)', text))
    missing = [s for s in _lib.header_symbols() if s not in bound]
    assert not missing, f"no Fortran interface for: {missing}"
    assert not bound - set(_lib.header_symbols()), "Fortran binds a name the header does not declare"
    assert max(len(line) for line in text.splitlines()) <= 132


def test_library_exports_every_header_symbol(lib):
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    missing = [s for s in _lib.header_symbols() if s not in exported]
    assert not missing, f"declared but not exported: {missing}"
    for s in _lib.header_symbols():
        assert hasattr(lib, s)


def test_calls_fail_loudly_without_setup(lib):
    # Before aero_init every entry point reports a state error (no silent path).
    lib.aero_finalize()
    out = (ctypes.c_double * 7)()
    assert lib.aero_residual(out) == _lib.__dict__.get("AERO_ERR_STATE", 2)
    assert b"aero_init" in lib.aero_last_error() or b"set-up" in lib.aero_last_error()


@pytest.mark.skipif(bool(glob.glob("/dev/nvidia[0-9]*")), reason="GPU present")
def test_no_gpu_means_error_not_fallback(lib):
    rc = lib.aero_init(ctypes.c_int(0))
    assert rc != 0
    assert lib.aero_last_error()
