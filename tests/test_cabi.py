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


def _header_prototypes():
    """name -> [(c_type, param_name)] for every function of the header."""
    import re
    text = open(_lib.HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"^\s*#.*$", "", text, flags=re.M)
    out = {}
    for m in re.finditer(r"\b(?:int|const char\*)\s+(aero_[a-z0-9_]+)\s*\(([^)]*)\)\s*;", text):
        params = []
        for p in m.group(2).split(","):
            p = " ".join(p.split())
            if not p or p == "void":
                continue
            pm = re.match(r"(.*?)(\w+)$", p)
            params.append((pm.group(1).strip(), pm.group(2)))
        out[m.group(1)] = params
    return out


def _fortran_dummies():
    """name -> {dummy: (type_spec, has_value, is_array)} for every bind(C)
    interface of the Fortran module."""
    import re
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "fortran", "aerocfd_gpu.f90")
    lines = open(path).read().splitlines()
    out, cur = {}, None
    joined = []
    for line in lines:  # join & continuations
        line = line.split("!")[0].rstrip()
        if joined and joined[-1].endswith("&"):
            joined[-1] = joined[-1][:-1] + " " + line.strip()
        else:
            joined.append(line)
    for line in joined:
        m = re.search(r'bind\(C,\s*name="(aero_[a-z0-9_]+)"\)', line)
        if m:
            cur = out.setdefault(m.group(1), {})
            continue
        if re.match(r"\s*end function", line):
            cur = None
            continue
        if cur is None or "::" not in line:
            continue
        spec, names = line.split("::", 1)
        attrs = [a.strip().lower() for a in re.split(r",(?![^()]*\))", spec)]
        has_value = "value" in attrs
        for nm in re.split(r",(?![^()]*\))", names):
            nm = nm.strip()
            if not nm:
                continue
            base = nm.split("(")[0].strip().lower()
            cur[base] = (attrs[0], has_value, "(" in nm)
    return out


def test_fortran_dummies_match_c_parameter_kinds():
    """Each C parameter has the Fortran dummy its kind needs: a C scalar is a
    `value` dummy; a C pointer is passed by reference (a host array or
    scalar), or as `type(c_ptr), value` where the caller passes an address
    itself: every pointer the header calls a DEVICE pointer or allows to be
    NULL must be `type(c_ptr), value`, since a Fortran array dummy can be
    neither a device address nor absent."""
    import re
    header_text = open(_lib.HEADER).read()
    # the comment that documents a function is the text since the previous
    # declaration; NULL / DEVICE wording applies to that function only
    special, last = {}, 0
    for m in re.finditer(r"\b(?:int|const char\*)\s+(aero_[a-z0-9_]+)\s*\([^)]*\)\s*;", header_text):
        doc = header_text[last:m.start()]
        names = set(re.findall(r"(\w+) \(may be NULL\)", doc))
        names |= set(re.findall(r"when (\w+) is not NULL", doc))
        names |= set(re.findall(r"(\w+) is a DEVICE pointer", doc))
        special[m.group(1)] = names
        last = m.end()
    protos, dummies = _header_prototypes(), _fortran_dummies()
    assert len(protos) >= 60
    bad = []
    for fn, params in protos.items():
        fd = dummies.get(fn)
        assert fd is not None, fn
        for ctype, name in params:
            d = fd.get(name.lower())
            if d is None:
                bad.append(f"{fn}: no dummy {name}")
                continue
            tspec, has_value, is_array = d
            if "*" not in ctype:
                if not has_value:
                    bad.append(f"{fn}({name}): C scalar {ctype!r} needs a value dummy")
                continue
            cptr_value = tspec == "type(c_ptr)" and has_value and not is_array
            if name in special.get(fn, ()):
                if not cptr_value:
                    bad.append(f"{fn}({name}): nullable or device pointer needs type(c_ptr), value")
            elif has_value and not cptr_value:
                bad.append(f"{fn}({name}): C pointer {ctype!r} passed by value as {tspec}")
    assert not bad, "\n".join(bad)
