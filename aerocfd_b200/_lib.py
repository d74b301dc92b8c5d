"""ctypes binding of libaerocfd_gpu.so (the C-ABI of include/aerocfd_gpu.h).

The library is built in-tree by ``python -m aerocfd_b200.build``.  There is no
fallback: if the shared object is missing or a call fails, an exception says
so.
"""
from __future__ import annotations

import ctypes
import os
import re
from typing import List

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libaerocfd_gpu.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "aerocfd_gpu.h")

AERO_OK = 0
_lib = None


class AeroError(RuntimeError):
    pass


def load() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AeroError(f"{LIB_PATH} is missing: build it with `python -m aerocfd_b200.build`")
        _lib = ctypes.CDLL(LIB_PATH)
        _lib.aero_last_error.restype = ctypes.c_char_p
        _lib.aero_sync_to_device.argtypes = [ctypes.c_ulonglong]
        _lib.aero_sync_to_host.argtypes = [ctypes.c_ulonglong]
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != AERO_OK:
        msg = load().aero_last_error().decode(errors="replace")
        raise AeroError(f"{what} failed with status {rc}: {msg}")


def header_symbols() -> List[str]:
    """Every function declared in include/aerocfd_gpu.h."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(aero_[a-z0-9_]+)\s*\(", text)))
