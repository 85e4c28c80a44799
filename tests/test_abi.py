"""The C-ABI library: it builds for sm_100a, loads, and exports every entry point include/lumen_b200.h declares;
argument errors come back as status codes (no GPU is touched for them)."""

import ctypes
import os
import re

from lumen_b200 import _abi as A
from lumen_b200 import detectors

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include", "lumen_b200.h")


def declared():
    return sorted(set(re.findall(r"\b(lumen_b200_\w+)\s*\(", open(HEADER).read())))


def test_library_exports_every_declared_entry_point(built):
    lib = ctypes.CDLL(built)
    names = declared()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert set(A.ENTRY_POINTS) <= set(names)


def test_abi_version_and_argument_errors(built):
    lib = A.engine()
    assert lib.lumen_b200_abi_version() == 1
    h = ctypes.c_void_p()
    assert lib.lumen_b200_scene_create(None, ctypes.byref(h)) == 1  # LUMEN_ERR_ARG before any device call
    assert b"null" in lib.lumen_b200_last_error()
    det = detectors.toy_tank()
    d, keep = det.desc()
    d.n_sensor = 1  # sensor indices past it: refused on the host
    assert lib.lumen_b200_scene_create(ctypes.byref(d), ctypes.byref(h)) == 1
    assert lib.lumen_b200_trace(None, None, None, 0, 0, 0, 1, None, None, None) == 1
