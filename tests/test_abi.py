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
    assert lib.lumen_b200_abi_version() == 12
    h = ctypes.c_void_p()
    assert lib.lumen_b200_scene_create(None, ctypes.byref(h)) == 1  # LUMEN_ERR_ARG before any device call
    assert b"null" in lib.lumen_b200_last_error()
    det = detectors.toy_tank()
    d, keep = det.desc()
    d.n_sensor = 1  # sensor indices past it: refused on the host
    assert lib.lumen_b200_scene_create(ctypes.byref(d), ctypes.byref(h)) == 1
    assert lib.lumen_b200_trace(None, None, None, 0, 0, 0, 1, None, None, None) == 1
    # a unified facet row needs the lobe's tables: refused on the host when they are missing
    fdet = detectors.cylinder_tank(n_pmt=20, wall_finish="ground", sigma_alpha=0.1)
    d, keep = fdet.desc()
    assert keep["unified"].size == A.UNI_WORDS
    d.unified = A.fptr(None)
    assert lib.lumen_b200_scene_create(ctypes.byref(d), ctypes.byref(h)) == 1
    assert b"unified tables" in lib.lumen_b200_last_error()


def test_header_constants_match_the_python_mirrors():
    from lumen_b200 import facets

    h = open(HEADER).read()

    def define(name):
        return float(re.search(rf"#define {name}\s+\(?(-?[0-9.]+)\)?", h).group(1))

    assert int(define("LUMEN_UNI_NX")) == A.UNI_NX == facets.NX
    assert int(define("LUMEN_UNI_NY")) == A.UNI_NY == facets.NY
    assert int(define("LUMEN_UNI_J_LO")) == facets.J_LO
    assert abs(define("LUMEN_UNI_Y0") - facets.Y0) < 1e-15 and abs(define("LUMEN_UNI_DY") - facets.DY) < 1e-15
    assert int(define("LUMEN_MAX_GRAD")) == A.MAX_GRAD
    assert facets.WORDS == A.UNI_WORDS
