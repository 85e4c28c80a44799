"""The C-ABI library: it builds for sm_100a, loads, and exports every entry point include/lumen_b200.h declares;
argument errors come back as status codes (no GPU is touched for them): malformed arrays and parameter values outside
their ranges are refused on the host."""

import ctypes
import os
import re

import numpy as np
import pytest

from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources
from lumen_b200.api import simulate
from lumen_b200.detector import InvalidValue

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
    assert lib.lumen_b200_abi_version() == 15
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


def _create(det, mutate=None):
    """scene_create on this detector's arrays (``mutate`` edits the host arrays first): the status and message. On
    a machine without a GPU a scene that passes every host check ends at LUMEN_ERR_NO_DEVICE."""
    lib = A.engine()
    d, keep = det.desc()
    if mutate is not None:
        mutate(d, keep)
    h = ctypes.c_void_p()
    st = lib.lumen_b200_scene_create(ctypes.byref(d), ctypes.byref(h))
    msg = lib.lumen_b200_last_error().decode()
    if st == 0:
        lib.lumen_b200_scene_destroy(h)
    return st, msg


def test_scene_create_refuses_a_corrupt_bvh_item(built):
    """A BVH item that is neither a volume nor a mesh chunk would make the traversal read past the volume records: it
    is refused on the host, before any device call."""
    det = detectors.cylinder_tank(n_pmt=20)

    def corrupt(d, keep):
        keep["items"][3] = 10**6

    st, msg = _create(det, corrupt)
    assert st == 1 and "BVH item" in msg


def test_scene_create_refuses_a_negative_leaf_count_and_missing_bvh_arrays(built):
    """A node count below 0 is neither a leaf (count > 0) nor an inner node (count 0), and BVH nodes or items without
    their arrays cannot be walked: both are refused on the host, before any device call."""
    det = detectors.cylinder_tank(n_pmt=20)
    leaf = int(np.flatnonzero(det.arrays["node_i"][:, 1] > 0)[0])

    def negative(d, keep):
        keep["node_i"][leaf, 1] = -1

    st, msg = _create(det, negative)
    assert st == 3 and "negative count" in msg  # LUMEN_ERR_SCENE

    def no_nodes(d, keep):
        d.node_i = ctypes.cast(None, A.c_i32p)

    st, msg = _create(det, no_nodes)
    assert st == 1 and "BVH nodes or items" in msg


@pytest.mark.parametrize("bad", [float("nan"), -1.0, float("inf")])
def test_scene_refuses_values_outside_their_range(bad, built):
    """A parameter value that is not finite or outside its range (src/lumen/_core/domains.py: a negative length, a
    reflectivity above 1) is refused, by the C ABI (LUMEN_ERR_ARG) and by simulate (InvalidValue, naming it), as the
    reference refuses a concrete value (src/lumen/build/values.py:235)."""
    det = detectors.toy_tank()
    t = det.params_index["media/Water/absorption"]
    off, k = det.arrays["tab"][t]

    def poison(d, keep):
        p = keep["pool"].copy()  # the detector's own pool stays as it is
        p[off + k] = bad
        keep["poisoned"] = p
        d.pool = A.fptr(p)

    st, msg = _create(det, poison)
    assert st == 1 and "not finite" in msg
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=1.0, lam=400.0)
    with pytest.raises(InvalidValue, match="media/Water/absorption"):
        simulate(det, src, {"media/Water/absorption": bad}, samples=16)
    with pytest.raises(InvalidValue, match="CathodeSurface/R"):
        simulate(det, src, {"surfaces/CathodeSurface/R": 1.5}, samples=16)


def test_every_detector_passes_the_host_checks(built):
    for make in (detectors.toy_tank, detectors.cylinder_tank, detectors.lar_box, detectors.solids_box,
                 detectors.readout_tank, detectors.mesh_tank, detectors.fog_box, detectors.glisur_tank):
        st, msg = _create(make())
        assert st in (0, 5), (make.__name__, st, msg)  # 5: LUMEN_ERR_NO_DEVICE, after every host check
