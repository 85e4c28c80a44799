"""Overlapping siblings (src/lumen/geometry/ownership.py:744 resolve: one owner per point, level by level) in the
checker: a volume proved inside a sibling is ahead of it in the rule's order (a plane lying in its active volume owns
its region), else the placement order decides (the first placed owns the shared part); an owner is a candidate of the
volumes it overlaps, so a ray leaves a region for its owner at the owner's face, and locate gives every point its
owner. Boxes that meet without their solids meeting add candidates and change nothing.
"""

import numpy as np
import pytest

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources


@pytest.fixture(scope="module")
def det():
    return detectors.overlap_box()


def _ids(det, *names):
    return [det.names.index(k) for k in names]


def test_the_rule_order(det):
    vi, n = det.arrays["vol_i"], det.arrays["n_vol"]
    ia, ip, iA, iB = _ids(det, "Active", "Plane", "A", "B")
    prio = vi[:n, 4]
    assert prio[ip] < prio[ia]  # proved inside its sibling: ahead of it
    assert prio[iA] < prio[iB]  # neither inside the other: the placement order
    cand = det.arrays["cand"]
    of = lambda v: set(cand[vi[v, 5]:vi[v, 5] + vi[v, 6]].tolist())  # noqa: E731
    assert ip in of(ia) and iA in of(iB) and ia not in of(ip) and iB not in of(iA)


def test_every_point_has_its_owner(det):
    ia, ip, iA, iB = _ids(det, "Active", "Plane", "A", "B")
    rng = np.random.default_rng(0)
    x = rng.uniform(-0.99, 0.99, (40000, 3))
    v = oracle.locate(det, x)
    # the plane: a 0.04 x 0.8 x 0.6 box at (0.1, 0, 0.45) turned 10 degrees about z
    c, s = np.cos(np.deg2rad(10.0)), np.sin(np.deg2rad(10.0))
    lp = (x - [0.1, 0.0, 0.45]) @ np.array([[c, -s, 0], [s, c, 0], [0, 0, 1.0]])
    in_plane = (np.abs(lp) < [0.02, 0.4, 0.3]).all(1)
    in_active = (np.abs(x - [0.0, 0.0, 0.45]) < [0.5, 0.5, 0.4]).all(1)
    in_a = (np.abs(x - [-0.2, 0.0, -0.5]) < [0.25, 0.25, 0.2]).all(1)
    in_b = (np.hypot(x[:, 0] - 0.15, x[:, 1] - 0.05) < 0.25) & (np.abs(x[:, 2] + 0.5) < 0.2)
    assert (v[in_plane] == ip).all()
    assert (v[in_active & ~in_plane] == ia).all()
    assert (v[in_a] == iA).all()  # the shared part is A's
    assert (v[in_b & ~in_a] == iB).all()
    assert in_plane.sum() > 50 and (in_a & in_b).sum() > 100


def test_rays_enter_the_owner_at_its_face(det):
    ia, ip, iA, iB = _ids(det, "Active", "Plane", "A", "B")
    n = 400
    rng = np.random.default_rng(1)
    y, z = rng.uniform(-0.1, 0.15, n), rng.uniform(-0.6, -0.4, n)
    o = np.stack([np.full(n, 0.32), y, z], 1)  # in B only (within 0.23 of its axis)
    d = np.tile([-1.0, 0.0, 0.0], (n, 1))
    oi, of = oracle.query(det, o, d)
    assert (oi[:, 1] == iB).all() and (oi[:, 2] == iA).all()  # into A at its face x = 0.05, inside B
    np.testing.assert_allclose(of[:, 0], 0.27, atol=2e-6)
    o2 = np.stack([np.full(n, -0.3), y, z], 1)  # in A only, heading +x: out of A at x = 0.05, into B
    oi2, of2 = oracle.query(det, o2, -d)
    assert (oi2[:, 2] == iB).all()
    np.testing.assert_allclose(of2[:, 0], 0.35, atol=2e-6)
    o3 = np.stack([np.full(n, 0.45), rng.uniform(-0.2, 0.2, n), 0.45 + rng.uniform(-0.2, 0.2, n)], 1)
    oi3, _ = oracle.query(det, o3, d)  # in Active, heading at the plane it holds: into the plane
    assert (oi3[:, 1] == ia).all() and (oi3[:, 2] == ip).all()


def test_photons_conserve_their_weight(det):
    n = 1 << 15
    T = oracle.trace(det, A.key_of_seed(1), n, source=sources.Point((0.0, 0.0, 0.0), 1.0, lam=400.0), samples=n,
                     controls=A.controls())[0]  # fmt: skip
    assert abs(T.health[:10].sum() - T.health[10]) < 1e-6 * T.health[10]
    assert T.arrival[0].sum() > 0


def test_a_protruding_daughter_is_clipped_by_its_mother():
    """A rod placed in a block and sticking out of its top face (src/lumen/geometry/ownership.py:679 clips): the block
    is a candidate of the rod whose face is its exit; the part outside the block is the water's."""
    det = detectors.protrusion_box()
    ib, ir, iw = _ids(det, "Block", "Rod", "Box")
    vi = det.arrays["vol_i"]
    cand = det.arrays["cand"]
    assert ib in cand[vi[ir, 5]:vi[ir, 5] + vi[ir, 6]]  # the clip
    assert vi[ib, 9] == 2 and vi[ir, 9] == 1  # the subtree sizes
    rng = np.random.default_rng(4)
    n = 300
    xy = np.stack([0.1 + rng.uniform(-0.05, 0.05, n), -0.05 + rng.uniform(-0.05, 0.05, n)], 1)
    v_in = oracle.locate(det, np.c_[xy, np.full(n, -0.1)])
    v_out = oracle.locate(det, np.c_[xy, np.full(n, 0.2)])  # in the rod's solid, above the block (top z = 0.1)
    assert (v_in == ir).all() and (v_out == iw).all()
    o = np.c_[xy, rng.uniform(-0.2, 0.0, n)]
    d = np.tile([0.0, 0.0, 1.0], (n, 1))
    oi, of = oracle.query(det, o, d)
    assert (oi[:, 1] == ir).all() and (oi[:, 2] == iw).all()  # out of the rod through the block's top face
    np.testing.assert_allclose(of[:, 0], 0.1 - o[:, 2], atol=2e-6)
    T = oracle.trace(det, A.key_of_seed(2), 1 << 14, source=sources.Point((0.1, -0.05, -0.1), 1.0, lam=400.0),
                     samples=1 << 14, controls=A.controls())[0]  # fmt: skip
    assert abs(T.health[:10].sum() - T.health[10]) < 1e-6 * T.health[10]


def test_frame_groups():
    """Daughters sharing a rotation whose world boxes are much larger than their own (the wire planes at +-60
    degrees) get a BVH in their frame; the vertical plane and the sensors stay in the world-frame BVH; parallel wires
    are proved apart (no owners among them)."""
    det = detectors.wire_planes()
    a = det.arrays
    assert a["n_group"] == 2 and (a["group_i"][:, 0] == 0).all()
    vi, n, cand = a["vol_i"], a["n_vol"], a["cand"]
    for v in range(1, n):
        ks = cand[vi[v, 5]:vi[v, 5] + vi[v, 6]]
        assert not [k for k in ks if k < n and vi[k, 1] != v]  # no owner: the wires are apart
    R = a["group_r64"].reshape(-1, 3, 3)
    ang = np.degrees(np.arctan2(R[:, 2, 1], R[:, 1, 1]))
    assert sorted(np.round(ang).tolist()) == [-60.0, 60.0]
    items = [set(a["items"][a["node_i"][g1:g2][:, 2][a["node_i"][g1:g2][:, 1] > 0]].tolist()) for _, g1, g2, _ in a["group_i"]]
    assert all(len(s) == 48 for s in items) and not (items[0] & items[1])
    world = a["items"][a["node_i"][vi[0, 7]:vi[0, 8]][:, 2][a["node_i"][vi[0, 7]:vi[0, 8]][:, 1] > 0]]
    assert len(world) == 48 + 8 and not (set(world.tolist()) & (items[0] | items[1]))
