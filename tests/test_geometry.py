"""Detector building and the checker's navigator on solids with known answers (box, sphere, hemisphere, tube,
CSG): locate, first crossings, surface codes and normals."""

import numpy as np

import oracle
from lumen_b200 import detectors, geometry as G, optics as O
from lumen_b200.detector import build


def one_solid(solid):
    top = G.Volume("World", G.Box(3, 3, 3), "Water")
    top.place(G.Volume("S", solid, "Glass"), (0.2, -0.1, 0.3), name="S")
    mats = {"Water": O.Material("Water", rindex=1.33), "Glass": O.Material("Glass", rindex=1.5)}
    return build(top, mats)


def test_box_and_sphere_distances():
    det = one_solid(G.Sphere(0.5))
    o = np.array([[0.2, -0.1, -1.0], [0.2, -0.1, 0.3], [2.0, 2.0, 2.0]], np.float32)
    d = np.array([[0, 0, 1], [1, 0, 0], [0, 0, 1]], np.float32)
    oi, of = oracle.query(det, o, d)
    assert oi[0, 0] == 1 and abs(of[0, 0] - (1.3 - 0.5)) < 2e-6  # entry
    assert oi[0, 2] == 1 and oi[0, 1] == 0  # into the sphere from the world
    assert oi[1, 0] == 1 and abs(of[1, 0] - 0.5) < 2e-6 and oi[1, 1] == 1  # exit from inside
    np.testing.assert_allclose(of[1, 1:], [-1, 0, 0], atol=1e-6)  # normal against the ray
    assert abs(of[2, 0] - 1.0) < 2e-6  # the world's own exit at z = 3
    assert (oracle.locate(det, o) == [0, 1, 0]).all()


def test_hemisphere_tube_and_csg():
    det = one_solid(G.Sphere(0.5, hemisphere=1))
    oi, of = oracle.query(det, [[0.2, -0.1, -1.0], [0.2, -0.1, 1.0]], [[0, 0, 1], [0, 0, -1]])
    assert abs(of[0, 0] - 1.3) < 2e-6 and abs(of[1, 0] - 0.2) < 2e-6  # the flat face, then the dome
    det = one_solid(G.Tube(rmax=0.4, dz=0.2, rmin=0.1))
    oi, of = oracle.query(det, [[0.2, -0.1, 0.3]], [[1, 0, 0]])  # from the hole's axis
    assert abs(of[0, 0] - 0.1) < 2e-6 and oi[0, 2] == 1
    det = one_solid(G.Boolean("subtraction", G.Box(0.5, 0.5, 0.5), G.Box(0.2, 0.2, 1.0)))
    assert (oracle.locate(det, [[0.2, -0.1, 0.3], [0.6, -0.1, 0.3]]) == [0, 1]).all()
    det = one_solid(G.Boolean("union", G.Box(0.5, 0.1, 0.1), G.Box(0.1, 0.5, 0.1)))
    assert (oracle.locate(det, [[0.2, 0.3, 0.3], [0.6, 0.3, 0.3]]) == [1, 0]).all()


def test_detectors_build():
    toy = detectors.toy_tank()
    assert toy.n_sensor == 8 and toy.arrays["n_vol"] == 9
    tank = detectors.cylinder_tank()
    assert tank.n_sensor == 2000 and tank.arrays["n_vol"] == 2001
    lar = detectors.lar_box()
    assert lar.n_sensor == 120
    # every PMT inside the tank: its centre is located in it or on its face
    v = oracle.locate(tank, tank.sensor_table().position + 0.05 * tank.sensor_table().axis)
    assert (v >= 1).all()
