"""The detectors of the benchmark and test workloads, built with ``lumen_b200.detector.build``.

- ``toy_tank()``: lumen's tutorial detector (examples/data/example_tank.gdml and examples/example_tank.py:21-35 of the
  reference): a 1 m cube of water (tabulated RINDEX and ABSLENGTH; Geant4's water Rayleigh table from RINDEX), 8 disc
  PMTs (radius 50 mm, 20 mm thick) behind a dielectric_metal cathode border (REFLECTIVITY 0, EFFICIENCY 1); light that
  leaves the water is absorbed.
- ``cylinder_tank()``: a water cylinder (radius 5 m, height 10 m) with 2000 inward-facing hemispherical PMTs (radius
  0.1 m) on a regular barrel and end-cap grid, black-sheet walls of reflectivity 0.1; water with absorption length
  50 m, Rayleigh length 80 m and a flat index of 1.34.
- ``lar_box()``: a 5 x 4 x 4 m liquid-argon box (index 1.38, Rayleigh 0.9 m, absorption 20 m) with a CSG cathode
  (a plate with a cut-out window, a box subtraction) and a field cage (a box shell with a union of two rails: box
  subtractions and unions) of reflectivity 0.9, and 120 flat discs (20 cm diameter) on one wall.
"""

from __future__ import annotations

import math

import numpy as np

from lumen_b200 import detector as D
from lumen_b200 import geometry as G
from lumen_b200 import optics as O

MM = 1e-3


def toy_tank() -> D.Detector:
    """Return the tutorial tank (values of examples/data/example_tank.gdml in the reference)."""
    water = O.Material("Water", rindex=([1.5, 2.5, 3.5, 5.0], [1.332, 1.336, 1.345, 1.366]),
                       abslength=([1.5, 2.5, 3.0, 3.5, 5.0], [5.0, 40.0, 60.0, 30.0, 2.0]))  # fmt: skip
    cathode = O.Material("Photocathode")
    pmt = G.Volume("PMT", G.Tube(rmax=50 * MM, dz=10 * MM), "Photocathode")
    tank = G.Volume("TankLV", G.Box(0.5, 0.5, 0.5), "Water")
    places = [((0, 0, -480), None), ((0, 0, 480), None), ((-480, 0, 0), ("y", 90)), ((480, 0, 0), ("y", 90)),
              ((0, -480, 0), ("x", 90)), ((0, 480, 0), ("x", 90)), ((-250, 0, -480), None), ((250, 0, -480), None)]
    for i, (p, r) in enumerate(places):
        rot = None if r is None else G.gdml_rotation(**{r[0]: r[1]})
        tank.place(pmt, np.asarray(p, float) * MM, rot, name=f"PMT_{i}", copy=i)
    surf = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    borders = [("TankLV", f"PMT_{i}", surf) for i in range(8)]
    return D.build(tank, {"Water": water, "Photocathode": cathode}, borders=borders, sensors={"pmt": "PMT"})


def readout_tank(after_tracking=True) -> D.Detector:
    """Return the scintillator cube's tank (Rayleigh, Mie and WLS in the bulk, a ground half-reflecting wall) with two
    sensor groups: six PMTs ("pmt") whose cathodes have a complex index (RINDEX 2.7, KINDEX 1.5: a photocathode
    reflecting specularly) and whose sensor model applies its QE after tracking (``after_tracking``: every absorption
    counted, deposits carrying 1 / A_n), and two reference PMTs ("ref") with a half-reflecting metal cathode of
    efficiency 0.8."""  # noqa: D205
    e_abs = [1.5, 2.5, 2.9, 3.0, 3.2, 5.0]
    lab = O.Material("LAB", rindex=([1.5, 2.5, 3.5, 5.0], [1.47, 1.48, 1.50, 1.53]), abslength=20.0, rayleigh=5.0,
                     mie=2.0, mie_forward=0.9, mie_backward=0.3, mie_forward_ratio=0.8,
                     wls=(e_abs, [100.0, 100.0, 20.0, 1.0, 1.0, 1.0]),
                     wls_spectrum=([2.3, 2.5, 2.7, 2.9, 3.1, 3.2], [0.0, 0.4, 1.0, 0.7, 0.1, 0.0]),
                     wls_mean=0.9, wls_tau=2.0, wls_profile="exponential")  # fmt: skip
    cathode = O.Material("Photocathode")
    pmt = G.Volume("PMT", G.Tube(rmax=50 * MM, dz=10 * MM), "Photocathode")
    ref = G.Volume("RefPMT", G.Tube(rmax=50 * MM, dz=10 * MM), "Photocathode")
    tank = G.Volume("TankLV", G.Box(0.5, 0.5, 0.5), "LAB")
    places = [((0, 0, -480), None), ((0, 0, 480), None), ((-480, 0, 0), ("y", 90)), ((480, 0, 0), ("y", 90)),
              ((0, -480, 0), ("x", 90)), ((0, 480, 0), ("x", 90)), ((-250, 0, -480), None), ((250, 0, -480), None)]
    for i, (p, r) in enumerate(places):
        rot = None if r is None else G.gdml_rotation(**{r[0]: r[1]})
        tank.place(ref if i in (2, 6) else pmt, np.asarray(p, float) * MM, rot, name=f"PMT_{i}", copy=i)
    photo = O.OpticalSurface("Cathode", "dielectric_metal", "polished", efficiency=0.9, rindex=2.7, kindex=1.5)
    metal = O.OpticalSurface("RefCathode", "dielectric_metal", "polished", reflectivity=0.5, efficiency=0.8)
    wall = O.OpticalSurface("Wall", "dielectric_metal", "ground", reflectivity=0.5, sigma_alpha=0.2, specularlobe=0.5)
    borders = [("TankLV", f"PMT_{i}", metal if i in (2, 6) else photo) for i in range(8)]
    return D.build(tank, {"LAB": lab, "Photocathode": cathode}, borders=borders, skins={"TankLV": wall},
                   sensors={"pmt": "PMT", "ref": "RefPMT"}, after_tracking=("pmt",) if after_tracking else ())


SCINT_COMPONENTS = ({"spectrum": ([2.5, 2.6, 2.8, 3.0, 3.3], [0.0, 0.0, 1.0, 1.0, 0.0]), "tau": 6.0, "rise": 1.0},
                    {"spectrum": ([2.5, 2.7, 3.1, 3.3], [0.2, 1.0, 0.5, 0.0]), "tau": 1500.0, "rise": 2.0})


def scintillating_tank() -> D.Detector:
    """Return the tutorial tank's geometry filled with a two-component scintillator (G4Scintillation, Geant4 11
    keys): 1000 photons / MeV shared 25 / 75 between a fast (6 ns decay, 1 ns rise) and a slow (1.5 us, 2 ns)
    component with their own spectra (each with intervals without mass); index 1.38, absorption 20 m."""  # noqa: D205
    scint = O.Material("Scint", rindex=([1.5, 5.0], [1.38, 1.38]), abslength=20.0, scint_yield=1000.0,
                       scint_components=SCINT_COMPONENTS, scint_shares=(0.25, 0.75))  # fmt: skip
    cathode = O.Material("Photocathode")
    pmt = G.Volume("PMT", G.Tube(rmax=50 * MM, dz=10 * MM), "Photocathode")
    tank = G.Volume("TankLV", G.Box(0.5, 0.5, 0.5), "Scint")
    places = [((0, 0, -480), None), ((0, 0, 480), None), ((-480, 0, 0), ("y", 90)), ((480, 0, 0), ("y", 90)),
              ((0, -480, 0), ("x", 90)), ((0, 480, 0), ("x", 90)), ((-250, 0, -480), None), ((250, 0, -480), None)]
    for i, (p, r) in enumerate(places):
        rot = None if r is None else G.gdml_rotation(**{r[0]: r[1]})
        tank.place(pmt, np.asarray(p, float) * MM, rot, name=f"PMT_{i}", copy=i)
    surf = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    borders = [("TankLV", f"PMT_{i}", surf) for i in range(8)]
    return D.build(tank, {"Scint": scint, "Photocathode": cathode}, borders=borders, sensors={"pmt": "PMT"})


def solids_box() -> D.Detector:
    """Return a 3 m water box holding one glass copy of each solid of the catalogue beyond the benchmarks' (tori,
    cones, sphere shells with phi and theta ranges, ellipsoids, elliptical tubes and cones, paraboloids, hyperboloids,
    polycones, polyhedra, trapezoids, tetrahedra, a phi-cut tube), each rotated, and 8 sensor discs on two walls."""  # noqa: D205
    water = O.Material("Water", rindex=1.33, abslength=30.0, rayleigh=10.0)
    glass = O.Material("Glass", rindex=1.5, abslength=5.0)
    cathode = O.Material("Photocathode")
    box = G.Volume("Box", G.Box(1.5, 1.5, 1.5), "Water")
    solids = [G.Torus(0.15, 0.35, 0.05, 0.5, 4.5), G.Torus(0.1, 0.3), G.Cons(0.1, 0.3, 0.05, 0.2, 0.3, 0.3, 4.0),
              G.SphereShell(0.35, 0.15, 0.5, 2.0, 0.3, 1.5), G.SphereShell(0.3, 0.0, 1.0, 5.0, 1.2, 1.4),
              G.Ellipsoid(0.3, 0.2, 0.35, -0.2, 0.3), G.EllipticalTube(0.3, 0.2, 0.3), G.EllipticalCone(0.5, 0.3, 0.5, 0.3),
              G.Paraboloid(0.1, 0.3, 0.3), G.Hype(0.1, 0.3, 0.3, 0.5, 0.3),
              G.Polycone(((0.0, 0.2, -0.3), (0.05, 0.3, 0.0), (0.0, 0.1, 0.3)), 0.2, 5.0),
              G.Polyhedra(((0.0, 0.2, -0.3), (0.05, 0.3, 0.3)), 6, 0.0, 5.0), G.Trd(0.2, 0.1, 0.3, 0.2, 0.3),
              G.Trap(0.3, 0.2, 0.3, 0.3, 0.2, 0.26, 0.1, 0.2, 0.15, 0.19, 0.1),
              G.Tet((0, 0, 0), (0.4, 0, 0), (0, 0.4, 0), (0, 0, 0.4)), G.Tube(0.3, 0.3, 0.1, 1.0, 2.0)]  # fmt: skip
    for k, s in enumerate(solids):
        i, j = divmod(k, 4)
        rot = G.rotation("x", 17.0 * k) @ G.rotation("z", 31.0 * k)
        box.place(G.Volume(f"S{k}", s, "Glass"), ((i - 1.5) * 0.7, (j - 1.5) * 0.7, 0.0), rot, name=f"S{k}")
    pmt = G.Volume("PMT", G.Tube(rmax=0.15, dz=0.01), "Photocathode")
    for i in range(4):
        box.place(pmt, (-0.75 + 0.5 * i, 0.0, -1.48), None, name=f"PMT_{i}", copy=i)
        box.place(pmt, (-0.75 + 0.5 * i, 0.0, 1.48), None, name=f"PMT_{4 + i}", copy=4 + i)
    surf = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    wall = O.OpticalSurface("Wall", "dielectric_metal", "ground", reflectivity=0.6, sigma_alpha=0.2, specularlobe=0.5)
    borders = [("Box", f"PMT_{i}", surf) for i in range(8)]
    return D.build(box, {"Water": water, "Glass": glass, "Photocathode": cathode}, borders=borders,
                   skins={"Box": wall}, sensors={"pmt": "PMT"})  # fmt: skip


def mesh_tank() -> D.Detector:
    """Return a 3 m water box holding two opaque tessellated parts (G4TessellatedSolid): a polished steel icosphere
    (r 0.4 m, 320 triangles, reflectivity 0.8) and a rotated black box mesh (12 triangles), beside a glass orb, and 8
    sensor discs on two walls."""  # noqa: D205
    water = O.Material("Water", rindex=1.33, abslength=30.0, rayleigh=10.0)
    glass = O.Material("Glass", rindex=1.5, abslength=5.0)
    steel = O.Material("Steel")
    black = O.Material("Black")
    cathode = O.Material("Photocathode")
    box = G.Volume("Box", G.Box(1.5, 1.5, 1.5), "Water")
    box.place(G.Volume("Ball", G.Mesh(G.icosphere(0.4, 2)), "Steel"), (-0.5, 0.2, 0.1), G.rotation("x", 20.0),
              name="Ball")  # fmt: skip
    box.place(G.Volume("Block", G.Mesh(G.box_mesh(0.3, 0.2, 0.25)), "Black"), (0.6, -0.3, -0.2),
              G.rotation("z", 30.0) @ G.rotation("y", 15.0), name="Block")  # fmt: skip
    box.place(G.Volume("Orb", G.Orb(0.25), "Glass"), (0.3, 0.6, 0.4), None, name="Orb")
    pmt = G.Volume("PMT", G.Tube(rmax=0.15, dz=0.01), "Photocathode")
    for i in range(4):
        box.place(pmt, (-0.75 + 0.5 * i, 0.0, -1.48), None, name=f"PMT_{i}", copy=i)
        box.place(pmt, (-0.75 + 0.5 * i, 0.0, 1.48), None, name=f"PMT_{4 + i}", copy=4 + i)
    surf = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    shiny = O.OpticalSurface("Shiny", "dielectric_metal", "polished", reflectivity=0.8)
    wall = O.OpticalSurface("Wall", "dielectric_metal", "ground", reflectivity=0.6, sigma_alpha=0.2, specularlobe=0.5)
    borders = [("Box", f"PMT_{i}", surf) for i in range(8)]
    return D.build(box, {"Water": water, "Glass": glass, "Steel": steel, "Black": black, "Photocathode": cathode},
                   borders=borders, skins={"Box": wall, "Ball": shiny}, sensors={"pmt": "PMT"})  # fmt: skip


def overlap_box() -> D.Detector:
    """Return a 2 m water box with overlapping siblings, resolved as the reference's ownership rule does (one owner per
    point): an argon-like "Active" box with a glass "Plane" placed after it inside it (proved inside, so ahead of it:
    the plane owns its region, as a wire plane lying in its active volume), and two partly overlapping glass-like boxes
    "A" and "B" (A placed first owns the shared part); 4 sensor discs on one wall."""  # noqa: D205
    water = O.Material("Water", rindex=1.33, abslength=30.0, rayleigh=10.0)
    active = O.Material("Active", rindex=1.25, abslength=20.0)
    glass = O.Material("Glass", rindex=1.5, abslength=5.0)
    acryl = O.Material("Acrylic", rindex=1.45, abslength=5.0)
    cathode = O.Material("Photocathode")
    box = G.Volume("Box", G.Box(1.0, 1.0, 1.0), "Water")
    box.place(G.Volume("Active", G.Box(0.5, 0.5, 0.4), "Active"), (0.0, 0.0, 0.45), None, name="Active")
    box.place(G.Volume("Plane", G.Box(0.02, 0.4, 0.3), "Glass"), (0.1, 0.0, 0.45), G.rotation("z", 10.0), name="Plane")
    box.place(G.Volume("A", G.Box(0.25, 0.25, 0.2), "Glass"), (-0.2, 0.0, -0.5), None, name="A")
    box.place(G.Volume("B", G.Tube(rmax=0.25, dz=0.2), "Acrylic"), (0.15, 0.05, -0.5), None, name="B")
    pmt = G.Volume("PMT", G.Tube(rmax=0.15, dz=0.01), "Photocathode")
    for i in range(4):
        box.place(pmt, (-0.6 + 0.4 * i, 0.0, -0.98), None, name=f"PMT_{i}", copy=i)
    surf = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    wall = O.OpticalSurface("Wall", "dielectric_metal", "ground", reflectivity=0.6, sigma_alpha=0.2, specularlobe=0.5)
    borders = [("Box", f"PMT_{i}", surf) for i in range(4)]
    return D.build(box, {"Water": water, "Active": active, "Glass": glass, "Acrylic": acryl, "Photocathode": cathode},
                   borders=borders, skins={"Box": wall}, sensors={"pmt": "PMT"})  # fmt: skip


def protrusion_box() -> D.Detector:
    """Return a 2 m water box holding an acrylic block with a glass rod placed in it that sticks out through the
    block's top face (the reference's protrusion: the rod holds only what lies inside the block; a photon in the rod
    leaves it at the block's face), and 4 sensor discs above."""  # noqa: D205
    water = O.Material("Water", rindex=1.33, abslength=30.0, rayleigh=10.0)
    acryl = O.Material("Acrylic", rindex=1.45, abslength=5.0)
    glass = O.Material("Glass", rindex=1.6, abslength=5.0)
    cathode = O.Material("Photocathode")
    box = G.Volume("Box", G.Box(1.0, 1.0, 1.0), "Water")
    block = G.Volume("Block", G.Box(0.4, 0.4, 0.3), "Acrylic")
    block.place(G.Volume("Rod", G.Tube(rmax=0.08, dz=0.25), "Glass"), (0.1, -0.05, 0.2), None, name="Rod")
    box.place(block, (0.0, 0.0, -0.2), None, name="Block")
    pmt = G.Volume("PMT", G.Tube(rmax=0.15, dz=0.01), "Photocathode")
    for i in range(4):
        box.place(pmt, (-0.6 + 0.4 * i, 0.0, 0.98), None, name=f"PMT_{i}", copy=i)
    surf = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    wall = O.OpticalSurface("Wall", "dielectric_metal", "ground", reflectivity=0.6, sigma_alpha=0.2, specularlobe=0.5)
    borders = [("Box", f"PMT_{i}", surf) for i in range(4)]
    return D.build(box, {"Water": water, "Acrylic": acryl, "Glass": glass, "Photocathode": cathode}, borders=borders,
                   skins={"Box": wall}, sensors={"pmt": "PMT"})  # fmt: skip


def wire_planes(n_wires=48, frame_groups=True) -> D.Detector:
    """Return a 2 m argon-like box with two planes of ``n_wires`` thin steel wires (r 1.5 mm) at +60 and -60 degrees
    about x (the induction planes of a wire chamber), a collection plane of vertical wires, and 8 sensor discs on one
    wall: daughters sharing a rotation whose world boxes are much larger than their own (frame groups)."""  # noqa: D205
    lar = O.Material("LAr", rindex=1.38, abslength=20.0, rayleigh=0.9)
    steel = O.Material("Steel")
    cathode = O.Material("Photocathode")
    box = G.Volume("Box", G.Box(1.0, 1.0, 1.0), "LAr")
    wire = G.Volume("Wire", G.Tube(rmax=0.0015, dz=0.55), "Steel")
    for p_, (x, ang) in enumerate(((0.3, 60.0), (0.4, -60.0), (0.5, 0.0))):
        for k in range(n_wires):
            y = -0.45 + 0.9 * k / (n_wires - 1)
            box.place(wire, (x, y, 0.0), G.rotation("x", ang), name=f"W{p_}_{k}", copy=p_ * n_wires + k)
    pmt = G.Volume("PMT", G.Tube(rmax=0.12, dz=0.01), "Photocathode")
    rot = G.rotation("y", 90.0)
    for i in range(8):
        box.place(pmt, (0.98, -0.6 + 0.4 * (i % 4), -0.3 + 0.6 * (i // 4)), rot, name=f"PMT_{i}", copy=i)
    surf = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    shiny = O.OpticalSurface("WireSurface", "dielectric_metal", "polished", reflectivity=0.5)
    borders = [("Box", f"PMT_{i}", surf) for i in range(8)]
    return D.build(box, {"LAr": lar, "Steel": steel, "Photocathode": cathode}, borders=borders,
                   skins={"Wire": shiny}, sensors={"pmt": "PMT"}, frame_groups=frame_groups)  # fmt: skip


def coated_panel(thickness=3e-6, distance=5.0, precision="float32") -> D.Detector:
    """Return a 12 m water box with a 2 x 2 m acrylic backing 20 cm thick at x = ``distance`` m, coated on its front
    face with a TPB-like layer ``thickness`` m thick (rindex 1.6), and 4 photocathode discs (r 0.3 m) behind it: the
    case the reference's float64 navigator is for (docs/dev/decisions.md:340): float32's band at 5 m is 4.8 um, so
    float32 steps over a 3 um coating that float64 enters."""  # noqa: D205
    water = O.Material("Water", rindex=1.33, abslength=40.0, rayleigh=40.0)
    acrylic = O.Material("Acrylic", rindex=1.49, abslength=5.0)
    tpb = O.Material("TPB", rindex=1.6, abslength=1.0)
    cathode = O.Material("Photocathode")
    world = G.Volume("World", G.Box(6.0, 6.0, 6.0), "Water")
    world.place(G.Volume("Backing", G.Box(0.1, 1.0, 1.0), "Acrylic"), (distance + 0.1, 0.0, 0.0), None, name="Backing")
    world.place(G.Volume("Coating", G.Box(0.5 * thickness, 1.0, 1.0), "TPB"), (distance - 0.5 * thickness, 0.0, 0.0),
                None, name="Coating")  # fmt: skip
    pmt = G.Volume("PMT", G.Tube(rmax=0.3, dz=0.01), "Photocathode")
    rot = G.rotation("y", 90.0)  # the discs' axis along x
    for k, (y, z) in enumerate(((-0.45, -0.45), (-0.45, 0.45), (0.45, -0.45), (0.45, 0.45))):
        world.place(pmt, (distance + 0.25, y, z), rot, name=f"PMT_{k}", copy=k)
    surf = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    borders = [("World", f"PMT_{k}", surf) for k in range(4)]
    return D.build(world, {"Water": water, "Acrylic": acrylic, "TPB": tpb, "Photocathode": cathode}, borders=borders,
                   sensors={"pmt": "PMT"}, precision=precision)  # fmt: skip


def scintillator_cube(mie=2.0, wls=1.0, rayleigh=5.0, profile="exponential") -> D.Detector:
    """Return the tutorial tank's geometry filled with a synthetic liquid scintillator whose bulk has all three of
    Geant4's channels: Rayleigh, Mie (G4OpMieHG, MIEHG ``mie`` m, forward 0.9, backward 0.3, forward ratio 0.8) and a
    wavelength shifter (G4OpWLS, WLSABSLENGTH ``wls`` m: absorbs below ~410 nm, re-emits a 390-500 nm band with 0.9
    photons per absorbed one after a ``profile`` 2 ns delay)."""  # noqa: D205
    e_abs = [1.5, 2.5, 2.9, 3.0, 3.2, 5.0]
    lab = O.Material("LAB", rindex=([1.5, 2.5, 3.5, 5.0], [1.47, 1.48, 1.50, 1.53]), abslength=20.0,
                     rayleigh=rayleigh, mie=mie, mie_forward=0.9, mie_backward=0.3, mie_forward_ratio=0.8,
                     wls=(e_abs, [100.0 * wls, 100.0 * wls, 20.0 * wls, wls, wls, wls]),
                     wls_spectrum=([2.3, 2.5, 2.7, 2.9, 3.1, 3.2], [0.0, 0.4, 1.0, 0.7, 0.1, 0.0]),
                     wls_mean=0.9, wls_tau=2.0, wls_profile=profile)  # fmt: skip
    cathode = O.Material("Photocathode")
    pmt = G.Volume("PMT", G.Tube(rmax=50 * MM, dz=10 * MM), "Photocathode")
    tank = G.Volume("TankLV", G.Box(0.5, 0.5, 0.5), "LAB")
    places = [((0, 0, -480), None), ((0, 0, 480), None), ((-480, 0, 0), ("y", 90)), ((480, 0, 0), ("y", 90)),
              ((0, -480, 0), ("x", 90)), ((0, 480, 0), ("x", 90)), ((-250, 0, -480), None), ((250, 0, -480), None)]
    for i, (p, r) in enumerate(places):
        rot = None if r is None else G.gdml_rotation(**{r[0]: r[1]})
        tank.place(pmt, np.asarray(p, float) * MM, rot, name=f"PMT_{i}", copy=i)
    surf = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    wall = O.OpticalSurface("Wall", "dielectric_metal", "ground", reflectivity=0.5, sigma_alpha=0.2, specularlobe=0.5)
    borders = [("TankLV", f"PMT_{i}", surf) for i in range(8)]
    return D.build(tank, {"LAB": lab, "Photocathode": cathode}, borders=borders, skins={"TankLV": wall},
                   sensors={"pmt": "PMT"})  # fmt: skip


def glisur_tank(polish_wall=0.8, polish_block=0.7) -> D.Detector:
    """Return the tutorial tank with GLISUR ground surfaces: the walls a GLISUR metal (R 0.7, polish ``polish_wall``)
    and an acrylic block (n 1.49, 30 x 30 x 20 cm) inside behind GLISUR ground dielectric borders both ways (polish
    ``polish_block``: facets that reflect or refract with Fresnel's shares)."""  # noqa: D205
    water = O.Material("Water", rindex=([1.5, 2.5, 3.5, 5.0], [1.332, 1.336, 1.345, 1.366]), abslength=30.0,
                       rayleigh=20.0)  # fmt: skip
    acrylic = O.Material("Acrylic", rindex=1.49, abslength=5.0)
    cathode = O.Material("Photocathode")
    pmt = G.Volume("PMT", G.Tube(rmax=50 * MM, dz=10 * MM), "Photocathode")
    tank = G.Volume("TankLV", G.Box(0.5, 0.5, 0.5), "Water")
    block = G.Volume("Block", G.Box(0.15, 0.15, 0.1), "Acrylic")
    tank.place(block, (0.0, 0.0, -0.2), name="Block")
    places = [((0, 0, -480), None), ((0, 0, 480), None), ((-480, 0, 0), ("y", 90)), ((480, 0, 0), ("y", 90)),
              ((0, -480, 0), ("x", 90)), ((0, 480, 0), ("x", 90)), ((-250, 0, -480), None), ((250, 0, -480), None)]
    for i, (p, r) in enumerate(places):
        rot = None if r is None else G.gdml_rotation(**{r[0]: r[1]})
        tank.place(pmt, np.asarray(p, float) * MM, rot, name=f"PMT_{i}", copy=i)
    surf = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    wall = O.OpticalSurface("Wall", "dielectric_metal", "ground", model="glisur", polish=polish_wall,
                            reflectivity=0.7)  # fmt: skip
    into = O.OpticalSurface("BlockIn", "dielectric_dielectric", "ground", model="glisur", polish=polish_block)
    out = O.OpticalSurface("BlockOut", "dielectric_dielectric", "ground", model="glisur", polish=polish_block)
    borders = [("TankLV", f"PMT_{i}", surf) for i in range(8)] + [("TankLV", "Block", into), ("Block", "TankLV", out)]
    return D.build(tank, {"Water": water, "Acrylic": acrylic, "Photocathode": cathode}, borders=borders,
                   skins={"TankLV": wall}, sensors={"pmt": "PMT"})  # fmt: skip


def fog_box(half=4.0, rayleigh=0.5, abs_len=30.0) -> D.Detector:
    """Return a cube of half-width ``half`` m filled with a strongly scattering medium (Rayleigh length ``rayleigh``
    m: the diffusion jump's domain, a volume at least 4 scattering lengths across), a dark 1 m block inside, and
    sensor discs (r 0.3 m) on four of its faces."""  # noqa: D205
    fog = O.Material("Fog", rindex=1.33, abslength=abs_len, rayleigh=rayleigh)
    steel = O.Material("Steel")
    box = G.Volume("FogBox", G.Box(half, half, half), "Fog")
    block = G.Volume("Block", G.Box(0.5, 0.5, 0.5), "Steel")
    box.place(block, (1.5, -1.0, 0.5), name="Block")
    disc = G.Volume("Sensor", G.Tube(rmax=0.3, dz=0.01), "Steel")
    faces = [((-half + 0.02, 0.0, 0.0), (1.0, 0.0, 0.0)), ((half - 0.02, 1.0, 0.0), (-1.0, 0.0, 0.0)),
             ((0.0, -half + 0.02, 1.0), (0.0, 1.0, 0.0)), ((0.5, 0.0, half - 0.02), (0.0, 0.0, -1.0))]
    for i, (p, ax) in enumerate(faces):
        box.place(disc, p, _frame_z(ax), name=f"Sensor_{i}", copy=i)
    sens = O.OpticalSurface("SensorSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    borders = [("FogBox", f"Sensor_{i}", sens) for i in range(len(faces))]
    return D.build(box, {"Fog": fog, "Steel": steel}, borders=borders, sensors={"sensor": "Sensor"})


def _grid_tank(n_pmt, radius, half_h, r_pmt, inset):
    """Return (positions, inward axes) of n_pmt PMTs on a regular barrel and end-cap grid."""
    area = 2 * math.pi * radius * 2 * half_h + 2 * math.pi * radius**2
    s = math.sqrt(area / n_pmt)
    while True:
        n_phi = max(int(round(2 * math.pi * radius / s)), 1)
        n_z = max(int(round(2 * half_h / s)), 1)
        pos, ax = [], []
        rr = radius - inset
        for iz in range(n_z):
            z = -half_h + (iz + 0.5) * (2 * half_h / n_z)
            for ip in range(n_phi):
                ph = 2 * math.pi * (ip + 0.5) / n_phi
                c, si = math.cos(ph), math.sin(ph)
                pos.append((rr * c, rr * si, z))
                ax.append((-c, -si, 0.0))
        cap = []
        m = int(math.ceil(radius / s)) + 1
        for i in range(-m, m + 1):
            for j in range(-m, m + 1):
                x, y = (i + 0.5) * s, (j + 0.5) * s
                if math.hypot(x, y) + r_pmt < radius - 2 * r_pmt:
                    cap.append((x, y))
        cap.sort(key=lambda p: (math.hypot(*p), p))
        need = n_pmt - len(pos)
        if 0 <= need <= 2 * len(cap):
            top = cap[: (need + 1) // 2]
            bot = cap[: need // 2]
            for x, y in top:
                pos.append((x, y, half_h - inset))
                ax.append((0.0, 0.0, -1.0))
            for x, y in bot:
                pos.append((x, y, -half_h + inset))
                ax.append((0.0, 0.0, 1.0))
            return np.asarray(pos), np.asarray(ax)
        s *= 0.99 if need > 2 * len(cap) else 1.01


def _frame_z(axis):
    """Return a rotation whose local z is ``axis``."""
    z = np.asarray(axis, float)
    z = z / np.linalg.norm(z)
    a = np.array([1.0, 0, 0]) if abs(z[0]) < 0.9 else np.array([0, 1.0, 0])
    x = np.cross(a, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    return np.stack([x, y, z], 1)


def cylinder_tank(n_pmt=2000, radius=5.0, half_h=5.0, r_pmt=0.1, wall_r=0.1, wall_finish="polished",
                  sigma_alpha=0.0, abs_len=50.0, ray_len=80.0, rindex=1.34) -> D.Detector:
    """Return the synthetic water tank of the plain-forward workload (see the module docstring)."""
    water = O.Material("Water", rindex=rindex, abslength=abs_len, rayleigh=ray_len)
    pmt = G.Volume("PMT", G.Sphere(r_pmt, hemisphere=+1), "Photocathode")
    tank = G.Volume("Tank", G.Tube(rmax=radius, dz=half_h), "Water")
    # the hemisphere's flat face 1.5 mm inside the wall: the disc's rim clears the curved barrel wall
    pos, ax = _grid_tank(n_pmt, radius, half_h, r_pmt, inset=1.5 * MM)
    for i in range(len(pos)):
        tank.place(pmt, pos[i], _frame_z(ax[i]), name=f"PMT_{i}", copy=i)
    cath = O.OpticalSurface("Cathode", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    if wall_finish == "polished":
        wall = O.OpticalSurface("BlackSheet", "dielectric_metal", "polished", reflectivity=wall_r)
    else:
        wall = O.OpticalSurface("BlackSheet", "dielectric_metal", "ground", reflectivity=wall_r,
                                sigma_alpha=sigma_alpha, specularlobe=1.0 if sigma_alpha > 0 else 0.0)  # fmt: skip
    borders = [("Tank", f"PMT_{i}", cath) for i in range(len(pos))]
    return D.build(tank, {"Water": water, "Photocathode": O.Material("Photocathode")}, borders=borders,
                   skins={"Tank": wall}, sensors={"pmt": "PMT"})  # fmt: skip


def lar_box(n_x=12, n_y=10, cage_r=0.9, sigma_alpha=0.0, ray_len=0.9, abs_len=20.0, rindex=1.38) -> D.Detector:
    """Return the synthetic liquid-argon box of the scintillation workload (see the module docstring)."""
    lar = O.Material("LAr", rindex=rindex, abslength=abs_len, rayleigh=ray_len)
    steel = O.Material("Steel")
    box = G.Volume("LArBox", G.Box(2.5, 2.0, 2.0), "LAr")
    # field cage: a box shell 2 cm thick inside the walls, minus the sensor wall's face, plus two rails (union)
    shell = G.Boolean("subtraction", G.Box(2.45, 1.95, 1.95), G.Box(2.43, 1.93, 1.93))
    open_face = G.Boolean("subtraction", shell, G.Box(0.02, 1.94, 1.94), pos=(-2.44, 0.0, 0.0))
    cage_solid = G.Boolean("union", open_face, G.Box(2.0, 0.02, 0.02), pos=(0.0, 1.9, 0.0))
    cage = G.Volume("FieldCage", cage_solid, "Steel")
    # cathode: a plate at x = +0.5 m with a window cut out (a box subtraction)
    plate = G.Boolean("subtraction", G.Box(0.01, 1.5, 1.5), G.Box(0.02, 0.3, 0.3))
    cathode = G.Volume("Cathode", plate, "Steel")
    box.place(cage, (0.0, 0.0, 0.0), name="FieldCage")
    box.place(cathode, (0.5, 0.0, 0.0), name="Cathode")
    disc = G.Volume("Sensor", G.Tube(rmax=0.1, dz=0.005), "Steel")
    rot = _frame_z((1.0, 0.0, 0.0))
    k = 0
    for iy in range(n_x):
        for iz in range(n_y):
            y = -1.65 + 3.3 * (iy + 0.5) / n_x
            z = -1.6 + 3.2 * (iz + 0.5) / n_y
            box.place(disc, (-2.49, y, z), rot, name=f"Sensor_{k}", copy=k)
            k += 1
    if sigma_alpha > 0.0:
        refl = O.OpticalSurface("CageSurface", "dielectric_metal", "ground", reflectivity=cage_r,
                                sigma_alpha=sigma_alpha, specularlobe=1.0)  # fmt: skip
    else:
        refl = O.OpticalSurface("CageSurface", "dielectric_metal", "ground", reflectivity=cage_r)
    sens = O.OpticalSurface("SensorSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    borders = [("LArBox", f"Sensor_{i}", sens) for i in range(k)]
    # the box's own walls absorb (the detector volume's boundary)
    return D.build(box, {"LAr": lar, "Steel": steel}, borders=borders,
                   skins={"FieldCage": refl, "Cathode": refl}, sensors={"sensor": "Sensor"})  # fmt: skip
