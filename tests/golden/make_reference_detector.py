"""Detectors exported from the reference's own host pipeline (run where the reference is mounted).

    python tests/golden/make_reference_detector.py /path/to/lumen   # writes tests/golden/refdet_<name>.json

The reference converts and loads its two shipped example detectors under the numpy-backed ``jax`` stub
(``refstub.py``): the tutorial's toy tank (examples/data/example_tank.gdml with the recipe of
examples/example_tank.py: detector volume TankLV, the PMT placements counted across CathodeSurface) and the YAML toy
(examples/data/yaml_toy), and the scintillator cube of ``tests/golden/yaml_scint`` (this repository's YAML, in the
reference's format: Rayleigh, Mie and a WLS with an exponential profile in one medium, a ground unified wall), and
``detectors.mesh_tank`` written out in the same format by ``mesh_tank_yaml`` (tessellated parts, an orb, skins), and
a water cube that is an ``any_entry`` sensor counting the photons born inside it (``born_cube_yaml``), and a comb
of 17 bars in one union solid, which the reference places as its pieces (``comb_yaml``).
``lumen_b200.reference.export`` then writes what the reference's photon loop runs on: the
navigator scene's instances and flattened solids, the compiled optics, the packed parameters, the defensive rows.
The tests rebuild the detectors from these files with ``lumen_b200.reference.detector``.
"""

from __future__ import annotations

import os
import shutil
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)


def _num(x):
    return repr(float(x))


def mesh_tank_yaml(where):
    """Write ``lumen_b200.detectors.mesh_tank`` (a water box holding a tessellated steel icosphere, a tessellated
    black box, a glass orb and eight sensor discs) in the reference's YAML detector format into the directory
    ``where``: its triangles and rotation matrices written out from this package's own geometry helpers."""  # noqa: D205, D209
    from lumen_b200 import geometry as G

    ball, block = G.icosphere(0.4, 2), G.box_mesh(0.3, 0.2, 0.25)
    rb, rk = G.rotation("x", 20.0), G.rotation("z", 30.0) @ G.rotation("y", 15.0)

    def tris(t):
        return "[" + ", ".join("[" + ", ".join("[" + ", ".join(_num(c) for c in v) + "]" for v in tri) + "]"
                               for tri in t) + "]"  # fmt: skip

    def mat(m):
        return "{matrix: [" + ", ".join("[" + ", ".join(_num(c) for c in row) + "]" for row in m) + "]}"

    flat = "{energy: [1.5, 5.0], value: [%s, %s]}"
    lines = ["schema: lumen-detector-yaml/3", "name: yaml_mesh", "detector_volume: Box", "solids:",
             "  WorldBox: {type: box, params: {x: 4*m, y: 4*m, z: 4*m}}",
             "  BoxSolid: {type: box, params: {x: 3*m, y: 3*m, z: 3*m}}",
             "  OrbSolid: {type: orb, params: {r: 0.25*m}}",
             "  PMTDisc: {type: tube, params: {rmax: 0.15*m, z: 0.02*m}}",
             "  BallMesh: {type: tessellated, mesh: ball}", "  BlockMesh: {type: tessellated, mesh: block}",
             f"meshes:\n  ball: {tris(ball)}\n  block: {tris(block)}", "volumes:",
             "  World: {solid: WorldBox, material: Air}", "  Box: {solid: BoxSolid, material: Water}",
             "  Ball: {solid: BallMesh, material: Steel}", "  Block: {solid: BlockMesh, material: Black}",
             "  Orb: {solid: OrbSolid, material: Glass}", "  PMT: {solid: PMTDisc, material: Photocathode}",
             "placements:", "  - {name: BoxPV, volume: Box, mother: World}",
             f"  - {{name: Ball, volume: Ball, mother: Box, position: [-0.5, 0.2, 0.1], rotation: {mat(rb)}}}",
             f"  - {{name: Block, volume: Block, mother: Box, position: [0.6, -0.3, -0.2], rotation: {mat(rk)}}}",
             "  - {name: Orb, volume: Orb, mother: Box, position: [0.3, 0.6, 0.4]}"]  # fmt: skip
    for i in range(4):
        x = _num(-0.75 + 0.5 * i)
        lines.append(f"  - {{name: PMT_{i}, volume: PMT, mother: Box, copy: {i}, position: [{x}, 0.0, -1.48]}}")
        lines.append(f"  - {{name: PMT_{4 + i}, volume: PMT, mother: Box, copy: {4 + i}, position: [{x}, 0.0, 1.48]}}")
    lines += ["materials:",
              "  Water: {state: liquid, composition: {density_g_cm3: 1.0, components: [{ref: H, atoms: 2}, "
              "{ref: O, atoms: 1}]}, properties: {RINDEX: " + flat % (1.33, 1.33) + ", ABSLENGTH: " + flat % (30.0, 30.0) +
              ", RAYLEIGH: " + flat % (10.0, 10.0) + "}}",
              "  Glass: {state: solid, composition: {density_g_cm3: 2.2, components: [{ref: Si, atoms: 1}, "
              "{ref: O, atoms: 2}]}, properties: {RINDEX: " + flat % (1.5, 1.5) + ", ABSLENGTH: " + flat % (5.0, 5.0) +
              "}}"]
    for name in ("Air", "Steel", "Black", "Photocathode"):
        lines.append(f"  {name}: {{state: solid, composition: {{density_g_cm3: 1.0, components: "
                     f"[{{ref: O, fraction: 1.0}}]}}}}")
    lines += ["surfaces:",
              "  CathodeSurface: {type: dielectric_metal, model: unified, finish: polished, value: 0, properties: "
              "{REFLECTIVITY: " + flat % (0.0, 0.0) + ", EFFICIENCY: " + flat % (1.0, 1.0) + "}}",
              "  Shiny: {type: dielectric_metal, model: unified, finish: polished, value: 0, properties: "
              "{REFLECTIVITY: " + flat % (0.8, 0.8) + "}}",
              "  Wall: {type: dielectric_metal, model: unified, finish: ground, value: 0.2, properties: "
              "{REFLECTIVITY: " + flat % (0.6, 0.6) + ", SPECULARLOBECONSTANT: " + flat % (0.5, 0.5) + "}}",
              "skins:", "  - {name: WallSkin, surface: Wall, volume: Box}",
              "  - {name: ShinySkin, surface: Shiny, volume: Ball}", "borders:"]  # fmt: skip
    lines += [f"  - {{name: Cathode_{i}, surface: CathodeSurface, pv1: BoxPV, pv2: PMT_{i}}}" for i in range(8)]
    lines += ["sensors:", "  - {name: pmt, rule: border_into, lv: PMT, values: examples/data/toy_pmt.json, "
              "readout: {gate: [-10.0, 60.0]}}"]  # fmt: skip
    os.makedirs(where, exist_ok=True)
    with open(os.path.join(where, "detector.yaml"), "w") as f:
        f.write("\n".join(lines) + "\n")


def born_cube_yaml(where):
    """Write a 2 m water box holding a 0.4 m water cube that is a sensor of an ``any_entry`` group (counted on every
    entry, and counting the photons born inside it: src/lumen/rules/sensors.py:39 counts_born), in the reference's
    YAML detector format, into the directory ``where``."""  # noqa: D205, D209
    flat = "{energy: [1.5, 5.0], value: [%s, %s]}"
    text = "\n".join([
        "schema: lumen-detector-yaml/3", "name: yaml_born", "detector_volume: Box", "solids:",
        "  WorldBox: {type: box, params: {x: 3*m, y: 3*m, z: 3*m}}",
        "  BoxSolid: {type: box, params: {x: 2*m, y: 2*m, z: 2*m}}",
        "  CubeSolid: {type: box, params: {x: 0.4*m, y: 0.4*m, z: 0.4*m}}",
        "volumes:", "  World: {solid: WorldBox, material: Air}", "  Box: {solid: BoxSolid, material: Water}",
        "  Cube: {solid: CubeSolid, material: Water}",
        "placements:", "  - {name: BoxPV, volume: Box, mother: World}",
        "  - {name: CubePV, volume: Cube, mother: Box, position: [0.3, 0.0, 0.0]}",
        "materials:",
        "  Water: {state: liquid, composition: {density_g_cm3: 1.0, components: [{ref: H, atoms: 2}, {ref: O, "
        "atoms: 1}]}, properties: {RINDEX: " + flat % (1.33, 1.33) + ", ABSLENGTH: " + flat % (20.0, 20.0) +
        ", RAYLEIGH: " + flat % (5.0, 5.0) + "}}",
        "  Air: {state: gas, composition: {density_g_cm3: 0.0012, components: [{ref: N, fraction: 1.0}]}}",
        "sensors:", "  - {name: s, rule: any_entry, lv: Cube, values: examples/data/toy_pmt.json, "
        "readout: {gate: [-10.0, 60.0]}}", ""])  # fmt: skip
    os.makedirs(where, exist_ok=True)
    with open(os.path.join(where, "detector.yaml"), "w") as f:
        f.write(text)


COMB_BARS = 17  # a union of this many bars: past the reference's SPLIT_LEAVES (16), so it is placed as its pieces


def comb_yaml(where):
    """Write a 2 m water box holding a comb (a union of ``COMB_BARS`` steel bars, one solid: the reference places it
    as its pieces) and two disc sensors, in the reference's YAML detector format, into the directory ``where``."""  # noqa: D205, D209
    flat = "{energy: [1.5, 5.0], value: [%s, %s]}"
    lines = ["schema: lumen-detector-yaml/3", "name: yaml_comb", "detector_volume: Box", "solids:",
             "  WorldBox: {type: box, params: {x: 3*m, y: 3*m, z: 3*m}}",
             "  BoxSolid: {type: box, params: {x: 2*m, y: 2*m, z: 2*m}}",
             "  BarSolid: {type: box, params: {x: 0.04*m, y: 0.04*m, z: 1.2*m}}",
             "  PMTDisc: {type: tube, params: {rmax: 0.15*m, z: 0.02*m}}"]  # fmt: skip
    prev = "BarSolid"
    for k in range(1, COMB_BARS):
        x = -0.85 + 0.1 * k  # -0.75 .. 0.75 beside the first bar at 0: no two bars meet
        name = "Comb" if k == COMB_BARS - 1 else f"Comb{k}"
        lines.append(f"  {name}: {{type: union, refs: [{prev}, BarSolid], transforms: [{{}}, "
                     f"{{position: [{x!r}, 0.0, 0.0]}}]}}")
        prev = name
    lines += ["volumes:", "  World: {solid: WorldBox, material: Air}", "  Box: {solid: BoxSolid, material: Water}",
              "  Comb: {solid: Comb, material: Steel}", "  PMT: {solid: PMTDisc, material: Photocathode}",
              "placements:", "  - {name: BoxPV, volume: Box, mother: World}",
              "  - {name: CombPV, volume: Comb, mother: Box, position: [0.0, 0.0, 0.0]}",
              "  - {name: PMT_0, volume: PMT, mother: Box, copy: 0, position: [0.0, 0.0, 0.95]}",
              "  - {name: PMT_1, volume: PMT, mother: Box, copy: 1, position: [0.0, 0.0, -0.95]}",
              "materials:",
              "  Water: {state: liquid, composition: {density_g_cm3: 1.0, components: [{ref: H, atoms: 2}, {ref: O, "
              "atoms: 1}]}, properties: {RINDEX: " + flat % (1.33, 1.33) + ", ABSLENGTH: " + flat % (20.0, 20.0) +
              ", RAYLEIGH: " + flat % (5.0, 5.0) + "}}"]  # fmt: skip
    for name in ("Air", "Steel", "Photocathode"):
        lines.append(f"  {name}: {{state: solid, composition: {{density_g_cm3: 1.0, components: "
                     f"[{{ref: O, fraction: 1.0}}]}}}}")
    lines += ["surfaces:",
              "  CathodeSurface: {type: dielectric_metal, model: unified, finish: polished, value: 0, properties: "
              "{REFLECTIVITY: " + flat % (0.0, 0.0) + ", EFFICIENCY: " + flat % (1.0, 1.0) + "}}",
              "borders:", "  - {name: Cathode_0, surface: CathodeSurface, pv1: BoxPV, pv2: PMT_0}",
              "  - {name: Cathode_1, surface: CathodeSurface, pv1: BoxPV, pv2: PMT_1}",
              "sensors:", "  - {name: pmt, rule: border_into, lv: PMT, values: examples/data/toy_pmt.json, "
              "readout: {gate: [-10.0, 60.0]}}", ""]  # fmt: skip
    os.makedirs(where, exist_ok=True)
    with open(os.path.join(where, "detector.yaml"), "w") as f:
        f.write("\n".join(lines))


def main(ref_root):
    import refstub

    api = refstub.install(os.path.join(ref_root, "src"))
    from lumen.format.sensorsets import SensorGroup
    from lumen.recipe import Recipe

    from lumen_b200 import reference

    data = os.path.join(ref_root, "examples", "data")
    recipe = Recipe(name="example_tank", detector_volume="TankLV",
                    groups=(SensorGroup("pmt", rule="border_into", lv="PMT", values=os.path.join(data, "toy_pmt.json"),
                                        readout={"gate": (-10.0, 60.0)}),))  # fmt: skip
    tmp = tempfile.mkdtemp(dir=HERE)
    cwd = os.getcwd()
    try:
        os.chdir(ref_root)  # the YAML toy names its sensor values relative to the reference's root
        made = {"example_tank": api.convert(os.path.join(data, "example_tank.gdml"), os.path.join(tmp, "t.lumen"),
                                            recipe=recipe),
                "yaml_toy": api.convert(os.path.join(data, "yaml_toy"), os.path.join(tmp, "y.lumen")),
                "yaml_scint": api.convert(os.path.join(HERE, "yaml_scint"), os.path.join(tmp, "s.lumen"))}  # fmt: skip
        mesh_tank_yaml(os.path.join(tmp, "yaml_mesh"))
        made["yaml_mesh"] = api.convert(os.path.join(tmp, "yaml_mesh"), os.path.join(tmp, "m.lumen"))
        born_cube_yaml(os.path.join(tmp, "yaml_born"))
        made["yaml_born"] = api.convert(os.path.join(tmp, "yaml_born"), os.path.join(tmp, "b.lumen"))
        comb_yaml(os.path.join(tmp, "yaml_comb"))
        made["yaml_comb"] = api.convert(os.path.join(tmp, "yaml_comb"), os.path.join(tmp, "c.lumen"))
        for name, path in made.items():
            x = reference.export(api.load(path))
            reference.save(x, os.path.join(HERE, f"refdet_{name}.json"))
            print(f"{name}: {len(x['volumes'])} volumes, {x['n_classes']} classes, {len(x['rows'])} rows, "
                  f"{len(x['sensors']['name'])} sensors")
    finally:
        os.chdir(cwd)
        shutil.rmtree(tmp)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the lumen source tree (the directory holding src/lumen)>")
    main(sys.argv[1])
