"""Detectors exported from the reference's own host pipeline (run where the reference is mounted).

    python tests/golden/make_reference_detector.py /path/to/lumen   # writes tests/golden/refdet_<name>.json

The reference converts and loads its two shipped example detectors under the numpy-backed ``jax`` stub
(``refstub.py``): the tutorial's toy tank (examples/data/example_tank.gdml with the recipe of
examples/example_tank.py: detector volume TankLV, the PMT placements counted across CathodeSurface) and the YAML toy
(examples/data/yaml_toy), and the scintillator cube of ``tests/golden/yaml_scint`` (this repository's YAML, in the
reference's format: Rayleigh, Mie and a WLS with an exponential profile in one medium, a ground unified wall).
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
