"""Extract the reference's Geant4 golden histograms of the facet paths into small fixtures.

    python tests/golden/make_g4_fixture.py /path/to/lumen
    # writes tests/golden/g4_unified_metal.npz and tests/golden/g4_glisur_dielectric.npz

The reference's tests/data/g4_boundary holds Geant4 11.3.0 runs of G4OpBoundaryProcess on one flat interface
(tools/g4ref/boundary.cc: 10^6 photons per case, MANIFEST.json with settings and sha256): for a unified ground
dielectric_metal surface with R = 1 and SPECULARLOBECONSTANT 1, the histogram of the last direction in (dz, |phi|).
This keeps those of the unified metal cases, with their incidence angle and sigma_alpha, and of the GLISUR ground
dielectric_dielectric cases launched with random linear polarisation (R = 1, T = 0: the facet loop of
DielectricDielectric), with their incidence angle, polish and indices.
"""

import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    d = os.path.join(ref, "tests", "data", "g4_boundary")
    man = json.load(open(os.path.join(d, "MANIFEST.json")))
    out = {}
    names = sorted(k for k, c in man["cases"].items() if c["model"] == "unified" and c["type"] == "dielectric_metal")
    for i, name in enumerate(names):
        c = man["cases"][name]
        path = os.path.join(d, c["file"])
        assert hashlib.sha256(open(path, "rb").read()).hexdigest() == c["sha256"]
        z = np.load(path)
        out[f"c{i}_hist"] = z["hist"]
        out[f"c{i}_edges_z"] = z["edges_z"]
        out[f"c{i}_edges_phi"] = z["edges_phi"]
        out[f"c{i}_theta_deg"] = np.float64(c["theta"])
        out[f"c{i}_sigma"] = np.float64(c["value"])
    out["names"] = np.asarray(names)
    np.savez_compressed(os.path.join(HERE, "g4_unified_metal.npz"), **out)
    print(names)
    out = {}
    names = sorted(k for k, c in man["cases"].items()
                   if c["model"] == "glisur" and c["type"] == "dielectric_dielectric" and c["pol"] == "random")
    for i, name in enumerate(names):
        c = man["cases"][name]
        path = os.path.join(d, c["file"])
        assert hashlib.sha256(open(path, "rb").read()).hexdigest() == c["sha256"]
        z = np.load(path)
        out[f"c{i}_hist"] = z["hist"]
        out[f"c{i}_edges_z"] = z["edges_z"]
        out[f"c{i}_edges_phi"] = z["edges_phi"]
        for k in ("theta", "value", "n1", "n2"):
            out[f"c{i}_{k}"] = np.float64(c[k])
    out["names"] = np.asarray(names)
    np.savez_compressed(os.path.join(HERE, "g4_glisur_dielectric.npz"), **out)
    print(names)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the lumen source tree (the directory holding src/lumen)>")
    main(sys.argv[1])
