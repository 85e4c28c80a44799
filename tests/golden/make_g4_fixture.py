"""Extract the reference's Geant4 golden histograms of the unified facet path into a small fixture.

    python tests/golden/make_g4_fixture.py /path/to/lumen     # writes tests/golden/g4_unified_metal.npz

The reference's tests/data/g4_boundary holds Geant4 11.3.0 runs of G4OpBoundaryProcess on one flat interface
(tools/g4ref/boundary.cc: 10^6 photons per case, MANIFEST.json with settings and sha256): for a unified ground
dielectric_metal surface with R = 1 and SPECULARLOBECONSTANT 1, the histogram of the last direction in (dz, |phi|).
This keeps those of the unified metal cases, with their incidence angle and sigma_alpha.
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


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
