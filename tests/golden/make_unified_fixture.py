"""Sample the reference's unified facet tables into a small fixture.

    python tests/golden/make_unified_fixture.py /path/to/lumen     # writes tests/golden/unified_tables.npz

The reference computes the tables with numpy alone (src/lumen/surfaces/facets.py:127 ``unified_tables``); its module
imports JAX, so the numpy-backed stand-in of make_golden.py is installed first. Kept: log zeta and its derivative at
every node, and F, Fx, Fy, Fxy at 1024 seeded (i, j) nodes with their indices.
"""

import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_golden  # noqa: E402


def main(ref):
    make_golden.install_stub()
    make_golden.register_lumen(os.path.join(ref, "src"))
    T = importlib.import_module("lumen.surfaces.facets").unified_tables()
    nx, ny = T["F"].shape
    rng = np.random.default_rng(5)
    i = rng.integers(0, nx, 1024)
    j = rng.integers(0, ny, 1024)
    i[:4], j[:4] = [0, nx - 1, 0, nx - 1], [0, 0, ny - 1, ny - 1]  # the corners
    out = {k: np.asarray(T[k], np.float32)[i, j] for k in ("F", "Fx", "Fy", "Fxy")}
    out.update(i=i.astype(np.int32), j=j.astype(np.int32), lz=np.asarray(T["lz"], np.float32),
               lzy=np.asarray(T["lzy"], np.float32), shape=np.asarray([nx, ny]))  # fmt: skip
    np.savez_compressed(os.path.join(HERE, "unified_tables.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the lumen source tree (the directory holding src/lumen)>")
    main(sys.argv[1])
