"""Build the CUDA engine in-tree: ``lumen_b200/liblumen_b200.so`` for sm_100a (B200).

    python -m lumen_b200.make          # or __graft_entry__.build()

nvcc compiles the engine with -fmad=false (no fused multiply-add the source does not spell out: the engine's
arithmetic is the CPU checker's, operation for operation) and -lineinfo for the profiler.
"""

from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc", "lumen_b200.cu")
OUT = os.path.join(HERE, "liblumen_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
FLAGS = ["-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-fmad=false",
         "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC",
         "-shared", "-cudart", "static"]  # fmt: skip


def sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d))] + [os.path.join(HERE, "..", "include", "lumen_b200.h")]


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(f) > t for f in sources())


def build(force: bool = False, verbose: bool = False, out: str = OUT, defines=()) -> str:
    """Compile the engine if a source is newer than the library; return the library's path."""
    if not force and not stale() and out == OUT:
        return OUT
    cmd = [NVCC, *FLAGS, *(["-Xptxas", "-v"] if verbose else []), *[f"-D{d}" for d in defines], "-o", out + ".tmp",
           SRC]  # fmt: skip
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}):\n{r.stderr[-8000:]}")
    if verbose:
        print(r.stderr)
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
