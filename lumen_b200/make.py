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
         "-prec-div=true", "-prec-sqrt=true", "-ftz=false", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC"]  # fmt: skip
LINK = ["-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler", "-fPIC"]
PART = os.path.join(HERE, "csrc", "k_part.cu")
N_PARTS = 12  # LUMEN_N_PARTS in csrc/engine.cuh: the kernel instantiations' parts, compiled in parallel
OBJ = os.path.join(HERE, "_build")


def sources():
    d = os.path.join(HERE, "csrc")
    return [os.path.join(d, f) for f in sorted(os.listdir(d))] + [os.path.join(HERE, "..", "include", "lumen_b200.h")]


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(f) > t for f in sources())


def _compile(job):
    cmd, out = job
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed ({r.returncode}) on {out}:\n{r.stderr[-8000:]}")
    return r.stderr


def build(force: bool = False, verbose: bool = False, out: str = OUT, defines=()) -> str:
    """Compile the engine if a source is newer than the library; return the library's path.

    The host side (csrc/lumen_b200.cu) and the parts of the kernel instantiations (csrc/k_part.cu, one object per
    part) compile in parallel, then link into one shared library with the CUDA runtime linked statically.
    """
    if not force and not stale() and out == OUT:
        return OUT
    from concurrent.futures import ThreadPoolExecutor

    tag = "" if out == OUT else f"_{abs(hash(out)) & 0xFFFFFF:06x}"
    odir = OBJ + tag
    os.makedirs(odir, exist_ok=True)
    extra = [*(["-Xptxas", "-v"] if verbose else []), *[f"-D{d}" for d in defines]]
    jobs = [([NVCC, *FLAGS, *extra, "-c", "-o", os.path.join(odir, "host.o"), SRC], "host.o")]
    jobs += [([NVCC, *FLAGS, *extra, f"-DLUMEN_PART={k}", "-c", "-o", os.path.join(odir, f"part{k}.o"), PART],
              f"part{k}.o") for k in range(N_PARTS)]  # fmt: skip
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as ex:
        logs = list(ex.map(_compile, jobs))
    objs = [os.path.join(odir, j[1]) for j in jobs]
    r = subprocess.run([NVCC, *LINK, "-o", out + ".tmp", *objs], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc link failed ({r.returncode}):\n{r.stderr[-8000:]}")
    if verbose:
        print("\n".join(logs))
    os.replace(out + ".tmp", out)
    return out


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
