"""Generate golden vectors from the reference's own Python (run in a container where the reference is mounted).

    python tests/golden/make_golden.py /path/to/lumen     # writes tests/golden/reference_vectors.npz

The reference's device functions are JAX; JAX is not installed here, so a minimal numpy-backed ``jax`` module stands
in for the few calls these functions make (jnp = numpy; lax.stop_gradient = identity; jit = identity), and the
``lumen`` package is registered by path so that its ``__init__`` (which imports the JAX runtime) does not run.
Only pure elementwise functions are evaluated: Fresnel amplitudes (src/lumen/surfaces/fresnel.py:25), the Rayleigh
inverse CDFs (src/lumen/media/phase.py:43-50), the orthonormal basis (src/lumen/_core/frames.py:14), Geant4's water
Rayleigh table (src/lumen/rules/optics.py:208) and the GROUPVEL group index (src/lumen/media/laws.py:156-183).
The vectors are then the reference's outputs on fixed inputs, in float64 numpy arithmetic.
"""

from __future__ import annotations

import contextlib
import importlib
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def install_stub():
    jax = types.ModuleType("jax")
    jnp = np
    lax = types.ModuleType("jax.lax")
    lax.stop_gradient = lambda x: x
    lax.cond = lambda p, a, b, *ops: a(*ops) if p else b(*ops)
    lax.switch = lambda i, brs, *ops: brs[int(i)](*ops)
    jax.numpy = jnp
    jax.lax = lax
    jax.jit = lambda f=None, **kw: (f if f is not None else (lambda g: g))
    jax.vmap = lambda f, *a, **k: np.vectorize(f)

    class _CJ:
        def __init__(self, f, **kw):
            self.f = f

        def __call__(self, *a, **k):
            return self.f(*a, **k)

        def defjvp(self, g):
            return g

    jax.custom_jvp = lambda f=None, **kw: _CJ(f) if f is not None else (lambda g: _CJ(g))
    jax.ensure_compile_time_eval = contextlib.nullcontext
    jax.Array = np.ndarray
    jax.tree_util = types.ModuleType("jax.tree_util")
    jax.tree_util.tree_map = lambda f, *t: f(*t)
    jax.tree_util.register_pytree_node = lambda *a, **k: None
    jax.tree_util.register_pytree_node_class = lambda c: c
    jax.tree_util.register_dataclass = lambda c, *a, **k: c
    jax.tree_util.tree_leaves = lambda t, **k: [t]
    jax.tree = jax.tree_util
    jax.random = types.ModuleType("jax.random")
    jax.scipy = types.ModuleType("jax.scipy")
    jax.nn = types.ModuleType("jax.nn")
    jax.core = types.ModuleType("jax.core")
    jax.core.Tracer = type("Tracer", (), {})
    jax.dtypes = types.ModuleType("jax.dtypes")
    for name, mod in (("jax", jax), ("jax.numpy", jnp), ("jax.lax", lax), ("jax.tree_util", jax.tree_util),
                      ("jax.random", jax.random), ("jax.scipy", jax.scipy), ("jax.nn", jax.nn),
                      ("jax.core", jax.core), ("jax.dtypes", jax.dtypes)):  # fmt: skip
        sys.modules[name] = mod


def register_lumen(src):
    pkg = types.ModuleType("lumen")
    pkg.__path__ = [os.path.join(src, "lumen")]
    sys.modules["lumen"] = pkg


def main(ref_root):
    install_stub()
    register_lumen(os.path.join(ref_root, "src"))
    out = {}
    fresnel = importlib.import_module("lumen.surfaces.fresnel")
    rng = np.random.default_rng(11)
    cos_i = np.concatenate([rng.uniform(0, 1, 64), [0.0, 1.0, 0.05, 0.999]])
    n1 = np.concatenate([rng.uniform(1.0, 1.6, 64), [1.33, 1.33, 1.5, 1.0]])
    n2 = np.concatenate([rng.uniform(1.0, 1.6, 64), [1.0, 1.5, 1.0, 1.33]])
    nk = np.concatenate([np.zeros(48), rng.uniform(0.0, 2.0, 16), [0.0, 0.0, 0.0, 1.5]])
    amps = []
    for c, a, b, k in zip(cos_i, n1, n2, nk, strict=True):
        r = fresnel.amplitudes(np.float64(c), np.complex128(a), np.complex128(b + 1j * k))
        amps.append([z for x in r for z in (np.real(x), np.imag(x))])
    out.update(fresnel_in=np.stack([cos_i, n1, n2, nk], 1), fresnel_out=np.asarray(amps, np.float64))
    frames = importlib.import_module("lumen._core.frames")
    v = rng.normal(size=(256, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    t1, t2 = frames.basis(v)
    out.update(basis_in=v, basis_t1=np.asarray(t1), basis_t2=np.asarray(t2))
    phase = importlib.import_module("lumen.media.phase")
    u = np.concatenate([rng.uniform(0, 1, 256), [1e-6, 0.5, 1 - 1e-6]])
    out.update(phase_u=u, rayleigh_mu=np.asarray(phase.rayleigh_mu(u)), dipole_cos=np.asarray(phase.dipole_cos(u)))
    optics = importlib.import_module("lumen.rules.optics")
    e = np.array([1.5, 2.5, 3.5, 5.0])
    n = np.array([1.332, 1.336, 1.345, 1.366])
    c1 = optics.WATER_COMPRESSIBILITY * optics.WATER_TEMPERATURE * optics.K_BOLTZMANN / (6.0 * np.pi)
    out.update(water_e=e, water_n=n, water_rayleigh=np.asarray(optics._rayleigh_length_f32(np.float32(e),
                                                                                           np.float32(n),
                                                                                           np.float32(c1))))
    laws = importlib.import_module("lumen.media.laws")
    lam = np.linspace(230.0, 860.0, 64)
    out.update(groupvel_lam=lam, groupvel_ng=np.asarray(laws.geant4_group_index(e, n, lam), np.float64))
    np.savez_compressed(os.path.join(HERE, "reference_vectors.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the lumen source tree (the directory holding src/lumen)>")
    main(sys.argv[1])
