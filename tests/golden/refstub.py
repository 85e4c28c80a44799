"""The numpy-backed ``jax`` stub of ``make_golden.py``, widened so that the reference's whole host pipeline runs:
``lumen.convert`` (GDML or YAML -> a detector file) and ``lumen.load`` (-> ``Detector``: its ``parts``, the
navigator's scene and the compiled optics) and ``lumen.build.pack.pack``. Used by the fixture scripts only, where
the reference is mounted; the reference's photon loop (JAX on a device) is never run under it.

What it adds to ``make_golden.install_stub``: pytrees (dicts, lists, tuples, named tuples, registered classes and
dataclasses) for ``tree_map`` / ``tree_leaves``; ``vmap`` as a loop over the mapped axis; ``custom_jvp.defjvp`` with
keyword options; ``jax.scipy.special`` from scipy; ``jax.config`` (64-bit mode on); ``jax.errors``.
"""

from __future__ import annotations

import dataclasses
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

from make_golden import install_stub, register_lumen  # noqa: E402

_REG: dict = {}  # registered pytree class -> (flatten, unflatten)


def _tree_map(f, t, *rest, is_leaf=None):
    if is_leaf is not None and is_leaf(t):
        return f(t, *rest)
    ty = type(t)
    if ty in _REG:
        flat, unflat = _REG[ty]
        ch, aux = flat(t)
        rch = [flat(r)[0] for r in rest]
        return unflat(aux, [_tree_map(f, x, *[r[i] for r in rch], is_leaf=is_leaf) for i, x in enumerate(ch)])
    if isinstance(t, dict):
        return {k: _tree_map(f, t[k], *[r[k] for r in rest], is_leaf=is_leaf) for k in t}
    if isinstance(t, tuple) and hasattr(t, "_fields"):
        return ty(*[_tree_map(f, x, *[r[i] for r in rest], is_leaf=is_leaf) for i, x in enumerate(t)])
    if isinstance(t, (list, tuple)):
        return ty(_tree_map(f, x, *[r[i] for r in rest], is_leaf=is_leaf) for i, x in enumerate(t))
    if t is None:
        return None
    return f(t, *rest)


def _tree_leaves(t, is_leaf=None):
    out = []
    _tree_map(out.append, t, is_leaf=is_leaf)
    return out


def _register_class(c):
    _REG[c] = (lambda x: x.tree_flatten(), lambda aux, ch, c=c: c.tree_unflatten(aux, ch))
    return c


def _register_node(c, flatten, unflatten, *a, **k):
    _REG[c] = (flatten, unflatten)


def _register_dataclass(c, data_fields=None, meta_fields=None, *a, **k):
    names = list(data_fields) if data_fields is not None else [f.name for f in dataclasses.fields(c)]

    def flatten(x):
        return [getattr(x, n) for n in names], x

    def unflatten(x, ch):
        return dataclasses.replace(x, **dict(zip(names, ch, strict=True)))

    _REG[c] = (flatten, unflatten)
    return c


def _vmap(f, in_axes=0, out_axes=0, **kw):
    def g(*args):
        axes = in_axes if isinstance(in_axes, (list, tuple)) else [in_axes] * len(args)
        n = next(len(_tree_leaves(a)[0]) if not hasattr(a, "shape") else a.shape[ax]
                 for a, ax in zip(args, axes, strict=True) if ax is not None)  # fmt: skip
        outs = [f(*[_tree_map(lambda x, i=i, ax=ax: np.take(np.asarray(x), i, axis=ax), a) if ax is not None else a
                    for a, ax in zip(args, axes, strict=True)]) for i in range(n)]  # fmt: skip
        return _tree_map(lambda *xs: np.stack([np.asarray(x) for x in xs]), outs[0], *outs[1:])

    return g


class _CustomJVP:
    def __init__(self, f, **kw):
        self.f = f

    def __call__(self, *a, **k):
        return self.f(*a, **k)

    def defjvp(self, g, **kw):
        return g


def install(ref_src):
    """Install the stub and register the reference's ``lumen`` package from ``ref_src`` (its ``src`` directory)."""
    import scipy.special as ss

    install_stub()
    jax = sys.modules["jax"]
    jax.tree_util.tree_map = _tree_map
    jax.tree_util.tree_leaves = _tree_leaves
    jax.tree_util.register_pytree_node_class = _register_class
    jax.tree_util.register_pytree_node = _register_node
    jax.tree_util.register_dataclass = _register_dataclass
    jax.vmap = _vmap
    jax.custom_jvp = lambda f=None, **kw: _CustomJVP(f) if f is not None else (lambda g: _CustomJVP(g))
    special = types.ModuleType("jax.scipy.special")
    for name in ("log_ndtr", "ndtr", "erf", "erfc", "gammaln", "xlogy", "logsumexp"):
        setattr(special, name, getattr(ss, name))
    jax.scipy.__path__ = []
    jax.scipy.special = special
    jax.scipy.stats = types.ModuleType("jax.scipy.stats")
    sys.modules["jax.scipy.special"] = special
    sys.modules["jax.scipy.stats"] = jax.scipy.stats
    jax.config = types.SimpleNamespace(jax_enable_x64=True, update=lambda *a: None)
    errs = ("UnexpectedTracerError", "TracerArrayConversionError", "ConcretizationTypeError")
    jax.errors = types.SimpleNamespace(**{e: type(e, (Exception,), {}) for e in errs})
    jax.device_put = lambda x, *a, **k: x
    jax.devices = lambda *a: []
    jax.block_until_ready = lambda x: x
    register_lumen(ref_src)
    from lumen import api

    api._placement_report = lambda r: r  # the placement check imports the device runtime
    return api
