"""The run as a ``torch.autograd.Function``: forward ``lumen_b200_trace``, backward ``lumen_b200_adjoint``.

The reference puts the whole run behind one derivative rule (src/lumen/api.py:748-787 ``_with_rule``, a
``jax.custom_jvp``): its value is ``runner.trace`` + ``rebuild`` (src/lumen/run.py:693, :534), its derivative the
tangent run of the same photons. Here the value is one trace launch, and the vector-Jacobian product is one adjoint
launch that replays the same photons from their counter-based keys (no stored path) and contracts every deposit's
tangent with the incoming cotangent. Both are at the run's values with every draw at the reference (the reweighting
estimator, src/lumen/transport/estimator.py): with the reference held, repeated calls trace the same photons.

A parameter is a table whose values move together (``Detector.pool_with``): its value here is the constant the table is
set to, and its derivative is that of the arrivals in it.

    values = torch.tensor([50.0, 0.1], dtype=torch.float64, requires_grad=True)
    arr = lumen_b200.autograd.simulate(det, src, values, ["media/Water/absorption", "surfaces/BlackSheet/R"],
                                       samples=2**20, seed=0)
    arr.sum().backward()       # values.grad: d(sum of arrivals) / d values, one adjoint launch
"""

from __future__ import annotations

import torch

from lumen_b200 import _abi as A
from lumen_b200.engine import DeviceRows, DeviceSource, DeviceTallies
from lumen_b200.sources import FromArrays


class Simulate(torch.autograd.Function):
    """``apply(values, det, source, names, samples, seed, reference, controls, device)`` -> arrivals (float64 on the
    device; (S,) for one event, (E, S) for several). ``values``: the parameters ``names``' values (a float64 tensor
    (P,)); ``reference``: {name: value} of the values the draws are made at (None: ``values``, as the reference's
    ``simulate(reference=None)``); ``controls``: as ``lumen_b200.simulate``'s (roulette, max_distance, max_vertices,
    variant, jump). Backward: d(cotangent . arrivals) / d values by the adjoint replay of the same photons."""  # noqa: D205

    @staticmethod
    def forward(ctx, values, det, source, names, samples, seed, reference=None, controls=None, device=None):
        from lumen_b200 import api

        names = list(names)
        if values.ndim != 1 or values.shape[0] != len(names):
            raise ValueError(f"Simulate: values ({tuple(values.shape)}) must hold one value per name ({len(names)})")
        if len(names) > A.MAX_GRAD:
            raise ValueError(f"Simulate: at most {A.MAX_GRAD} parameters per run")
        vals = {k: float(v) for k, v in zip(names, values.detach().cpu().tolist(), strict=True)}
        live = det.pool_with(vals)
        ref = None if reference is None else det.pool_with({**vals, **reference})
        det.check_values(live, "Simulate")
        if ref is not None:
            det.check_values(ref, "Simulate: reference")
        eng = api._engine(det, device)
        ctl = dict(roulette=0.01, max_distance=0.0, max_vertices=1 << 22, variant=0, jump=True) | (controls or {})
        ctl["flags"] = A.F_JUMP if ctl["jump"] else 0  # the diffusion jump, on as in lumen.simulate
        if isinstance(source, FromArrays):
            host = source.rows()
            src, rows, n_ev, n = None, DeviceRows(host, eng.device), source.events(), len(host["x"])
        else:
            src, rows, n_ev = DeviceSource(source, int(samples), eng.device, det), None, source.events()
            n = src.total
        key = A.key_of_seed(seed)
        c = A.controls(ctl["max_distance"] or 0.0, ctl["roulette"], ctl["max_vertices"], variant=ctl["variant"],
                       flags=ctl["flags"])  # fmt: skip
        eng.set_pools(live, ref)
        T = DeviceTallies(det.n_sensor, n_ev, 0, 0.0, 1.0, 0, eng.device)
        eng.trace(key, n, source=src, rows=rows, controls=c, tallies=T)
        ctx.run = (eng, det, names, live, ref, src, rows, n, key, ctl, n_ev)
        ctx.like = (values.device, values.dtype)
        out = T.arrival if n_ev > 1 else T.arrival[0]
        return out.clone()

    @staticmethod
    def backward(ctx, grad_out):
        eng, det, names, live, ref, src, rows, n, key, ctl, n_ev = ctx.run
        gt = [det.params_index[k] for k in names]
        # the adjoint's launch is the persistent loop (its replay needs no slots); the pools again, as another run on
        # this engine may have set its own since the forward
        c = A.controls(ctl["max_distance"] or 0.0, ctl["roulette"], ctl["max_vertices"], gt, variant=0, flags=ctl["flags"])
        eng.set_pools(live, ref)
        cot = grad_out.to(device=eng.device, dtype=torch.float64).reshape(max(n_ev, 1), -1).contiguous()
        g = eng.adjoint(key, n, cot, source=src, rows=rows, controls=c)
        return (g.to(*ctx.like), None, None, None, None, None, None, None, None)


def simulate(det, source, values, names, *, samples=None, seed=0, reference=None, controls=None, device=None):
    """Return the arrivals of ``samples`` photons of ``source`` at the parameters ``names`` set to ``values`` (a
    float64 tensor that may require grad): ``Simulate.apply`` (its docstring)."""  # noqa: D205
    if not torch.is_tensor(values):
        values = torch.as_tensor(values, dtype=torch.float64)
    return Simulate.apply(values, det, source, list(names), samples, seed, reference, controls, device)
