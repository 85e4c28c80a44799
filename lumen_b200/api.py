"""The public call: ``simulate(det, source, params, *, samples, seed, ...) -> Light``, lumen's signature.

Mirrors ``lumen.simulate`` (src/lumen/api.py:876) and its outputs ``Light`` (:515) and ``Health`` (:445): per sensor
the expected photon arrivals, their Monte Carlo error from the per-photon second moment
(src/lumen/readout/grid.py:48 ``moment_error``), the mean arrival time, optional 1 ns (or any width) arrival-time
histograms, the health fates, and, when asked, the arrivals' derivatives in named parameters. Photon i of a run is
keyed ``fold_in(PRNGKey(seed), i)`` (src/lumen/run.py:309), so a run is the same whatever its chunking. ``params``
are the run's live values, ``reference`` the values every draw is made at (src/lumen/transport/estimator.py): with a
reference held, runs at nearby values share their random numbers (common random numbers for finite differences).
"""

from __future__ import annotations

import hashlib
import math
import warnings
from dataclasses import dataclass, field

import numpy as np
import torch

from lumen_b200 import _abi as A
from lumen_b200 import readout as RO
from lumen_b200 import truth as TR
from lumen_b200.engine import DeviceRows, DeviceSource, DeviceTallies, Engine
from lumen_b200.sources import FromArrays

MAX_ID = 2**31 - 1  # photon ids are int32 (src/lumen/_core/rng.py:23)


@dataclass
class Health:
    """What no sensor counted (src/lumen/api.py:445): the fates every start weight ends in, and the counts."""

    lost: float
    abandoned: float
    escaped: float
    distance_cut: float
    truncated: float
    absorbed_bulk: float
    absorbed_surface: float
    rouletted: float
    reweighted: float
    pushed: float
    records: int
    photons: int
    steps: int
    start: float
    records_dropped: int = 0
    records_mismatch: int = 0
    nonfinite: int = 0
    invalid: int = 0

    FATES = ("absorbed_bulk", "absorbed_surface", "lost", "escaped", "distance_cut", "abandoned", "truncated",
             "rouletted", "reweighted")  # fmt: skip

    def balance(self, start=None) -> float:
        """Return the start weight minus every fate: 0 to float32 rounding per step at the reference values."""
        s = self.start if start is None else start
        return float(s) - sum(float(getattr(self, k)) for k in self.FATES)


@dataclass
class Light:
    """What ``simulate`` returns (src/lumen/api.py:515); with several events every array has a leading event axis."""

    arrivals: np.ndarray
    arrivals_error: np.ndarray
    mean_arrival_time: np.ndarray
    health: Health
    provenance: dict = field(default_factory=dict)
    groups: dict | None = None  # {readout group: lumen_b200.readout.Histograms} (the run's ``groups``)
    gradients: dict | None = None  # {parameter: d arrivals / d value}
    diagnostics: dict | None = None  # "time" (.., S, bins) arrival-time histograms and "time_edges" (``time_bins``)
    truth: object = None

    @property
    def events(self) -> int:
        return self.arrivals.shape[0] if self.arrivals.ndim == 2 else 0


def moment_error(x2, x, n):
    """Return sqrt(n / (n - 1) (sum x^2 - (sum x)^2 / n)): the standard error of a sum of n i.i.d. photons
    (src/lumen/readout/grid.py:48)."""  # noqa: D205, D209
    n = np.asarray(n, np.float64)
    v = np.maximum(np.asarray(x2) - np.asarray(x) ** 2 / np.maximum(n, 1.0), 0.0)
    return np.sqrt(n / np.maximum(n - 1.0, 1.0) * v)


def _check_values(det, pool, what):
    """``Detector.check_values``, once per detector and pool values (a run repeated at the same values checks once:
    the digests of the values found admissible are kept on the detector)."""  # noqa: D205, D209
    key = hashlib.blake2b(np.ascontiguousarray(pool).tobytes(), digest_size=16).digest()
    seen = det.__dict__.setdefault("_admissible", set())
    if key not in seen:
        det.check_values(pool, what)
        seen.add(key)


def _engine(det, device=None) -> Engine:
    cache = det.__dict__.setdefault("_engines", {})
    dev = torch.device(device if device is not None else "cuda", torch.cuda.current_device()) if device is None \
        else torch.device(device)  # fmt: skip
    if dev not in cache:
        cache[dev] = Engine(det, dev)
    return cache[dev]


def simulate(det, source, params=None, *, samples=None, seed=0, reference=None, controls=None, chunk=None,
             gradients=(), time_bins=None, groups=None, records=None, truth=None, device=None, stream=None) -> Light:
    """Return the Light of ``samples`` photons of ``source`` in detector ``det`` (lumen.simulate's signature).

    ``params``: {parameter name: value} overriding the detector's values (``det.params()``); ``reference``: the
    values the draws are made at (default: ``params``). ``controls``: ``dict(roulette=0.01, max_distance=None,
    max_vertices=2**22, variant=None, jump=True)``; ``jump`` the diffusion jump (on, as lumen.simulate's default: where a
    medium and volume allow it; the same estimator in law as the plain walk); ``variant`` picks the launch
    (``LumenControls.variant``; default: the wavefront, measured the faster on the tank and LAr workloads, forward and
    with tangents; scenes it does not serve run the persistent loop). ``chunk``: photons per launch (default: all in one launch). ``gradients``: parameter names
    whose derivatives of the arrivals are returned (forward tangents of the reweighting estimator along each path).
    ``time_bins``: (bins, t0, width) ns of the per-sensor arrival-time histograms (``Light.diagnostics``).
    ``groups``: the readout groups' histograms to fill ({name: lumen_b200.readout.Grid or Group}: a Grid's sensors
    are the detector's group of that name, else every sensor) into ``Light.groups`` (src/lumen/readout/grid.py
    Histograms); ``records``: the deposit records one launch may keep for them (default 2 per photon, at least 2^16;
    a launch that outgrows it is re-run with room for what it needed, as the reference's RecordsOverflow retry).
    ``truth``: a ``lumen_b200.truth.Truth``: the run's truth rows in ``Light.truth`` (``TruthHits``: each photon's
    analog record thinned by detection at the groups' efficiency and acceptance). Not differentiable; at one set of
    values (no ``reference``); each source row at most one photon (samples >= the photons emitted).
    """
    live = det.pool_with(params)
    ref = None if reference is None else det.pool_with({**(params or {}), **reference})
    _check_values(det, live, "simulate")  # a concrete value outside its range is refused (build/values.py:203)
    if ref is not None:
        _check_values(det, ref, "simulate: reference")
    eng = _engine(det, device)
    eng.set_pools(live, ref)
    ctl = dict(roulette=0.01, max_distance=0.0, max_vertices=1 << 22, variant=None, jump=True) | (controls or {})
    gnames = list(gradients)
    gt = [det.params_index[k] for k in gnames]
    variant = ctl["variant"] if ctl["variant"] is not None else A.VARIANT_WAVEFRONT
    flags = A.F_JUMP if ctl["jump"] else 0  # the diffusion jump on, as lumen.simulate (src/lumen/api.py:1157)
    if truth is not None:  # src/lumen/api.py:1296 _truth_setup
        if not isinstance(truth, TR.Truth):
            raise ValueError(f"simulate: truth is a lumen_b200.truth.Truth, got {truth!r}")
        if gt:
            raise ValueError("simulate: truth rows are not differentiable; take the derivative of a run without truth=")
        if reference is not None:
            raise ValueError("simulate: truth rows decide each photon's fate at the run's own values; leave reference out")
        if not ctl["roulette"] <= 1.0:
            raise ValueError("simulate: with truth rows the roulette must be <= 1")
        flags |= A.F_TRUTH
    c = A.controls(ctl["max_distance"] or 0.0, ctl["roulette"], ctl["max_vertices"], gt, variant=variant, flags=flags)
    if isinstance(source, FromArrays):
        rows = source.rows()
        n = len(rows["x"])
        dsrc, drows, n_ev = None, DeviceRows(rows, eng.device), source.events()
        total = n
    else:
        if samples is None:
            raise ValueError("simulate: give samples")
        n = int(samples)
        dsrc, drows, n_ev = DeviceSource(source, n, eng.device, det), None, source.events()
        total = dsrc.total
    if total > MAX_ID:
        raise ValueError(f"a run traces at most {MAX_ID} photons (int32 ids)")
    if truth is not None:
        if isinstance(source, FromArrays):
            TR.check_weights(drows.w.cpu().numpy() if hasattr(drows, "w") else source.rows()["w"])
        elif dsrc.c.kind in (A.SRC_CHERENKOV, A.SRC_SCINT_MATERIAL):
            raise ValueError("simulate: truth rows need row weights known before the run (<= 1 photon each); a "
                             "Cherenkov or material scintillation source weighs its rows on the device")
        else:
            TR.check_weights(source.arrays(n, det)["ev_w"])
    nb, t0, tw = (0, 0.0, 1.0) if time_bins is None else time_bins
    T = DeviceTallies(det.n_sensor, n_ev, nb, t0, tw, len(gt), eng.device)
    G = None
    step = int(chunk) if chunk else total
    if groups:
        G = RO.GroupCells(det, groups, n_ev, eng.device)
        T.attach_groups(G, int(records) if records else max(1 << 16, 2 * min(step, total)))
    key = A.key_of_seed(seed)
    hits = None
    for _attempt in range(4):
        try:
            hits = []
            for first in range(0, total, max(step, 1)):
                m = min(step, total - first)
                if drows is not None and first > 0:
                    raise ValueError("explicit rows run in one launch")
                before = int(T.counts[A.C_RECORDS].item()) if G is not None else 0
                if truth is not None:
                    T.attach_truth(m)
                eng.trace(key, m, source=dsrc, rows=drows, first_id=first, controls=c, tallies=T, stream=stream)
                if truth is not None:
                    hits.append(TR.rows(truth, det, T.truth.cpu().numpy()[:m], key, first,
                                        _labels(source, dsrc, first, m, n_ev),
                                        dict(zip(G.names, G.groups)) if G is not None else None))  # fmt: skip
            break
        except A.RecordsOverflow:  # the launch's records outgrew the scratch: every tally again with room for them
            need = int(T.counts[A.C_RECORDS].item()) - before
            T.zero_()
            T.attach_groups(G, need + need // 4 + 1024)
    else:
        raise A.RecordsOverflow(A.ERR_RECORDS, "the deposit records kept outgrowing the scratch")
    light = _light(det, T, n_ev, total, seed, gnames, (nb, t0, tw), source, G)
    if truth is not None:
        light.truth = TR.join(hits, total)
    return light


def _labels(source, dsrc, first, m, n_ev):
    """The events of photons first .. first + m - 1 (None with one event: label -1)."""
    if n_ev <= 1:
        return None
    ids = first + np.arange(m)
    if isinstance(source, FromArrays):
        return np.asarray(source.event, np.int32)[ids]
    ev_first = dsrc.ev_first.cpu().numpy()
    return (np.searchsorted(ev_first, ids, side="right") - 1).astype(np.int32)


def _host_tallies(T):
    """The tallies on the host in one device-to-host copy: {name: array} of the FP64 tallies, "counts" and
    "nonfinite" (the output cells that are not finite, counted on the device)."""  # noqa: D205, D209
    names = [k for k in ("arrival", "arrival_t", "arrival2", "hist", "jac", "health") if getattr(T, k) is not None]
    cells = [getattr(T, k) for k in ("arrival", "arrival_t", "arrival2", "hist", "jac") if getattr(T, k) is not None]
    nonfinite = sum((~torch.isfinite(c)).sum() for c in cells).to(torch.float64).reshape(1)
    dev = torch.cat([getattr(T, k).reshape(-1) for k in names] + [nonfinite, T.counts.view(torch.float64)])
    if dev.is_cuda:  # into page-locked memory (torch's caching host allocator keeps it for the next call)
        flat = torch.empty(dev.shape, dtype=dev.dtype, pin_memory=True)
        flat.copy_(dev)
    else:
        flat = dev
    out, o = {}, 0
    for k in names:
        t = getattr(T, k)
        out[k] = flat[o:o + t.numel()].numpy().reshape(tuple(t.shape))
        o += t.numel()
    out["nonfinite"] = int(flat[o].item())
    out["counts"] = flat[o + 1:].numpy().view(np.int64)
    return out


def _light(det, T, n_ev, samples, seed, gnames, bins, source, G=None):
    host = _host_tallies(T)
    arr, arr_t, arr2 = host["arrival"], host["arrival_t"], host["arrival2"]
    h = host["health"]
    cnt = host["counts"]
    if n_ev > 1:
        per_ev = np.diff(source.arrays(samples, det)["ev_first"]) if not isinstance(source, FromArrays) else \
            np.bincount(np.asarray(source.event), minlength=n_ev)  # fmt: skip
        nn = per_ev[:, None].astype(np.float64)
    else:
        arr, arr_t, arr2 = arr[0], arr_t[0], arr2[0]
        nn = float(samples)
    err = moment_error(arr2, arr, nn)
    with np.errstate(invalid="ignore", divide="ignore"):
        mt = np.where(arr > 0, arr_t / np.where(arr > 0, arr, 1.0), np.nan)
    # the output cells that are not finite (the reference's exact-sum cells that are NaN, src/lumen/api.py:469)
    nonfinite = host["nonfinite"]
    health = Health(lost=h[0], abandoned=h[1], escaped=h[2], distance_cut=h[3], absorbed_bulk=h[4],
                    absorbed_surface=h[5], rouletted=h[6], reweighted=h[7], truncated=h[8], pushed=h[9],
                    start=h[10], records=int(cnt[2]), photons=int(cnt[0]), steps=int(cnt[1]),
                    nonfinite=nonfinite)  # fmt: skip
    diag = None
    if bins[0]:
        hist = host["hist"]
        diag = {"time": hist if n_ev > 1 else hist[0], "time_edges": bins[1] + bins[2] * np.arange(bins[0] + 1)}
    groups = G.histograms(nn) if G is not None else None
    grads = None
    if gnames:
        jac = host["jac"]
        grads = {k: (jac[..., i] if n_ev > 1 else jac[0, :, i]) for i, k in enumerate(gnames)}
    prov = dict(seed=seed, samples=samples, engine="lumen_b200", steps_per_photon=cnt[1] / max(cnt[0], 1),
                moment_table_sums=int(cnt[A.C_MULTI]))  # fmt: skip
    if cnt[A.C_MOMENT_LOST]:  # sums that found the moment table full were squared alone: the errors are not exact
        warnings.warn(f"simulate: {int(cnt[A.C_MOMENT_LOST])} per-photon sensor sums found the moment table full; "
                      "arrivals_error is approximate (run fewer photons per launch: chunk=)", RuntimeWarning,
                      stacklevel=3)  # fmt: skip
        prov["moment_lost"] = int(cnt[A.C_MOMENT_LOST])
    return Light(arr, err, mt, health, prov, groups, grads, diag)


def pe(light: Light, values=None, *, qe=None, efficiency=1.0, lam=None):
    """Return expected photoelectrons per sensor (src/lumen/readout/detection.py:91 ``pe``).

    With readout groups: ``values`` = {group: {"tables": [(axis names, values over those axes' cells), ...] (the sensor
    model's acceptance tables, e.g. the QE on the wavelength knots), "efficiency": scalar or per sensor}}; each
    group's charge histogram contracted with its tables, times the efficiency, at its sensors (0 at a sensor of no
    group). Without: efficiency x QE(lam) x arrivals for a source of one wavelength ``lam`` (nm); ``qe`` =
    (wavelengths nm, values).
    """
    if values is not None:
        out = np.zeros(light.arrivals.shape, np.float64)
        for name, h in (light.groups or {}).items():
            v = values.get(name)
            if v is None:
                continue
            acc = RO.tables_acceptance(h.grid, v.get("tables", ()))
            ids = np.arange(out.shape[-1]) if h.sensors is None else np.asarray(h.sensors, np.int64)
            out[..., ids] = RO.expected_pe(h, acc, v.get("efficiency", 1.0))
        return out
    q = 1.0 if qe is None else float(np.interp(lam, np.asarray(qe[0], float), np.asarray(qe[1], float)))
    return np.asarray(efficiency) * q * light.arrivals


def pe_error(light: Light):
    """Return each sensor's pe Monte Carlo error at the groups' acceptance the run was given (``Group.weights`` and
    ``efficiency``; src/lumen/readout/detection.py:106 ``pe_error``); 0 at a sensor of no such group."""  # noqa: D205, D209
    out = np.zeros(light.arrivals.shape, np.float64)
    for h in (light.groups or {}).values():
        if h.pe_error is None:
            continue
        ids = np.arange(out.shape[-1]) if h.sensors is None else np.asarray(h.sensors, np.int64)
        out[..., ids] = h.pe_error
    return out


def seed_key(seed: int):
    """Return the run key of a seed: jax.random.PRNGKey(seed)'s key data."""
    return A.key_of_seed(seed)


def ceil_pow2(n: int) -> int:
    return 1 << max(int(math.ceil(math.log2(max(n, 1)))), 0)
