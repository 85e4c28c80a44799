"""Photon sources: emission rows drawn on the device from each photon's own key.

Mirrors ``lumen.sources`` (src/lumen/sources/point.py:37 ``Point``, _base.py:312 ``photon_uniforms``, :318
``gaussian``): photon i of a run takes its uniforms from vertex 0 of ``fold_in(fold_in(key, SOURCE_STREAM), i)`` and a
point source draws an isotropic direction as a normalised Gaussian triple; a source stands for ``n_photons`` physical
photons shared by the run's samples (row weight n_photons / samples). Events: a source with several events (a batch)
assigns photon ids to events by contiguous ranges of uneven sizes (``counts``), every photon tallied into its event.

- ``Point(position, n_photons, lam | lam_range, time)``: isotropic points, one per event.
- ``Tracks(start, direction, length, cone_angle, ...)``: straight tracks emitting on a cone of fixed half-angle about
  their direction (a Cherenkov-like source; linear polarisation in the plane of track and photon, polar.py:89).
- ``Scintillation(position, tau=(tau1, tau2), fraction)``: isotropic points with a two-exponential time profile.
- ``CherenkovSegment(material, start, direction, length, beta, charge, time)``: the Frank-Tamm light of charged
  segments (src/lumen/sources/cherenkov.py:65), one event per segment, on the medium's live RINDEX.
- ``ScintillationPoint(material, position, energy, time)`` / ``ScintillationSegment(material, start, end, t_start,
  t_end, energy, birks)``: a material's scintillation light (src/lumen/sources/scintillation.py:172, :182), one event
  per deposit: its components, spectra, decay and rise times and yield from the detector's tables.
- ``FromArrays(x, d, t, lam, w, pol)``: explicit rows (src/lumen/sources/arrays.py:24).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from lumen_b200 import _abi as A


def _events(v, n_ev, width):
    a = np.asarray(v, np.float32)
    return np.broadcast_to(a, (n_ev, width)) if a.ndim <= 1 else a


@dataclass
class Source:
    """Base: ``arrays()`` gives the LumenSource layout (kind, per-event records, event ranges and row weights)."""

    def events(self) -> int:
        return 1

    def counts(self, samples: int) -> np.ndarray:
        """Return the photons of each event in a run of ``samples`` photons."""
        return np.asarray([samples], np.int64)


@dataclass
class Point(Source):
    """Isotropic points (src/lumen/sources/point.py:37): ``position`` (3,) or (E, 3) m, one event each."""

    position: object
    n_photons: object = 1.0
    lam: float | None = None
    lam_range: tuple | None = None
    time: object = 0.0
    counts_: object = None

    def events(self):
        p = np.asarray(self.position, np.float32)
        return 1 if p.ndim == 1 else len(p)

    def counts(self, samples):
        if self.counts_ is not None:
            return np.asarray(self.counts_, np.int64)
        e = self.events()
        base = np.full(e, samples // e, np.int64)
        base[: samples - base.sum()] += 1
        return base

    def arrays(self, samples, det=None):
        e = self.events()
        pos = _events(self.position, e, 3)
        ev_f = np.zeros((e, A.EV_F), np.float32)
        ev_f[:, 0:3] = pos
        ev_f[:, 3] = np.broadcast_to(np.asarray(self.time, np.float32), (e,))
        cnt = self.counts(samples)
        return _common(self, A.SRC_POINT, ev_f, cnt, self.n_photons)


@dataclass
class Tracks(Source):
    """Straight tracks emitting on a cone about their direction, one event per track."""

    start: object
    direction: object
    length: object
    cone_angle: float = math.radians(42.0)
    n_photons: object = 1.0
    lam: float | None = None
    lam_range: tuple | None = None
    time: object = 0.0
    counts_: object = None

    def events(self):
        return len(np.asarray(self.start, np.float32).reshape(-1, 3))

    def counts(self, samples):
        if self.counts_ is not None:
            return np.asarray(self.counts_, np.int64)
        e = self.events()
        base = np.full(e, samples // e, np.int64)
        base[: samples - base.sum()] += 1
        return base

    def arrays(self, samples, det=None):
        e = self.events()
        ev_f = np.zeros((e, A.EV_F), np.float32)
        ev_f[:, 0:3] = _events(self.start, e, 3)
        u = np.asarray(_events(self.direction, e, 3), np.float64)
        ev_f[:, 3:6] = u / np.linalg.norm(u, axis=1, keepdims=True)
        ev_f[:, 6] = np.broadcast_to(np.asarray(self.length, np.float32), (e,))
        ev_f[:, 7] = np.broadcast_to(np.asarray(self.time, np.float32), (e,))
        out = _common(self, A.SRC_TRACK, ev_f, self.counts(samples), self.n_photons)
        out["cone_cos"] = float(np.float32(math.cos(self.cone_angle)))
        return out


@dataclass
class Scintillation(Source):
    """Isotropic scintillation points with a two-exponential time profile, one event per point."""

    position: object
    tau: tuple = (6.0, 1500.0)
    fraction: float = 0.25
    n_photons: object = 1.0
    lam: float | None = None
    lam_range: tuple | None = None
    time: object = 0.0
    counts_: object = None

    def events(self):
        return len(np.asarray(self.position, np.float32).reshape(-1, 3))

    def counts(self, samples):
        if self.counts_ is not None:
            return np.asarray(self.counts_, np.int64)
        e = self.events()
        base = np.full(e, samples // e, np.int64)
        base[: samples - base.sum()] += 1
        return base

    def arrays(self, samples, det=None):
        e = self.events()
        ev_f = np.zeros((e, A.EV_F), np.float32)
        ev_f[:, 0:3] = _events(self.position, e, 3)
        ev_f[:, 3] = np.broadcast_to(np.asarray(self.time, np.float32), (e,))
        out = _common(self, A.SRC_SCINT, ev_f, self.counts(samples), self.n_photons)
        out.update(tau1=float(self.tau[0]), tau2=float(self.tau[1]), frac1=float(self.fraction))
        return out


HC = 1239.84198433200208  # eV nm (src/lumen/units.py:20)


@dataclass
class CherenkovSegment(Source):
    """A charge ``charge`` (e) from ``start`` (m) along the unit ``direction`` for ``length`` m at ``beta`` in
    ``material``, at ``time`` ns at the start (src/lumen/sources/cherenkov.py:65): cos theta = 1 / (beta n(lam)), the
    wavelength ~ 1 / lam^2 over the span of the medium's RINDEX table, the weight Frank-Tamm's photons per sample
    2 pi alpha z^2 L (1 - 1 / (beta n)^2)_+ (1 / lam_min - 1 / lam_max) / samples, Geant4's polarisation. Several
    segments (rows of start, direction, length, beta, charge, time): one event each."""  # noqa: D205

    material: str
    start: object = (0.0, 0.0, 0.0)
    direction: object = (0.0, 0.0, 1.0)
    length: object = 1.0
    beta: object = 1.0
    charge: object = 1.0
    time: object = 0.0
    counts_: object = None

    def events(self):
        return len(np.asarray(self.start, np.float32).reshape(-1, 3))

    def counts(self, samples):
        if self.counts_ is not None:
            return np.asarray(self.counts_, np.int64)
        e = self.events()
        base = np.full(e, samples // e, np.int64)
        base[: samples - base.sum()] += 1
        return base

    def arrays(self, samples, det=None):
        if det is None:
            raise ValueError("CherenkovSegment: the detector holds its medium's RINDEX (pass det)")
        name = f"media/{self.material}/index"
        if name not in det.params_index:
            raise ValueError(f"CherenkovSegment: no medium {self.material!r} with an index in the detector")
        tab = det.params_index[name]
        off, k = (int(v) for v in det.arrays["tab"][tab])
        e = np.asarray(det.pool[off:off + k], np.float32)  # the table's knots (energies, eV)
        lam0, lam1 = np.float32(HC) / e.max(), np.float32(HC) / e.min()  # cherenkov.py:56 bounds
        n_ev = self.events()
        cnt = self.counts(samples)
        ev_f = np.zeros((n_ev, A.EV_F), np.float32)
        ev_f[:, 0:3] = _events(self.start, n_ev, 3)
        u = np.asarray(_events(self.direction, n_ev, 3), np.float64)
        ev_f[:, 3:6] = u / np.linalg.norm(u, axis=1, keepdims=True)
        for col, v in ((6, self.length), (7, self.time), (8, self.beta), (9, self.charge)):
            ev_f[:, col] = np.broadcast_to(np.asarray(v, np.float32), (n_ev,))
        ev_f[:, 10] = cnt.astype(np.float32)  # the event's samples (the weight's divisor)
        first = np.zeros(n_ev + 1, np.int64)
        first[1:] = np.cumsum(cnt)
        return dict(kind=A.SRC_CHERENKOV, ev_f=ev_f, ev_first=first, ev_w=np.ones(n_ev, np.float32),
                    lam0=float(lam0), lam1=float(lam1), cone_cos=1.0, tau1=0.0, tau2=0.0, frac1=0.0, rindex_tab=tab)  # fmt: skip


def _scint_mat(det, material):
    """The LumenSource.mat words of a material's scintillation tables in the detector."""
    pi = det.params_index
    m = f"media/{material}/"
    if m + "scint_yield" not in pi:
        raise ValueError(f"{material}: no scintillation (SCINTILLATIONYIELD and its components) in the detector")
    n = sum(1 for i in (1, 2, 3) if f"{m}scint_spectrum{i}" in pi)
    words = np.full(A.SM_WORDS, -1, np.int32)
    rises = all(f"{m}scint_rise{i}" in pi for i in range(1, n + 1))
    words[A.SM_N], words[A.SM_SEGMENT], words[A.SM_RISES], words[A.SM_YIELD] = n, 0, int(rises), pi[m + "scint_yield"]
    for i in range(n):
        words[A.SM_SPEC + i] = pi[f"{m}scint_spectrum{i + 1}"]
        words[A.SM_TAU + i] = pi[f"{m}scint_tau{i + 1}"]
        if rises:
            words[A.SM_RISE + i] = pi[f"{m}scint_rise{i + 1}"]
    for i in range(3):
        words[A.SM_SHARE + i] = pi.get(f"{m}scint_share{i + 1}", -1)
    return words


@dataclass
class ScintillationPoint(Source):
    """``energy`` (MeV) deposited at ``position`` (m) at ``time`` (ns) in ``material`` (src/lumen/sources/
    scintillation.py:172): its light's photons are the yield times the energy; rows of position, energy and time are
    one event each."""  # noqa: D205

    material: str
    position: object = (0.0, 0.0, 0.0)
    energy: object = 1.0
    time: object = 0.0
    counts_: object = None
    SEGMENT = False

    def events(self):
        return len(np.asarray(self.position, np.float32).reshape(-1, 3))

    def counts(self, samples):
        if self.counts_ is not None:
            return np.asarray(self.counts_, np.int64)
        e = self.events()
        base = np.full(e, samples // e, np.int64)
        base[: samples - base.sum()] += 1
        return base

    def _ev(self, n_ev):
        ev_f = np.zeros((n_ev, A.EV_F), np.float32)
        ev_f[:, 0:3] = _events(self.position, n_ev, 3)
        ev_f[:, 3] = np.broadcast_to(np.asarray(self.time, np.float32), (n_ev,))
        ev_f[:, 8] = np.broadcast_to(np.asarray(self.energy, np.float32), (n_ev,))
        return ev_f

    def arrays(self, samples, det=None):
        if det is None:
            raise ValueError("a scintillation source reads its material's tables from the detector (pass det)")
        n_ev = self.events()
        cnt = self.counts(samples)
        ev_f = self._ev(n_ev)
        ev_f[:, 10] = cnt.astype(np.float32)  # the event's samples (the weight's divisor)
        mat = _scint_mat(det, self.material)
        mat[A.SM_SEGMENT] = int(self.SEGMENT)
        first = np.zeros(n_ev + 1, np.int64)
        first[1:] = np.cumsum(cnt)
        return dict(kind=A.SRC_SCINT_MATERIAL, ev_f=ev_f, ev_first=first, ev_w=np.ones(n_ev, np.float32), lam0=0.0,
                    lam1=0.0, cone_cos=1.0, tau1=0.0, tau2=0.0, frac1=0.0, mat=mat)  # fmt: skip


@dataclass
class ScintillationSegment(ScintillationPoint):
    """A charged step from ``start`` (at ``t_start`` ns) to ``end`` (``t_end``) depositing ``energy`` MeV, quenched by
    Birks' law with ``birks`` (m / MeV) (src/lumen/sources/scintillation.py:182); photons uniform along it."""  # noqa: D205

    start: object = (0.0, 0.0, 0.0)
    end: object = (0.0, 0.0, 0.0)
    t_start: object = 0.0
    t_end: object = 0.0
    birks: object = 0.0
    SEGMENT = True

    def events(self):
        return len(np.asarray(self.start, np.float32).reshape(-1, 3))

    def _ev(self, n_ev):
        ev_f = np.zeros((n_ev, A.EV_F), np.float32)
        ev_f[:, 0:3] = _events(self.start, n_ev, 3)
        ev_f[:, 3] = np.broadcast_to(np.asarray(self.t_start, np.float32), (n_ev,))
        ev_f[:, 4:7] = _events(self.end, n_ev, 3)
        ev_f[:, 7] = np.broadcast_to(np.asarray(self.t_end, np.float32), (n_ev,))
        ev_f[:, 8] = np.broadcast_to(np.asarray(self.energy, np.float32), (n_ev,))
        ev_f[:, 9] = np.broadcast_to(np.asarray(self.birks, np.float32), (n_ev,))
        return ev_f


def _common(src, kind, ev_f, cnt, n_photons):
    e = len(cnt)
    first = np.zeros(e + 1, np.int64)
    first[1:] = np.cumsum(cnt)
    nph = np.broadcast_to(np.asarray(n_photons, np.float64), (e,))
    ev_w = np.where(cnt > 0, nph / np.maximum(cnt, 1), 0.0).astype(np.float32)
    if src.lam is not None:
        lam0, lam1 = float(src.lam), 0.0
    elif src.lam_range is not None:
        lam0, lam1 = float(src.lam_range[0]), float(src.lam_range[1])
    else:
        raise ValueError("a source needs lam or lam_range")
    return dict(kind=kind, ev_f=ev_f, ev_first=first, ev_w=ev_w, lam0=lam0, lam1=lam1, cone_cos=1.0, tau1=0.0,
                tau2=0.0, frac1=0.0)  # fmt: skip


@dataclass
class FromArrays(Source):
    """Explicit emission rows (src/lumen/sources/arrays.py:24): x (n, 3), d (n, 3), t, lam, w (n,), pol (n, 2, 3)."""

    x: object
    d: object
    t: object = 0.0
    lam: object = 400.0
    w: object = 1.0
    pol: object = None
    event: object = None

    def rows(self):
        x = np.asarray(self.x, np.float32).reshape(-1, 3)
        n = len(x)
        d = np.asarray(self.d, np.float32).reshape(-1, 3)
        return dict(x=x, d=d, t=np.broadcast_to(np.float32(self.t), (n,)).copy(),
                    lam=np.broadcast_to(np.asarray(self.lam, np.float32), (n,)).copy(),
                    w=np.broadcast_to(np.asarray(self.w, np.float32), (n,)).copy(),
                    pol=None if self.pol is None else np.asarray(self.pol, np.float32).reshape(-1, 6),
                    event=None if self.event is None else np.asarray(self.event, np.int32))  # fmt: skip

    def events(self):
        return 1 if self.event is None else int(np.max(self.event)) + 1
