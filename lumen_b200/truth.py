"""Truth rows: the analog (Geant4-like) record of a run, one row per absorbed or detected photon (lumen.readout.truth).

Each traced photon carries one analog photon (src/lumen/transport/state.py:30 Analog): open with probability k (its
row's physical photons, <= 1) from one uniform of its own stream, absorbed on a cathode at most once, at the crossing
where its place in the weight falls in the crossing's reached share (src/lumen/transport/step.py:625), and kept by the
roulette while its fate is open (step.py:649), so the record is exact and the expected values are unchanged in law.
The engine writes each photon's record (LUMEN_F_TRUTH); here, as src/lumen/readout/truth.py:150 does, the absorbed
photons are thinned by detection: a second uniform of the photon's own (its key folded with DETECT_STREAM) against
the sensor's detection probability (the group's efficiency times its acceptance read at the deposit's features, as
the binned readout reads it; 1 on a sensor of no modelled group) times the row's 1 / A_n.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from lumen_b200 import _abi as A

DETECT_STREAM = 0x7A4A1062  # the photon key's fold of its detection uniform (src/lumen/_core/rng.py:24)
KEEPS = ("detected", "absorbed")
_ROT = (13, 15, 26, 6, 17, 29, 16, 24)


def _rotl(x, r):
    return ((x << np.uint32(r)) | (x >> np.uint32(32 - r))).astype(np.uint32)


def threefry(k0, k1, x0, x1):
    """Threefry2x32-20 (Salmon et al., SC'11) of counters (x0, x1) under keys (k0, k1), elementwise on uint32 arrays."""
    k0, k1, x0, x1 = (np.asarray(v, np.uint32) for v in (k0, k1, x0, x1))
    with np.errstate(over="ignore"):
        ks = (k0, k1, k0 ^ k1 ^ np.uint32(0x1BD11BDA))
        a, b = (x0 + ks[0]).astype(np.uint32), (x1 + ks[1]).astype(np.uint32)
        for i in range(5):
            for r in _ROT[(i % 2) * 4:(i % 2) * 4 + 4]:
                a = (a + b).astype(np.uint32)
                b = _rotl(b, r) ^ a
            a = (a + ks[(i + 1) % 3]).astype(np.uint32)
            b = (b + ks[(i + 2) % 3] + np.uint32(i + 1)).astype(np.uint32)
    return a, b


def fold_in(key, d):
    """JAX's fold_in of a key pair by data d (elementwise)."""
    return threefry(key[0], key[1], np.zeros_like(np.asarray(d, np.uint32)), d)


def uniform(key, i=0):
    """The i-th uniform in (0, 1) of a key pair: 23 bits of the partitionable block, centred."""
    y0, y1 = threefry(key[0], key[1], 0, i)
    return (((y0 ^ y1) >> np.uint32(9)).astype(np.float32) + np.float32(0.5)) * np.float32(1.1920928955078125e-7)


@dataclass(frozen=True)
class Truth:
    """What truth rows a run keeps (src/lumen/readout/truth.py:46): ``keep`` "detected" or "absorbed" (every cathode
    absorption, with its ``detected`` flag); ``angle``, ``position``: the hit angle and hit point columns."""  # noqa: D205, D209

    keep: str = "detected"
    angle: bool = False
    position: bool = False

    def __post_init__(self):
        if self.keep not in KEEPS:
            raise ValueError(f"Truth: keep is one of {KEEPS}, got {self.keep!r}")


@dataclass
class TruthHits:
    """The truth rows of a run, one per photon, in photon order (src/lumen/readout/truth.py:57): ``photon`` its id,
    ``label`` its event (-1 with one), ``sensor``, ``time`` (ns, at the cathode), ``detected``; ``angle`` (rad, the
    cathode position angle) and ``position`` ((n, 3) m, in the sensor placement's frame) when asked for."""  # noqa: D205, D209

    photon: np.ndarray
    label: np.ndarray
    sensor: np.ndarray
    time: np.ndarray
    detected: np.ndarray
    angle: np.ndarray | None = None
    position: np.ndarray | None = None
    n_photons: int = 0

    def select(self, mask) -> TruthHits:
        pick = lambda v: None if v is None else v[mask]  # noqa: E731
        return TruthHits(self.photon[mask], self.label[mask], self.sensor[mask], self.time[mask], self.detected[mask],
                         pick(self.angle), pick(self.position), self.n_photons)  # fmt: skip

    def sum_by(self, keys=("label", "sensor"), *, detected: bool = True) -> dict:
        """Return per distinct key the rows ``n`` and the first time ``t_first`` (sorted by the keys)."""
        hits = self.select(self.detected) if detected else self
        cols = [np.asarray(getattr(hits, k), np.int64) for k in keys]
        if not len(hits.photon):
            return {k: np.zeros(0, np.int64) for k in keys} | {"n": np.zeros(0, np.int64), "t_first": np.zeros(0)}
        order = np.lexsort(cols[::-1])
        key = np.stack([c[order] for c in cols], 1)
        start = np.flatnonzero(np.r_[True, (key[1:] != key[:-1]).any(1)])
        t = np.asarray(hits.time, np.float64)[order]
        return {k: c[order][start] for k, c in zip(keys, cols)} | {"n": np.diff(np.r_[start, len(order)]),
                                                                     "t_first": np.minimum.reduceat(t, start)}


def _local(arrays, vol, pos):
    """The points pos (world) in the frames of the placements vol: R^T (x - t)."""
    vf = np.asarray(arrays["vol_f"], np.float64)[np.maximum(vol, 0)]
    R, t = vf[:, 0:9].reshape(-1, 3, 3), vf[:, 9:12]
    return np.einsum("nij,ni->nj", R, np.asarray(pos, np.float64) - t)


def _acceptance(group, lam, loc):
    """A group's efficiency times its acceptance at the records' features (hats on knots, cells between edges)."""
    gr = group.grid
    feats = {"wavelength": lam, "theta": np.arctan2(np.sqrt(loc[:, 0] ** 2 + loc[:, 1] ** 2 + 1e-30), loc[:, 2]),
             "x": loc[:, 0], "y": loc[:, 1], "z": loc[:, 2], "rho": np.hypot(loc[:, 0], loc[:, 1])}  # fmt: skip
    cells = [(np.zeros(len(lam), np.int64), np.ones(len(lam)))]
    for ax in gr.axes:
        if ax.feature not in feats:
            raise ValueError(f"truth rows: a detection read of {ax.feature!r} is not recorded by the analog photon")
        v, x = np.asarray(ax.values), feats[ax.feature]
        c = np.searchsorted(v, x, side="right")
        if ax.knots is not None:
            i = np.clip(c - 1, 0, len(v) - 2)
            f = np.clip((x - v[i]) / (v[i + 1] - v[i]), 0.0, 1.0)
            pieces = [(i, 1.0 - f), (i + 1, f)]
        else:
            b = c - 1
            pieces = [(np.where((b >= 0) & (b < len(v) - 1), b, -1), np.ones(len(x)))]
        cells = [(np.where((p >= 0) & (j >= 0), p * ax.size + j, -1), w * u) for p, w in cells for j, u in pieces]
    acc = np.zeros(len(lam))
    tab = np.asarray(group.weights, np.float64).ravel()
    for idx, w in cells:
        acc += np.where(idx >= 0, w * tab[np.maximum(idx, 0)], 0.0)
    return float(group.efficiency) * acc


def rows(spec: Truth, det, rec, key, first_id, labels, groups=None) -> TruthHits:
    """Return the TruthHits of one call's photon records ``rec`` ((n, LUMEN_TRUTH_WORDS) float32, photons first_id ..)
    thinned by detection; ``labels`` each photon's event (None: -1); ``groups`` the run's readout groups ({name:
    lumen_b200.readout.Group}) whose efficiency and acceptance the detection reads."""  # noqa: D205, D209
    rec = np.asarray(rec, np.float32)
    sensor = rec[:, 0].view(np.int32)
    n = len(rec)
    ids = np.uint32(first_id) + np.arange(n, dtype=np.uint32)
    pk = fold_in(key, ids)
    u = uniform(fold_in(pk, np.full(n, DETECT_STREAM, np.uint32)), 0)
    absorbed = sensor >= 0
    lam, scale = rec[:, 2].astype(np.float64), rec[:, 3].astype(np.float64)
    vol = rec[:, 7].view(np.int32)
    loc = _local(det.arrays, vol, rec[:, 4:7])
    p = np.ones(n)
    for g in (groups or {}).values():
        if getattr(g, "weights", None) is None:
            continue
        sens = np.arange(det.n_sensor) if g.sensors is None else np.asarray(g.sensors, np.int64)
        mine = absorbed & np.isin(sensor, sens)
        if mine.any():
            p[mine] = _acceptance(g, lam[mine], loc[mine])
    detected = absorbed & (u < (p * scale).astype(np.float32))
    keep = detected if spec.keep == "detected" else absorbed
    idx = np.flatnonzero(keep)
    lab = np.full(n, -1, np.int32) if labels is None else np.asarray(labels, np.int32)
    out = TruthHits(photon=np.int64(first_id) + idx, label=lab[idx], sensor=sensor[idx].copy(),
                    time=rec[idx, 1].copy(), detected=detected[idx], n_photons=n)  # fmt: skip
    if spec.angle:
        out.angle = np.arctan2(np.sqrt(loc[idx, 0] ** 2 + loc[idx, 1] ** 2 + 1e-30), loc[idx, 2]).astype(np.float32)
    if spec.position:
        out.position = loc[idx].astype(np.float32)
    return out


def join(parts: list, n_photons: int) -> TruthHits:
    """Return the TruthHits of a run's calls, in photon order."""
    if not parts:
        return TruthHits(*(np.zeros(0, d) for d in (np.int64, np.int32, np.int32, np.float32, bool)), n_photons=n_photons)
    cat = lambda k: None if getattr(parts[0], k) is None else np.concatenate([getattr(p, k) for p in parts])  # noqa: E731
    return TruthHits(cat("photon"), cat("label"), cat("sensor"), cat("time"), cat("detected"), cat("angle"),
                     cat("position"), n_photons)  # fmt: skip


def check_weights(w, what="a source row"):
    """Refuse rows standing for more than one photon (a truth row is one photon: src/lumen/api.py:1287)."""
    top = float(np.max(w)) if np.size(w) else 0.0
    if top > 1.0 + 1e-6:
        raise ValueError(f"simulate: {what} stands for {top:.9g} photons; a truth row is one photon: run samples >= "
                         "the photons emitted")  # fmt: skip
    if not math.isfinite(top):
        raise ValueError("simulate: a non-finite row weight")
