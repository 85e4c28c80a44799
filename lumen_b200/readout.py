"""The readout groups: histograms of the deposits per sensor group, filled during tracking (lumen.readout).

The reference bins its deposit records after tracking (src/lumen/readout/fill.py:88 ``readout``) into two histograms
per sensor group (src/lumen/readout/grid.py): ``charge`` (S, *axes) on features of the deposit (wavelength, the
cathode angle, the incidence, ...: src/lumen/sensors/features.py) with its per-photon second moment ``charge2``, and on
a timed grid ``time`` (S, *delay_axes, nt) on nodes t0 + j dt with the cubic Lagrange split, plus ``late`` / ``early``
(S, *delay_axes, 2: q and q t beyond the last / before the first node). Here the engine appends a record per deposit
during the trace and a second kernel bins them (``include/lumen_b200.h`` LumenGroup); the grids are the reference's
``Axis`` / ``Grid`` restated, the sensor model's tables are the caller's (``pe``).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from lumen_b200 import _abi as A

FEATURES = {name: i for i, name in enumerate(A.FEATURES)}


@dataclass(frozen=True)
class Axis:
    """One histogram axis (grid.py:63): a deposit feature on ``knots`` (hat functions, constant beyond the end knots) or
    between ``edges`` (one cell between each pair, none outside)."""  # noqa: D205, D209

    name: str
    feature: str
    knots: tuple | None = None
    edges: tuple | None = None

    def __post_init__(self):
        if self.feature not in FEATURES:
            raise ValueError(f"Axis {self.name!r}: feature {self.feature!r} is not one of {tuple(FEATURES)}")
        v = self.knots if self.knots is not None else self.edges
        if (self.knots is None) == (self.edges is None) or v is None or len(v) < 2 or \
                any(b <= a for a, b in zip(v, v[1:])):  # fmt: skip
            raise ValueError(f"Axis {self.name!r}: exactly one of knots or edges, at least two ascending values")

    @property
    def values(self) -> tuple:
        return tuple(float(x) for x in (self.knots if self.knots is not None else self.edges))

    @property
    def size(self) -> int:
        return len(self.knots) if self.knots is not None else len(self.edges) - 1


@dataclass(frozen=True)
class Grid:
    """The static grid of one group's histograms (grid.py:100 Grid); times in ns."""

    axes: tuple = ()
    delay_axes: tuple = ()
    t0: float = 0.0
    dt: float = 1.0
    nt: int = 0
    weighted: bool = False  # the time histogram weighted by the group's acceptance read at the deposit's charge cells
    normalise: bool = False  # each deposit times 1 / A_n of its surface (rows read per normal incidence)

    def __post_init__(self):
        for axes in (self.axes, self.delay_axes):
            if len({a.name for a in axes}) != len(axes):
                raise ValueError(f"Grid: distinct axis names, got {[a.name for a in axes]}")
        if len(self.axes) + len(self.delay_axes) > A.MAX_AXES:
            raise ValueError(f"Grid: at most {A.MAX_AXES} axes in all")
        if self.nt < 0 or (self.nt and not self.dt > 0):
            raise ValueError("Grid: nt >= 0 and dt > 0")

    @classmethod
    def bands(cls, edges, **kw) -> Grid:
        """A grid of wavelength bands between ``edges`` (nm)."""
        return cls(axes=(Axis("wavelength", "wavelength", edges=tuple(float(e) for e in edges)),), **kw)

    @property
    def shape(self) -> tuple:
        return tuple(a.size for a in self.axes)

    @property
    def n_cells(self) -> int:
        return math.prod(self.shape)

    @property
    def delay_shape(self) -> tuple:
        return tuple(a.size for a in self.delay_axes)

    @property
    def n_delay(self) -> int:
        return math.prod(self.delay_shape)


@dataclass
class Group:
    """A readout group: its grid, the detector sensors in it (None: every sensor, in order) and the acceptance per
    charge cell at the run's values (``weights``, shape ``grid.shape``: the product of the sensor model's tables; a
    weighted grid reads it, and with it the pe moment ``pe2`` is kept), with the efficiency ``pe_error`` scales by."""  # noqa: D205, D209

    grid: Grid
    sensors: tuple | None = None
    weights: np.ndarray | None = None
    efficiency: float = 1.0


@dataclass
class Histograms:
    """One group's histograms (grid.py:272 Histograms): with several events every array leads with the event axis."""

    charge: np.ndarray
    charge2: np.ndarray | None = None
    time: np.ndarray | None = None
    late: np.ndarray | None = None
    early: np.ndarray | None = None
    pe_error: np.ndarray | None = None
    grid: Grid = field(default_factory=Grid)
    group: str = ""
    sensors: tuple | None = None


class GroupCells:
    """The cells of a run's readout groups in the LumenGroup layout: on the device (``device`` a torch device) or on
    the host (``device`` None: numpy, the checker's)."""  # noqa: D205, D209

    def __init__(self, det, groups: dict, n_events: int = 1, device=None):
        if len(groups) > A.MAX_GROUPS:
            raise ValueError(f"at most {A.MAX_GROUPS} readout groups")
        self.names = list(groups)
        self.groups = [self._group(det, name, g) for name, g in groups.items()]
        seen = set()
        for name, g in zip(self.names, self.groups):
            ids = set(range(det.n_sensor)) if g.sensors is None else set(g.sensors)
            if seen & ids:
                raise ValueError(f"readout group {name!r}: a sensor is in one group at most")
            seen |= ids
        self.E, self.S = max(n_events, 1), max(det.n_sensor, 1)
        self.device = device
        self.keep = []
        self.outs = []  # the FP64 cells (zeroed by zero_)
        arr = self._dev if device is not None else self._host  # kept alive with the cells (the pointers are raw)
        self.cells = []
        cs = (A.LumenGroup * A.MAX_GROUPS)()
        for k, g in enumerate(self.groups):
            gr = g.grid
            ns = det.n_sensor if g.sensors is None else len(g.sensors)
            c = cs[k]
            c.n_axes, c.n_delay, c.nt = len(gr.axes), len(gr.delay_axes), gr.nt
            c.weighted, c.normalise, c.n_sensors = int(gr.weighted), int(gr.normalise), ns
            c.t0, c.dt = gr.t0, gr.dt
            for i, ax in enumerate((*gr.axes, *gr.delay_axes)):
                v = arr(np.asarray(ax.values, np.float32), np.float32)
                c.axes[i].feature, c.axes[i].n, c.axes[i].knots = FEATURES[ax.feature], len(ax.values), int(ax.knots is not None)
                c.axes[i].values = self._ptr(v, A.c_f32p)
            if g.sensors is not None:
                idx = np.full(det.n_sensor, -1, np.int32)
                idx[np.asarray(g.sensors, np.int64)] = np.arange(ns, dtype=np.int32)
                c.index = self._ptr(arr(idx, np.int32), A.c_i32p)
            if g.weights is not None:
                w = np.asarray(g.weights, np.float32)
                if w.shape != gr.shape and w.size != gr.n_cells:
                    raise ValueError(f"readout group: weights of shape {gr.shape}, got {w.shape}")
                c.weights = self._ptr(arr(w.ravel(), np.float32), A.c_f32p)
            elif gr.weighted:
                raise ValueError("readout group: a weighted grid reads its acceptance: give weights")
            z = self._zeros
            out = dict(charge=z(self.E * ns * gr.n_cells), charge2=z(self.E * ns * gr.n_cells))
            if gr.nt:
                out |= dict(time=z(self.E * ns * gr.n_delay * gr.nt), over_q=z(self.E * ns * gr.n_delay * 2),
                            over_qt=z(self.E * ns * gr.n_delay * 2))  # fmt: skip
            for k2, a in out.items():
                setattr(c, k2, self._ptr(a, A.c_f64p))
            self.cells.append(out)
        self.c = cs
        self.pe2 = self._zeros(self.E * self.S) if any(g.weights is not None for g in self.groups) else None

    @staticmethod
    def _group(det, name, g) -> Group:
        if isinstance(g, Grid):
            g = Group(g, tuple(det.groups[name]) if name in getattr(det, "groups", {}) else None)
        if not isinstance(g, Group):
            raise TypeError(f"readout group {name!r}: a Grid or a Group")
        return g

    def _host(self, a, dt):
        h = np.ascontiguousarray(a, dt)
        self.keep.append(h)
        return h

    def _dev(self, a, dt):
        import torch

        t = torch.as_tensor(np.ascontiguousarray(a, dt), device=self.device)
        self.keep.append(t)
        return t

    def _zeros(self, n):
        if self.device is None:
            a = np.zeros(n)
        else:
            import torch

            a = torch.zeros(n, dtype=torch.float64, device=self.device)
        self.keep.append(a)
        self.outs.append(a)
        return a

    @staticmethod
    def _ptr(a, typ):
        p = a.data_ptr() if hasattr(a, "data_ptr") else a.ctypes.data
        return ctypes_cast(p, typ)

    def attach(self, t, records=None, capacity=0):
        """Point the LumenTallies ``t`` at these groups (and at the records scratch, device runs)."""
        import ctypes

        t.n_groups = len(self.groups)
        t.groups = ctypes.cast(self.c, ctypes.POINTER(A.LumenGroup))
        t.pe2 = self._ptr(self.pe2, A.c_f64p) if self.pe2 is not None else ctypes.cast(None, A.c_f64p)
        t.records = None if records is None else (records.data_ptr() if hasattr(records, "data_ptr") else
                                                  records.ctypes.data)  # fmt: skip
        t.rec_capacity = int(capacity)

    def zero_(self):
        for a in self.outs:
            if isinstance(a, np.ndarray):
                a.fill(0.0)
            else:
                a.zero_()
        return self

    def _np(self, a):
        return a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)

    def histograms(self, n_photons) -> dict:
        """Return {group name: Histograms} (event axis first with several events; pe_error where weights are given)."""
        out = {}
        ev = (self.E,) if self.E > 1 else ()
        pe2 = self._np(self.pe2).reshape(self.E, self.S) if self.pe2 is not None else None
        for name, g, cells in zip(self.names, self.groups, self.cells):
            gr = g.grid
            ns = len(g.sensors) if g.sensors is not None else self.S
            charge = self._np(cells["charge"]).reshape(*ev, ns, *gr.shape)
            charge2 = self._np(cells["charge2"]).reshape(*ev, ns, *gr.shape)
            h = Histograms(charge, charge2, grid=gr, group=name, sensors=g.sensors)
            if gr.nt:
                h.time = self._np(cells["time"]).reshape(*ev, ns, *gr.delay_shape, gr.nt)
                q = self._np(cells["over_q"]).reshape(*ev, ns, *gr.delay_shape, 2)
                qt = self._np(cells["over_qt"]).reshape(*ev, ns, *gr.delay_shape, 2)
                h.late, h.early = (np.stack([q[..., i], qt[..., i]], -1) for i in (0, 1))
            if g.weights is not None and pe2 is not None:
                ids = np.arange(self.S) if g.sensors is None else np.asarray(g.sensors, np.int64)
                q2 = pe2[:, ids] if self.E > 1 else pe2[0, ids]
                h.pe_error = g.efficiency * moment_error(q2, expected_pe(h, g.weights, 1.0), n_photons)
            out[name] = h
        return out


def ctypes_cast(p, typ):
    import ctypes

    return ctypes.cast(ctypes.c_void_p(int(p)), typ)


def moment_error(q2, s, n):
    """sqrt(n / (n - 1) (q2 - s^2 / n)), clipped at 0 (src/lumen/readout/grid.py:48)."""
    n = np.asarray(n, np.float64)
    v = np.maximum(np.asarray(q2) - np.asarray(s) ** 2 / np.maximum(n, 1.0), 0.0)
    return np.sqrt(n / np.maximum(n - 1.0, 1.0) * v)


def expected_pe(h: Histograms, acceptance, efficiency=1.0):
    """Return the expected photoelectrons per sensor of a group's histograms: efficiency x the charge histogram
    contracted with the acceptance per charge cell (src/lumen/readout/detection.py:86 expected_pe)."""  # noqa: D205, D209
    acc = np.asarray(acceptance, np.float64).reshape(h.grid.shape)
    k = len(h.grid.shape)
    s = (h.charge * acc).reshape(*h.charge.shape[: h.charge.ndim - k], -1).sum(-1) if k else h.charge
    return np.asarray(efficiency) * s


def tables_acceptance(grid: Grid, tables) -> np.ndarray:
    """Return the acceptance per charge cell of a sensor model's tables: [(axis names, values over those axes'
    cells), ...] multiplied in order and broadcast over the grid's axes (the reference's ``model.tables`` einsum)."""  # noqa: D205, D209
    names = [a.name for a in grid.axes]
    acc = np.ones(grid.shape, np.float64)
    for axes, values in tables:
        v = np.asarray(values, np.float64)
        order = [names.index(a) for a in axes]
        shape = [1] * len(names)
        for i, ax in enumerate(order):
            shape[ax] = v.shape[i]
        acc = acc * np.transpose(v, np.argsort(order)).reshape(shape)
    return acc
