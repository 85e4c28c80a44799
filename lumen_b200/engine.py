"""The engine on one CUDA device: a scene handle of the C ABI and device buffers held as torch tensors.

PyTorch is the plumbing here (device memory, streams); every photon is traced by the CUDA library
``liblumen_b200.so`` through its C ABI (include/lumen_b200.h). There is no CPU path: without the library or a GPU the
engine raises.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from lumen_b200 import _abi as A


def _f32p(t):
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), A.c_f32p) if t is not None else ctypes.cast(None, A.c_f32p)


def _i32p(t):
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), A.c_i32p) if t is not None else ctypes.cast(None, A.c_i32p)


def _f64p(t):
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), A.c_f64p) if t is not None else ctypes.cast(None, A.c_f64p)


def _i64p(t):
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), A.c_i64p) if t is not None else ctypes.cast(None, A.c_i64p)


class DeviceTallies:
    """FP64 tallies on the device in the LumenTallies layout (added to by each trace call)."""

    def __init__(self, n_sensor, n_events=1, n_bins=0, bin0=0.0, bin_w=1.0, n_grad=0, device="cuda"):
        S, E = max(n_sensor, 1), max(n_events, 1)
        z = lambda *s: torch.zeros(*s, dtype=torch.float64, device=device)  # noqa: E731
        self.arrival, self.arrival_t, self.arrival2 = z(E, S), z(E, S), z(E, S)
        self.hist = z(E, S, n_bins) if n_bins else None
        self.jac = z(E, S, n_grad) if n_grad else None
        self.health = z(A.N_HEALTH)
        self.counts = torch.zeros(A.N_COUNT, dtype=torch.int64, device=device)
        t = A.LumenTallies()
        t.n_events, t.n_bins, t.bin0, t.bin_w = E, n_bins, bin0, bin_w
        t.arrival, t.arrival_t, t.arrival2 = _f64p(self.arrival), _f64p(self.arrival_t), _f64p(self.arrival2)
        t.hist, t.jac, t.health = _f64p(self.hist), _f64p(self.jac), _f64p(self.health)
        t.counts = ctypes.cast(ctypes.c_void_p(self.counts.data_ptr()), A.c_u64p)
        self.c = t

    def attach_truth(self, n: int):
        """Keep each of the next call's ``n`` photons' analog records (LUMEN_F_TRUTH) in ``self.truth``."""
        self.truth = torch.zeros((max(int(n), 1), A.TRUTH_WORDS), dtype=torch.float32, device=self.arrival.device)
        self.c.truth = _f32p(self.truth)
        return self

    def attach_groups(self, groups, capacity: int):
        """Fill the readout groups ``groups`` (a ``lumen_b200.readout.GroupCells`` on this device) from a records
        scratch of ``capacity`` deposits (a trace whose deposits outgrow it raises ``RecordsOverflow``)."""  # noqa: D205, D209
        self.groups = groups
        self.records = torch.empty((max(int(capacity), 1), A.REC_WORDS), dtype=torch.int32,
                                   device=self.arrival.device)  # fmt: skip
        groups.attach(self.c, self.records, self.records.shape[0])
        return self

    def zero_(self):
        for v in (self.arrival, self.arrival_t, self.arrival2, self.hist, self.jac, self.health, self.counts):
            if v is not None:
                v.zero_()
        if getattr(self, "groups", None) is not None:
            self.groups.zero_()
        return self


class DeviceSource:
    """A procedural source's arrays on the device (LumenSource layout)."""

    def __init__(self, src, samples, device="cuda", det=None):
        a = src.arrays(samples, det)
        self.ev_f = torch.as_tensor(np.ascontiguousarray(a["ev_f"], np.float32), device=device)
        self.ev_first = torch.as_tensor(np.ascontiguousarray(a["ev_first"], np.int64), device=device)
        self.ev_w = torch.as_tensor(np.ascontiguousarray(a["ev_w"], np.float32), device=device)
        s = A.LumenSource()
        s.kind, s.n_events = a["kind"], len(a["ev_w"])
        s.ev_f, s.ev_first, s.ev_w = _f32p(self.ev_f), _i64p(self.ev_first), _f32p(self.ev_w)
        s.lam0, s.lam1, s.cone_cos = a["lam0"], a["lam1"], a["cone_cos"]
        s.tau1, s.tau2, s.frac1 = a["tau1"], a["tau2"], a["frac1"]
        s.rindex_tab = a.get("rindex_tab", -1)
        if "mat" in a:
            s.mat[:] = [int(v) for v in a["mat"]]
        self.c = s
        self.n_events = len(a["ev_w"])
        self.total = int(a["ev_first"][-1])


class DeviceRows:
    """Explicit emission rows on the device (LumenRows layout): a dict of numpy / torch arrays."""

    def __init__(self, rows: dict, device="cuda"):
        def f32(v):
            return torch.as_tensor(np.ascontiguousarray(v, np.float32) if not torch.is_tensor(v) else v,
                                   dtype=torch.float32, device=device).contiguous()  # fmt: skip

        x, d = f32(rows["x"]).reshape(-1, 3), f32(rows["d"]).reshape(-1, 3)
        self.cols = {k: x[:, i].contiguous() for i, k in enumerate("xyz")}
        self.cols.update({"d" + k: d[:, i].contiguous() for i, k in enumerate("xyz")})
        for k in ("t", "lam", "w"):
            self.cols[k] = f32(rows[k]).reshape(-1)
        self.pol = f32(rows["pol"]).reshape(-1, 6) if rows.get("pol") is not None else None
        ev = rows.get("event")
        self.event = torch.as_tensor(np.asarray(ev, np.int32), device=device) if ev is not None else None
        r = A.LumenRows()
        for k in ("x", "y", "z", "dx", "dy", "dz", "t", "lam", "w"):
            setattr(r, k, _f32p(self.cols[k]))
        r.pol = _f32p(self.pol)
        r.event = _i32p(self.event)
        self.c = r
        self.n = int(x.shape[0])


class Engine:
    """The detector uploaded to one CUDA device (``lumen_b200_scene_create``)."""

    def __init__(self, det, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("lumen_b200 needs a CUDA device (there is no CPU path)")
        self.det = det
        self.device = torch.device(device if device is not None else "cuda", torch.cuda.current_device()) \
            if device is None else torch.device(device)  # fmt: skip
        self.lib = A.engine()
        desc, keep = det.desc()
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            A.check(self.lib.lumen_b200_scene_create(ctypes.byref(desc), ctypes.byref(h)))
        self.h = h
        self.n_sensor = det.n_sensor
        self.pool = np.ascontiguousarray(det.pool, np.float32)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.lumen_b200_scene_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def set_pools(self, live=None, ref=None):
        """Set the live and reference parameter pools (None: the detector's own values)."""
        lv = np.ascontiguousarray(self.pool if live is None else live, np.float32)
        rf = None if ref is None else np.ascontiguousarray(ref, np.float32)
        self._pools = (lv, rf)
        A.check(self.lib.lumen_b200_scene_set_pools(self.h, A.fptr(lv), A.fptr(rf)))

    def _stream(self, stream):
        s = stream if stream is not None else torch.cuda.current_stream(self.device)
        return ctypes.c_void_p(s.cuda_stream)

    def trace(self, key, n, *, source=None, rows=None, first_id=0, controls=None, tallies=None, stream=None):
        """Trace photons first_id .. first_id + n - 1 into ``tallies`` (DeviceTallies, added to)."""
        c = controls or A.controls()
        src = ctypes.byref(source.c) if source is not None else None
        rw = ctypes.byref(rows.c) if rows is not None else None
        with torch.cuda.device(self.device):
            st = self.lib.lumen_b200_trace(self.h, rw, src, key[0], key[1], first_id, n, ctypes.byref(c),
                                           ctypes.byref(tallies.c), self._stream(stream))  # fmt: skip
            self.launches = int(self.lib.lumen_b200_last_launches())  # the kernels the call launched
            A.check(st)
        return tallies

    def adjoint(self, key, n, cotangent, *, source=None, rows=None, first_id=0, controls=None, stream=None):
        """Return d(sum cotangent * arrival) / d parameters (float64, n_grad) by replaying the photons."""
        c = controls
        cot = torch.as_tensor(cotangent, dtype=torch.float64, device=self.device).contiguous()
        grads = torch.zeros(c.n_grad, dtype=torch.float64, device=self.device)
        n_ev = cot.shape[0] if cot.ndim == 2 else 1
        src = ctypes.byref(source.c) if source is not None else None
        rw = ctypes.byref(rows.c) if rows is not None else None
        with torch.cuda.device(self.device):
            A.check(self.lib.lumen_b200_adjoint(self.h, rw, src, key[0], key[1], first_id, n, ctypes.byref(c),
                                                _f64p(cot), n_ev, _f64p(grads), self._stream(stream)))  # fmt: skip
        return grads

    def trace_photons(self, key, n, *, source=None, rows=None, first_id=0, controls=None):
        c = controls or A.controls()
        out_i = torch.zeros((n, 5), dtype=torch.int32, device=self.device)
        out_f = torch.zeros((n, 4), dtype=torch.float32, device=self.device)
        src = ctypes.byref(source.c) if source is not None else None
        rw = ctypes.byref(rows.c) if rows is not None else None
        with torch.cuda.device(self.device):
            A.check(self.lib.lumen_b200_trace_photons(self.h, rw, src, key[0], key[1], first_id, n, ctypes.byref(c),
                                                      _i32p(out_i), _f32p(out_f), self._stream(None)))  # fmt: skip
        return out_i, out_f

    def query(self, o, d, vol=None, srf=None, t_max=None):
        """The navigator query per ray (lumen_b200_query; lumen_b200_query64 in float64 on a float64 detector)."""
        f64 = self.det.precision == "float64"
        dt, tt = (np.float64, torch.float64) if f64 else (np.float32, torch.float32)
        o = torch.as_tensor(np.asarray(o, dt).reshape(-1, 3), device=self.device)
        d = torch.as_tensor(np.asarray(d, dt).reshape(-1, 3), device=self.device)
        n = o.shape[0]
        ray = torch.cat([o, d], 1).contiguous()
        vol = torch.full((n,), -1, dtype=torch.int32, device=self.device) if vol is None else \
            torch.as_tensor(np.asarray(vol, np.int32), device=self.device)  # fmt: skip
        srf = torch.full((n,), -1, dtype=torch.int32, device=self.device) if srf is None else \
            torch.as_tensor(np.asarray(srf, np.int32), device=self.device)  # fmt: skip
        out_i = torch.zeros((n, 8), dtype=torch.int32, device=self.device)
        out_f = torch.zeros((n, 4), dtype=tt, device=self.device)
        tm = self.det.arrays["reach"] if t_max is None else t_max
        with torch.cuda.device(self.device):
            if f64:
                A.check(self.lib.lumen_b200_query64(self.h, _f64p(ray), _i32p(vol), _i32p(srf), ctypes.c_double(tm),
                                                    n, _i32p(out_i), _f64p(out_f), self._stream(None)))  # fmt: skip
            else:
                A.check(self.lib.lumen_b200_query(self.h, _f32p(ray), _i32p(vol), _i32p(srf), ctypes.c_float(tm), n,
                                                  _i32p(out_i), _f32p(out_f), self._stream(None)))  # fmt: skip
        return out_i, out_f

    def locate(self, pts):
        """The volume holding each point (lumen_b200_locate; lumen_b200_locate64 on a float64 detector)."""
        f64 = self.det.precision == "float64"
        dt = np.float64 if f64 else np.float32
        p = torch.as_tensor(np.asarray(pts, dt).reshape(-1, 3), device=self.device).contiguous()
        vol = torch.zeros(p.shape[0], dtype=torch.int32, device=self.device)
        with torch.cuda.device(self.device):
            if f64:
                A.check(self.lib.lumen_b200_locate64(self.h, _f64p(p), p.shape[0], _i32p(vol), self._stream(None)))
            else:
                A.check(self.lib.lumen_b200_locate(self.h, _f32p(p), p.shape[0], _i32p(vol), self._stream(None)))
        return vol
