"""Benchmark: photons/s of the photon-transport hot path on B200 (one JSON line on rank 0).

Workload (the plain-forward tank): a water cylinder of radius 5 m and height 10 m with 2000 inward-facing
hemispherical PMTs (radius 0.1 m) on a barrel and end-cap grid, black-sheet walls of reflectivity 0.1, water with
absorption length 50 m, Rayleigh length 80 m and index 1.34; 2^24 photons per GPU per step, wavelength uniform in
300-600 nm, isotropic from one point drawn uniformly in the inner volume with a fixed host seed; outputs per-PMT
arrivals, their second moments and 1 ns arrival-time histograms over [0, 200) ns. Synthetic: the detector is built
from these numbers, the photons drawn from the reference's counter-based stream (seed 0).

A step is one pass of the photon loop over the step's photons (the trace kernel with its FP64 tallies), inputs
resident on the device. ``e2e`` times the same metric through the public call ``lumen_b200.simulate`` with host
inputs and outputs (parameter pool and source records host-to-device, tallies device-to-host, every step).
Multi-GPU: each rank traces its own photon-id range (weak scaling) and the tallies are summed by one NCCL all-reduce.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl lumen_b200|reference] [--photons P]
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

BYTES_STEP = 208  # canonical per photon-step: SoA FP32 photon state read + written (104 B each way)
BYTES_PHOTON = 60  # per photon: its emission row (15 float32)
BYTES_DEPOSIT = 24  # per sensor deposit: the reference's record (sensor, q, w0, time, lam, photon)
METRIC = "photons/s on 1 B200 (fwd; batched fwd+adjoint) at matched per-PMT MC error"
L2_FLUSH_BYTES = 256 << 20


# DRAM bytes per photon-step of the tank workload, from ncu's dram__bytes_read.sum + dram__bytes_write.sum: the
# persistent loop k_trace<0,256,4,2,0,0> on one launch of 2^20 photons (2.76 steps each; local memory almost all of
# it), and the wavefront's k_wave_query<0,2> + k_wave_step<0> summed over every round of seven calls of 2^20 photons
# (2.76 steps each; 2.613 GB read + 2.090 GB written per call: the slots' state and the kernels' local memory)
TRAFFIC_PER_STEP = {0: (0.253087e9 + 1.570654e9) / (1048576 * 2.760), 3: (2.613e9 + 2.090e9) / (1048576 * 2.760)}


def workload_point(seed=12345):
    rng = np.random.default_rng(seed)
    while True:
        p = rng.uniform([-4.8, -4.8, -4.8], [4.8, 4.8, 4.8])
        if np.hypot(p[0], p[1]) < 4.8:
            return p


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """The SM clock and throttle reasons sampled by one ``nvidia-smi -lms 200`` process (started once, before the
    warm-up, so that no process start-up falls in the timed region); ``mark()`` and ``close()`` bound the rows kept."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")  # fmt: skip

    def __init__(self, index):
        self.index, self.rows, self.t0, self.t1 = index, [], None, None

    def _read(self):
        for line in self.p.stdout:
            self.rows.append((time.monotonic(), [x.strip() for x in line.strip().split(",")]))

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)  # fmt: skip
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.p = None
        return self

    def mark(self):
        self.t0 = time.monotonic()

    def __exit__(self, *a):
        self.t1 = time.monotonic()
        if self.p is not None:
            time.sleep(0.25)  # one more sample after the timed region
            self.p.terminate()
            self.p.wait(timeout=10)
            self.t.join(timeout=10)

    def per_step(self, bounds):
        """The median SM clock (MHz) sampled inside each (start, end) host-time interval of ``bounds`` (None: no
        sample fell in it: a step shorter than the 200 ms sampling period)."""  # noqa: D205, D209
        out = []
        for a, b in bounds:
            v = [float(r[0]) for t, r in self.rows if a <= t <= b and len(r) >= 6 and r[0].replace(".", "").isdigit()]
            out.append(float(np.median(v)) if v else None)
        return out

    def summary(self):
        t0, t1 = self.t0 or 0.0, (self.t1 or time.monotonic()) + 0.25
        rows = [r for t, r in self.rows if t0 <= t <= t1 and len(r) >= 6]
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[k] for r in rows for k in range(4) if r[2 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm), "sampler": "nvidia-smi -lms 200 (one process)"}  # fmt: skip


def dist_setup(args):
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    return world, rank, local


def cpu_reference(args, det, src, n_total):
    """The reference arm / CPU baseline: the C++ restatement of the photon loop on every host thread."""
    import oracle
    from lumen_b200 import _abi as A

    threads = os.cpu_count() or 1
    key = A.key_of_seed(0)
    oracle.lib()
    sample = args.cpu_photons
    oracle.trace(det, key, 1024, source=src, samples=n_total, threads=threads)  # warm-up
    ts = []
    for _ in range(max(args.cpu_steps, 1)):
        t0 = time.perf_counter()
        oracle.trace(det, key, sample, source=src, samples=n_total, threads=threads)
        ts.append(time.perf_counter() - t0)
    dt = float(np.median(ts))
    return dict(value=sample / dt, unit="photons/s", cores=threads, kind="port",
                sample=f"{sample} photons of the workload (photon ids 0..{sample - 1}), median of {len(ts)} runs")


def batched_events(seed=2024, n_events=256):
    """256 Cherenkov-like tracks in the tank: starts uniform in the volume, isotropic directions, lengths uniform in
    0.5-3 m (resampled until the track stays inside), cone half-angle 42 degrees, photons per event log-uniform in
    [1e3, 1e6]."""  # noqa: D205
    rng = np.random.default_rng(seed)
    st, dr, ln = [], [], []
    while len(st) < n_events:
        p = rng.uniform(-4.7, 4.7, 3)
        u = rng.normal(size=3)
        u /= np.linalg.norm(u)
        L = rng.uniform(0.5, 3.0)
        e = p + L * u
        if np.hypot(p[0], p[1]) < 4.7 and np.hypot(e[0], e[1]) < 4.7 and abs(e[2]) < 4.7:
            st.append(p), dr.append(u), ln.append(L)
    counts = np.exp(rng.uniform(np.log(1e3), np.log(1e6), n_events)).astype(np.int64)
    return np.asarray(st), np.asarray(dr), np.asarray(ln), counts


def per_sensor(arrival, arrival2, photons_per_event):
    """Per-sensor arrivals summed over events and their MC errors (each event's moment error, src/lumen/readout/
    grid.py:48, added in quadrature)."""  # noqa: D205, D209
    from lumen_b200.api import moment_error

    n = np.asarray(photons_per_event, np.float64).reshape(-1, 1)
    err = moment_error(arrival2, arrival, n)
    return arrival.sum(0), np.sqrt((err**2).sum(0))


def chi2_vs_checker(eng, det, src, n_ev, gt=(), m=1 << 17, flags=0):
    """The GPU's arrivals of photon ids 0 .. m - 1 (seed 0) against the checker's of the same ids drawn with seed 1:
    two independent samples of the same photons' law. Returns chi^2 / ndf over the sensors that see light (per-sensor
    sums over events, combined MC errors), ndf, and the largest relative difference of the GPU and the checker on the
    SAME photons (seed 0), which parity makes ~1e-12."""  # noqa: D205, D209
    import torch

    import oracle
    from lumen_b200 import _abi as A
    from lumen_b200.engine import DeviceSource, DeviceTallies

    ds = DeviceSource(src, m, eng.device, det)
    c = A.controls(grad_tabs=list(gt), flags=flags)
    T = DeviceTallies(det.n_sensor, n_ev, 0, 0.0, 1.0, len(gt), eng.device)
    eng.trace(A.key_of_seed(0), m, source=ds, controls=c, tallies=T)
    torch.cuda.synchronize(eng.device)
    ev_first = ds.ev_first.cpu().numpy()
    per_ev = np.diff(np.clip(ev_first, 0, m))
    threads = os.cpu_count() or 1
    a0, e0 = per_sensor(T.arrival.cpu().numpy(), T.arrival2.cpu().numpy(), per_ev)
    O1, _ = oracle.trace(det, A.key_of_seed(1), m, source=src, samples=m, controls=c, n_events=n_ev, threads=threads)
    a1, e1 = per_sensor(O1.arrival, O1.arrival2, per_ev)
    O0, _ = oracle.trace(det, A.key_of_seed(0), m, source=src, samples=m, controls=c, n_events=n_ev, threads=threads)
    var = e0**2 + e1**2
    ok = var > 0
    chi2 = float(((a0 - a1)[ok] ** 2 / var[ok]).sum())
    ndf = int(ok.sum())
    same = float(np.max(np.abs(T.arrival.cpu().numpy() - O0.arrival) / np.maximum(np.abs(O0.arrival), 1e-300)))
    return {"chi2_ndf": chi2 / max(ndf, 1), "ndf": ndf, "photons": m, "checker_seed": 1,
            "same_photons_max_rel_diff": same}


def mc_error(arrival, arrival2, per_ev):
    """The median relative per-PMT MC error over the sensors that see light (per-sensor sums over events)."""
    a, e = per_sensor(arrival, arrival2, per_ev)
    ok = a > 0
    return float(np.median(e[ok] / a[ok])) if ok.any() else None


# the reference's published run of the tutorial tank (docs/tutorial/first-hour.md:101-111): arrivals and their errors
PUBLISHED_TOY = ([394.54, 913.75, 547.76, 501.74, 515.31, 528.14, 320.36, 340.68],
                 [17.22, 26.23, 20.30, 19.43, 19.69, 19.94, 15.51, 16.03])  # fmt: skip


def run_toy(dev, reps=10, with_cpu=True):
    """The shipped toy tank (8 PMTs): one isotropic 400 nm point at (0, 0, 0.1) m, n_photons 2e5, 2^18 photons, seed 0,
    plain forward; arrivals +- MC error per PMT and their chi^2 / ndf against the reference's published table."""  # noqa: D205
    import torch

    from lumen_b200 import _abi as A
    from lumen_b200 import detectors, sources
    from lumen_b200.api import moment_error
    from lumen_b200.engine import DeviceSource, DeviceTallies, Engine

    det = detectors.toy_tank()
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=2e5, lam=400.0)
    n = 1 << 18
    eng = Engine(det, dev)
    ds = DeviceSource(src, n, dev)
    c = A.controls()
    T = DeviceTallies(det.n_sensor, 1, 0, 0.0, 1.0, 0, dev)
    eng.trace(A.key_of_seed(0), n, source=ds, controls=c, tallies=T)
    ms = []
    for _ in range(reps):
        T.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.trace(A.key_of_seed(0), n, source=ds, controls=c, tallies=T)
        e1.record()
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    arr = T.arrival.cpu().numpy()[0]
    err = moment_error(T.arrival2.cpu().numpy()[0], arr, n)
    cnt = T.counts.cpu().numpy()
    pa, pe = np.asarray(PUBLISHED_TOY[0]), np.asarray(PUBLISHED_TOY[1])
    m = float(np.median(ms))
    out = {"value": n / (m * 1e-3), "unit": "photons/s", "photons_per_launch": n, "ms_per_launch": m,
           "steps_per_photon": float(cnt[1] / cnt[0]), "records": int(cnt[2]),
           "arrivals": [round(float(x), 2) for x in arr], "arrivals_error": [round(float(x), 2) for x in err],
           "mc_error": float(np.median(err / arr)),
           "chi2_ndf_vs_published": float((((arr - pa) ** 2) / (err**2 + pe**2)).sum() / len(pa)),
           "published": "docs/tutorial/first-hour.md:101-111 (lumen 0.2.0)"}  # fmt: skip
    if with_cpu:
        out["vs_checker"] = chi2_vs_checker(eng, det, src, 1, m=n)
    eng.close()
    return out


def run_batched(dev, det, reps=3, with_cpu=True):
    """The batched forward + adjoint: one fused launch (arrivals and their Jacobian per event) under a CUDA graph."""
    import torch

    from lumen_b200 import _abi as A
    from lumen_b200 import autotune, sources
    from lumen_b200.engine import DeviceSource, DeviceTallies, Engine

    st, dr, ln, counts = batched_events()
    src = sources.Tracks(start=st, direction=dr, length=ln, cone_angle=np.radians(42.0), n_photons=counts.astype(float),
                         lam_range=(300.0, 600.0), counts_=counts)  # fmt: skip
    n = int(counts.sum())
    eng = Engine(det, dev)
    ds = DeviceSource(src, n, dev)
    names = ["media/Water/absorption", "media/Water/rayleigh", "surfaces/BlackSheet/R"]
    gt = [det.params_index[k] for k in names]
    shape, times = autotune.tune(eng, ds, 1 << 20, gt, ds.n_events, A.key_of_seed(0), asynchronous=True)
    c = shape.controls(n, gt, A.F_ASYNC)
    T = DeviceTallies(det.n_sensor, ds.n_events, 0, 0.0, 1.0, len(gt), dev)
    key = A.key_of_seed(0)
    stream = torch.cuda.Stream(dev)
    with torch.cuda.stream(stream):  # warm-up on the side stream before capture
        T.zero_()
        eng.trace(key, n, source=ds, controls=c, tallies=T, stream=stream)
    torch.cuda.synchronize(dev)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        T.zero_()
        eng.trace(key, n, source=ds, controls=c, tallies=T, stream=stream)
    g.replay()
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    cnt = T.counts.cpu().numpy()
    jac = T.jac.cpu().numpy()
    m = float(np.median(ms))
    per_ev = np.diff(ds.ev_first.cpu().numpy())
    err = mc_error(T.arrival.cpu().numpy(), T.arrival2.cpu().numpy(), per_ev)
    vs = chi2_vs_checker(eng, det, src, ds.n_events, gt) if with_cpu else None
    del g
    # the reverse mode over the same photons: one adjoint replay with a cotangent per event and sensor
    cot = np.random.default_rng(10).normal(size=jac.shape[:2])
    ca = shape.controls(n, gt)  # the tuned shape, synchronous
    eng.adjoint(key, n, cot, source=ds, controls=ca)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ga = eng.adjoint(key, n, cot, source=ds, controls=ca)
    e1.record()
    torch.cuda.synchronize(dev)
    ma = e0.elapsed_time(e1)
    want = np.einsum("es,esp->p", cot, jac)
    adj = {"value": n / (ma * 1e-3), "unit": "photons/s", "ms_per_launch": ma,
           "max_rel_diff_to_cot_jac": float(np.max(np.abs(ga.cpu().numpy() - want) / np.abs(want)))}  # fmt: skip
    eng.close()
    return {"value": n / (m * 1e-3), "unit": "photons/s", "events": int(ds.n_events), "photons_per_launch": n,
            "mc_error": err, "vs_checker": vs, "adjoint_replay": adj,
            "ms_per_launch": m, "photon_steps_per_s": float(cnt[1]) / (m * 1e-3), "gradients": names,
            "graph": True, "autotune": {"shape": shape.label(), "ms_sample": {k: round(v, 3) for k, v in times.items()}},
            "jacobian_norm": float(np.abs(jac).sum()), "aborted": int(cnt[5])}  # fmt: skip


def run_tank_adjoint(dev, src, n, reps=2, with_cpu=True):
    """The tank forward + Jacobian with its wall switched to ground unified, sigma_alpha 0.1: derivatives in the
    absorption and Rayleigh lengths, the wall reflectivity and its sigma_alpha (the facet path's score) in the same
    launch (the 2000 PMT efficiencies' derivatives are the arrivals: after tracking)."""  # noqa: D205
    import torch

    from lumen_b200 import _abi as A
    from lumen_b200 import autotune, detectors
    from lumen_b200.engine import DeviceSource, DeviceTallies, Engine

    det = detectors.cylinder_tank(wall_finish="ground", sigma_alpha=0.1)
    eng = Engine(det, dev)
    ds = DeviceSource(src, n, dev)
    names = ["media/Water/absorption", "media/Water/rayleigh", "surfaces/BlackSheet/R",
             "surfaces/BlackSheet/sigma_alpha"]  # fmt: skip
    gt = [det.params_index[k] for k in names]
    # a sample of several pool fills: the wavefront's last rounds run few photons, a cost a one-fill sample overstates
    shape, times = autotune.tune(eng, ds, min(n, 1 << 23), gt, ds.n_events, A.key_of_seed(0), reps=1)
    c = shape.controls(n, gt)
    T = DeviceTallies(det.n_sensor, ds.n_events, 200, 0.0, 1.0, len(gt), dev)
    key = A.key_of_seed(0)
    eng.trace(key, min(n, 1 << 20), source=ds, controls=c, tallies=T)
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(reps):
        T.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.trace(key, n, source=ds, controls=c, tallies=T)
        e1.record()
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    cnt = T.counts.cpu().numpy()
    m = float(np.median(ms))
    jac = T.jac.cpu().numpy()[0]
    err = mc_error(T.arrival.cpu().numpy(), T.arrival2.cpu().numpy(), [n])
    vs = chi2_vs_checker(eng, det, src, 1, gt) if with_cpu else None
    adj = adjoint_replay(eng, ds, n, c, jac, key, dev)
    fd = fd_check(eng, det, ds, names, gt, key, dev)
    eng.close()
    return {"value": n / (m * 1e-3), "unit": "photons/s", "photons_per_launch": n, "ms_per_launch": m,
            "photon_steps_per_s": float(cnt[1]) / (m * 1e-3), "steps_per_photon": float(cnt[1] / max(cnt[0], 1)),
            "mc_error": err, "vs_checker": vs, "adjoint_replay": adj, "fd_check": fd,
            "wall": "ground unified, sigma_alpha 0.1", "gradients": names,
            "autotune": {"shape": shape.label(), "ms_sample": {k: round(v, 3) for k, v in times.items()}},
            "jacobian_abs_sum": [float(x) for x in np.abs(jac).sum(0)]}  # fmt: skip


def adjoint_replay(eng, ds, n, c, jac, key, dev, reps=2):
    """The reverse mode timed: lumen_b200_adjoint replays the run's photons from their keys (in the launch shape of
    the controls ``c``, the forward's) and contracts every deposit's tangent with a cotangent (one per sensor); the
    result must be cotangent @ the Jacobian the forward tangents gave on the same photons."""  # noqa: D205, D209
    import torch

    cot = np.random.default_rng(9).normal(size=(1, jac.shape[0]))
    g = eng.adjoint(key, n, cot, source=ds, controls=c)
    ms = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g = eng.adjoint(key, n, cot, source=ds, controls=c)
        e1.record()
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    want = cot[0] @ jac
    rel = float(np.max(np.abs(g.cpu().numpy() - want) / np.maximum(np.abs(want), 1e-300)))
    m = float(np.median(ms))
    return {"value": n / (m * 1e-3), "unit": "photons/s", "ms_per_launch": m, "max_rel_diff_to_cot_jac": rel}


def fd_check(eng, det, ds, names, gt, key, dev, n=1 << 20, h=0.01, seeds=(0, 1, 2, 3)):
    """Each parameter's derivative of the summed arrivals against central differences of +-1 % with the reference
    held (common random numbers), over independent seeds: the mean difference in units of its standard error."""  # noqa: D205, D209
    import torch

    from lumen_b200 import _abi as A
    from lumen_b200.engine import DeviceTallies

    base = {k: float(det.params()[k][1][0]) for k in names}
    c = A.controls(grad_tabs=gt)
    c0 = A.controls()
    rows = []
    for seed in seeds:
        k = A.key_of_seed(seed)
        T = DeviceTallies(det.n_sensor, 1, 0, 0.0, 1.0, len(gt), dev)
        eng.set_pools(det.pool, None)
        eng.trace(k, n, source=ds, controls=c, tallies=T)
        d = T.jac.cpu().numpy()[0].sum(0)
        fd = []
        for name in names:
            s = []
            for sgn in (1.0, -1.0):
                Tp = DeviceTallies(det.n_sensor, 1, 0, 0.0, 1.0, 0, dev)
                eng.set_pools(det.pool_with({name: base[name] * (1.0 + sgn * h)}), det.pool)
                eng.trace(k, n, source=ds, controls=c0, tallies=Tp)
                s.append(float(Tp.arrival.sum().item()))
            fd.append((s[0] - s[1]) / (2.0 * h * base[name]))
        rows.append((d, np.asarray(fd)))
    eng.set_pools(det.pool, None)
    torch.cuda.synchronize(dev)
    D = np.array([r[0] for r in rows])
    F = np.array([r[1] for r in rows])
    diff = (D - F).mean(0)
    se = np.sqrt(D.var(0, ddof=1) / len(seeds) + F.var(0, ddof=1) / len(seeds))
    return {"photons": n, "seeds": len(seeds), "step": h, "derivative": [float(x) for x in D.mean(0)],
            "central_difference": [float(x) for x in F.mean(0)],
            "diff_in_standard_errors": [float(x) for x in diff / np.maximum(se, 1e-300)],
            "rel_diff": [float(x) for x in diff / np.abs(F.mean(0))]}  # fmt: skip


def run_lar(dev, n, reps=1, with_cpu=True):
    """The liquid-argon box: 10^4 scintillation points, forward + Jacobian over the cage reflectivity and the
    Rayleigh length (the sensor efficiencies' derivatives are the arrivals: after tracking). The cage and cathode are
    ground unified with sigma_alpha 0.1."""  # noqa: D205
    import torch

    from lumen_b200 import _abi as A
    from lumen_b200 import autotune, detectors, sources
    from lumen_b200.engine import DeviceSource, DeviceTallies, Engine

    det = detectors.lar_box(sigma_alpha=0.1)
    pts = np.random.default_rng(77).uniform([-2.4, -1.9, -1.9], [2.4, 1.9, 1.9], (10000, 3))
    src = sources.Scintillation(position=pts, lam=128.0, tau=(6.0, 1500.0), fraction=0.25, n_photons=1.0)
    eng = Engine(det, dev)
    ds = DeviceSource(src, n, dev)
    names = ["surfaces/CageSurface/R", "media/LAr/rayleigh"]
    gt = [det.params_index[k] for k in names]
    shape, times = autotune.tune(eng, ds, min(n, 1 << 22), gt, ds.n_events, A.key_of_seed(0), reps=1)
    c = shape.controls(n, gt)
    T = DeviceTallies(det.n_sensor, ds.n_events, 0, 0.0, 1.0, len(gt), dev)
    key = A.key_of_seed(0)
    eng.trace(key, min(n, 1 << 18), source=ds, controls=c, tallies=T)
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(reps):
        T.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        eng.trace(key, n, source=ds, controls=c, tallies=T)
        e1.record()
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
    cnt = T.counts.cpu().numpy()
    m = float(np.median(ms))
    err = mc_error(T.arrival.cpu().numpy(), T.arrival2.cpu().numpy(), np.diff(ds.ev_first.cpu().numpy()))
    vs = chi2_vs_checker(eng, det, src, ds.n_events, gt) if with_cpu else None
    eng.close()
    return {"value": n / (m * 1e-3), "unit": "photons/s", "photons_per_launch": n, "ms_per_launch": m,
            "photon_steps_per_s": float(cnt[1]) / (m * 1e-3), "steps_per_photon": float(cnt[1] / max(cnt[0], 1)),
            "mc_error": err, "vs_checker": vs, "moment_table_sums": int(cnt[4]), "moment_lost": int(cnt[7]),
            "points": 10000, "gradients": names, "arrivals_sum": float(T.arrival.sum().item()),
            "autotune": {"shape": shape.label(), "ms_sample": {k: round(v, 3) for k, v in times.items()}}}  # fmt: skip


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="lumen_b200")
    ap.add_argument("--photons", type=int, default=1 << 24)
    ap.add_argument("--cpu-photons", type=int, default=1 << 17)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the batched and liquid-argon workloads")
    ap.add_argument("--lar-photons", type=int, default=1 << 26)
    ap.add_argument("--variant", type=int, default=-1,
                    help="the headline's launch variant (3: wavefront; default: the autotuner's pick)")
    args = ap.parse_args()

    from lumen_b200 import detectors, sources

    det = detectors.cylinder_tank()
    point = workload_point()
    n = args.photons
    src = sources.Point(position=point, n_photons=1.0, lam_range=(300.0, 600.0))
    cfg = {"workload": "cylinder water tank, 2000 hemispherical PMTs, plain forward, 1 ns time histograms",
           "photons_per_gpu_per_step": n, "radius_m": 5.0, "height_m": 10.0, "pmts": 2000, "wall_reflectivity": 0.1,
           "abs_length_m": 50.0, "rayleigh_length_m": 80.0, "rindex": 1.34, "lambda_nm": [300, 600],
           "source_point_m": [round(float(v), 4) for v in point], "time_bins": [200, 0.0, 1.0],
           "l2": "flushed between timed steps (256 MiB write)"}  # fmt: skip

    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return
        cb = cpu_reference(args, det, src, n)
        line = {"metric": METRIC, "value": cb["value"], "unit": "photons/s", "n_gpus": args.gpus,
                "steps": args.cpu_steps, "warmup": 1, "ms_per_step": 1e3 * args.cpu_photons / cb["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": cfg, "impl": "reference", "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "photons/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch

    from lumen_b200 import _abi as A
    from lumen_b200 import api, distributed
    from lumen_b200 import make as engine_build
    from lumen_b200.engine import DeviceSource, DeviceTallies, Engine

    world, rank, local = dist_setup(args)
    engine_build.build()
    dev = torch.device("cuda", local)
    eng = Engine(det, dev)
    key = A.key_of_seed(0)
    first, n_rank = distributed.shard_range(n * world, rank, world)  # this rank's contiguous photon ids
    ds = DeviceSource(src, n * world, dev)
    T = DeviceTallies(det.n_sensor, 1, 200, 0.0, 1.0, 0, dev)
    from lumen_b200 import autotune

    if args.variant < 0:  # the autotuner's pick on a sample of this rank's photons (src: the same photon law)
        shape, tune_ms = autotune.tune(eng, ds, min(n_rank, 1 << 22), (), 1, key)
    else:
        shape, tune_ms = autotune.Shape(args.variant), {}
    c = shape.controls(n_rank)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

    launches = []

    def one_step():
        T.zero_()
        distributed.trace_shard(eng, key, first, n_rank, source=ds, controls=c, tallies=T, stream=stream)
        launches.append(eng.launches)  # the library's own kernels this call launched
        distributed.all_reduce_tallies(T)  # one NCCL all-reduce of every tally (nothing with one rank)

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    # the clock sampler starts before the warm-up and samples on through the timed steps
    with Clocks(local) as clk:
        for k in range(args.warmup):
            flush.fill_(float(k))
            one_step()
        torch.cuda.synchronize(dev)
        clk.mark()
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize(dev)
        bounds = []  # each step's host-time interval (the device is idle between steps: a sync after each)
        for k in range(args.steps):
            flush.fill_(float(k))
            t_a = time.monotonic()
            ev[k][0].record(stream)
            one_step()
            ev[k][1].record(stream)
            torch.cuda.synchronize(dev)
            bounds.append((t_a, time.monotonic()))
        torch.cuda.synchronize(dev)
    ms = [a.elapsed_time(b) for a, b in ev]
    timed_launches = int(sum(launches[args.warmup:]))
    cnt = T.counts.cpu().numpy()
    ms_step = float(np.mean(ms))
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([ms_step], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_step = float(t.item())
    value = world * n / (ms_step * 1e-3)
    steps_pp = cnt[1] / max(cnt[0], 1)
    # the trace kernel's algorithmic bytes per launch (its own duration: the step without the all-reduce)
    alg = float(cnt[1]) * BYTES_STEP + float(cnt[0]) * BYTES_PHOTON + float(cnt[2]) * BYTES_DEPOSIT
    pk, pk_kind = peaks()
    ach = alg / (ms_step * 1e-3) / 1e9
    # e2e through the public call, host buffers in and out each step
    # (N > 1: the sharded call, every rank its share of world x n photons and one all-reduce; the slowest rank's time)
    e2e_ms = []
    for k in range(max(4, args.steps) + 1):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        if world > 1:
            light = distributed.simulate_sharded(det, src, samples=n * world, seed=0, time_bins=(200, 0.0, 1.0),
                                                 device=dev)  # fmt: skip
        else:
            light = api.simulate(det, src, samples=n, seed=0, time_bins=(200, 0.0, 1.0), device=dev)
        torch.cuda.synchronize(dev)
        if k:
            e2e_ms.append(1e3 * (time.perf_counter() - t0))
    e2e_med = float(np.median(e2e_ms))
    if world > 1:
        import torch.distributed as dist

        t = torch.tensor([e2e_med], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_med = float(t.item())
    h2d = det.pool.nbytes + 8 * 4 + 8 + 8 + 4  # the parameter pool and the source's event records
    d2h = (3 * det.n_sensor + det.n_sensor * 200 + 11) * 8 + 5 * 8
    e2e_v = world * n / (e2e_med * 1e-3)
    line = {"metric": METRIC, "value": value, "unit": "photons/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": cfg,
            "photon_steps_per_s": world * float(cnt[1]) / (ms_step * 1e-3), "steps_per_photon": steps_pp,
            "roofline": {"bound": "hbm", "achieved": ach, "peak": pk, "unit": "GB/s", "frac": ach / pk,
                         "traffic": (TRAFFIC_PER_STEP[shape.variant] * float(cnt[1])
                                     if shape.variant in TRAFFIC_PER_STEP else None), "peak_kind": pk_kind,
                         "algorithmic_bytes": alg,
                         "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum of this launch shape on "
                                         "2^20-photon calls of this workload (profiles/k_wave_cylinder_tank.md), per "
                                         "photon-step, times this step's photon-steps"},
            "e2e": {"value": e2e_v, "unit": "photons/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
            # the library's kernels launched in the timed steps (lumen_b200_last_launches: the trace's kernels or the
            # wavefront's rounds, and the moment table's pass)
            "gpu_launches": timed_launches, "launch_shape": shape.label(),
            "autotune_ms": {k: round(v, 3) for k, v in tune_ms.items()},
            "clocks": clk.summary(), "ms_steps": [round(x, 3) for x in ms],
            "sm_mhz_steps": clk.per_step(bounds), "mc_error": mc_error(T.arrival.cpu().numpy(),
                                                                       T.arrival2.cpu().numpy(), [n * world]),
            "arrivals_sum": float(light.arrivals.sum())}  # fmt: skip
    # the checker's comparisons, the other workloads and the CPU baseline: one GPU only (at N > 1 the other ranks would
    # wait for rank 0 in the closing barrier, and the GPUs are held for nothing)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["vs_checker"] = chi2_vs_checker(eng, det, src, 1)
    if rank == 0 and world == 1 and not args.no_extra:
        cpu = not args.no_cpu
        line["toy_tank"] = run_toy(dev, with_cpu=cpu)
        line["tank_fwd_adjoint"] = run_tank_adjoint(dev, src, n, with_cpu=cpu)
        line["batched_fwd_adjoint"] = run_batched(dev, det, with_cpu=cpu)
        line["lar_fwd_adjoint"] = run_lar(dev, args.lar_photons, with_cpu=cpu)
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_reference(args, det, src, n)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


if __name__ == "__main__":
    main()
