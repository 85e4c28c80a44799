"""The unified facet lobe's tables: the facing share F and log zeta = log(Z / sigma^2), float64 quadrature stored
float32 with the grid derivatives a C1 bicubic (F) and cubic (log zeta) Hermite reads.

Geant4's unified facet draw (G4OpBoundaryProcess::GetFacetNormal) tilts the facet by alpha ~ N(0, sigma) kept where
``u f_max <= sin alpha`` and alpha < pi / 2, f_max = min(1, 4 sigma), azimuth uniform, redrawn while the facet faces
away from the photon. Per solid angle of the facet m the photon meets

    D(m) [V . m > 0] / F(theta, sigma),   D(m) = exp(-alpha^2 / 2 sigma^2) min(1, f_max / sin alpha) / (2 pi Z),

Z(sigma) = int_0^{pi/2} exp(-a^2 / 2 sigma^2) min(sin a, f_max) da and F the share of facets that face a photon at
incidence theta. One mirror reflection off a facet then has density D(h) / (4 F V . h) in the outgoing direction
(h the half vector). The reference tabulates F and log zeta on one grid (src/lumen/surfaces/facets.py:127
``unified_tables``, resolution in src/lumen/rules/choices.py:101 ``UNIFIED_TABLE``):

- x = (2 / pi) atan2(cos theta, sigma sin theta) on NX = 257 uniform nodes of [0, 1];
- y = log sigma = log(1/4) + j log(2) / 8, j in [-52, 16] (sigma in [0.00276, 1] rad);
- the node derivatives by central differences of the quadrature (step 1e-5, one-sided 1e-6 at the x ends), the
  mixed one by second-order differences of Fx along y.

This module computes the same tables with its own composite Gauss-Legendre quadrature of the same integrals (16
points on 64 panels for Z, 16 on 16 panels for each of F's two pieces, the integrands cut at 14 sigma), in the same
layout, so that a caller may pass either these or the reference's own ``unified_tables()`` to the engine.
"""

from __future__ import annotations

import functools
import math

import numpy as np

NX = 257
J_LO, J_HI = -52, 16
NY = J_HI - J_LO + 1
Y0 = math.log(0.25)
DY = math.log(2.0) / 8.0
SIGMA_MIN = math.exp(Y0 + DY * J_LO)  # 0.00276 rad
SIGMA_MAX = math.exp(Y0 + DY * J_HI)  # 1 rad
ORDER, PANELS_Z, PANELS_F, CUT = 16, 64, 16, 14.0
FD, FD_END = 1e-5, 1e-6
WORDS = 4 * NX * NY + 2 * NY  # the engine's flat layout: F, Fx, Fy, Fxy (NX x NY, row-major), lz, lzy (NY)


def _nodes(a, b, panels):
    """Composite Gauss-Legendre on [a, b] for arrays a, b: (nodes, weights), the quadrature on the last axis."""
    g, gw = np.polynomial.legendre.leggauss(ORDER)
    a = np.asarray(a, np.float64)[..., None]
    b = np.asarray(b, np.float64)[..., None]
    k = np.arange(panels)
    h = (b - a) / panels  # panel width
    c = a + (k + 0.5) * h  # panel centres
    x = c[..., :, None] + 0.5 * h[..., :, None] * g
    w = np.broadcast_to(0.5 * h[..., :, None] * gw, x.shape)
    return x.reshape(*x.shape[:-2], -1), w.reshape(*w.shape[:-2], -1)


def _tilt(a, sigma):
    """The unnormalised tilt density exp(-a^2 / 2 sigma^2) min(sin a, f_max)."""
    return np.exp(-(a * a) / (2.0 * sigma * sigma)) * np.minimum(np.sin(a), min(1.0, 4.0 * sigma))


def norm_z(sigma: float) -> float:
    """Z(sigma): the tilt density's integral over (0, pi/2), split where min(sin a, f_max) switches branch."""
    top = min(0.5 * math.pi, CUT * sigma)
    kink = min(math.asin(min(1.0, 4.0 * sigma)), top)
    z = 0.0
    for a, b in ((0.0, kink), (kink, top)):
        if b > a:
            x, w = _nodes(a, b, PANELS_Z)
            z += float(np.sum(w * _tilt(x, sigma)))
    return z


def facing(x, sigma: float):
    """F at table coordinate x (array) and width sigma: the share of facets facing a photon at incidence theta.

    With c = cot theta = sigma tan(pi x / 2), every facet tilted below a_k = atan(c) faces the photon; a facet tilted
    by a > a_k faces away on the azimuth share acos(c cot a) / pi. Over a = a_k + (top - a_k) t^2 the square-root edge
    at a_k is smooth in t, and the f_max kink (a = asin f_max) is a panel edge.
    """
    x = np.asarray(x, np.float64)
    inf = x >= 1.0
    c = np.where(inf, np.inf, sigma * np.tan(0.5 * math.pi * np.minimum(x, 1.0)))
    ak = np.arctan(c)
    span = np.minimum(0.5 * math.pi, ak + CUT * sigma) - ak
    kink = math.asin(min(1.0, 4.0 * sigma))
    tk = np.sqrt(np.clip((kink - ak) / np.where(span > 0.0, span, 1.0), 0.0, 1.0))
    away = np.zeros_like(x)
    for lo, hi in ((np.zeros_like(x), tk), (tk, np.ones_like(x))):
        t, w = _nodes(lo, hi, PANELS_F)
        a = ak[..., None] + span[..., None] * t * t
        cot = np.cos(a) / np.sin(a)
        arg = np.where(inf[..., None], 1.0, np.clip(c[..., None] * cot, -1.0, 1.0))
        away += np.sum(w * _tilt(a, sigma) * (np.arccos(arg) / math.pi) * (2.0 * span[..., None] * t), -1)
    return 1.0 - away / norm_z(sigma)


def _log_zeta(y: float) -> float:
    return math.log(norm_z(math.exp(y)) / math.exp(2.0 * y))


@functools.lru_cache(maxsize=None)
def tables() -> dict:
    """The float32 tables {F, Fx, Fy, Fxy: (NX, NY); lz, lzy: (NY,)} (a few seconds; cached per process)."""
    xs = np.linspace(0.0, 1.0, NX)
    ys = Y0 + DY * np.arange(J_LO, J_HI + 1)
    xp = np.minimum(xs + FD, 1.0)
    xm = np.maximum(xs - FD, 0.0)
    xp[0], xm[-1] = FD_END, 1.0 - FD_END
    F = np.empty((NX, NY))
    Fx = np.empty((NX, NY))
    Fy = np.empty((NX, NY))
    lz = np.empty(NY)
    lzy = np.empty(NY)
    for j, y in enumerate(ys):
        s = math.exp(y)
        F[:, j] = facing(xs, s)
        Fx[:, j] = (facing(xp, s) - facing(xm, s)) / (xp - xm)
        Fy[:, j] = (facing(xs, math.exp(y + FD)) - facing(xs, math.exp(y - FD))) / (2.0 * FD)
        lz[j] = _log_zeta(y)
        lzy[j] = (_log_zeta(y + FD) - _log_zeta(y - FD)) / (2.0 * FD)
    Fxy = np.gradient(Fx, DY, axis=1, edge_order=2)
    out = dict(F=F, Fx=Fx, Fy=Fy, Fxy=Fxy, lz=lz, lzy=lzy)
    return {k: np.ascontiguousarray(v, np.float32) for k, v in out.items()}


def flat(t: dict | None = None) -> np.ndarray:
    """The tables in the engine's flat layout (WORDS float32): F, Fx, Fy, Fxy (i * NY + j), then lz, lzy.

    ``t`` may be the reference's own ``lumen.surfaces.facets.unified_tables()`` (the same keys and shapes).
    """
    t = tables() if t is None else t
    parts = [np.asarray(t[k], np.float32).reshape(-1) for k in ("F", "Fx", "Fy", "Fxy", "lz", "lzy")]
    f = np.concatenate(parts)
    if f.size != WORDS:
        raise ValueError(f"unified tables: {f.size} values, expected {WORDS}")
    return f
