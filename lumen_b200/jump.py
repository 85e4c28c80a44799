"""The diffusion jump's data: a proven clearance grid per medium the jump can act in.

The jump (src/lumen/transport/fastpath.py) lets a photon at a bulk Rayleigh event walk its own scatterings inside a
ball around it with no geometry query; the ball must cross no surface. Its radius is read from a grid of lower bounds
of the distance to every surface (src/lumen/geometry/clearance.py:224 ``bound``), built here in float64 from the
navigator's own arrays:

- a volume whose box does not hold the node: the distance to that box (the solid lies inside it);
- else the minimum over the volume's leaves of a lower bound of the distance to the leaf's surfaces (a boolean's
  surface lies in the union of its leaves'): a plane's distance |n . y - h| / |n| (exact), a quadric
  f = y'Ay + 2b'y + c's the root r >= 0 of ||A|| r^2 + |grad f| r = |f| (f keeps its sign within r); a torus's
  |sqrt((rho - R)^2 + z^2) - r| in its canonical coordinates u = M (x - og), over ||M||;

minus the navigator's band at the grid's scale, rounded down to float32, at most ``cap`` (the largest half-width of
the medium's volumes: no point of it is farther from a surface). The device reads c(x) = clear[node] - |x - node| at
the node nearest x, again a lower bound (the distance is 1-Lipschitz), so any spacing gives a proven bound.

Which media and where (fastpath.py:116 ``prepare``): a medium whose only channel is Rayleigh; its volumes whose box
half-width is at least R_0 = 4 of its shortest Rayleigh lengths; spacing h = 2 R_0 lambda / sqrt(3) (coarsened until
the grid fits 64 MB of float32 nodes); not built where the largest clearance holds no ball of R_0 lambda.
"""

from __future__ import annotations

import math

import numpy as np

from lumen_b200 import geometry as G

R_0 = 4.0  # scattering lengths: the smallest ball a grid is built for (speed only)
GRID_BYTES = 1 << 26
GRID_COARSEN = 1.0 + 2.0**-20


def _leaf_bound(arrays, g, xl):
    """A lower bound of the distance from points xl (N, 3; the volume's frame) to leaf g's surfaces (float64)."""
    lf = np.asarray(arrays["leaf_f"][g], np.float64)
    li = arrays["leaf_i"][g]
    out = np.full(len(xl), np.inf)
    og = lf[0:3]
    if int(li[0]) == 2:  # a torus: |sqrt((rho - R)^2 + z^2) - r| in u = M (x - og), over ||M|| (clearance.py:17)
        M = lf[6:15].reshape(3, 3)
        u = (xl - og) @ M.T
        rho = np.hypot(u[:, 0], u[:, 1])
        du = np.abs(np.hypot(rho - lf[15], u[:, 2]) - lf[16])
        return du / float(np.linalg.norm(M, 2))
    for k in range(int(li[2])):
        p = np.asarray(arrays["plane_f"][int(li[1]) + k], np.float64)
        nn = max(float(np.linalg.norm(p[:3])), 1e-300)
        out = np.minimum(out, np.abs((xl - og) @ p[:3] - p[3]) / nn)
    if int(li[0]) == 1:
        A = lf[6:15].reshape(3, 3)
        b, c = lf[15:18], float(lf[18])
        y = xl - lf[3:6]
        f = np.einsum("ni,ij,nj->n", y, A, y) + 2.0 * (y @ b) + c
        gr = np.linalg.norm(2.0 * (y @ A.T + b), axis=1)
        an = float(np.max(np.abs(np.linalg.eigvalsh(0.5 * (A + A.T)))))
        af = np.abs(f)
        if an > 0.0:
            r = 2.0 * af / (gr + np.sqrt(gr * gr + 4.0 * an * af))
        else:
            r = np.where(gr > 0.0, af / np.maximum(gr, 1e-300), np.where(af > 0.0, np.inf, 0.0))
        out = np.minimum(out, r)
    return out


def clearance(arrays, lo, h, n, cap) -> np.ndarray:
    """The proven clearance (float32, shape n) at the nodes lo + h i, at most ``cap`` before the band."""
    n = np.asarray(n, np.int64)
    ijk = np.stack(np.meshgrid(*[np.arange(int(m)) for m in n], indexing="ij"), -1).reshape(-1, 3)
    x = np.asarray(lo, np.float64) + h * ijk
    out = np.full(len(x), float(cap))
    vf = np.asarray(arrays["vol_f"], np.float64)
    vi = arrays["vol_i"]
    kind_i = arrays["kind_i"]
    for v in range(int(arrays["n_vol"])):
        blo, bhi = vf[v, 12:15], vf[v, 15:18]
        o = np.maximum(np.maximum(blo - x, x - bhi), 0.0)
        d = np.sqrt(np.sum(o * o, 1))
        out = np.minimum(out, np.where(d > 0.0, d, np.inf))
        inside = np.flatnonzero(d == 0.0)
        if not len(inside):
            continue
        R, t = vf[v, 0:9].reshape(3, 3), vf[v, 9:12]
        xl = (x[inside] - t) @ R  # R^T (x - t): the volume's frame
        k = int(vi[v, 0])
        l0, nl = int(kind_i[k, 0]), int(kind_i[k, 1])
        cv = np.full(len(inside), np.inf)
        for g in range(l0, l0 + nl):
            cv = np.minimum(cv, _leaf_bound(arrays, g, xl))
        out[inside] = np.minimum(out[inside], cv)
    tri = np.asarray(arrays.get("mesh_tri64", np.zeros((0, 12))), np.float64)
    for s, c, _, _ in np.asarray(arrays.get("mesh_chunk", np.zeros((0, 4))), np.int64):
        # a mesh chunk: the distance to its box outside it, to its triangles' planes (a lower bound) inside it
        T = tri[s:s + c]
        blo, bhi = T[:, 0:9].reshape(-1, 3).min(0), T[:, 0:9].reshape(-1, 3).max(0)
        o = np.maximum(np.maximum(blo - x, x - bhi), 0.0)
        d = np.sqrt(np.sum(o * o, 1))
        inside = np.flatnonzero(d == 0.0)
        out = np.minimum(out, np.where(d > 0.0, d, np.inf))
        if len(inside):
            pl = np.abs(np.einsum("nki,ki->nk", x[inside, None, :] - T[None, :, 0:3], T[:, 9:12]))
            out[inside] = np.minimum(out[inside], pl.min(1))
    scale = float(np.max(np.abs(np.concatenate([lo, np.asarray(lo) + h * (n - 1)])))) + float(cap)
    band = G.BAND_ULPS_EPS * scale + G.BAND_FLOOR
    c = np.maximum(out - band, 0.0)
    c32 = c.astype(np.float32)
    up = c32.astype(np.float64) > c
    c32[up] = np.nextafter(c32[up], np.float32(0))
    return c32.reshape(tuple(n))


def prepare(arrays, vol_medium, media) -> dict:
    """The jump's arrays (``include/lumen_b200.h`` LumenSceneDesc jump fields) and a report per medium.

    ``vol_medium``: each volume's medium index; ``media``: per medium (eligible, shortest Rayleigh length m).
    """
    vf = np.asarray(arrays["vol_f"], np.float64)
    nv = int(arrays["n_vol"])
    lo_w, hi_w = vf[:nv, 12:15], vf[:nv, 15:18]
    half = 0.5 * np.min(hi_w - lo_w, 1)
    jf, ji, clear, report = [], [], [], []
    for m, (eligible, lam) in enumerate(media):
        if not eligible:
            continue
        vols = np.flatnonzero(np.asarray(vol_medium) == m)
        if lam <= 0.0 or not len(vols):
            report.append(dict(medium=m, built=False, why="no volume"))
            continue
        fire = vols[half[vols] >= R_0 * lam]
        if not len(fire):
            report.append(dict(medium=m, built=False, why="no volume holds the smallest jump"))
            continue
        h = 2.0 * R_0 * lam / math.sqrt(3.0)
        lo, hi = lo_w[fire].min(0), hi_w[fire].max(0)
        while True:
            n = np.floor((hi - lo) / h).astype(np.int64) + 2
            if 4 * int(np.prod(n)) <= GRID_BYTES:
                break
            h *= max((4.0 * float(np.prod(n)) / GRID_BYTES) ** (1.0 / 3.0), GRID_COARSEN)
        cap = float(half[vols].max())
        c = clearance(arrays, lo, h, n, cap)
        if float(c.max()) < R_0 * lam:
            report.append(dict(medium=m, built=False, why="the largest clearance holds no jump"))
            continue
        jf.append([*np.asarray(lo, np.float32), np.float32(h)])
        ji.append([m, *[int(x) for x in n], sum(x.size for x in clear), 0, 0, 0])
        clear.append(c.ravel())
        report.append(dict(medium=m, built=True, h=h, nodes=int(np.prod(n)), cap=cap, clear_max=float(c.max())))
    return dict(jump_f=np.asarray(jf, np.float32).reshape(-1, 4), jump_i=np.asarray(ji, np.int32).reshape(-1, 8),
                clear=np.concatenate(clear).astype(np.float32) if clear else np.zeros(0, np.float32),
                report=report)  # fmt: skip
