"""A built detector: geometry + optics flattened into the arrays of the C ABI, with its parameters by name.

``Detector`` mirrors what the reference's ``lumen.load`` gives (src/lumen/api.py:70 ``Detector``, ``params()``,
``sensor_table()``): the navigator arrays, the optics tables and the packed parameter values. The class rule follows
the reference's surface lookup (src/lumen/build/lookup.py:394 Optics: a class per placed volume's optical role, a row
per crossed class pair, a medium per class) and src/lumen/build/tracked.py:181 (sensor per volume).

    det = build(top, materials, borders=[...], skins={...}, sensors={"pmt": "PMT"})
    det.params()["media/Water/absorption"]      # a table (energies, values)
"""

from __future__ import annotations

import ctypes
import dataclasses
from dataclasses import dataclass, field

import numpy as np

from lumen_b200 import facets
from lumen_b200 import geometry as G
from lumen_b200 import jump as J
from lumen_b200 import optics as O

OUTSIDE = "OUT"
PRECISIONS = ("float32", "float64")


@dataclass
class SensorTable:
    """The sensors in the order of ``Light.arrivals`` (src/lumen/api.py:498 SensorTable)."""

    name: list
    group: list
    position: np.ndarray
    axis: np.ndarray


class InvalidValue(ValueError):  # noqa: N818 (the reference's name, src/lumen/build/values.py:52)
    """A parameter value outside what the detector's structure holds: outside its range, or not finite."""


# the admissible ranges of the values a run reads (src/lumen/_core/domains.py: FRACTION, POSITIVE / LENGTH, INDEX;
# a Mie asymmetry within MIE_G_MAX, src/lumen/rules/choices.py:99), by the table's role: a medium's tables (LUMEN_MI_*)
# and a surface row's columns (LUMEN_COL_*)
_DOMAINS = {"fraction": (0.0, 1.0), "positive": (0.0, np.inf), "index": (1.0, np.inf), "mie_g": (-0.999, 0.999)}
_MED_ROLES = {0: "index", 1: "positive", 2: "positive", 3: "positive", 4: "mie_g", 5: "mie_g", 6: "fraction",
              7: "positive", 8: "positive", 9: "positive", 10: "positive"}  # fmt: skip
_COL_ROLES = ("fraction", "fraction", "fraction", "fraction", "fraction", "fraction", "positive", "fraction", "index",
              "positive")  # fmt: skip


@dataclass
class Detector:
    """The flattened detector (see the module docstring)."""

    arrays: dict
    pool: np.ndarray
    params_index: dict  # parameter name -> table index
    sensors: SensorTable
    names: list
    classes: dict = field(default_factory=dict)
    groups: dict = field(default_factory=dict)  # sensor group -> sensor indices
    precision: str = "float32"  # the navigator's: "float32" or "float64" (src/lumen/rules/navigation.py:96)

    def with_precision(self, precision: str) -> Detector:
        """Return this detector with the navigator in ``precision`` ("float32" or "float64"): the reference's load
        option ``precision=`` (docs/dev/decisions.md:332). float64 runs the navigator (frames, boxes, leaves, roots,
        intervals, the band) and the photon's position in float64, the physics in float32."""
        if precision not in PRECISIONS:
            raise ValueError(f"precision {precision!r} is not one of {PRECISIONS}")
        return dataclasses.replace(self, precision=precision)

    @property
    def n_sensor(self) -> int:
        return len(self.sensors.name)

    def params(self) -> dict:
        """Return {name: (energies, values)} of every parameter table (src/lumen/api.py:70 Detector.params)."""
        out = {}
        for k, t in self.params_index.items():
            off, n = self.arrays["tab"][t]
            out[k] = (self.pool[off:off + n].copy(), self.pool[off + n:off + 2 * n].copy())
        return out

    def check_values(self, pool: np.ndarray, what: str = "values") -> None:
        """Raise ``InvalidValue`` naming the first parameter of ``pool`` outside its admissible range, or not finite
        (src/lumen/build/values.py:235 ``_check_params``: a concrete value is refused; the ranges of
        src/lumen/_core/domains.py, both ends included). The C ABI refuses the same values (LUMEN_ERR_ARG)."""  # noqa: D205
        a = self.arrays
        tab = np.asarray(a["tab"]).reshape(-1, 2)
        med = np.asarray(a["med_i"]).reshape(-1, 16)
        rows = np.asarray(a["row_i"]).reshape(-1, 16)
        name = {t: k for k, t in self.params_index.items()}
        roles = [(t, r) for m in med for t, r in zip(m[list(_MED_ROLES)], _MED_ROLES.values(), strict=True)]
        roles += [(t, r) for ri in rows for t, r in zip(ri[6:6 + len(_COL_ROLES)], _COL_ROLES, strict=True)]
        for t, role in roles:
            if t < 0:
                continue
            off, k = tab[t]
            e, v = pool[off:off + k], pool[off + k:off + 2 * k]
            label = name.get(int(t), f"table {int(t)}")
            if not (np.all(np.isfinite(e)) and np.all(np.diff(e) > 0)):
                raise InvalidValue(f"{what}: {label}: its knot energies must be finite and strictly ascending")
            lo, hi = _DOMAINS[role]
            if not np.all(np.isfinite(v) & (v >= lo) & (v <= hi)):
                bad = v[~(np.isfinite(v) & (v >= lo) & (v <= hi))][0]
                raise InvalidValue(f"{what}: {label} has a value outside [{lo}, {hi}] or not finite ({bad})")

    def pool_with(self, values: dict | None) -> np.ndarray:
        """Return the pool with some parameters replaced: {name: constant or values array (same knots)}."""
        p = self.pool.copy()
        for k, v in (values or {}).items():
            t = self.params_index[k]
            off, n = self.arrays["tab"][t]
            p[off + n:off + 2 * n] = np.broadcast_to(np.asarray(v, np.float32), (n,))
        return p

    def sensor_table(self) -> SensorTable:
        return self.sensors

    # ------------------------------------------------------------------------------------ the C ABI's descriptor
    def desc(self):
        """Return (LumenSceneDesc, keepalive) over this detector's arrays (host pointers)."""
        from lumen_b200._abi import LumenSceneDesc, dptr, fptr, iptr

        a = self.arrays
        keep = {k: np.ascontiguousarray(v) for k, v in a.items() if isinstance(v, np.ndarray)}
        keep["pool"] = np.ascontiguousarray(self.pool, np.float32)
        d = LumenSceneDesc()
        d.n_vol, d.n_kind, d.n_leaf = a["n_vol"], len(keep["kind_i"]), len(keep["leaf_i"])
        d.n_plane, d.n_prog, d.n_node = len(keep["plane_f"]), len(keep["prog_i"]), len(keep["node_i"])
        d.n_item, d.n_cand = len(keep["items"]), len(keep["cand"])
        d.vol_i, d.vol_f, d.cand = iptr(keep["vol_i"]), fptr(keep["vol_f"]), iptr(keep["cand"])
        d.node_f, d.node_i, d.items = fptr(keep["node_f"]), iptr(keep["node_i"]), iptr(keep["items"])
        d.kind_i, d.leaf_f, d.leaf_i = iptr(keep["kind_i"]), fptr(keep["leaf_f"]), iptr(keep["leaf_i"])
        d.plane_f, d.prog_i = fptr(keep["plane_f"]), iptr(keep["prog_i"])
        if a.get("n_mesh", 0):  # tessellated meshes: triangles, chunks and the chunks' boxes
            d.n_mesh, d.n_chunk, d.n_tri = a["n_mesh"], len(keep["mesh_chunk"]), len(keep["mesh_tri"])
            d.mesh_tri, d.mesh_tri64 = fptr(keep["mesh_tri"]), dptr(keep["mesh_tri64"])
            d.mesh_chunk, d.chunk_box, d.chunk_box64 = iptr(keep["mesh_chunk"]), fptr(keep["chunk_box"]), dptr(keep["chunk_box64"])
        if a.get("n_group", 0):  # frame groups: their node ranges and frames
            d.n_group = a["n_group"]
            d.group_i, d.group_r, d.group_r64 = iptr(keep["group_i"]), fptr(keep["group_r"]), dptr(keep["group_r64"])
        if self.precision == "float64":  # the float64 navigator's arrays
            d.precision = 1
            d.vol_f64, d.node_f64 = dptr(keep["vol_f64"]), dptr(keep["node_f64"])
            d.leaf_f64, d.plane_f64 = dptr(keep["leaf_f64"]), dptr(keep["plane_f64"])
        d.reach = ctypes.c_float(a["reach"])
        if a.get("cls_born") is not None:  # sensors counting the photons born inside them: each class's entry class
            d.cls_born = iptr(keep["cls_born"])
        if a.get("pair_pre") is not None:  # exit sensors: the class pairs whose deposit goes to the volume left
            d.pair_pre = iptr(keep["pair_pre"])
        d.n_cls, d.n_med, d.n_row = a["n_cls"], len(keep["med_i"]), len(keep["row_i"])
        d.n_tab, d.n_pool, d.n_sensor = len(keep["tab"]), len(keep["pool"]), self.n_sensor
        d.cls_medium, d.row_of, d.med_i = iptr(keep["cls_medium"]), iptr(keep["row_of"]), iptr(keep["med_i"])
        d.row_i, d.tab, d.pool = iptr(keep["row_i"]), iptr(keep["tab"]), fptr(keep["pool"])
        if self.draws_facets:  # a unified facet row (reflect, not about the global normal): the lobe's tables
            keep["unified"] = facets.flat()
            d.unified = fptr(keep["unified"])
        r = G.reach_arrays(a)  # the sensor reach of bulk steps' queries
        for k, v in r.items():
            keep[k] = v
        d.n_comp, d.n_fnode = len(r["comp_box"]), len(r["fnode_i"])
        d.comp, d.comp_box = iptr(keep["comp"]), fptr(keep["comp_box"])
        d.fnode_f, d.fnode_i = fptr(keep["fnode_f"]), iptr(keep["fnode_i"])
        d.n_jump, d.n_clear = len(keep["jump_i"]), len(keep["clear"])
        d.jump_f, d.jump_i, d.clear = fptr(keep["jump_f"]), iptr(keep["jump_i"]), fptr(keep["clear"])
        return d, keep

    @property
    def draws_facets(self) -> bool:
        """Whether a surface row draws the unified facet lobe (its density reads the unified tables)."""
        r = self.arrays["row_i"].reshape(-1, 16)
        return bool(((r[:, 0] == 0) & (r[:, 1] == 0) & (r[:, 2] == 0)).any())


def build(top: G.Volume, materials: dict, *, borders=(), skins=None, sensors=None, prio=None,
          after_tracking=(), precision="float32", frame_groups=True, born=()) -> Detector:
    """Return the Detector of the volume tree ``top`` (the detector volume, placed at the origin).

    ``materials``: {name: Material}. ``borders``: [(pv from, pv to, OpticalSurface)] (Geant4 border surfaces, ordered);
    ``skins``: {lv name: OpticalSurface}. ``sensors``: {group: lv name}: every placement of that logical volume is a
    sensor, counted where a crossing's surface into it deposits (the ``border_into`` rule), and where a border out of
    it whose surface has an EFFICIENCY detects (an exit sensor, credited to the volume left). Light that leaves ``top``
    is absorbed there (the detector volume's boundary, as the reference's recipe ``detector_volume``).
    ``after_tracking``: sensor groups whose sensor model applies its QE after tracking: their rows detect every
    absorption (eff 1) and are read per normal incidence (types.py:576 per_normal: a deposit carries 1 / A_n, by
    which a normalising readout grid divides it). ``precision``: the navigator's ("float32", or "float64":
    ``Detector.with_precision``). ``frame_groups``: daughters sharing a rotation get a BVH in its frame where that
    pays (the navigator's speed only; the same results). ``born``: sensor groups that count a photon emitted inside
    their volumes at its emission, with what their entry from the mother volume detects (Geant4's sensitive detector
    counting every step in the volume: src/lumen/rules/sensors.py:39 counts_born, Optics.born_pair).
    """
    skins = skins or {}
    sensors = sensors or {}
    sensor_lv = {lv: g for g, lv in sensors.items()}
    # the volumes, then the meshes (G4TessellatedSolid placements: navigator pseudo-volumes after the outside)
    flat = G.flatten(top)
    is_mesh = [isinstance(p.lv.solid, G.Mesh) for p in flat]
    vol_idx = [i for i, m in enumerate(is_mesh) if not m]
    mesh_idx = [i for i, m in enumerate(is_mesh) if m]
    new_of = {old: new for new, old in enumerate(vol_idx)}
    for i in mesh_idx:
        p = flat[i]
        if p.lv.daughters:
            raise ValueError(f"mesh {p.name!r} has daughters: a mesh holds no point (src/lumen/geometry/navigator_build.py:131)")
        if p.lv.name in sensor_lv:
            raise ValueError(f"mesh {p.name!r} is a sensor: a mesh reports only its first hit")
        if materials[p.lv.material].rindex is not None:
            raise ValueError(f"mesh {p.name!r}: its material {p.lv.material!r} has a RINDEX; the navigator does not track "
                             "inside a mesh (an opaque part: no RINDEX, its surfaces reflect or absorb)")
        if p.parent < 0:
            raise ValueError("the top volume is a mesh")
    placed = [dataclasses.replace(flat[i], parent=new_of.get(flat[i].parent, -1)) for i in vol_idx]
    meshes = [(np.einsum("ij,nkj->nki", flat[i].R, flat[i].lv.solid.tris) + flat[i].t, new_of[flat[i].parent])
              for i in mesh_idx]  # fmt: skip
    everything = placed + [flat[i] for i in mesh_idx]
    n = len(placed)
    names = [p.name for p in placed]
    by_name = {p.name: i for i, p in enumerate(everything)}
    # optical roles -> classes (the outside is class 0's neighbour: its own class)
    roles = [set() for _ in everything]
    for a, b, s in borders:
        roles[by_name[a]].add((s.name, "from"))
        roles[by_name[b]].add((s.name, "to"))
    keys = []
    for i, p in enumerate(everything):
        keys.append((p.lv.name, p.lv.material, tuple(sorted(roles[i])), p.lv.name in skins, p.lv.name in sensor_lv))
    cls_of_key, vol_cls, cls_lv, cls_mat = {}, [], [], []
    for i, k in enumerate(keys):
        if k not in cls_of_key:
            cls_of_key[k] = len(cls_of_key)
            cls_lv.append(everything[i].lv)
            cls_mat.append(everything[i].lv.material)
        vol_cls.append(cls_of_key[k])
    out_cls = len(cls_of_key)
    n_cls = out_cls + 1
    # sensors: every placement of a sensor LV, in the walk's order
    vol_sensor = np.full(len(placed), -1, np.int32)
    s_name, s_group, s_pos, s_axis, groups = [], [], [], [], {}
    for i, p in enumerate(placed):
        g = sensor_lv.get(p.lv.name)
        if g is not None:
            vol_sensor[i] = len(s_name)
            groups.setdefault(g, []).append(len(s_name))
            s_name.append(p.name)
            s_group.append(g)
            s_pos.append(p.t)
            s_axis.append(p.R[:, 2])
    if prio is not None:  # the rule's order given per placement of the walk (and the outside last)
        prio = np.asarray([prio[i] for i in vol_idx] + [prio[len(flat)]])
    nav = G.navigator_arrays(placed, vol_cls[:n], out_cls, vol_sensor, prio, meshes=meshes, mesh_cls=vol_cls[n:],
                             use_frame_groups=frame_groups)  # fmt: skip
    # media
    pool = O.Pool()
    med_names = sorted(set(cls_mat))
    med_i = np.full((len(med_names), 16), -1, np.int32)
    opaque = {}
    for m, name in enumerate(med_names):
        mat = materials[name]
        opaque[name] = mat.rindex is None
        if mat.rindex is not None:
            med_i[m, 0] = pool.add(mat.rindex, f"media/{name}/index")
        if mat.abslength is not None:
            med_i[m, 1] = pool.add(mat.abslength, f"media/{name}/absorption")
        ray = mat.rayleigh
        if ray is None and name.split("0x")[0] == "Water" and mat.rindex is not None:
            ray = O.water_rayleigh(O.table(mat.rindex))
        if ray is not None and mat.rindex is not None:
            med_i[m, 2] = pool.add(ray, f"media/{name}/rayleigh")
        if mat.mie is not None and mat.rindex is not None:  # G4OpMieHG: the length and the lobe's constants
            med_i[m, 3] = pool.add(mat.mie, f"media/{name}/mie")
            med_i[m, 4] = pool.add(float(mat.mie_forward), f"media/{name}/mie_g_forward")
            med_i[m, 5] = pool.add(float(mat.mie_backward), f"media/{name}/mie_g_backward")
            med_i[m, 6] = pool.add(float(mat.mie_forward_ratio), f"media/{name}/mie_forward_ratio")
            med_i[m, 12] = 1  # the ratio is a parameter: the lobe choice is a defensive part (api.py:797 _edge_rows)
        if mat.wls is not None and mat.rindex is not None:  # G4OpWLS: the absorption length and the emission
            med_i[m, 7] = pool.add(mat.wls, f"media/{name}/wls")
            med_i[m, 8] = pool.add(float(mat.wls_mean), f"media/{name}/wls_yield")
            med_i[m, 9] = pool.add(float(mat.wls_tau), f"media/{name}/wls_tau")
            med_i[m, 10] = pool.add(tuple(np.asarray(x, np.float64) for x in mat.wls_spectrum), f"media/{name}/wls_spectrum")
            med_i[m, 11] = 1 if mat.wls_profile == "exponential" else 0
        if mat.scint_components:  # a scintillation source's tables (sources.ScintillationPoint reads them by name)
            pool.add(float(mat.scint_yield), f"media/{name}/scint_yield")
            for i, comp in enumerate(mat.scint_components, 1):
                pool.add(tuple(np.asarray(x, np.float64) for x in comp["spectrum"]), f"media/{name}/scint_spectrum{i}")
                pool.add(float(comp["tau"]), f"media/{name}/scint_tau{i}")
                if comp.get("rise") is not None:
                    pool.add(float(comp["rise"]), f"media/{name}/scint_rise{i}")
            for i, y in enumerate(mat.scint_shares or (), 1):
                pool.add(float(y), f"media/{name}/scint_share{i}")
    mi_of = {n: i for i, n in enumerate(med_names)}
    cls_medium = np.asarray([mi_of[m] for m in cls_mat] + [mi_of[cls_mat[0]] if cls_mat else 0], np.int32)
    # surface rows per crossed class pair
    neutral = {c: pool.add(v) for c, v in O.NEUTRAL.items()}
    rows, row_key, row_of = [], {}, np.full((n_cls, n_cls), -1, np.int32)
    # (mother class, daughter class) of every placement: a volume's and a mesh's (whose mother is a volume)
    daughter_of = {(vol_cls[p.parent], vol_cls[i]) for i, p in enumerate(placed) if p.parent >= 0}
    daughter_of |= {(vol_cls[new_of[flat[j].parent]], vol_cls[n + k]) for k, j in enumerate(mesh_idx)}
    border_of = {}
    # exit sensors: a border out of a sensor's volume whose surface has an EFFICIENCY detects there, its deposit
    # credited to the volume left (src/lumen/rules/boundary.py:92, the surface's own EFFICIENCY)
    exit_pairs = set()
    for a, b, s in borders:
        border_of[(vol_cls[by_name[a]], vol_cls[by_name[b]])] = s
        if everything[by_name[a]].lv.name in sensor_lv and s.efficiency is not None:
            exit_pairs.add((vol_cls[by_name[a]], vol_cls[by_name[b]]))
    pair_pre = np.zeros((n_cls, n_cls), np.int32)
    for ca, cb in exit_pairs:
        pair_pre[ca, cb] = 1
    for ca in range(n_cls):
        for cb in range(n_cls):
            if ca == cb:
                continue
            into_out = cb == out_cls
            from_out = ca == out_cls
            far_opq = into_out or opaque[cls_mat[cb]]
            surf = border_of.get((ca, cb))
            # the skins: the entered daughter's first, then its mother's; otherwise the volume left's first
            # (G4OpBoundaryProcess's enteredDaughter; src/lumen/rules/boundary.py:61-66)
            sides = [(cb, into_out), (ca, from_out)] if (ca, cb) in daughter_of else [(ca, from_out), (cb, into_out)]
            for c, out in sides:
                if surf is None and not out and cls_lv[c].name in skins:
                    surf = skins[cls_lv[c].name]
            is_sensor = (not into_out) and cls_lv[cb].name in sensor_lv
            per_normal = int(is_sensor and sensor_lv[cls_lv[cb].name] in set(after_tracking))
            if (ca, cb) in exit_pairs:  # an exit sensor's crossing: the surface's EFFICIENCY, no entry rule
                is_sensor, per_normal = True, 0
            if surf is not None and far_opq and O.kills_far_side(surf):  # NoRINDEX before the draw: the absorber
                surf, is_sensor, per_normal = O.ABSORBER, False, 0
            if surf is None:
                if into_out or from_out or opaque[cls_mat[cb]] or opaque[cls_mat[ca]]:
                    surf = O.ABSORBER  # the detector volume's boundary; Geant4's NoRINDEX
                else:
                    surf = O.OpticalSurface("__fresnel__", "dielectric_dielectric", "polished")
            key = (surf.name, is_sensor, far_opq, id(surf), per_normal)
            if key not in row_key:
                row = O.surface_row(surf, is_sensor, far_opq, 1.0 if per_normal else None)
                row.sensor = is_sensor
                row.per_normal = per_normal
                if surf is O.ABSORBER:  # the reference's ABSORBER type: no outcome, no parameter (types.py:441)
                    row.cover = 0
                row_key[key] = len(rows)
                rows.append(row)
            row_of[ca, cb] = row_key[key]
    row_i = np.zeros((len(rows), 16), np.int32)
    col_tab = {}  # one table per (surface, column): every row of a surface reads (and moves with) the same values
    for r, row in enumerate(rows):
        row_i[r, 0:6] = [row.model, row.normal, row.glisur, row.far_opaque, row.per_normal, row.cover]
        for c, col in enumerate(O.COLUMNS):
            if col not in row.cols or (col == "eff" and not row.sensor):
                row_i[r, 6 + c] = neutral[col]
                continue
            if col == "eff" and row.per_normal:  # every absorption entering is counted: eff 1, not a parameter
                row_i[r, 6 + c] = pool.add(1.0)
                continue
            k = (row.name, col)
            if k not in col_tab:
                col_tab[k] = pool.add(row.cols[col], None if row.name.startswith("__") else f"surfaces/{row.name}/{col}")
            row_i[r, 6 + c] = col_tab[k]
    st = SensorTable(s_name, s_group, np.asarray(s_pos).reshape(-1, 3), np.asarray(s_axis).reshape(-1, 3))
    cls_names = {i: cls_lv[i].name for i in range(out_cls)} | {out_cls: OUTSIDE}
    # sensors counting the photons born inside them: each such sensor class's entry, the class of its volumes'
    # mother (the crossing whose detection the emission deposits)
    cls_born = np.full(n_cls, -1, np.int32)
    for g in born:
        lv = sensors[g]
        for c in range(out_cls):
            if cls_lv[c].name != lv:
                continue
            mothers = sorted(b for b, d in daughter_of if d == c)
            if not mothers:
                raise ValueError(f"sensor group {g!r}: its volumes have no mother volume to enter from")
            cls_born[c] = mothers[0]
    return assemble(nav, vol_cls[:n], n_cls, cls_medium, row_of, med_i, row_i, pool, st, names, cls_names, groups,
                    precision, cls_born, pair_pre)  # fmt: skip


def assemble(nav: dict, vol_cls, n_cls: int, cls_medium, row_of, med_i, row_i, pool: O.Pool, sensors: SensorTable,
             names: list, cls_names: dict, groups: dict, precision: str = "float32", cls_born=None,
             pair_pre=None) -> Detector:
    """Return the Detector of navigator arrays ``nav`` (``geometry.navigator_arrays``, volumes of classes ``vol_cls``)
    and the surface lookup's tables: per class its medium (``cls_medium``), per crossed class pair its surface row
    (``row_of`` (C, C), -1 never crossed), the media's (``med_i``) and rows' (``row_i``) table indices into ``pool``;
    then the diffusion jump's clearance grids of the media whose only channel is Rayleigh
    (src/lumen/transport/fastpath.py:96). ``cls_born``: per class the entry class of a sensor that counts the photons
    born inside it (-1 none; None: no such sensor); ``pair_pre`` (C, C): 1 where a crossing's deposit goes to the
    sensor of the volume left (an exit sensor; None: none)."""  # noqa: D205, D209
    params_index = dict(pool.names)
    tab, data = pool.arrays()
    arrays = dict(nav)
    arrays.update(n_cls=int(n_cls), cls_medium=np.asarray(cls_medium, np.int32),
                  row_of=np.asarray(row_of).ravel().astype(np.int32), med_i=np.asarray(med_i, np.int32),
                  row_i=np.asarray(row_i, np.int32), tab=tab)  # fmt: skip
    if cls_born is not None and np.any(np.asarray(cls_born) >= 0):
        arrays["cls_born"] = np.asarray(cls_born, np.int32)
    if pair_pre is not None and np.any(np.asarray(pair_pre)):
        arrays["pair_pre"] = np.asarray(pair_pre, np.int32).ravel()
    media = []
    for m in range(len(med_i)):
        ok = med_i[m, 0] >= 0 and med_i[m, 2] >= 0 and med_i[m, 3] < 0 and med_i[m, 7] < 0
        lam = 0.0
        if ok:
            off, k = tab[med_i[m, 2]]
            lam = float(np.min(data[off + k:off + 2 * k].astype(np.float64)))
        media.append((ok, lam))
    jp = J.prepare(arrays, arrays["cls_medium"][np.asarray(vol_cls, np.int64)], media)
    arrays.update(jump_f=jp["jump_f"], jump_i=jp["jump_i"], clear=jp["clear"], jump_report=jp["report"])
    return Detector(arrays, data, params_index, sensors, names, cls_names, groups).with_precision(precision)
