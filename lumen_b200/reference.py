"""Detectors from the reference's own host pipeline: a loaded ``lumen.Detector`` as this package's ``Detector``.

    data = reference.export(ref_det)     # the reference's compiled products as plain data (JSON-able)
    det = reference.detector(data)       # a lumen_b200.detector.Detector: simulate(det, ...) runs it
    det = reference.from_reference(ref_det)

``ref_det`` is what ``lumen.load(path)`` returns (src/lumen/api.py:310). ``export`` reads the products the reference's
photon loop is built from, and re-derives none of them:

- the navigator's scene (``Parts.nav_scene``; ``scene.instances``, src/lumen/geometry/scene.py:151): every instance
  of a definition with a member is a navigator volume (its world pose composed by the reference's walk, its parent
  the nearest such ancestor), each member's solid as the reference flattens it (``solids.Compiled``,
  src/lumen/geometry/solids.py:200: the transforms baked into the leaves, one origin for the solid's quadric leaves,
  coplanar planes made identical) with its box (``solids.node_bbox``); a tessellated member (``scene.Mesh``) as its
  world triangles and mother, the navigator's opaque pseudo-volume;
- the compiled optics (``lookup.Optics``, src/lumen/build/lookup.py:394): the class of every placed volume by its PV
  path, the medium of every class, the surface row of every crossed class pair (``row_of``), each row's Interaction,
  flags and outcome support (``lookup.SurfaceTable``, lookup.py:360), the sensor tags;
- the packed parameters at the detector's own values (``pack.pack``, src/lumen/build/pack.py:84): each row's column
  and each medium's tables, float32 as the reference's step reads them;
- the defensive rows (``api._edge_rows``, src/lumen/api.py:797): a row the estimator covers gets its support as its
  cover mask;
- the parameter keys (``Parts.key_rows``): a table read directly from a key is named by the key
  ("materials/Water/ABSLENGTH", "surfaces/Liner/REFLECTIVITY"), so ``simulate(det, src, params={key: ...})`` and its
  ``gradients`` take the reference's names; a table with no key of its own keeps this package's name
  ("media/Water/rayleigh": a table derived from RINDEX; "surfaces/<surface>/<column>").

``detector`` then builds this package's navigator arrays (a BVH per volume over the same leaves and poses) and the C
ABI's tables from that data: the reference's classes, media, rows and values, one table per key. The leaves and
values are the reference's bits; the navigator's arrays are this package's layout of them.

A split union's pieces (``Definition.piece_of``: a union of many leaves placed as its pieces) are volumes of their
union's class. Refused (``NotImplementedError`` naming the part), where the photon loop here has no counterpart: a
medium channel other than Rayleigh, Mie (G4OpMieHG) and a WLS (G4OpWLS) with its
own spectrum and a delta or exponential profile, and a vertex on the class table's diagonal (a skin between touching
volumes of one class). Sensors that count the photons born inside them (``Optics.born_pair``) carry their entry
class per class (``LumenSceneDesc.cls_born``), exit sensors (``Optics.deposit_pre``) the class pairs whose deposit
goes to the volume left (``LumenSceneDesc.pair_pre``). A pass row
(``types.PASS``: two classes of one medium split by a role elsewhere) becomes a row that carries the photon straight
on: the reference steps over such a crossing, this navigator stops at it and continues it unchanged, so the two draw
other random numbers for the same law (the same expected values).
"""

from __future__ import annotations

import gzip
import json

import numpy as np

from lumen_b200 import detector as D
from lumen_b200 import geometry as G
from lumen_b200 import optics as O

FORMAT = "lumen_b200-reference-detector/1"
OUTSIDE_PV = "<outside>"  # the outside's PV name in the reference's class table (src/lumen/build/tree.py OUTSIDE_PV)
MODELS = {"g4.reflect": O.MODEL_REFLECT, "g4.dielectric": O.MODEL_DIELECTRIC, "g4.complex": O.MODEL_COMPLEX}
GLISUR_LOBES = {"glisur": 1, "glisur_dielectric": 2}  # GLISUR_METAL, GLISUR_DIELECTRIC (src/lumen/surfaces/types.py)
OPS = {"union": 1, "inter": 2, "sub": 3}  # the postfix program's opcodes (include/lumen_b200.h)
DIRECT = ("value", "constant", "setting", "default")  # key_rows columns read from a key as they are (build/pack.py)
# the medium record's table slots in order (include/lumen_b200.h LUMEN_MI_*; this package's names of the tables)
MEDIUM_PARTS = ("index", "absorption", "rayleigh", "mie", "mie_g_forward", "mie_g_backward", "mie_forward_ratio", "wls",
                "wls_yield", "wls_tau", "wls_spectrum")


# ------------------------------------------------------------------------------------------------------ export
def _f(x):
    return np.asarray(x, np.float64).tolist()


def _leaf_data(lf) -> dict:
    if lf.kind == "q":
        return {"kind": "q", "A": _f(lf.A), "b": _f(lf.b), "c": float(lf.c), "has_q": bool(lf.has_q), "N": _f(lf.N),
                "H": _f(lf.H), "origin": _f(lf.origin), "qo": _f(lf.qo)}  # fmt: skip
    if lf.kind == "torus":
        return {"kind": "torus", "R": float(lf.R), "r": float(lf.r), "lin": _f(lf.lin), "origin": _f(lf.origin)}
    raise NotImplementedError(f"a leaf of kind {lf.kind!r}")


def _solid_data(node) -> dict:
    from lumen.geometry import solids

    comp = solids.Compiled(node)
    lo, hi = solids.node_bbox(node)
    return {"leaves": [_leaf_data(lf) for lf in comp.leaves], "expr": comp.expr, "lo": _f(lo), "hi": _f(hi)}


def _table(t) -> list:
    """A packed (energy, value) table, or a constant, as [energies, values] (float32 values as float64 numbers)."""
    if isinstance(t, dict):
        return [_f(np.asarray(t["energy"], np.float32)), _f(np.asarray(t["value"], np.float32))]
    return float(np.float32(t))


def export_scene(scene, meshes=None) -> tuple:
    """Return (solids, volumes) of a reference ``Scene``: per definition with a member its flattened solid, per
    navigator volume (an instance of such a definition, in the reference's instance order) its PV path, definition,
    parent volume, world pose and label (the member's (medium, sensor)). A tessellated member (``scene.Mesh``, an
    opaque part the navigator meets as a pseudo-volume) goes to ``meshes`` (a list: its PV path, world triangles in
    the reference's instance order, mother volume, world pose, label); without the list a mesh is refused."""  # noqa: D205, D209
    from lumen.geometry import scene as sc

    T = sc.instances(scene)
    solids, volumes, vol_of_inst = {}, [], {}
    for i, dname in enumerate(T.defn):
        d = scene.definitions[dname]
        if d.member is None:
            continue
        if isinstance(d.member.solid, sc.Mesh):
            if meshes is None:
                raise NotImplementedError(f"{dname}: a mesh (tessellated solid) is not converted here")
            p = int(T.parent[i])
            while p >= 0 and p not in vol_of_inst:
                p = int(T.parent[p])
            seg = sc.member_segment(d, dname)
            tris = np.einsum("ij,nkj->nki", T.R[i], np.asarray(d.member.solid.tris, float)) + T.t[i]
            meshes.append({"pv": f"{T.path[i]}/{seg}" if T.path[i] else seg, "tris": _f(tris),
                           "mother": vol_of_inst[p] if p >= 0 else -1, "R": _f(T.R[i]), "t": _f(T.t[i]),
                           "label": [int(d.member.label.medium), int(d.member.label.sensor)]})  # fmt: skip
            continue
        if dname not in solids:
            solids[dname] = _solid_data(d.member.solid)
        p = int(T.parent[i])
        while p >= 0 and p not in vol_of_inst:  # an assembly places its daughters in the nearest ancestor volume
            p = int(T.parent[p])
        vol_of_inst[i] = len(volumes)
        # a piece of a split union (Definition.piece_of) takes its union's placement as its PV, the union instance
        # being its parent (src/lumen/build/tracked.py:129 classes)
        j = int(T.parent[i]) if d.piece_of else i
        seg = sc.member_segment(d, d.piece_of or dname)
        lab = d.member.label
        volumes.append({"pv": f"{T.path[j]}/{seg}" if T.path[j] else seg, "path": T.path[i], "definition": dname,
                        "parent": vol_of_inst[p] if p >= 0 else -1, "R": _f(T.R[i]), "t": _f(T.t[i]),
                        "label": [int(lab.medium), int(lab.sensor)], "piece": bool(d.piece_of)})  # fmt: skip
    return solids, volumes


def export(det) -> dict:
    """Return the products of a loaded reference detector (``lumen.load``) that its photon loop runs on, as plain
    data (lists, numbers and strings: ``json.dumps`` keeps every float64 exactly); the module docstring says which."""  # noqa: D205, D209
    from lumen import api
    from lumen.build import pack
    from lumen.geometry import scene as sc

    parts = det.parts
    optics = parts.optics
    meshes = []
    solids, volumes = export_scene(parts.nav_scene, meshes)
    packed = pack.pack(det, det.params())
    keys = {}  # packed path -> the key it is read from directly
    for path, src in parts.key_rows.items():
        if src.key is not None and src.column in DIRECT:
            keys["/".join(str(x) for x in path)] = src.key
    tab = optics.table
    edge_rows = api._edge_rows(det)
    edge, lobes = set(edge_rows.surfaces), set(edge_rows.lobes)
    rows = []
    for r, row in enumerate(optics.rows):
        model = tab.models[int(tab.flags.model[r])].name
        glisur = 0
        if bool(tab.flags.glisur[r]):
            glisur = GLISUR_LOBES[tab.lobes[int(tab.lobe_of[r])]]
        cols, col_keys = {}, {}
        for c in O.COLUMNS:
            v = packed["surfaces"].get(c)
            reads = c in tab.reads[r]
            if v is None or (isinstance(v, dict) and not reads):
                cols[c] = float(np.float32(tab.consts[c][r]))
            elif isinstance(v, dict):
                cols[c] = [_f(np.asarray(v["energy"], np.float32)[r]), _f(np.asarray(v["value"], np.float32)[r])]
            else:
                cols[c] = float(np.float32(np.asarray(v)[r]))
            if reads and row.origin is not None:
                section, _, entry = row.origin.partition(":")
                base = f"{'surfaces' if section == 'surface' else 'sensors'}/{entry}/{tab.reads[r][c]}"
                key = keys.get(base + "/value", keys.get(base))
                if key is not None:
                    col_keys[c] = key
        rows.append({"type": row.surface_type.name, "origin": row.origin, "model": model, "reads": sorted(tab.reads[r]),
                     "normal": bool(tab.flags.normal[r]), "glisur": glisur, "far_opaque": bool(tab.flags.far_opaque[r]),
                     "per_normal": bool(tab.flags.per_normal[r]), "support": [bool(x) for x in tab.support[r]],
                     "edge": r in edge, "cols": cols, "keys": col_keys})  # fmt: skip
    media = []
    for m, name in zip(optics.media, optics.media_names, strict=True):
        pm = packed["media"][name]
        entry = {"name": name, "opaque": bool(m.opaque), "tables": {}, "keys": {}}
        for part in ("index", "absorption"):
            if part in pm:
                entry["tables"][part] = _table(pm[part])
                key = keys.get(f"media/{name}/{part}/value")
                if key is not None:
                    entry["keys"][part] = key
        for ch in m.channels:
            pc = pm[ch.name]
            if ch.name == "rayleigh" and ch.emission is None:
                parts_of = {"rayleigh": ("length",)}
            elif ch.name == "mie" and ch.emission is None:
                parts_of = {"mie": ("length",), "mie_g_forward": ("lobe", "g_forward"),
                            "mie_g_backward": ("lobe", "g_backward"), "mie_forward_ratio": ("lobe", "forward_ratio")}  # fmt: skip
                entry["mie_cover"] = (name, "mie", "forward_ratio") in lobes
            elif ch.name == "wls" and ch.emission is not None and ch.emission.spectrum is None:
                parts_of = {"wls": ("length",), "wls_yield": ("yield",), "wls_tau": ("tau",),
                            "wls_spectrum": ("spectrum",)}  # fmt: skip
                comps = tuple(ch.emission.profile.components)
                if comps not in (("delta",), ("decay",)):
                    raise NotImplementedError(f"medium {name}: WLS time profile {comps} is not converted")
                entry["wls_profile"] = int(comps == ("decay",))
            else:
                raise NotImplementedError(f"medium {name}: channel {ch.name!r} is not converted")
            for part, path in parts_of.items():
                leaf = pc
                for k in path:
                    leaf = leaf[k]
                entry["tables"][part] = _table(leaf)
                key = keys.get("/".join(("media", name, ch.name, *path)) + ("/value" if isinstance(leaf, dict) else ""))
                if key is not None:
                    entry["keys"][part] = key
        media.append(entry)
    row_of = np.asarray(optics.row_of, np.int64)
    if np.any(np.diag(row_of) >= 0):
        raise NotImplementedError("a vertex between two volumes of one class (a skin of touching siblings) is not "
                                  "converted")  # fmt: skip
    st = det.sensor_table()
    return {"format": FORMAT, "name": det.name, "precision": det.precision, "solids": solids, "volumes": volumes,
            "meshes": meshes,
            "n_classes": int(optics.n_classes), "class_names": list(optics.class_names),
            "class_of": {k: int(v) for k, v in optics.class_of.items()},
            "medium_of": [int(x) for x in optics.medium_of], "media": media, "row_of": row_of.tolist(), "rows": rows,
            "sensor_index": {k: int(v) for k, v in optics.sensor_index.items()},
            "born_pair": None if optics.born_pair is None else [int(x) for x in optics.born_pair],
            "deposit_pre": None if optics.deposit_pre is None else np.asarray(optics.deposit_pre, int).tolist(),
            "sensors": {"name": list(st.name), "sensor": list(st.sensor), "position": _f(st.position),
                        "axis": _f(st.axis)}}  # fmt: skip


def _open(path, mode):
    return gzip.open(path, mode + "t") if str(path).endswith(".gz") else open(path, mode)


def save(data: dict, path) -> None:
    """Write exported data as JSON (every float64 round-trips exactly; gzip-compressed where the name ends in .gz)."""
    with _open(path, "w") as f:
        json.dump(data, f, separators=(",", ":"))


def load_scene(path) -> dict:
    """Read exported scene data ({"solids", "volumes"}: ``export_scene``) written by ``save``."""
    with _open(path, "r") as f:
        return json.load(f)


def load(path) -> dict:
    with _open(path, "r") as f:
        data = json.load(f)
    if data.get("format") != FORMAT:
        raise ValueError(f"{path}: not exported reference detector data ({FORMAT})")
    return data


# ------------------------------------------------------------------------------------------------------ import
class Flattened(G.Solid):
    """A solid given as the reference flattened it: leaves in the solid's frame and its boolean expression."""

    def __init__(self, data: dict):
        self.data = data
        self._low = None

    def lower(self) -> G.Lowered:
        if self._low is None:
            self._low = _lowered(self.data)
        return self._low


def _leaf(d: dict) -> G.Leaf:
    """This package's leaf of a reference leaf: a quadric about origin + qo in its own frame (``solids.quad_frame``),
    the planes about origin; a torus in the canonical coordinates u = lin^-1 (x - origin)."""  # noqa: D205, D209
    og = np.asarray(d["origin"], float)
    if d["kind"] == "torus":
        return G.Leaf(False, og=og, oq=og.copy(), torus=(float(d["R"]), float(d["r"])),
                      M=np.linalg.inv(np.asarray(d["lin"], float)))  # fmt: skip
    A, b, c = np.asarray(d["A"], float), np.asarray(d["b"], float), float(d["c"])
    qo = np.asarray(d["qo"], float)
    bq, cq = b + A @ qo, float(qo @ A @ qo + 2.0 * b @ qo + c)
    N = np.asarray(d["N"], float).reshape(-1, 3)
    return G.Leaf(bool(d["has_q"]), A, bq, cq, og + qo, og, N, np.asarray(d["H"], float).reshape(-1))


def _program(expr) -> list:
    if isinstance(expr, int):
        return [(0, expr)]
    op, a, b = expr
    return _program(a) + _program(b) + [(OPS[op], 0)]


def _lowered(data: dict) -> G.Lowered:
    return G.Lowered([_leaf(d) for d in data["leaves"]], _program(data["expr"]), np.asarray(data["lo"], float),
                     np.asarray(data["hi"], float))  # fmt: skip


def _add(pool: O.Pool, t, name=None) -> int:
    if isinstance(t, list):
        return pool.add((np.asarray(t[0], np.float64), np.asarray(t[1], np.float64)), name)
    return pool.add(float(t), name)


def placed_volumes(solids: dict, vols: list, material) -> list:
    """This package's placed volumes (``geometry.Placed``) of exported solids and volumes, in their order; one
    logical volume per definition, of ``material(volume)``."""  # noqa: D205, D209
    flat = {k: Flattened(v) for k, v in solids.items()}
    lvs, placed = {}, []
    for v in vols:
        dn = v["definition"]
        if dn not in lvs:
            lvs[dn] = G.Volume(dn, flat[dn], material(v))
        depth = 0 if v["parent"] < 0 else placed[v["parent"]].depth + 1
        placed.append(G.Placed(v["pv"], lvs[dn], np.asarray(v["R"], float), np.asarray(v["t"], float),
                               int(v["parent"]), depth))  # fmt: skip
    return placed


def scene_detector(solids: dict, vols: list) -> D.Detector:
    """The navigator of an exported scene alone (``export_scene``), for navigation checks: a class per volume
    label (medium, sensor) and the outside, every class's medium transparent (index 1), every crossing the absorber.
    ``Detector.names`` are the PV paths; ``arrays["vol_i"]`` holds each volume's class and sensor."""  # noqa: D205, D209
    labels = sorted({tuple(v["label"]) for v in vols})
    cls_of = {lab: c for c, lab in enumerate(labels)}
    placed = placed_volumes(solids, vols, lambda v: f"m{v['label'][0]}")
    vol_cls = [cls_of[tuple(v["label"])] for v in vols]
    out_cls = len(labels)
    vol_sensor = np.asarray([v["label"][1] if v["label"][1] >= 0 else -1 for v in vols], np.int32)
    nav = G.navigator_arrays(placed, vol_cls, out_cls, vol_sensor)
    pool = O.Pool()
    med_i = np.full((1, 16), -1, np.int32)
    med_i[0, 0] = pool.add(1.0)
    row = O.surface_row(O.ABSORBER, False, True)
    row_i = np.zeros((1, 16), np.int32)
    row_i[0, 0:6] = [row.model, row.normal, row.glisur, row.far_opaque, row.per_normal, 0]
    for c, col in enumerate(O.COLUMNS):
        row_i[0, 6 + c] = pool.add(float(O.table(row.cols[col])[1][0]) if col in row.cols else O.NEUTRAL[col])
    n_cls = out_cls + 1
    row_of = np.zeros((n_cls, n_cls), np.int32)
    np.fill_diagonal(row_of, -1)
    n_sensor = int(vol_sensor.max()) + 1 if len(vol_sensor) and vol_sensor.max() >= 0 else 0
    st = D.SensorTable([f"s{i}" for i in range(n_sensor)], ["s"] * n_sensor, np.zeros((n_sensor, 3)),
                       np.tile([0.0, 0.0, 1.0], (n_sensor, 1)))  # fmt: skip
    return D.assemble(nav, vol_cls, n_cls, np.zeros(n_cls, np.int32), row_of, med_i, row_i, pool, st,
                      [v["pv"] for v in vols], {c: str(lab) for lab, c in cls_of.items()}, {})  # fmt: skip


def detector(data: dict, precision: str | None = None) -> D.Detector:
    """Return this package's Detector of exported reference data (``export``, ``load``); ``precision``: the
    navigator's (default: the reference detector's)."""  # noqa: D205, D209
    if data.get("format") != FORMAT:
        raise ValueError(f"not exported reference detector data ({FORMAT})")
    vols = data["volumes"]
    med_names = [m["name"] for m in data["media"]]
    medium_of = np.asarray(data["medium_of"], np.int32)
    class_of = data["class_of"]
    placed = placed_volumes(data["solids"], vols, lambda v: med_names[medium_of[class_of[v["pv"]]]])
    vol_cls = [int(class_of[v["pv"]]) for v in vols]
    out_cls = int(class_of[OUTSIDE_PV])
    sensor_index = data["sensor_index"]
    vol_sensor = np.asarray([sensor_index.get(v["pv"], -1) for v in vols], np.int32)
    meshes = [(np.asarray(m["tris"], float).reshape(-1, 3, 3), int(m["mother"])) for m in data.get("meshes", ())]
    mesh_cls = [int(class_of[m["pv"]]) for m in data.get("meshes", ())]
    nav = G.navigator_arrays(placed, vol_cls, out_cls, vol_sensor, meshes=meshes, mesh_cls=mesh_cls)
    pool = O.Pool()
    by_key = {}  # key -> table: one table per key, shared by every row reading it

    def keyed(t, key, name):
        if key is None:
            return _add(pool, t, name)
        if key not in by_key:
            by_key[key] = _add(pool, t, key)
        else:
            off, k = pool.tabs[by_key[key]]
            e, y = O.table(tuple(np.asarray(x, np.float64) for x in t) if isinstance(t, list) else t)
            have = np.asarray(pool.data[off:off + 2 * k], np.float32)
            if len(e) != k or not np.array_equal(have, np.concatenate([np.float32(e), np.float32(y)])):
                raise ValueError(f"key {key}: read with different values by two rows")
        return by_key[key]

    med_i = np.full((len(data["media"]), 16), -1, np.int32)
    for m, med in enumerate(data["media"]):
        for slot, part in enumerate(MEDIUM_PARTS):
            if part in med["tables"]:
                med_i[m, slot] = keyed(med["tables"][part], med["keys"].get(part), f"media/{med['name']}/{part}")
        if "wls" in med["tables"]:
            med_i[m, 11] = int(med["wls_profile"])
        if "mie" in med["tables"]:
            med_i[m, 12] = int(bool(med["mie_cover"]))
    rows = data["rows"]
    row_i = np.zeros((len(rows), 16), np.int32)
    for r, row in enumerate(rows):
        cover = 0
        if row["edge"]:
            for o, s in enumerate(row["support"]):
                cover |= int(s) << o
        if row["type"] == "pass":  # straight on, unchanged (the module docstring)
            row = dict(row, cols=dict(row["cols"], T=1.0, R=0.0))
        row_i[r, 0:6] = [MODELS[row["model"]], int(row["normal"]), int(row["glisur"]), int(row["far_opaque"]),
                         int(row["per_normal"]), cover]  # fmt: skip
        section, _, entry = (row["origin"] or "").partition(":")
        for c, col in enumerate(O.COLUMNS):
            name = None  # a column the row reads as a parameter, with no key of its own: this package's name
            if col in row["reads"] and row["origin"]:
                name = f"{'surfaces' if section == 'surface' else 'sensors'}/{entry}/{col}"
            row_i[r, 6 + c] = keyed(row["cols"][col], row["keys"].get(col), name)
    s = data["sensors"]
    groups = {}
    for i, entry in enumerate(s["sensor"]):
        groups.setdefault(entry.split(":", 1)[0], []).append(i)
    st = D.SensorTable(list(s["name"]), [e.split(":", 1)[0] for e in s["sensor"]],
                       np.asarray(s["position"], float).reshape(-1, 3), np.asarray(s["axis"], float).reshape(-1, 3))  # fmt: skip
    names = [v["pv"] for v in vols]
    cls_names = dict(enumerate(data["class_names"]))
    return D.assemble(nav, vol_cls, int(data["n_classes"]), medium_of, np.asarray(data["row_of"]), med_i, row_i, pool,
                      st, names, cls_names, groups, precision or data.get("precision", "float32"),
                      data.get("born_pair"), data.get("deposit_pre"))  # fmt: skip


def from_reference(det, precision: str | None = None) -> D.Detector:
    """Return this package's Detector of a loaded reference detector (``lumen.load``): ``detector(export(det))``."""
    return detector(export(det), precision)
