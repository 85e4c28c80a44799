"""Optics on the host: materials, optical surfaces, the surface lookup's classes and rows, and the parameter pool.

The reference compiles a detector's optics into a class per placed volume, a surface row per crossed class pair
(``row_of[C, C]``), a medium per class and packed parameter tables (src/lumen/build/lookup.py:360-500 SurfaceTable,
Optics, pack; src/lumen/build/pack.py:84). This module builds the same structure for the C ABI
(include/lumen_b200.h): every value a run reads is a table, linear in photon energy between its knots and held beyond
(src/lumen/media/laws.py:86), stored in one float32 pool that a call may replace (live and reference values).

Surface types follow Geant4's chain as the reference restates it (src/lumen/surfaces/types.py:445-493):
``dielectric_metal`` polished = a specular metal (R into the spike), ground unified = the reflection constants
(spike, lobe, backscatter, Lambertian), ``dielectric_dielectric`` polished = the Fresnel interface, and the absorber
(nothing continues). A sensor's surface reads EFFICIENCY as its detected share; on any other surface it is fixed at 0
(types.py:557 no_detection).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from lumen_b200 import facets

HC = 1239.8419843320025  # h c in eV nm (src/lumen/units.py:20)
HC_EV_M = HC * 1e-9
# G4OpRayleigh::CalculateRayleighMeanFreePaths for a material named "Water" (src/lumen/rules/optics.py:98-103)
WATER_COMPRESSIBILITY = 7.658e-23  # m3 / MeV
WATER_TEMPERATURE = 283.15  # K
K_BOLTZMANN = 8.617333e-11  # MeV / K

# the columns of a surface row and their neutral values (src/lumen/surfaces/types.py:72 COLUMNS)
COLUMNS = ("R", "T", "eff", "p_spike", "p_lobe", "p_back", "sigma_alpha", "polish", "nr", "nk")
NEUTRAL = {"R": 0.0, "T": 0.0, "eff": 0.0, "p_spike": 0.0, "p_lobe": 0.0, "p_back": 0.0, "sigma_alpha": 0.1,
           "polish": 0.0, "nr": 1.0, "nk": 0.0}  # fmt: skip
MODEL_REFLECT, MODEL_DIELECTRIC, MODEL_COMPLEX = 0, 1, 2
# the outcomes, in the reference's order (src/lumen/surfaces/outcomes.py:30 NAMES)
STRAIGHT, REFRACT, SPECULAR, BACKSCATTER, GLOSSY, DIFFUSE = range(6)


def table(v, energy=None):
    """Return a table (energies eV ascending, values) from a constant or from (energies, values)."""
    if energy is None:
        if isinstance(v, tuple) and len(v) == 2:
            e, y = np.asarray(v[0], float), np.asarray(v[1], float)
        else:
            return np.array([1.0]), np.array([float(v)])
    else:
        e, y = np.asarray(energy, float), np.asarray(v, float)
    o = np.argsort(e)
    return e[o], y[o]


def water_rayleigh(rindex):
    """Return Geant4's Rayleigh-length table of water on the RINDEX knots (src/lumen/rules/optics.py:208-254)."""
    e, n = rindex
    c1 = WATER_COMPRESSIBILITY * WATER_TEMPERATURE * K_BOLTZMANN / (6.0 * math.pi)
    e32, n32 = np.float32(e), np.float32(n)
    k = np.float32(2.0 * math.pi / HC_EV_M) * e32
    n2 = n32 * n32
    L = np.float32(1.0) / (np.float32(c1) * k**4 * ((n2 - 1.0) * (n2 + 2.0) / np.float32(3.0)) ** 2)
    return e, np.asarray(L, float)


@dataclass
class Material:
    """A medium: RINDEX (None: opaque), ABSLENGTH (m, None: no absorption), RAYLEIGH (m; None: Geant4's water
    table for a material named Water, else no scattering). Tables are (energies eV, values) or constants.

    Mie scattering (G4OpMieHG, src/lumen/rules/optics.py:357 mie_constants): ``mie`` the length MIEHG (m) with the
    constants ``mie_forward`` (MIEHG_FORWARD), ``mie_backward`` (MIEHG_BACKWARD), ``mie_forward_ratio``
    (MIEHG_FORWARD_RATIO). Wavelength shifting (G4OpWLS, optics.py:337 _wls_channel): ``wls`` the absorption length
    WLSABSLENGTH (m), ``wls_spectrum`` the WLSCOMPONENT table (energies eV, intensities), ``wls_mean`` the mean
    photons per absorbed one (WLSMEANNUMBERPHOTONS, 1 when absent), ``wls_tau`` WLSTIMECONSTANT (ns, 0 when absent),
    ``wls_profile`` "delta" (Geant4's default) or "exponential".

    Scintillation (G4Scintillation, Geant4 11 keys, src/lumen/sources/scintillation.py): ``scint_yield``
    SCINTILLATIONYIELD (photons / MeV); ``scint_components`` up to three dicts, in order, with ``spectrum``
    (SCINTILLATIONCOMPONENTi: energies eV, intensities), ``tau`` (SCINTILLATIONTIMECONSTANTi, ns) and ``rise``
    (SCINTILLATIONRISETIMEi, ns; all or none of the components); ``scint_shares`` the SCINTILLATIONYIELDi (None:
    Geant4's defaults 1, 0, 0). The material's light is a source's (``sources.ScintillationPoint``), not the bulk's.
    """  # noqa: D205

    name: str
    rindex: object = None
    abslength: object = None
    rayleigh: object = None
    mie: object = None
    mie_forward: float = 0.0
    mie_backward: float = 0.0
    mie_forward_ratio: float | None = None
    wls: object = None
    wls_spectrum: object = None
    wls_mean: float = 1.0
    wls_tau: float = 0.0
    wls_profile: str = "delta"
    scint_yield: float | None = None
    scint_components: tuple = ()
    scint_shares: tuple | None = None

    def __post_init__(self):
        """Refuse what G4OpMieHG / G4OpWLS would abort on or the reference refuses (optics.py:337-380)."""
        if self.mie is not None:
            if self.mie_forward_ratio is None:
                raise ValueError(f"{self.name}: MIEHG without MIEHG_FORWARD_RATIO (G4OpMieHG aborts at the first Mie "
                                 "event)")  # fmt: skip
            if not 0.0 <= self.mie_forward_ratio <= 1.0:
                raise ValueError(f"{self.name}: MIEHG_FORWARD_RATIO {self.mie_forward_ratio} outside [0, 1]")
            for g in (self.mie_forward, self.mie_backward):
                if not abs(g) <= MIE_G_MAX:
                    raise ValueError(f"{self.name}: a Mie asymmetry |g| above {MIE_G_MAX}")
        if self.scint_components:
            if self.scint_yield is None or not 1 <= len(self.scint_components) <= 3:
                raise ValueError(f"{self.name}: scintillation needs SCINTILLATIONYIELD and one to three components")
            rises = [c.get("rise") is not None for c in self.scint_components]
            if any(rises) and not all(rises):
                raise ValueError(f"{self.name}: a rise time for every component or for none")
            for c in self.scint_components:
                if c.get("spectrum") is None or c.get("tau") is None:
                    raise ValueError(f"{self.name}: a component without its spectrum or decay time (Geant4 aborts)")
        if self.wls is not None:
            if self.wls_spectrum is None:
                raise ValueError(f"{self.name}: WLSABSLENGTH without WLSCOMPONENT (G4OpWLS absorbs and emits nothing)")
            e, v = (np.asarray(x, np.float64) for x in self.wls_spectrum)
            if np.any(v < 0) or not np.sum(0.5 * (v[1:] + v[:-1]) * np.diff(e)) > 0:
                raise ValueError(f"{self.name}: WLSCOMPONENT needs a non-negative intensity with positive integral")
            if self.wls_profile not in ("delta", "exponential"):
                raise ValueError(f"{self.name}: wls_profile {self.wls_profile!r} is not 'delta' or 'exponential'")
            if not (self.wls_mean >= 0.0 and self.wls_tau >= 0.0):
                raise ValueError(f"{self.name}: WLSMEANNUMBERPHOTONS and WLSTIMECONSTANT must be >= 0")


MIE_G_MAX = 0.999  # the largest |g| of a Mie lobe (src/lumen/rules/choices.py:99)


@dataclass
class OpticalSurface:
    """A Geant4 optical surface (G4OpticalSurface + its property table)."""

    name: str
    type: str = "dielectric_metal"  # or "dielectric_dielectric"
    finish: str = "polished"  # or "ground"
    model: str = "unified"
    sigma_alpha: float = 0.0
    polish: float = 1.0  # GLISUR's polish (its facet radius is 1 - polish)
    reflectivity: object = None
    efficiency: object = None
    transmittance: object = None
    specularspike: object = None
    specularlobe: object = None
    backscatter: object = None
    rindex: object = None  # a dielectric_metal surface's complex index (RINDEX, KINDEX): a photocathode
    kindex: object = None


ABSORBER = OpticalSurface("__absorber__", "dielectric_metal", "polished", reflectivity=0.0)


@dataclass
class Row:
    """One surface row: model, flags and a value per column."""

    model: int
    normal: int = 0
    glisur: int = 0
    far_opaque: int = 0
    cols: dict = field(default_factory=dict)  # column -> table
    name: str = ""
    sensor: bool = False
    per_normal: int = 0  # read for a sensor model applying its QE after tracking: eff 1, deposits carry 1 / A_n
    cover: int = 0  # the defensive mixture's outcomes (bit per outcome) of an edge row, else 0 (``edge_cover``)


def edge_cover(surf: OpticalSurface, sensor: bool, support) -> int:
    """Return the cover mask of a surface row: the bits of ``support`` (the row type's possible outcomes,
    src/lumen/surfaces/types.py:413-513 and their ``fixed`` / ``transmitting`` rules) when the row reads a parameter
    with a defensive role, else 0.

    The reference decides edge rows by structure (src/lumen/api.py:797 ``_edge_rows``): a row is one when a property
    the detector gives (a parameter key; an omitted Geant4 default is no key) is read through a column whose role is
    "zero" (R, T, eff, the unified constants; types.py:329-336) or "support" (GLISUR's polish, read wherever a facet
    path is). EFFICIENCY is read on a sensor only (types.py:557 ``no_detection``).
    """
    keyed = (surf.reflectivity is not None or surf.transmittance is not None
             or (sensor and surf.efficiency is not None)
             or any(v is not None for v in (surf.specularspike, surf.specularlobe, surf.backscatter)))  # fmt: skip
    glisur_path = surf.model == "glisur" and surf.finish != "polished" and surf.polish < 1.0
    if not (keyed or glisur_path):
        return 0
    m = 0
    for o in support:
        m |= 1 << o
    return m


FAR_SIDE = (STRAIGHT, REFRACT)  # the outcomes that end beyond the surface (src/lumen/surfaces/outcomes.py:33)


def kills_far_side(surf: OpticalSurface) -> bool:
    """Whether Geant4 kills a photon meeting ``surf`` into a medium without RINDEX before its draw (NoRINDEX): a
    polished or ground dielectric_dielectric surface (src/lumen/rules/boundary.py:21-27 ``FAR_KILL``; the row is the
    absorber). A frontpainted finish and a dielectric_metal surface with a TRANSMITTANCE transmit and are absorbed
    where they land instead (``FAR_ABSORB``, ``surface_row``)."""  # noqa: D205, D209
    return surf.type == "dielectric_dielectric" and surf.finish not in ("polishedfrontpainted", "groundfrontpainted")


def _finish(row: Row, support, surf: OpticalSurface, sensor: bool, far_opaque: bool) -> Row:
    """Return ``row`` with its far side and cover: into an opaque medium a row with far-side outcomes loses them
    (src/lumen/surfaces/types.py:543 ``into_opaque``: the flag zeroes their shares, and they leave the outcomes the
    cover is made of); a row without any keeps the flag off (src/lumen/rules/boundary.py:100)."""  # noqa: D205, D209
    if far_opaque and any(o in FAR_SIDE for o in support):
        row.far_opaque = 1
        support = tuple(o for o in support if o not in FAR_SIDE)
    row.cover = edge_cover(surf, sensor, support)
    return row


def surface_row(surf: OpticalSurface, sensor: bool, far_opaque: bool, entry_eff=None) -> Row:
    """Return the row of a Geant4 surface (types.py:445-493 types, :557 no_detection); ``entry_eff``: a sensor's
    detection on entry instead of EFFICIENCY (1 where its sensor model applies the QE after tracking,
    src/lumen/rules/sensors.py:29 entry_efficiency)."""
    eff = surf.efficiency if (sensor and surf.efficiency is not None) else 0.0
    if sensor and entry_eff is not None:
        eff = float(entry_eff)
    if surf.type == "dielectric_dielectric" and surf.finish in ("polishedfrontpainted", "groundfrontpainted"):
        # PAINTED_T (types.py:483): R specular (polished) or Lambertian (ground), T straight, the rest absorbed
        cols = {"R": 1.0 if surf.reflectivity is None else surf.reflectivity,
                "T": 0.0 if surf.transmittance is None else surf.transmittance, "eff": eff,
                "p_spike": 1.0 if surf.finish == "polishedfrontpainted" else 0.0, "p_lobe": 0.0, "p_back": 0.0}  # fmt: skip
        # support: the straight share (T is read at its default), and the finish's half of the split (types.py:425)
        sup = (STRAIGHT, SPECULAR if surf.finish == "polishedfrontpainted" else DIFFUSE)
        return _finish(Row(MODEL_REFLECT, normal=1, cols=cols, name=surf.name), sup, surf, sensor, far_opaque)
    if surf.type == "dielectric_metal" and (surf.rindex is not None or surf.kindex is not None):
        # PHOTOCATHODE (types.py:455): the complex index's Fresnel reflectance, specular; the rest detected with eff
        if surf.rindex is None or surf.kindex is None or surf.finish != "polished":
            raise NotImplementedError(f"surface {surf.name}: a complex index needs RINDEX and KINDEX, polished")
        cols = {"nr": surf.rindex, "nk": surf.kindex, "eff": eff,
                "T": 0.0 if surf.transmittance is None else surf.transmittance}  # fmt: skip
        sup = (SPECULAR,) + ((STRAIGHT,) if surf.transmittance is not None else ())  # types.py:455, :494
        return _finish(Row(MODEL_COMPLEX, cols=cols, name=surf.name), sup, surf, sensor, far_opaque)
    if surf.type == "dielectric_dielectric":
        if surf.finish != "polished" and surf.model == "glisur" and surf.polish < 1.0:
            # GLISUR_DIELECTRIC (types.py:463): the cuts, then below R the GLISUR facet path that reflects or refracts
            # at each facet, between R and R + T straight on
            cols = {"R": 1.0 if surf.reflectivity is None else surf.reflectivity,
                    "T": 0.0 if surf.transmittance is None else surf.transmittance, "eff": eff, "p_spike": 0.0,
                    "p_lobe": 1.0, "p_back": 0.0, "polish": float(surf.polish)}  # fmt: skip
            row = Row(MODEL_REFLECT, glisur=2, cols=cols, name=surf.name)
            return _finish(row, (GLOSSY, STRAIGHT), surf, sensor, far_opaque)
        if surf.finish != "polished" and not (surf.model == "glisur" and surf.polish >= 1.0):
            raise NotImplementedError("dielectric_dielectric ground with the unified model is not built")
        cols = {"R": 1.0 if surf.reflectivity is None else surf.reflectivity,
                "T": 0.0 if surf.transmittance is None else surf.transmittance, "eff": eff}  # fmt: skip
        # DIELECTRIC_RT (types.py:444): refract, specular, straight
        row = Row(MODEL_DIELECTRIC, cols=cols, name=surf.name)
        return _finish(row, (REFRACT, SPECULAR, STRAIGHT), surf, sensor, far_opaque)
    # dielectric_metal
    R = 1.0 if surf.reflectivity is None else surf.reflectivity
    cols = {"R": R, "eff": eff, "T": 0.0 if surf.transmittance is None else surf.transmittance}
    tr = (STRAIGHT,) if surf.transmittance is not None else ()  # types.transmitting (types.py:494)
    if surf.model == "glisur" and surf.finish != "polished" and surf.polish < 1.0:
        # GLISUR_METAL (types.py:459): R into the GLISUR facet path of radius 1 - polish
        cols.update({"p_spike": 0.0, "p_lobe": 1.0, "p_back": 0.0, "polish": float(surf.polish)})
        row = Row(MODEL_REFLECT, glisur=1, cols=cols, name=surf.name)
        return _finish(row, (GLOSSY, *tr), surf, sensor, far_opaque)
    if surf.finish == "polished" or surf.model == "glisur":
        cols["p_spike"] = 1.0  # polished, or GLISUR at polish 1: the mirror (types.py:573 SPECULAR_METAL)
        row = Row(MODEL_REFLECT, normal=1, cols=cols, name=surf.name)
        return _finish(row, (SPECULAR, *tr), surf, sensor, far_opaque)
    ss = 0.0 if surf.specularspike is None else surf.specularspike
    sl = 0.0 if surf.specularlobe is None else surf.specularlobe
    bs = 0.0 if surf.backscatter is None else surf.backscatter
    cols.update({"p_spike": ss, "p_lobe": sl, "p_back": bs, "sigma_alpha": surf.sigma_alpha})
    normal = int(surf.sigma_alpha == 0.0)  # sigma_alpha 0: the lobe reflects about the global normal (types.py:471)
    if not normal and not (facets.SIGMA_MIN <= surf.sigma_alpha <= facets.SIGMA_MAX):
        raise ValueError(f"surface {surf.name}: sigma_alpha {surf.sigma_alpha} outside the unified tables' span "
                         f"[{facets.SIGMA_MIN:.5f}, {facets.SIGMA_MAX}] rad (or exactly 0)")  # fmt: skip
    # UNIFIED_METAL_NORMAL (types.py:471: its support rule reads fixed constants only, and these are read values)
    # or UNIFIED_METAL (types.py:467)
    sup = (SPECULAR, BACKSCATTER, DIFFUSE) if normal else (SPECULAR, BACKSCATTER, GLOSSY, DIFFUSE)
    row = Row(MODEL_REFLECT, normal=normal, cols=cols, name=surf.name)
    return _finish(row, (*sup, *tr), surf, sensor, far_opaque)


class Pool:
    """The parameter pool: every table's knots and values in one float32 array (include/lumen_b200.h tables)."""

    def __init__(self):
        self.tabs = []  # (offset, k)
        self.data = []
        self.names = {}

    def add(self, tab, name=None) -> int:
        e, y = table(tab)
        k = len(e)
        self.tabs.append((len(self.data), k))
        self.data.extend(np.float32(e).tolist())
        self.data.extend(np.float32(y).tolist())
        t = len(self.tabs) - 1
        if name is not None:
            self.names[name] = t
        return t

    def arrays(self):
        return np.asarray(self.tabs, np.int32).reshape(-1, 2), np.asarray(self.data, np.float32)
