"""Param mirror and BG_param.txt key reader for the flow-step path.

Mirrors the members of the reference ``Param`` class (src/Param.h:10-239) that
the flow step reads, with the reference's names and defaults, and a reader for
the matching subset of ``BG_param.txt`` keys.  The reader follows the
reference's rules (src/ReadInput.cu:1689-1742): one ``key = value`` per line,
keys are case-insensitive and have aliases, ``#`` starts a comment and the
value stops at ``;``.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass, field, fields

__all__ = ["Param", "read_param_text", "BndSegmentSpec", "CParam"]


class CParam(ctypes.Structure):
    """ctypes image of ``bgf_param`` (include/bg_flood_b200.h)."""
    _fields_ = [(n, ctypes.c_double) for n in (
        "g", "eps", "dt", "CFL", "theta", "cf", "dx", "delta", "xo", "yo", "lat", "zsinit", "zsoffset",
        "bndtaper", "bndrelaxtime", "bndfiltertime", "inittime", "dtmin", "dtinit", "mask")] + \
        [(n, ctypes.c_int) for n in (
            "engine", "frictionmodel", "ForceMassConserve", "wetdryfix", "conserveElevation",
            "doubleprecision", "minlevel", "maxlevel", "initlevel", "aoibnd", "rainbnd", "GPUDEVICE", "fastmath",
            "splitprecision")]


@dataclass
class BndSegmentSpec:
    """A boundary segment as declared by the reference's ``left``/``right``/``top``/``bot``
    keys (readbndlineside, src/ReadInput.cu:1952-2005): a side polygon, a type and an
    optional uniform water-level series."""
    side: str  # "left", "right", "top", "bot" or "all"
    type: int
    times: list = field(default_factory=list)
    levels: list = field(default_factory=list)
    file: str = ""  # uniform water-level series file ("time value" lines)


@dataclass
class Param:
    """Flow-step subset of the reference Param class, same names and defaults.

    Key aliases follow readparamstr (src/ReadInput.cu:162-890)."""
    g: float = 9.81
    rho: float = 1025.0
    eps: float = 0.0001
    dt: float = 0.0
    CFL: float = 0.5
    theta: float = 1.3
    VelThreshold: float = -1.0
    frictionmodel: int = 0
    cf: float = 0.0001
    lat: float = 0.0
    GPUDEVICE: int = 0
    doubleprecision: int = 0
    fastmath: int = 0  # library option, not a reference key: 1 selects the fast-math kernels
    splitprecision: int = 0  # library option: FP32 depths as deviations from per-block datums (deep water)
    engine: int = 1
    dx: float = math.nan
    xo: float = math.nan
    yo: float = math.nan
    xmax: float = math.nan
    ymax: float = math.nan
    mask: float = 9999.0
    initlevel: int = 0
    maxlevel: int = -99999
    minlevel: int = -99999
    membuffer: float = 1.05
    outputtimestep: float = 0.0
    endtime: float = float(1.7976931348623157e308)
    totaltime: float = 0.0
    inittime: float = 0.0
    dtinit: float = -1.0
    dtmin: float = 0.0005
    aoibnd: int = 0
    bndrelaxtime: float = 3600.0
    bndfiltertime: float = 60.0
    bndtaper: float = 0.0
    rainbnd: bool = False
    zsinit: float = math.nan
    zsoffset: float = math.nan
    conserveElevation: bool = False
    wetdryfix: bool = True
    ForceMassConserve: bool = False
    adaptmaxiteration: int = 20
    AdaptCrit: str = ""
    Adapt_args: list = field(default_factory=list)
    posdown: int = 0
    grdalpha: float = math.nan
    reftime: str = ""
    # forcing-side keys the path uses (reference Forcing class)
    segments: list = field(default_factory=list)
    rain: str = ""
    bathy: list = field(default_factory=list)  # bathymetry files, first one the base grid
    rivers: list = field(default_factory=list)  # (discharge file, xstart, xend, ystart, yend)
    cf_file: str = ""  # a roughness map named by the cf key (not read by this library)

    @property
    def delta(self) -> float:
        return self.dx

    def to_c(self) -> CParam:
        c = CParam()
        for n, _ in CParam._fields_:
            if n == "delta":
                v = self.dx
            elif n in ("maxlevel", "minlevel"):
                v = getattr(self, n)
                v = self.initlevel if v == -99999 else v
            elif n == "zsoffset":
                v = 0.0 if math.isnan(self.zsoffset) else self.zsoffset
            else:
                v = getattr(self, n)
            setattr(c, n, type(getattr(c, n))(v))
        return c


# key -> (attribute, type, aliases); from the reference reader src/ReadInput.cu:162-890
_KEYS = [
    ("test", None, ["test"]),
    ("g", float, ["g"]),
    ("rho", float, ["rho"]),
    ("eps", float, ["eps"]),
    ("dt", float, ["dt"]),
    ("CFL", float, ["CFL"]),
    ("theta", float, ["theta"]),
    ("VelThreshold", float, ["VelThreshold", "vthresh", "vmax", "velmax"]),
    ("frictionmodel", int, ["frictionmodel"]),
    ("cf", float, ["cf", "roughness", "cfmap"]),
    ("lat", float, ["lat"]),
    ("GPUDEVICE", int, ["GPUDEVICE", "gpu"]),
    ("doubleprecision", int, ["doubleprecision"]),
    ("dx", float, ["dx"]),
    ("xo", float, ["xo", "xmin"]),
    ("yo", float, ["yo", "ymin"]),
    ("xmax", float, ["xmax"]),
    ("ymax", float, ["ymax"]),
    ("mask", float, ["mask"]),
    ("initlevel", int, ["initlevel"]),
    ("maxlevel", int, ["maxlevel"]),
    ("minlevel", int, ["minlevel"]),
    ("membuffer", float, ["membuffer"]),
    ("outputtimestep", float, ["outputtimestep", "outtimestep", "outputstep"]),
    ("endtime", float, ["endtime", "stoptime", "end", "stop", "end_time", "stop_time"]),
    ("totaltime", float, ["totaltime", "inittime", "starttime", "start_time", "init_time", "start", "init"]),
    ("dtinit", float, ["dtinit"]),
    ("dtmin", float, ["dtmin"]),
    ("aoibnd", int, ["aoibnd", "remainderbnd", "remainbndtype", "aoibndtype"]),
    ("bndrelaxtime", float, ["bndrelaxtime"]),
    ("bndfiltertime", float, ["bndfiltertime"]),
    ("bndtaper", float, ["bndtaper"]),
    ("rainbnd", bool, ["rainbnd", "rainonbnd"]),
    ("zsinit", float, ["zsinit", "initzs"]),
    ("zsoffset", float, ["zsoffset"]),
    ("conserveElevation", bool, ["conserveElevation"]),
    ("wetdryfix", bool, ["wetdryfix", "reminstab", "fixinstab"]),
    ("ForceMassConserve", bool, ["ForceMassConserve", "MassConservation", "MassCon", "forcemassconservation",
                                  "forcevolumeconservation", "Volumeconservation", "VolumeCon", "ForceVolConserve"]),
    ("adaptmaxiteration", int, ["adaptmaxiteration", "maxiterationadapt"]),
    ("posdown", int, ["posdown"]),
    ("grdalpha", float, ["grdalpha"]),
    ("reftime", str, ["reftime", "referencetime", "timeref"]),
]

# bathymetry file keys (readparamstr for Forcing, src/ReadInput.cu:899-906)
_BATHY_KEYS = ("bathy", "bathyfile", "bathymetry", "depfile", "depthfile", "topofile", "topo", "dem")


def _split_line(line: str):
    """Key/value split as findparameter does: cut comments at '#', split at the first
    '=', cut the value at ';', trim blanks."""
    line = line.split("#", 1)[0]
    if "=" not in line:
        return None, None
    key, val = line.split("=", 1)
    val = val.split(";", 1)[0]
    return key.strip(), val.strip()


def _is_number(v: str) -> bool:
    try:
        float(v)
        return True
    except ValueError:
        return False


def _parse_bool(v: str) -> bool:
    # readparambool (src/ReadInput.cu): "1", "true", "yes", "on" (any case) are true
    return v.strip().lower() in ("1", "true", "yes", "on", "t", "y")


def read_param_text(text: str, param: Param | None = None) -> Param:
    """Applies ``BG_param.txt``-style lines to a Param (defaults if None)."""
    p = param if param is not None else Param()
    for raw in text.splitlines():
        key, val = _split_line(raw)
        if not key or val == "":
            continue
        k = key.lower()
        if k == "engine":
            # only "b", "butt", "buttinger" or "1" select engine 1; every other value
            # selects engine 5 in the reference (src/ReadInput.cu:193-213).  Engine 2
            # (Kurganov) is exposed here under the values "2", "kurganov" and "k".
            v = val.lower()
            if v in ("b", "butt", "buttinger", "1"):
                p.engine = 1
            elif v in ("2", "kurganov", "k", "kurg"):
                p.engine = 2
            else:
                p.engine = 5
            continue
        if k in ("left", "leftbndfile", "leftbnd", "right", "rightbndfile", "rightbnd", "top", "topbndfile",
                 "topbnd", "bot", "botbndfile", "botbnd", "bottom"):
            side = {"l": "left", "r": "right", "t": "top", "b": "bot"}[k[0]]
            # readbndlineside (src/ReadInput.cu:1952-2005): "type" or "type,file" / "file,type"
            items = [s.strip() for s in val.split(",") if s.strip()]
            if len(items) == 1:
                p.segments.append(BndSegmentSpec(side, int(items[0])))
            else:
                if items[1][:1].isdigit():
                    typ, fname = int(items[1]), items[0]
                else:
                    typ, fname = int(items[0]), items[1]
                p.segments.append(BndSegmentSpec(side, typ, file=fname))
            continue
        if k in _BATHY_KEYS:
            p.bathy.append(val)
            continue
        if k in ("river", "rivers"):
            # "file, xstart, xend, ystart, yend" (src/ReadInput.cu:1020-1045)
            items = [s for s in val.split(",") if s]
            if len(items) != 5:
                raise ValueError(f"river needs 5 comma-separated items (file, xstart, xend, ystart, yend): {val!r}")
            p.rivers.append((items[0].strip(), float(items[1]), float(items[2]), float(items[3]), float(items[4])))
            continue
        if k in ("adaptation", "adapt"):
            items = [s.strip() for s in val.split(",")]
            p.AdaptCrit = items[0]
            p.Adapt_args = items[1:]
            continue
        if k in ("rain", "rainfile"):
            p.rain = val
            continue
        for attr, typ, aliases in _KEYS:
            if k in (a.lower() for a in aliases):
                if typ is None:
                    pass
                elif typ is bool:
                    setattr(p, attr, _parse_bool(val))
                elif attr == "cf" and not _is_number(val):
                    p.cf_file = val  # a roughness map file: not read by this library
                else:
                    setattr(p, attr, typ(val))
                break
    return p


def param_names() -> list[str]:
    return [f.name for f in fields(Param)]
