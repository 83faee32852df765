"""Input files of a BG_Flood scenario: bathymetry grids and uniform time series.

Readers for the file formats a ``BG_param.txt`` points at, with the reference's
rules:

* ESRI ASCII grids (``.asc``) through the native readers ``bgf_read_asc_head``
  and ``bgf_read_asc`` (readbathyASCHead / readbathyASCzb,
  src/ReadForcing.cu:2067-2220), then the positive-down flip and NaN fill of
  readforcing / readbathydata (src/ReadForcing.cu:38-53, 575-593);
* uniform series (rain in mm/h, boundary water levels in m): one ``time value``
  pair per line, tab, blank or comma separated, ``#`` lines skipped
  (readINfileUNI, src/ReadForcing.cu:1363-1425); times are seconds or
  ``YYYY-MM-DDTHH:MM:SS`` dates relative to ``reftime`` (readinputtimetxt,
  src/utctime.cu:341-366).

One deliberate difference: the reference leaves the y spacing of an ``.asc``
grid at 0 (only its ``.md`` reader sets ``dy = dx``, src/ReadForcing.cu:1788),
and its bilinear interp2BUQ divides by that spacing, which turns every bed value
into inf.  Here ``dy = dx`` for ``.asc`` grids, the value the reference's other
readers and its own tests (src/Testing.cu:501) use.
"""
from __future__ import annotations

import ctypes
import datetime as _dt
import os
from dataclasses import dataclass

import numpy as np

from ._native import lib

__all__ = ["BathyGrid", "read_asc_header", "read_asc", "read_bathy", "read_uniform_series", "readinputtimetxt",
           "read_flow_file"]


class CGrid(ctypes.Structure):
    """ctypes image of ``bgf_grid`` (include/bg_flood_b200.h)."""
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("xo", ctypes.c_double), ("yo", ctypes.c_double),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("xmax", ctypes.c_double),
                ("ymax", ctypes.c_double), ("val", ctypes.c_void_p)]


@dataclass
class BathyGrid:
    """A regular grid of nodes as the reference holds a static forcing
    (StaticForcingP<float>): val is (ny, nx) float32 with row 0 at yo."""
    nx: int
    ny: int
    xo: float
    yo: float
    dx: float
    dy: float
    val: np.ndarray
    grdalpha: float = 0.0
    path: str = ""

    @property
    def xmax(self) -> float:
        return self.xo + (self.nx - 1) * self.dx

    @property
    def ymax(self) -> float:
        return self.yo + (self.ny - 1) * self.dx

    def to_c(self) -> CGrid:
        """The bgf_grid view of this grid (valid while self.val lives)."""
        self.val = np.ascontiguousarray(self.val, dtype=np.float32)
        return CGrid(self.nx, self.ny, self.xo, self.yo, self.dx, self.dy, self.xmax, self.ymax,
                     self.val.ctypes.data)


def _check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().bgf_last_error()
        raise ValueError(f"{what}: {msg.decode() if msg else rc}")


def read_asc_header(path: str) -> tuple:
    """(nx, ny, dx, xo, yo, grdalpha) of an ESRI ASCII grid; xo, yo are the first
    node's position as readbathyASCHead leaves them."""
    nx, ny = ctypes.c_int(0), ctypes.c_int(0)
    dx, xo, yo, ga = (ctypes.c_double(0.0) for _ in range(4))
    _check(lib().bgf_read_asc_head(os.fsencode(path), ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(dx),
                                   ctypes.byref(xo), ctypes.byref(yo), ctypes.byref(ga)), f"reading {path}")
    return nx.value, ny.value, dx.value, xo.value, yo.value, ga.value


def read_asc(path: str) -> BathyGrid:
    """An ESRI ASCII grid as a BathyGrid (dy = dx)."""
    nx, ny, dx, xo, yo, ga = read_asc_header(path)
    val = np.empty((ny, nx), np.float32)
    _check(lib().bgf_read_asc(os.fsencode(path), nx, ny, val.ctypes.data), f"reading {path}")
    return BathyGrid(nx, ny, xo, yo, dx, dx, val, ga, path)


def read_bathy(path: str, posdown: int = 0, first: bool = True) -> BathyGrid:
    """readbathydata for one bathymetry file: the grid, negated when ``posdown == 1``;
    the first (base) grid has its NaNs set to 0 (src/ReadForcing.cu:44-53)."""
    ext = path.rsplit(".", 1)[-1].lower() if "." in os.path.basename(path) else ""
    if ext != "asc":
        raise ValueError(f"bathymetry format '.{ext}' is not supported by this library (ESRI ASCII .asc only): {path}")
    g = read_asc(path)
    if posdown == 1:
        g.val = (g.val * np.float32(-1.0)).astype(np.float32)
    if first:
        g.val = np.where(np.isnan(g.val), np.float32(0.0), g.val).astype(np.float32)
    return g


def _date_seconds(text: str) -> float:
    t = _dt.datetime.fromisoformat(text.strip())
    if t.tzinfo is None:
        t = t.replace(tzinfo=_dt.timezone.utc)
    return t.timestamp()


def readinputtimetxt(text: str, reftime: list) -> float:
    """Seconds for a time item (readinputtimetxt, src/utctime.cu:341-366): a number,
    or a date ``YYYY-MM-DDTHH:MM:SS`` counted from ``reftime[0]`` (set to the date
    itself when empty, as the reference does)."""
    s = text.strip()
    if "T" in s:
        if not reftime[0]:
            reftime[0] = s
        return _date_seconds(s) - _date_seconds(reftime[0])
    return float(s)


def read_uniform_series(path: str, reftime: list | None = None) -> tuple:
    """(times, values) of a uniform series file as readINfileUNI reads it."""
    ref = reftime if reftime is not None else [""]
    times, vals = [], []
    with open(path, "r") as fh:
        for line in fh:
            line = line.rstrip("\n")
            if not line or line.startswith("#"):
                continue
            el = [e for e in line.split("\t") if e]
            if len(el) < 2:
                el = [e for e in line.split(" ") if e]
            if len(el) < 2:
                el = [e for e in line.split(",") if e]
            if len(el) < 2:
                raise ValueError(f"{path}: format error, at least 2 items expected per line: {line!r}")
            times.append(readinputtimetxt(el[0], ref))
            vals.append(float(el[1]))
    if not times:
        raise ValueError(f"{path}: no samples")
    return np.asarray(times, np.float64), np.asarray(vals, np.float64)


def read_flow_file(path: str, reftime: list | None = None) -> tuple:
    """(times, discharges) of a river discharge file as readFlowfile reads it
    (src/ReadForcing.cu:1277-1345): exactly two items per line, tab, blank or
    comma separated, ``#`` lines skipped."""
    ref = reftime if reftime is not None else [""]
    times, q = [], []
    with open(path, "r") as fh:
        for line in fh:
            line = line.rstrip("\n")
            if not line or line.startswith("#"):
                continue
            el = [e for e in line.split("\t") if e]
            if len(el) != 2:
                el = [e for e in line.split(" ") if e]
            if len(el) != 2:
                el = [e for e in line.split(",") if e]
            if len(el) != 2:
                raise ValueError(f"{path}: flow file format error, 2 items expected per line: {line!r}")
            times.append(readinputtimetxt(el[0], ref))
            q.append(float(el[1]))
    if len(times) < 2:
        raise ValueError(f"{path}: a discharge series needs at least 2 samples")
    return np.asarray(times, np.float64), np.asarray(q, np.float64)
