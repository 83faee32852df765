"""Host mirror of the reference's adaptation pass (src/AdaptCriteria.cu,
src/Adaptation.cu): criteria parsing and the table-level entry points of the C ABI.

``parse_criterion`` reads the reference's ``Adaptation`` key ("Threshold,<z>,<var>",
"Inrange,<zmin>,<zmax>,<var>" or "Targetlevel,<file>,...", src/ReadInput.cu:830-850,
1155-1172).  ``refine_sanity`` and
``refine_tables`` call bgf_refine_sanity / bgf_refine_tables on block-id indexed
host tables; ``adapt_sanity`` / ``adapt_tables`` are their forms with coarsening
(an extension: the reference cancels coarsening, src/Adaptation.cu:173-175)."""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from ._native import lib

THRESHOLD, INRANGE, TARGETLEVEL, HGRAD = 1, 2, 3, 4
VARS = {"h": 0, "zs": 1, "u": 2, "v": 3, "zb": 4}


@dataclass
class Criterion:
    kind: int
    var: str
    arg1: float
    arg2: float = 0.0
    maps: tuple = ()  # Targetlevel: the target-level map files, in order

    def flags(self, z: np.ndarray, dtype=np.float32) -> np.ndarray:
        """Refine flag per block from the interior cells z (nblk, 16, 16), as
        Thresholdcriteria / inrangecriteria compare them (in the state precision)."""
        z = np.asarray(z, dtype)
        if self.kind == THRESHOLD:
            return np.any(z > dtype(self.arg1), axis=(1, 2)).astype(np.uint8)
        return np.any((z >= dtype(self.arg1)) & (z <= dtype(self.arg2)), axis=(1, 2)).astype(np.uint8)


def depth_or_slope(h_threshold: float, slope_threshold: float) -> Criterion:
    """The depth-or-slope criterion (an extension, no key in the reference's
    parameter file): refine where h > h_threshold or the wet-surface slope exceeds
    slope_threshold, coarsen where every cell stays below half of both."""
    return Criterion(HGRAD, "h", float(h_threshold), float(slope_threshold))


def parse_criterion(text: str) -> Criterion:
    parts = [p.strip() for p in text.split(",")]
    if parts[0] == "Threshold":
        return Criterion(THRESHOLD, parts[2], float(parts[1]))
    if parts[0] == "Inrange":
        return Criterion(INRANGE, parts[3], float(parts[1]), float(parts[2]))
    if parts[0].lower() == "targetlevel":
        return Criterion(TARGETLEVEL, "h", 0.0, 0.0, tuple(p for p in parts[1:] if p))
    raise ValueError(f"unsupported adaptation criterion: {text}")


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def refine_sanity(active, level, nbr8, nblkmem, minlevel, maxlevel, refine):
    """refinesanitycheck on block-id indexed tables; returns (refine, coarsen) copies."""
    act = np.ascontiguousarray(active, np.int32)
    lv = np.ascontiguousarray(level, np.int32)
    nb = np.ascontiguousarray(nbr8, np.int32).reshape(nblkmem, 8)
    r = np.ascontiguousarray(refine, np.uint8).copy()
    c = np.zeros(nblkmem, np.uint8)
    rc = lib().bgf_refine_sanity(len(act), _ip(act), _ip(lv), _ip(nb), nblkmem, minlevel, maxlevel,
                                 r.ctypes.data_as(ctypes.c_void_p), c.ctypes.data_as(ctypes.c_void_p))
    if rc:
        raise RuntimeError(f"bgf_refine_sanity: status {rc}")
    return r, c


def refine_tables(active, level, nbr8, xo, yo, nblkmem, dx, doubleprecision, refine):
    """Refined block tables (all indexed by block id, sized nblkmem).  Returns
    (active, level, nbr8 (nblkmem, 8), xo, yo, children (nblkmem, 3))."""
    n = ctypes.c_int(len(active))
    act = np.full(nblkmem, -1, np.int32)
    act[: len(active)] = active
    lv = np.ascontiguousarray(level, np.int32).copy()
    nb = np.ascontiguousarray(nbr8, np.int32).reshape(nblkmem, 8).copy()
    x = np.ascontiguousarray(xo, np.float64).copy()
    y = np.ascontiguousarray(yo, np.float64).copy()
    r = np.ascontiguousarray(refine, np.uint8)
    ch = np.zeros((nblkmem, 3), np.int32)
    rc = lib().bgf_refine_tables(ctypes.byref(n), _ip(act), _ip(lv), _ip(nb), _dp(x), _dp(y), nblkmem, float(dx),
                                 int(doubleprecision), r.ctypes.data_as(ctypes.c_void_p), _ip(ch))
    if rc:
        raise RuntimeError(f"bgf_refine_tables: status {rc}")
    return act[: n.value], lv, nb, x, y, ch


def adapt_sanity(active, level, nbr8, nblkmem, minlevel, maxlevel, refine, coarsen, xo, yo, dx,
                 allow_coarsen=True):
    """bgf_adapt_sanity on block-id indexed tables; returns (refine, coarsen) copies."""
    act = np.ascontiguousarray(active, np.int32)
    lv = np.ascontiguousarray(level, np.int32)
    nb = np.ascontiguousarray(nbr8, np.int32).reshape(nblkmem, 8)
    r = np.ascontiguousarray(refine, np.uint8).copy()
    c = np.ascontiguousarray(coarsen, np.uint8).copy()
    x = np.ascontiguousarray(xo, np.float64)
    y = np.ascontiguousarray(yo, np.float64)
    rc = lib().bgf_adapt_sanity(len(act), _ip(act), _ip(lv), _ip(nb), nblkmem, minlevel, maxlevel, _dp(x), _dp(y),
                                float(dx), 1 if allow_coarsen else 0, r.ctypes.data_as(ctypes.c_void_p),
                                c.ctypes.data_as(ctypes.c_void_p))
    if rc:
        raise RuntimeError(f"bgf_adapt_sanity: status {rc}")
    return r, c


def adapt_tables(active, level, nbr8, xo, yo, nblkmem, dx, doubleprecision, refine, coarsen):
    """Tables after merging the flagged quads and refining the flagged blocks.  Returns
    (active, level, nbr8 (nblkmem, 8), xo, yo, children (nblkmem, 3), siblings (nblkmem, 3))."""
    n = ctypes.c_int(len(active))
    act = np.full(nblkmem, -1, np.int32)
    act[: len(active)] = active
    lv = np.ascontiguousarray(level, np.int32).copy()
    nb = np.ascontiguousarray(nbr8, np.int32).reshape(nblkmem, 8).copy()
    x = np.ascontiguousarray(xo, np.float64).copy()
    y = np.ascontiguousarray(yo, np.float64).copy()
    r = np.ascontiguousarray(refine, np.uint8)
    c = np.ascontiguousarray(coarsen, np.uint8)
    ch = np.zeros((nblkmem, 3), np.int32)
    sb = np.zeros((nblkmem, 3), np.int32)
    rc = lib().bgf_adapt_tables(ctypes.byref(n), _ip(act), _ip(lv), _ip(nb), _dp(x), _dp(y), nblkmem, float(dx),
                                int(doubleprecision), r.ctypes.data_as(ctypes.c_void_p),
                                c.ctypes.data_as(ctypes.c_void_p), _ip(ch), _ip(sb))
    if rc:
        raise RuntimeError(f"bgf_adapt_tables: status {rc}")
    return act[: n.value], lv, nb, x, y, ch, sb
