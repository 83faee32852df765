"""Python bindings of the test oracle (test infrastructure only).

* ``Oracle`` wraps oracle/liboracle.so, the C restatement of the reference
  flow step (bgf_oracle.h).
* ``Reference`` wraps oracle/_ref/libbgf_ref.so, the reference BG_Flood sources
  compiled in place with a small harness (oracle/ref/ref_harness.cu).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module, and only as the checker or the timed CPU baseline.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libbgf_ref.so")

D = ctypes.POINTER(ctypes.c_double)
I = ctypes.POINTER(ctypes.c_int)


class OraParam(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "g", "rho", "eps", "dt", "CFL", "theta", "cf", "delta", "dx", "xo", "yo", "lat", "zsinit", "zsoffset",
        "bndtaper", "bndrelaxtime", "bndfiltertime", "inittime", "mask")] + \
        [(n, ctypes.c_int) for n in ("engine", "frictionmodel", "ForceMassConserve", "wetdryfix",
                                     "conserveElevation", "rainbnd", "maxlevel")] + [("dtinit", ctypes.c_double)]


_olib = None


def oracle_lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_LIB):
            raise RuntimeError(f"oracle not built: {ORACLE_LIB}")
        l = ctypes.CDLL(ORACLE_LIB)
        l.ora_create.restype = ctypes.c_void_p
        l.ora_create.argtypes = [ctypes.POINTER(OraParam), ctypes.c_int, ctypes.c_int]
        l.ora_destroy.argtypes = [ctypes.c_void_p]
        l.ora_set_blocks.argtypes = [ctypes.c_void_p, I, I, D, D]
        l.ora_set_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p, D]
        l.ora_get_field.argtypes = [ctypes.c_void_p, ctypes.c_char_p, D]
        l.ora_add_segment.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, D, D, I, ctypes.POINTER(I)]
        l.ora_set_rain.argtypes = [ctypes.c_void_p, ctypes.c_int, D, D]
        l.ora_init_bed.argtypes = [ctypes.c_void_p]
        l.ora_set_rain_map.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_float)]
        l.ora_add_river.restype = ctypes.c_double
        l.ora_add_river.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double, ctypes.c_int, D, D]
        l.ora_init_loop.restype = ctypes.c_double
        l.ora_init_loop.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double]
        l.ora_set_loop.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        l.ora_step.argtypes = [ctypes.c_void_p, ctypes.c_int, D]
        l.ora_totaltime.restype = ctypes.c_double
        l.ora_totaltime.argtypes = [ctypes.c_void_p]
        _olib = l
    return _olib


# the same sources built with the reference Makefile's own host flags (no -O)
REF_LIB_FAITHFUL = os.path.join(HERE, "_ref", "faithful", "libbgf_ref.so")
_rlibs = {}


def ref_available(faithful: bool = False) -> bool:
    return os.path.exists(REF_LIB_FAITHFUL if faithful else REF_LIB)


def ref_lib(path: str | None = None):
    path = path or REF_LIB
    if path in _rlibs:
        return _rlibs[path]
    l = ctypes.CDLL(path)
    l.ref_create.restype = ctypes.c_void_p
    l.ref_create.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                             ctypes.c_double, ctypes.c_double, D, D, D, D, D, ctypes.c_double]
    l.ref_step.argtypes = [ctypes.c_void_p, ctypes.c_int, D]
    l.ref_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, D]
    l.ref_get_blocks.argtypes = [ctypes.c_void_p, I, D, D, I]
    l.ref_nblk.argtypes = [ctypes.c_void_p]
    l.ref_nseg.argtypes = [ctypes.c_void_p]
    l.ref_set_segment_series.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, D, D]
    l.ref_set_rain_series.argtypes = [ctypes.c_void_p, ctypes.c_int, D, D]
    l.ref_destroy.argtypes = [ctypes.c_void_p]
    l.ref_adapt.argtypes = [ctypes.c_void_p]
    l.ref_set.argtypes = [ctypes.c_void_p, ctypes.c_char_p, D]
    l.ref_reinit.argtypes = [ctypes.c_void_p, ctypes.c_double]
    l.ref_get_active.argtypes = [ctypes.c_void_p, I]
    l.ref_adaptation.argtypes = [ctypes.c_void_p]
    l.ref_flags.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_ubyte), ctypes.POINTER(ctypes.c_ubyte)]
    l.ref_set_bathy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                ctypes.c_double, D]
    l.ref_add_target_map.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_int)]
    l.ref_nblkmem.argtypes = [ctypes.c_void_p]
    l.ref_create_from_file.restype = ctypes.c_void_p
    l.ref_create_from_file.argtypes = [ctypes.c_char_p, ctypes.c_int]
    l.ref_read_asc_head.argtypes = [ctypes.c_char_p, I, I, D, D, D, D]
    l.ref_read_asc.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]
    l.ref_param.argtypes = [ctypes.c_void_p, D]
    l.ref_rain.argtypes = [ctypes.c_void_p, D, D]
    l.ref_segment.argtypes = [ctypes.c_void_p, ctypes.c_int, I, D, D]
    l.ref_get_active_cell.argtypes = [ctypes.c_void_p, I]
    l.ref_set_rain_map.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                   ctypes.c_double, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float)]
    _rlibs[path] = l
    return l


def _dp(a):
    return a.ctypes.data_as(D)


class Oracle:
    """CPU restatement of the reference flow step on BUQ tiles (nblk, 18, 18)."""

    def __init__(self, param, nblk: int, use_double: bool = False):
        p = OraParam()
        p.g, p.rho, p.eps, p.dt, p.CFL, p.theta, p.cf = param.g, param.rho, param.eps, param.dt, param.CFL, \
            param.theta, param.cf
        p.delta = p.dx = param.dx
        p.xo = 0.0 if math.isnan(param.xo) else param.xo
        p.yo = 0.0 if math.isnan(param.yo) else param.yo
        p.lat = param.lat
        p.zsinit = param.zsinit
        p.zsoffset = 0.0 if math.isnan(param.zsoffset) else param.zsoffset
        p.bndtaper, p.bndrelaxtime, p.bndfiltertime = param.bndtaper, param.bndrelaxtime, param.bndfiltertime
        p.inittime, p.mask = param.inittime, param.mask
        p.engine, p.frictionmodel = param.engine, param.frictionmodel
        p.ForceMassConserve, p.wetdryfix, p.conserveElevation = int(param.ForceMassConserve), int(param.wetdryfix), \
            int(param.conserveElevation)
        p.rainbnd = int(param.rainbnd)
        p.maxlevel = param.initlevel if param.maxlevel == -99999 else param.maxlevel
        p.dtinit = param.dtinit
        self.nblk = nblk
        self._p = p
        self.h = oracle_lib().ora_create(ctypes.byref(p), 1 if use_double else 0, nblk)

    def __del__(self):
        if getattr(self, "h", None):
            oracle_lib().ora_destroy(self.h)
            self.h = None

    def set_blocks(self, level, nbr, xo=None, yo=None):
        lv = np.ascontiguousarray(level, np.int32)
        nb = np.ascontiguousarray(nbr, np.int32).reshape(-1)
        xo = np.ascontiguousarray(xo if xo is not None else np.zeros(self.nblk), np.float64)
        yo = np.ascontiguousarray(yo if yo is not None else np.zeros(self.nblk), np.float64)
        oracle_lib().ora_set_blocks(self.h, lv.ctypes.data_as(I), nb.ctypes.data_as(I), _dp(xo), _dp(yo))

    def set(self, name: str, buq):
        a = np.ascontiguousarray(buq, np.float64).reshape(-1)
        assert a.size == self.nblk * 324
        rc = oracle_lib().ora_set_field(self.h, name.encode(), _dp(a))
        if rc:
            raise KeyError(name)

    def get(self, name: str) -> np.ndarray:
        a = np.zeros(self.nblk * 324)
        rc = oracle_lib().ora_get_field(self.h, name.encode(), _dp(a))
        if rc:
            raise KeyError(name)
        return a.reshape(self.nblk, 18, 18)

    def add_segment(self, typ, times, levels, sides):
        t = np.ascontiguousarray(times, np.float64)
        w = np.ascontiguousarray(levels, np.float64)
        arrs = [np.ascontiguousarray(s, np.int32) for s in sides]
        cnt = (ctypes.c_int * 4)(*[len(a) for a in arrs])
        ptrs = (I * 4)(*[a.ctypes.data_as(I) for a in arrs])
        oracle_lib().ora_add_segment(self.h, int(typ), len(t), _dp(t), _dp(w), cnt, ptrs)

    def set_rain(self, times, rates):
        t = np.ascontiguousarray(times, np.float64)
        r = np.ascontiguousarray(rates, np.float64)
        oracle_lib().ora_set_rain(self.h, len(t), _dp(t), _dp(r))

    def set_rain_map(self, xo, yo, dx, dy, to, dt, frames):
        fr = np.ascontiguousarray(frames, np.float32)
        nt, ny, nx = fr.shape
        oracle_lib().ora_set_rain_map(self.h, nx, ny, xo, yo, dx, dy, nt, to, dt,
                                      fr.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
        self._rain_map = fr

    def add_river(self, xs, xe, ys, ye, times, q) -> float:
        t = np.ascontiguousarray(times, np.float64)
        qq = np.ascontiguousarray(q, np.float64)
        return oracle_lib().ora_add_river(self.h, xs, xe, ys, ye, len(t), _dp(t), _dp(qq))

    def init_bed(self):
        rc = oracle_lib().ora_init_bed(self.h)
        if rc:
            raise RuntimeError("oracle: unsupported mesh")

    def init_loop(self, totaltime: float, nextoutputtime: float) -> float:
        return oracle_lib().ora_init_loop(self.h, totaltime, nextoutputtime)

    def set_loop(self, totaltime, nextoutputtime, dtmax):
        oracle_lib().ora_set_loop(self.h, totaltime, nextoutputtime, dtmax)

    def step(self, n: int) -> np.ndarray:
        dts = np.zeros(n)
        rc = oracle_lib().ora_step(self.h, n, _dp(dts))
        if rc:
            raise RuntimeError("oracle: unsupported mesh")
        return dts

    @property
    def totaltime(self) -> float:
        return oracle_lib().ora_totaltime(self.h)


def ref_read_asc(path: str):
    """The reference's readbathyASCHead + readbathyASCzb<float> on a file:
    ((nx, ny, dx, xo, yo, grdalpha), values (ny, nx) float32)."""
    nx, ny = ctypes.c_int(0), ctypes.c_int(0)
    dx, xo, yo, ga = (ctypes.c_double(0.0) for _ in range(4))
    l = ref_lib()
    l.ref_read_asc_head(path.encode(), ctypes.byref(nx), ctypes.byref(ny), ctypes.byref(dx), ctypes.byref(xo),
                        ctypes.byref(yo), ctypes.byref(ga))
    val = np.zeros((ny.value, nx.value), np.float32)
    l.ref_read_asc(path.encode(), nx.value, ny.value, val.ctypes.data_as(ctypes.POINTER(ctypes.c_float)))
    return (nx.value, ny.value, dx.value, xo.value, yo.value, ga.value), val


# names of the scalars ref_param returns, in order
REF_PARAM_NAMES = ("xo", "yo", "xmax", "ymax", "dx", "delta", "nx", "ny", "nblk", "nblkmem", "doubleprecision",
                   "zsinit", "zsoffset", "endtime", "totaltime", "nextoutputtime", "dtmax", "CFL", "engine", "mask",
                   "initlevel", "minlevel", "maxlevel", "nrain", "nseg")


class Reference:
    """The reference BG_Flood flow step (FlowCPU, or FlowGPU with gpudevice >= 0)."""

    def __init__(self, paramtext: str, nx, ny, dx, xo, yo, zb, h, u, v, cf=None, nextoutputtime=0.0,
                 use_double=False, lib_path: str | None = None):
        self.lib = ref_lib(lib_path)
        cfa = None if cf is None else np.ascontiguousarray(cf, np.float64)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (zb, h, u, v)]
        self.h = self.lib.ref_create(paramtext.encode(), 1 if use_double else 0, nx, ny, dx, xo, yo,
                                     *[_dp(a) for a in arrs], None if cfa is None else _dp(cfa), nextoutputtime)
        self.nblk = self.lib.ref_nblk(self.h)

    @classmethod
    def from_file(cls, paramfile: str, fix_asc_dy: bool = True) -> "Reference":
        """The reference's own start-up from a BG_param.txt (paths in it relative to
        the working directory), on the CPU."""
        self = cls.__new__(cls)
        self.lib = ref_lib()
        self.h = self.lib.ref_create_from_file(paramfile.encode(), 1 if fix_asc_dy else 0)
        self.nblk = self.lib.ref_nblk(self.h)
        return self

    def params(self) -> dict:
        out = np.zeros(64)
        n = self.lib.ref_param(self.h, _dp(out))
        return dict(zip(REF_PARAM_NAMES, out[:n].tolist()))

    def rain(self):
        n = int(self.params()["nrain"])
        t, r = np.zeros(max(n, 1)), np.zeros(max(n, 1))
        self.lib.ref_rain(self.h, _dp(t), _dp(r))
        return t[:n], r[:n]

    def segment(self, iseg: int):
        typ = ctypes.c_int(0)
        cap = 4096
        t, w = np.zeros(cap), np.zeros(cap)
        n = self.lib.ref_segment(self.h, iseg, ctypes.byref(typ), _dp(t), _dp(w))
        return typ.value, t[:n], w[:n]

    def set_rain_map(self, xo, yo, dx, dy, to, dt, before, after):
        b = np.ascontiguousarray(before, np.float32)
        a = np.ascontiguousarray(after, np.float32)
        ny, nx = b.shape
        F = ctypes.POINTER(ctypes.c_float)
        self.lib.ref_set_rain_map(self.h, nx, ny, xo, yo, dx, dy, to, dt, b.ctypes.data_as(F), a.ctypes.data_as(F))

    def active_cell(self) -> np.ndarray:
        a = np.zeros(self.nblk * 324, np.int32)
        self.lib.ref_get_active_cell(self.h, a.ctypes.data_as(I))
        return a.reshape(self.nblk, 18, 18)

    def __del__(self):
        if getattr(self, "h", None):
            self.lib.ref_destroy(self.h)
            self.h = None

    def blocks(self):
        n = self.nblk
        lev = np.zeros(n, np.int32)
        xo = np.zeros(n)
        yo = np.zeros(n)
        nb = np.zeros(n * 8, np.int32)
        self.lib.ref_get_blocks(self.h, lev.ctypes.data_as(I), _dp(xo), _dp(yo), nb.ctypes.data_as(I))
        return lev, nb.reshape(n, 8), xo, yo

    def get(self, name: str) -> np.ndarray:
        a = np.zeros(self.nblk * 324)
        rc = self.lib.ref_get(self.h, name.encode(), _dp(a))
        if rc:
            raise KeyError(name)
        return a.reshape(self.nblk, 18, 18)

    def set_segment_series(self, iseg, times, levels):
        t = np.ascontiguousarray(times, np.float64)
        w = np.ascontiguousarray(levels, np.float64)
        self.lib.ref_set_segment_series(self.h, iseg, len(t), _dp(t), _dp(w))

    def set_rain(self, times, rates):
        t = np.ascontiguousarray(times, np.float64)
        r = np.ascontiguousarray(rates, np.float64)
        self.lib.ref_set_rain_series(self.h, len(t), _dp(t), _dp(r))

    def step(self, n: int) -> np.ndarray:
        dts = np.zeros(n)
        self.lib.ref_step(self.h, n, _dp(dts))
        return dts

    def adapt(self) -> int:
        """Runs the reference's own Adaptation() with the "Adaptation" key of paramtext."""
        self.nblk = self.lib.ref_adapt(self.h)
        return self.nblk

    def adaptation(self) -> int:
        """The reference's Adaptation() alone (no InitialConditions afterwards)."""
        self.nblk = self.lib.ref_adaptation(self.h)
        return self.nblk

    def flags(self):
        """(refine, coarsen) per active block of one AdaptCriteria + refinesanitycheck
        pass; the model is refined by that one iteration of Adaptation()."""
        r = np.zeros(self.nblk, np.uint8)
        c = np.zeros(self.nblk, np.uint8)
        self.lib.ref_flags(self.h, r.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)),
                           c.ctypes.data_as(ctypes.POINTER(ctypes.c_ubyte)))
        self.nblk = self.lib.ref_nblk(self.h)
        return r, c

    def set_bathy(self, xo: float, yo: float, dx: float, val: np.ndarray):
        """Bathymetry forcing grid (ny, nx) with node (0, 0) at (xo, yo)."""
        v = np.ascontiguousarray(val, np.float64)
        ny, nx = v.shape
        self.lib.ref_set_bathy(self.h, nx, ny, xo, yo, dx, _dp(v))

    def add_target_map(self, xo: float, yo: float, dx: float, levels: np.ndarray):
        """Appends a target-level map (ny, nx) of integers with node (0, 0) at (xo, yo)
        (the Targetlevel criterion; the last map decides)."""
        v = np.ascontiguousarray(levels, np.int32)
        ny, nx = v.shape
        if self.lib.ref_add_target_map(self.h, nx, ny, xo, yo, dx, v.ctypes.data_as(ctypes.POINTER(ctypes.c_int))):
            raise RuntimeError("ref_add_target_map failed")

    @property
    def nblkmem(self) -> int:
        return self.lib.ref_nblkmem(self.h)

    def active(self) -> np.ndarray:
        a = np.zeros(self.nblk, np.int32)
        self.lib.ref_get_active(self.h, a.ctypes.data_as(I))
        return a

    def set(self, name: str, buq):
        a = np.ascontiguousarray(buq, np.float64).reshape(-1)
        assert a.size == self.nblk * 324
        if self.lib.ref_set(self.h, name.encode(), _dp(a)):
            raise KeyError(name)

    def reinit(self, nextoutputtime: float):
        self.lib.ref_reinit(self.h, nextoutputtime)

    def mesh_active_order(self):
        """Block tables renumbered to active order: (level, nbr (nblk, 8), xo, yo)."""
        act = self.active()
        pos = {int(b): k for k, b in enumerate(act)}
        lev, nb, xo, yo = self.blocks()
        nbr = np.vectorize(lambda b: pos[int(b)])(nb).astype(np.int32)
        return lev, nbr, xo, yo
