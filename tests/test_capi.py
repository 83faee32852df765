"""Host-side checks that need no GPU: the C ABI library loads and exports every
entry point declared in include/*.h, fails cleanly without a GPU, and its mesh,
boundary and parameter helpers follow the reference."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from bg_flood_b200 import read_param_text
from bg_flood_b200._native import LIB_PATH, SIGNATURES, lib
from bg_flood_b200.mesh import boundary_segments, fill_halo, grid_to_buq, uniform_mesh
from bg_flood_b200.params import BndSegmentSpec

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(h).read()
        syms |= set(re.findall(r"\b(bgf_\w+)\s*\(", txt))
    return syms


def test_library_exports_every_declared_symbol():
    l = ctypes.CDLL(LIB_PATH)
    syms = declared_symbols()
    assert syms, "no declarations found"
    for s in syms:
        assert hasattr(l, s), s
    assert syms <= set(SIGNATURES), syms - set(SIGNATURES)


def test_strerror_and_create_fail_cleanly_without_gpu():
    l = lib()
    assert l.bgf_strerror(0) == b"ok"
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    from bg_flood_b200.params import Param
    p = Param(dx=1.0).to_c()
    h = ctypes.c_void_p()
    rc = l.bgf_create(ctypes.byref(p), 4, None, ctypes.byref(h))
    assert rc != 0 and not h.value


def test_invalid_arguments_are_rejected():
    l = lib()
    h = ctypes.c_void_p()
    assert l.bgf_create(None, 4, None, ctypes.byref(h)) == 1
    assert l.bgf_mesh_uniform(0, 3, 1.0, None, None, None, None, None, None, 0) == 1


def test_uniform_mesh_tables():
    m = uniform_mesh(64, 48, 2.0)
    assert m.nblk == 12
    ib = np.arange(12)
    bx, by = ib % 4, ib // 4
    left = np.where(bx > 0, ib - 1, ib)
    right = np.where(bx < 3, ib + 1, ib)
    bot = np.where(by > 0, ib - 4, ib)
    top = np.where(by < 2, ib + 4, ib)
    assert np.array_equal(m.nbr, np.stack([left, left, right, right, bot, bot, top, top], 1))
    assert np.allclose(m.xo, bx * 32 + 1.0) and np.allclose(m.yo, by * 32 + 1.0)


def test_masked_blocks_renumber_and_become_edges():
    present = np.ones((3, 3), np.uint8)
    present[1, 1] = 0
    m = uniform_mesh(48, 48, 1.0, present)
    assert m.nblk == 8
    # block (1,0) (id 1) sits below the hole: its top neighbour is itself
    assert m.nbr[1, 6] == 1 and m.nbr[1, 7] == 1
    # block (0,1) (id 3) is left of the hole: its right neighbour is itself
    assert m.nbr[3, 2] == 3


def test_halo_fill_and_grid_roundtrip():
    m = uniform_mesh(32, 32, 1.0)
    g = np.arange(32 * 32, dtype=np.float64).reshape(32, 32)
    b = fill_halo(grid_to_buq(g, m), m)
    # left halo of block 1 = last column of block 0; domain edge copies own edge
    assert np.array_equal(b[1, 1:17, 0], g[0:16, 15])
    assert np.array_equal(b[0, 1:17, 0], g[0:16, 0])
    assert np.array_equal(b[2, 0, 1:17], g[15, 0:16])


def test_boundary_segment_assignment():
    m = uniform_mesh(64, 64, 1.0)
    segs = boundary_segments(m, [BndSegmentSpec("left", 2)], aoibnd=0)
    assert [s[0] for s in segs] == [2, 0]
    left, right, top, bot = segs[0][3]
    # the west column (incl. both west corners) belongs to the declared segment
    assert sorted(left) == [0, 4, 8, 12]
    assert sorted(bot) == [0] and sorted(top) == [12]
    assert len(right) == 0
    rl, rr, rt, rb = segs[1][3]
    assert sorted(rr) == [3, 7, 11, 15] and sorted(rb) == [1, 2, 3] and len(rl) == 0


def test_param_reader_follows_reference_rules():
    p = read_param_text("""
    # comment line
    CFL = 0.4 ; trailing text
    ENGINE = buttinger
    theta=1.5   # inline comment
    frictionmodel = -1
    cf = 0.035
    left = 2, bnd.txt
    gpu = 3
    endtime = 7200
    ForceVolConserve = 1
    """)
    assert p.CFL == 0.4 and p.engine == 1 and p.theta == 1.5
    assert p.frictionmodel == -1 and p.cf == 0.035 and p.GPUDEVICE == 3
    assert p.endtime == 7200.0 and p.ForceMassConserve is True
    assert p.segments[0].side == "left" and p.segments[0].type == 2
    assert read_param_text("engine = 2").engine == 2
    assert read_param_text("engine = 9").engine == 5


def test_noalloc_rejects_a_misaligned_bed():
    """The allocation-free step copies bed tiles in 16-byte pieces: a bed pointer off
    a 16-byte boundary is refused with BGF_EINVAL before any device work (so this
    runs without a GPU; the other pointers are never dereferenced)."""
    import ctypes
    import cases
    from bg_flood_b200._native import lib
    from bg_flood_b200.flow import Loop

    class NoallocArgs(ctypes.Structure):
        _fields_ = [("nblk", ctypes.c_int), ("nblkmem", ctypes.c_int)] + \
            [(n, ctypes.c_void_p) for n in ("active", "level", "nbr", "bndtype", "zb", "dzbdx", "dzbdy",
                                            "h_in", "u_in", "v_in", "h_out", "u_out", "v_out")] + \
            [("reset_means", ctypes.c_int)]

    a = NoallocArgs()
    a.nblk = a.nblkmem = 9
    for k in ("active", "level", "nbr", "bndtype", "dzbdx", "dzbdy", "h_in", "u_in", "v_in",
              "h_out", "u_out", "v_out"):
        setattr(a, k, 0x10000)
    a.zb = 0x10004
    p = cases.gauss(48, 1, 3).param.to_c()
    c = Loop().to_c()
    rc = lib().bgf_flow_step_noalloc(ctypes.byref(p), ctypes.byref(a), ctypes.byref(c), None)
    assert rc == 1, rc  # BGF_EINVAL
    assert b"16-byte" in lib().bgf_last_error()
