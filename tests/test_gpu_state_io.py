"""bgf_set_state / bgf_get_state: the DMA path for page-locked host arrays and the
host-conversion path give the same arrays (interiors of active blocks, zeros
elsewhere), on a mesh with spare block slots."""
import numpy as np
import pytest
import torch

import cases
from bg_flood_b200.flow import FlowB200, Loop
from bg_flood_b200.mesh import boundary_segments, fill_halo, grid_to_buq, uniform_mesh

pytestmark = pytest.mark.gpu


def _pinned(shape, dtype):
    t = torch.zeros(shape, dtype=torch.float64 if dtype == np.float64 else torch.float32, pin_memory=True)
    return t, t.numpy()


@pytest.mark.parametrize("dbl", [0, 1])
def test_pinned_and_pageable_state_io_agree(dbl):
    c = cases.dam_break(48, 1)
    c.param.doubleprecision = dbl
    mesh = uniform_mesh(c.nx, c.ny, c.dx, doubleprecision=bool(dbl))
    nmem = mesh.nblk + 5  # spare slots: their tiles must come back as zeros
    f = FlowB200(c.param, nmem)
    f.set_blocks(mesh.active, mesh.level, mesh.nbr, mesh.xo, mesh.yo)
    zb = np.zeros((nmem, 18, 18))
    zb[: mesh.nblk] = fill_halo(grid_to_buq(c.zb, mesh), mesh)
    f.set_bed(zb)
    for typ, times, levels, sides in boundary_segments(mesh, c.param.segments, c.param.aoibnd):
        f.add_segment(typ, times, levels, sides)
    dt = f.dtype
    fields = []
    for a in (c.h, c.u, c.v):
        b = np.full((nmem, 18, 18), 7.0, dt)  # halo and spare entries are ignored on upload
        b[: mesh.nblk] = grid_to_buq(a, mesh, dt)
        fields.append(b)
    keep = []
    pin_in = []
    for b in fields:
        t, n = _pinned(b.shape, dt)
        n[...] = b
        keep.append(t)
        pin_in.append(n)
    f.set_state(*pin_in)                       # DMA path
    pin_out = []
    for _ in range(4):
        t, n = _pinned((nmem, 18, 18), dt)
        n[...] = 3.0                           # everything is overwritten
        keep.append(t)
        pin_out.append(n)
    f.get_state(out=pin_out)
    page = f.get_state(out=[np.full((nmem, 18, 18), 3.0, dt) for _ in range(4)])   # host path
    for a, b in zip(pin_out, page):
        assert np.array_equal(a, b)
    # interiors of the active blocks are the state, everything else 0
    for k, b in enumerate(fields):
        got = page[k + 1]
        assert np.array_equal(got[: mesh.nblk, 1:17, 1:17], b[: mesh.nblk, 1:17, 1:17])
        mask = np.ones_like(got, bool)
        mask[: mesh.nblk, 1:17, 1:17] = False
        assert not got[mask].any()
    # after steps, both paths still agree and the pageable upload gives the same run
    loop = Loop(nextoutputtime=1e30)
    f.init_dt(loop)
    for _ in range(5):
        loop.totaltime += f.flow_step(loop)
    f.get_state(out=pin_out)
    page = f.get_state()
    for a, b in zip(pin_out, page):
        assert np.array_equal(a, b)
    f.close()
