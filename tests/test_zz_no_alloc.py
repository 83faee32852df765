"""The allocation-free flow step (bgf_flow_step_noalloc) against the handle-based
bgf_flow_step on the same inputs, two calls in a row.

It serves callers that cannot allocate device memory once running (a service
with a pre-reserved GPU memory pool, or a host model that owns every device
array); here the test itself allocates the caller's arrays with torch, and the
entry point only uses its static scratch array.  This file is collected last so
that a failure here leaves every other test already run."""
import ctypes

import numpy as np
import pytest

import cases
from bg_flood_b200._native import lib
from bg_flood_b200.flow import CLoop, Loop
from bg_flood_b200.mesh import boundary_segments, fill_halo, grid_to_buq
from runners import interior, make_gpu, make_oracle

pytestmark = pytest.mark.gpu


class NoallocArgs(ctypes.Structure):
    _fields_ = [("nblk", ctypes.c_int), ("nblkmem", ctypes.c_int)] + \
        [(n, ctypes.c_void_p) for n in ("active", "level", "nbr", "bndtype", "zb", "dzbdx", "dzbdy",
                                        "h_in", "u_in", "v_in", "h_out", "u_out", "v_out")] + \
        [("reset_means", ctypes.c_int)]


def _device_inputs(case, mesh, torch):
    n = mesh.nblk
    dt = torch.float32
    o, _ = make_oracle(case)  # the bed gradients of the reference initialisation
    zb = torch.tensor(fill_halo(grid_to_buq(case.zb, mesh), mesh).reshape(n, 324), dtype=dt, device="cuda")
    gx = torch.tensor(o.get("dzbdx").reshape(n, 324), dtype=dt, device="cuda")
    gy = torch.tensor(o.get("dzbdy").reshape(n, 324), dtype=dt, device="cuda")
    bnd = np.full((n, 4), -1, np.int32)
    for typ, _, _, sides in boundary_segments(mesh, case.param.segments, case.param.aoibnd, case.xo, case.yo):
        for s, blks in enumerate(sides):
            bnd[blks, s] = typ
    state = [torch.tensor(interior(grid_to_buq(getattr(case, k), mesh)).reshape(n, 256), dtype=dt, device="cuda")
             for k in ("h", "u", "v")]
    t = {
        "active": torch.arange(n, dtype=torch.int32, device="cuda"),
        "level": torch.tensor(mesh.level, dtype=torch.int32, device="cuda"),
        "nbr": torch.tensor(np.ascontiguousarray(mesh.nbr.T), dtype=torch.int32, device="cuda"),
        "bndtype": torch.tensor(bnd, device="cuda"),
        "zb": zb, "dzbdx": gx, "dzbdy": gy,
    }
    return t, state


def _step(case, t, state_in, state_out, loop, reset=False):
    a = NoallocArgs()
    a.reset_means = 1 if reset else 0
    a.nblk = a.nblkmem = t["active"].numel()
    for k in ("active", "level", "nbr", "bndtype", "zb", "dzbdx", "dzbdy"):
        setattr(a, k, t[k].data_ptr())
    a.h_in, a.u_in, a.v_in = (x.data_ptr() for x in state_in)
    a.h_out, a.u_out, a.v_out = (x.data_ptr() for x in state_out)
    p = case.param.to_c()
    c = loop.to_c()
    rc = lib().bgf_flow_step_noalloc(ctypes.byref(p), ctypes.byref(a), ctypes.byref(c), None)
    assert rc == 0, (rc, lib().bgf_last_error())
    loop.from_c(c)
    return loop.dt


@pytest.mark.parametrize("mk", [lambda: cases.gauss(48, 1, 3), lambda: cases.hump_walls(64, 2)],
                         ids=["gauss48_e1_absorbing", "hump64_e2_walls"])
def test_noalloc_step_matches_handle_step(mk):
    torch = pytest.importorskip("torch")
    case = mk()
    f, mesh, loop = make_gpu(case)
    t, cur = _device_inputs(case, mesh, torch)
    nxt = [torch.empty_like(x) for x in cur]
    nloop = Loop(totaltime=loop.totaltime, dt=loop.dt, dtmax=loop.dtmax, nextoutputtime=loop.nextoutputtime)
    torch.cuda.synchronize()
    for step in range(2):  # two calls in a row: the static scratch is reused
        dt_ref = f.flow_step(loop)
        loop.totaltime += dt_ref
        dt_na = _step(case, t, cur, nxt, nloop, reset=step == 0)
        nloop.totaltime += dt_na
        assert dt_na == dt_ref, (step, dt_na, dt_ref)
        zs, h, u, v = f.get_state()
        for name, ref, got in (("h", h, nxt[0]), ("u", u, nxt[1]), ("v", v, nxt[2])):
            ref_i = interior(ref).reshape(mesh.nblk, 256)
            assert np.array_equal(got.cpu().numpy(), ref_i), (step, name)
        cur, nxt = nxt, cur


def test_noalloc_absorbing_means_carry_across_calls():
    """An absorbing edge with the dt key set: the boundary's running means (the time
    filter of ABS1DQ, src/Boundary.cu:481-537) carry from call to call in the static
    array, so 30 calls follow bgf_flow_step and the oracle step by step, bit for bit,
    while the wave leaves the domain."""
    torch = pytest.importorskip("torch")
    case = cases.gauss(48, 1, 3)
    case.param.dt = 0.01
    case.param.bndfiltertime = 0.05
    f, mesh, loop = make_gpu(case)
    o, _ = make_oracle(case)
    t, cur = _device_inputs(case, mesh, torch)
    init = [x.clone() for x in cur]
    nxt = [torch.empty_like(x) for x in cur]
    loop0 = (loop.totaltime, loop.dt, loop.dtmax, loop.nextoutputtime)
    nloop = Loop(*loop0)
    torch.cuda.synchronize()
    nsteps = 30
    for step in range(nsteps):
        dt_ref = f.flow_step(loop)
        loop.totaltime += dt_ref
        dt_na = _step(case, t, cur, nxt, nloop, reset=step == 0)
        nloop.totaltime += dt_na
        dt_o = float(o.step(1)[0])
        assert dt_na == dt_ref == dt_o, (step, dt_na, dt_ref, dt_o)
        zs, h, u, v = f.get_state()
        for name, ref, got in (("h", h, nxt[0]), ("u", u, nxt[1]), ("v", v, nxt[2])):
            ref_i = interior(ref).reshape(mesh.nblk, 256)
            assert np.array_equal(got.cpu().numpy(), ref_i), (step, name)
            assert np.array_equal(got.cpu().numpy(), interior(o.get(name)).reshape(mesh.nblk, 256)), (step, name)
        cur, nxt = nxt, cur
    final_h = cur[0].cpu().numpy().copy()
    # the case is sensitive to the running means: clearing them on every call
    # (what the step did before they were kept) ends elsewhere
    cur = [x.clone() for x in init]
    nxt = [torch.empty_like(x) for x in cur]
    nloop = Loop(*loop0)
    for step in range(nsteps):
        nloop.totaltime += _step(case, t, cur, nxt, nloop, reset=True)
        cur, nxt = nxt, cur
    assert not np.array_equal(cur[0].cpu().numpy(), final_h)


def test_noalloc_rejects_too_many_blocks():
    case = cases.hump_walls(64, 2)
    a = NoallocArgs()
    a.nblk = 16
    a.nblkmem = 513  # above BGF_NOALLOC_MAX_BLOCKS = 512
    p = case.param.to_c()
    c = CLoop(1e30, 0.0, 0.1, 0.0)
    assert lib().bgf_flow_step_noalloc(ctypes.byref(p), ctypes.byref(a), ctypes.byref(c), None) == 1
