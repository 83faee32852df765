"""Edge cases of the mesh and state on the B200, against the oracle: a single
block (every neighbour the block itself), one-block-wide strips in x and in y, an
all-dry domain, and meshes the library must reject."""
import numpy as np
import pytest

import cases
from bg_flood_b200.flow import BGFError, FlowB200
from bg_flood_b200.mesh import uniform_mesh
from bg_flood_b200.params import Param
from runners import interior, make_gpu, make_oracle

pytestmark = pytest.mark.gpu


def _case(nx, ny, kind, engine=1):
    dx = 0.5
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    X, Y = np.meshgrid(x, y)
    zb = (0.01 * X - 0.005 * Y).astype(np.float32)
    if kind == "hump":
        h = np.maximum(0.3 + 0.1 * np.exp(-((X - x.mean()) ** 2 + (Y - y.mean()) ** 2) / 4.0) - zb, 0.0)
    elif kind == "dam":
        h = np.where(X < x.mean(), 0.5 - zb, 0.0)
    else:  # dry
        h = np.zeros_like(X)
    h = h.astype(np.float32)
    z = np.zeros_like(h)
    p = Param(dx=dx, xo=0.0, yo=0.0, engine=engine, aoibnd=0, cf=0.001, frictionmodel=0)
    return cases.Case(f"{kind}{nx}x{ny}_e{engine}", p, cases._param_text(p), dx, 0.0, 0.0, zb, h, z, z.copy(),
                      nextoutputtime=1e30)


@pytest.mark.parametrize("nx,ny,kind,engine", [
    (16, 16, "hump", 1), (16, 16, "dam", 2),      # a single block
    (128, 16, "dam", 1), (16, 128, "dam", 2),     # strips one block wide
    (48, 32, "dry", 1),                           # nothing wet
])
def test_edge_meshes_bitexact_vs_oracle(nx, ny, kind, engine):
    c = _case(nx, ny, kind, engine)
    f, mesh, loop = make_gpu(c)
    o, _ = make_oracle(c)
    for _ in range(25):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        assert dt == o.step(1)[0]
    zs, h, u, v = f.get_state()
    for name, a in (("h", h), ("u", u), ("v", v)):
        assert np.array_equal(interior(a).astype(np.float64), interior(o.get(name))), name
    if kind == "dry":
        assert not interior(h).any()


def test_degenerate_meshes_are_rejected():
    with pytest.raises(ValueError):
        uniform_mesh(24, 16, 1.0)          # not whole blocks
    p = Param(dx=1.0, xo=0.0, yo=0.0)
    f = FlowB200(p, 4)
    with pytest.raises(BGFError) as e:
        f.set_blocks(np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros((0, 8), np.int32))
    assert e.value.status == 1            # BGF_EINVAL: no active block
    nbr = np.array([[0, 0, 7, 7, 0, 0, 0, 0]], np.int32)   # neighbour outside the slots
    with pytest.raises(BGFError):
        f.set_blocks(np.zeros(1, np.int32), np.zeros(1, np.int32), nbr)
    with pytest.raises(BGFError):
        f.flow_step(__import__("bg_flood_b200.flow", fromlist=["Loop"]).Loop())  # no bed or state yet
    f.close()
