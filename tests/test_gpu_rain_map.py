"""Gridded rain on the B200 against the oracle (pinned to the reference's rain-map
path on the CPU).  Within tolerances, as for uniform rain: the reference adds the
rain to h and to its stored zs separately, this library keeps zs = zb + h; the
case also uses Manning friction (cbrtf)."""
import numpy as np
import pytest

from rainmap_case import MAP, NSTEPS, rainmap_case
from runners import interior, make_gpu, make_oracle

pytestmark = pytest.mark.gpu
FIELD_TOL = 1e-5
DT_RTOL = 1e-5


@pytest.mark.parametrize("fast", [0, 1])
def test_rain_map_close_to_oracle(fast):
    c, before, after = rainmap_case()
    c.param.fastmath = fast
    frames = np.stack([before, after])
    f, _, loop = make_gpu(c)
    f.set_rain_map(MAP["xo"], MAP["yo"], MAP["dx"], MAP["dy"], MAP["to"], MAP["dt"], frames)
    o, _ = make_oracle(c)
    o.set_rain_map(MAP["xo"], MAP["yo"], MAP["dx"], MAP["dy"], MAP["to"], MAP["dt"], frames)
    tol = FIELD_TOL if not fast else 2e-4
    for _ in range(NSTEPS):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        do = o.step(1)[0]
        assert abs(dt - do) <= (DT_RTOL if not fast else 1e-4) * do
    zs, h, u, v = f.get_state()
    for k, a in (("h", h), ("u", u), ("v", v)):
        assert float(np.abs(interior(a).astype(np.float64) - interior(o.get(k))).max()) <= tol, k
    assert float(interior(h).sum()) > 0.0


def test_rain_map_replaces_uniform_series():
    # a uniform series set after the map replaces it, and the other way round
    c, before, after = rainmap_case()
    f, _, loop = make_gpu(c)
    f.set_rain_map(MAP["xo"], MAP["yo"], MAP["dx"], MAP["dy"], MAP["to"], MAP["dt"], np.stack([before, after]))
    f.set_rain([0.0, 1e9], [0.0, 0.0])
    v0 = f.volume()
    for _ in range(5):
        loop.totaltime += f.flow_step(loop)
    assert f.volume() == v0  # no rain: dry terrain stays dry
