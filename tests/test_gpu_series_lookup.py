"""Uniform series late in a long record: the boundary water level, the rain rate
and a river's discharge are looked up by bisection when the series' times are
non-decreasing and by the reference's forward scan otherwise; both give the
oracle's values bit for bit.
The run starts 400 s into a 601-sample record, where the forward scan walks
hundreds of samples per boundary cell and step."""
import numpy as np
import pytest

import cases
from bg_flood_b200.flow import BGFError, Loop
from bg_flood_b200.params import BndSegmentSpec
from runners import interior, make_gpu, make_oracle

pytestmark = pytest.mark.gpu

T0 = 400.0
NEXT = 1e9


def _river(sorted_times: bool):
    t = np.linspace(0.0, 600.0, 301)
    if not sorted_times:
        t[[100, 101]] = t[[101, 100]]
    return (-0.02, 0.02, -0.02, 0.02, t, 0.002 + 0.001 * np.sin(t / 30.0))


def _case(sorted_times: bool, rain: bool):
    case = cases.gauss(48, 1, 3)
    t = np.linspace(0.0, 600.0, 601)
    if not sorted_times:
        t[[200, 201]] = t[[201, 200]]   # two samples out of order, before T0
        t[[450, 451]] = t[[451, 450]]   # and two after
    wl = 0.1 + 0.01 * np.sin(t / 15.0)
    case.param.segments = [BndSegmentSpec("left", 2, list(t), list(wl))]
    if rain:
        rt = np.linspace(0.0, 3600.0, 3601)
        if not sorted_times:
            rt[[500, 501]] = rt[[501, 500]]
        case.rain = (list(rt), list(20.0 + 10.0 * np.sin(rt / 100.0)))
    case.nextoutputtime = NEXT
    return case


@pytest.mark.parametrize("sorted_times", [True, False], ids=["sorted", "unsorted"])
@pytest.mark.parametrize("rain,river", [(False, False), (True, False), (False, True)],
                         ids=["bnd", "bnd+rain", "bnd+river"])
def test_late_series_lookup_bitexact(sorted_times, rain, river):
    case = _case(sorted_times, rain)
    f, mesh, loop0 = make_gpu(case)
    o, _ = make_oracle(case)
    if river:
        xs, xe, ys, ye, t, q = _river(sorted_times)
        if not sorted_times:
            # discharge series must have increasing times (readFlowfile's files do)
            with pytest.raises(BGFError):
                f.add_river(xs, xe, ys, ye, t, q)
            return
        assert f.add_river(xs, xe, ys, ye, t, q) == o.add_river(xs, xe, ys, ye, t, q) > 0
    loop = Loop(totaltime=T0, dt=loop0.dt, dtmax=loop0.dtmax, nextoutputtime=NEXT)
    o.set_loop(T0, NEXT, loop0.dtmax)
    for s in range(20):
        dt = f.flow_step(loop)
        loop.totaltime += dt
        do = o.step(1)[0]
        assert dt == do, (s, dt, do)
    zs, h, u, v = f.get_state()
    for name, a in (("h", h), ("u", u), ("v", v)):
        assert np.array_equal(interior(a).astype(np.float64), interior(o.get(name))), name
