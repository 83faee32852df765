"""bgf_adapt's table work on the device (bgf_set_adapt_mode 1, the default) against
the host C++ tables (mode 0): the same flags, ids, active list, levels, origins,
neighbour tables, bed and state, bit for bit, over several passes of refinement
and of refinement with coarsening."""
import numpy as np
import pytest

from bg_flood_b200.adapt import Criterion, INRANGE, depth_or_slope, parse_criterion
from runners import interior
from test_gpu_adapt_coarsen import dam_handle, run_steps

pytestmark = pytest.mark.gpu


def _state(f):
    act, lv, nb, xo, yo = f.get_blocks()
    zs, h, u, v = f.get_state()
    return act, lv, nb, xo, yo, f.get_bed(), h, u, v


def _same(a, b):
    act_a, lv_a, nb_a, xo_a, yo_a, zb_a, h_a, u_a, v_a = a
    act_b, lv_b, nb_b, xo_b, yo_b, zb_b, h_b, u_b, v_b = b
    assert np.array_equal(act_a, act_b)
    assert np.array_equal(lv_a[act_a], lv_b[act_b])
    assert np.array_equal(nb_a[act_a], nb_b[act_b])
    assert np.array_equal(xo_a[act_a], xo_b[act_b]) and np.array_equal(yo_a[act_a], yo_b[act_b])
    assert np.array_equal(interior(zb_a)[act_a], interior(zb_b)[act_b])
    for x, y in ((h_a, h_b), (u_a, u_b), (v_a, v_b)):
        assert np.array_equal(interior(x)[act_a], interior(y)[act_b])


def _pair():
    out = []
    for mode in (0, 1):
        case, f = dam_handle()
        f.set_adapt_mode(mode)
        out.append((case, f))
    return out


def test_refinement_same_on_device_and_host():
    (case, fh), (_, fd) = _pair()
    for crit in (parse_criterion("Threshold,0.5,zs"), depth_or_slope(0.3, 0.05)):
        nh, ih = fh.adapt(crit, maxiteration=4)
        nd, idv = fd.adapt(crit, maxiteration=4)
        assert (nh, ih) == (nd, idv)
        _same(_state(fh), _state(fd))


@pytest.mark.parametrize("thr", [(10.0, 100.0), (1.0, 0.2), (0.6, 0.02)])
def test_coarsening_same_on_device_and_host(thr):
    """Refine, run, then adapt with coarsening allowed (merges, refinements or both)."""
    (case, fh), (_, fd) = _pair()
    for f in (fh, fd):
        f.adapt(depth_or_slope(0.3, 0.05), maxiteration=3)
        run_steps(f, case, 40)
    _same(_state(fh), _state(fd))
    for f in (fh, fd):
        f.adapt(depth_or_slope(*thr), maxiteration=4, allow_coarsen=True)
    _same(_state(fh), _state(fd))
    # and the flow continues identically on both
    for f in (fh, fd):
        run_steps(f, case, 20)
    _same(_state(fh), _state(fd))


def test_inrange_on_the_bed_same_on_device_and_host():
    (case, fh), (_, fd) = _pair()
    crit = Criterion(INRANGE, "zb", 0.2, 0.4)
    assert fh.adapt(crit, maxiteration=5) == fd.adapt(crit, maxiteration=5)
    _same(_state(fh), _state(fd))
