"""The refinement pass's table work (bgf_refine_sanity, bgf_refine_tables) against
the reference's own Adaptation(): refine/coarsen flags, the active list, levels,
all eight neighbour tables and the block origins, bit for bit, iteration by
iteration until the mesh stops changing (2 to 4 levels, reallocating meshes).

The reference-marked test runs the reference; the fixture test replays the
recorded iterations (tests/golden/adapt_tables.npz, written by
tests/golden/make_golden.py) without it."""
import os

import numpy as np
import pytest

from adapt_cases import ADAPT_CASES, MEM, criterion_of, id_tables, reference_with_bathy
from bg_flood_b200.adapt import refine_sanity, refine_tables

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "adapt_tables.npz")


def _mine(case, act, level, nbr, xo, yo, pre):
    fl = np.zeros(MEM, np.uint8)
    fl[act] = pre
    r, c = refine_sanity(act, level, nbr, MEM, case.param.minlevel, case.param.maxlevel, fl)
    out = refine_tables(act, level, nbr, xo, yo, MEM, case.dx, 0, r)
    return r[act], c[act], out


@pytest.mark.reference
@pytest.mark.parametrize("name", list(ADAPT_CASES))
def test_refinement_tables_match_reference(have_reference, name):
    case = ADAPT_CASES[name]()
    crit = criterion_of(case)
    r = reference_with_bathy(case)
    for it in range(8):
        act, level, nbr, xo, yo = id_tables(r)
        pre = crit.flags(r.get(crit.var)[:, 1:17, 1:17])
        rf_m, cf_m, (act2, lv2, nb2, x2, y2, _) = _mine(case, act, level, nbr, xo, yo, pre)
        rf, cf = r.flags()  # one reference iteration
        assert np.array_equal(rf_m, rf) and not cf.any() and not cf_m.any(), it
        act_r, level_r, nbr_r, xo_r, yo_r = id_tables(r)
        assert np.array_equal(act2, act_r), it
        assert np.array_equal(lv2[act_r], level_r[act_r]), it
        assert np.array_equal(nb2[act_r], nbr_r[act_r]), it
        assert np.array_equal(x2[act_r].astype(np.float32), xo_r[act_r].astype(np.float32)), it
        assert np.array_equal(y2[act_r].astype(np.float32), yo_r[act_r].astype(np.float32)), it
        if len(act_r) == len(act):
            break
    assert it >= 1


def test_refinement_tables_match_reference_fixture():
    g = np.load(GOLDEN)
    for key in sorted(k for k in g.files if k.endswith("_pre")):
        stem = key[: -len("_pre")]
        name = stem.rsplit("_it", 1)[0]
        case = ADAPT_CASES[name]()
        act, level, nbr, xo, yo = (g[f"{stem}_{k}"] for k in ("act", "level", "nbr", "xo", "yo"))
        rf_m, cf_m, (act2, lv2, nb2, x2, y2, _) = _mine(case, act, level, nbr, xo, yo, g[key])
        assert np.array_equal(rf_m, g[f"{stem}_refine"]) and not cf_m.any(), stem
        act_r = g[f"{stem}_act_out"]
        assert np.array_equal(act2, act_r), stem
        assert np.array_equal(lv2[act_r], g[f"{stem}_level_out"]), stem
        assert np.array_equal(nb2[act_r], g[f"{stem}_nbr_out"]), stem
        assert np.array_equal(x2[act_r].astype(np.float32), g[f"{stem}_xo_out"].astype(np.float32)), stem
        assert np.array_equal(y2[act_r].astype(np.float32), g[f"{stem}_yo_out"].astype(np.float32)), stem


def test_sanity_pass_balances_levels():
    """A block flagged next to a coarser block drags it along (2:1 balance)."""
    # 2x2 level-0 blocks; block 0 already refined into 0, 4, 5, 6 (level 1)
    from bg_flood_b200.mesh import uniform_mesh  # noqa: F401
    mem = 16
    act = np.array([0, 1, 2, 3], np.int32)
    level = np.zeros(mem, np.int32)
    nbr = np.zeros((mem, 8), np.int32)
    nbr[0] = [0, 0, 1, 1, 0, 0, 2, 2]
    nbr[1] = [0, 0, 1, 1, 1, 1, 3, 3]
    nbr[2] = [2, 2, 3, 3, 0, 0, 2, 2]
    nbr[3] = [2, 2, 3, 3, 1, 1, 3, 3]
    xo = np.array([0.5, 16.5, 0.5, 16.5] + [0.0] * 12)
    yo = np.array([0.5, 0.5, 16.5, 16.5] + [0.0] * 12)
    fl = np.zeros(mem, np.uint8)
    fl[0] = 1
    r, c = refine_sanity(act, level, nbr, mem, 0, 2, fl)
    act2, lv2, nb2, x2, y2, ch = refine_tables(act, level, nbr, xo, yo, mem, 1.0, 1, r)
    assert list(act2) == [0, 1, 2, 3, 4, 5, 6] and list(ch[0]) == [4, 5, 6]
    assert list(lv2[act2]) == [1, 0, 0, 0, 1, 1, 1]
    # right side of child 4 (bottom-right) is block 1 (coarser); block 1's left side is 4 then 6
    assert list(nb2[4][2:4]) == [1, 1] and list(nb2[1][0:2]) == [4, 6]
    # second pass: refining child 4 forces block 1 (coarser, level 0) to refine
    fl2 = np.zeros(mem, np.uint8)
    fl2[4] = 1
    r2, _ = refine_sanity(act2, lv2, nb2, mem, 0, 2, fl2)
    assert r2[4] and r2[1] and not r2[2] and not r2[3]
