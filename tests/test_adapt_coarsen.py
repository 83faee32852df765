"""Coarsening extension of the refinement pass, table level (no GPU): the C ABI's
bgf_adapt_sanity / bgf_adapt_tables against the CPU restatement in
coarsen_restate.py and against mesh invariants -- 2:1 balance, neighbour tables
equal to a brute-force search over block extents, the domain covered exactly once,
the reference's id and active-order rules (src/Adaptation.cu:535-596, 677-1015,
1762-1876)."""
import numpy as np
import pytest

import coarsen_restate as cr
from bg_flood_b200.adapt import adapt_sanity, adapt_tables, refine_sanity, refine_tables
from bg_flood_b200.mesh import uniform_mesh

DX = 2.0


def _tables(nbx, nby, mem):
    m = uniform_mesh(16 * nbx, 16 * nby, DX)
    act = np.arange(m.nblk, dtype=np.int32)
    level = np.zeros(mem, np.int32)
    nbr = np.zeros((mem, 8), np.int32)
    nbr[: m.nblk] = m.nbr
    xo = np.zeros(mem)
    yo = np.zeros(mem)
    xo[: m.nblk] = m.xo
    yo[: m.nblk] = m.yo
    return act, level, nbr, xo, yo


def _check_mesh(act, lev, nbr, xo, yo, area):
    assert cr.balanced(act, lev, nbr)
    assert np.array_equal(nbr[act], cr.brute_neighbours(act, lev, xo, yo, DX, nbr.shape)[act])
    assert cr.covered_area(act, lev, DX) == pytest.approx(area, rel=1e-12)
    assert len(set(act.tolist())) == len(act)


def test_refine_all_then_coarsen_all_restores_the_mesh():
    mem = 256
    act, lev, nbr, xo, yo = _tables(4, 4, mem)
    r = np.zeros(mem, np.uint8)
    r[act] = 1
    r, _ = refine_sanity(act, lev, nbr, mem, 0, 1, r)
    act1, lev1, nbr1, x1, y1, ch = refine_tables(act, lev, nbr, xo, yo, mem, DX, 0, r)
    assert len(act1) == 64
    c = np.zeros(mem, np.uint8)
    c[act1] = 1
    r2, c2 = adapt_sanity(act1, lev1, nbr1, mem, 0, 1, np.zeros(mem, np.uint8), c, x1, y1, DX)
    rr, cc = cr.sanity(act1, lev1, nbr1, 0, 1, x1, y1, DX, np.zeros(mem, np.uint8), c)
    assert np.array_equal(r2, rr) and np.array_equal(c2, cc)
    # exactly the 16 original ids are the quad parents
    assert sorted(np.flatnonzero(c2).tolist()) == list(range(16))
    act2, lev2, nbr2, x2, y2, ch2, sb2 = adapt_tables(act1, lev1, nbr1, x1, y1, mem, DX, 0, r2, c2)
    assert np.array_equal(act2, act)
    assert np.array_equal(lev2[act], lev[act]) and np.array_equal(nbr2[act], nbr[act])
    assert np.array_equal(x2[act], xo[act]) and np.array_equal(y2[act], yo[act])
    assert np.array_equal(sb2[:16], ch[:16]) and (ch2 == -1).all()


def test_reference_mode_cancels_coarsening():
    mem = 64
    act, lev, nbr, xo, yo = _tables(4, 4, mem)
    fl = np.zeros(mem, np.uint8)
    fl[5] = 1
    c = np.ones(mem, np.uint8)
    r0, c0 = refine_sanity(act, lev, nbr, mem, -2, 2, fl)
    r1, c1 = adapt_sanity(act, lev, nbr, mem, -2, 2, fl, c, xo, yo, DX, allow_coarsen=False)
    assert np.array_equal(r0, r1) and not c1[act].any() and not c0[act].any()
    t0 = refine_tables(act, lev, nbr, xo, yo, mem, DX, 0, r0)
    t1 = adapt_tables(act, lev, nbr, xo, yo, mem, DX, 0, r1, np.zeros(mem, np.uint8))
    for a, b in zip(t0, t1):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("seed", range(12))
def test_random_refine_coarsen_sequences(seed):
    """Random refine / coarsen flags over several passes on a 6x4-block domain, maxlevel
    3: flags equal the restatement, and every resulting mesh is a valid quadtree."""
    rng = np.random.default_rng(seed)
    mem = 24 * 64 + 64
    act, lev, nbr, xo, yo = _tables(6, 4, mem)
    area = cr.covered_area(act, lev, DX)
    minlevel, maxlevel = 0, 3
    merged = refined = 0
    for it in range(8):
        r = np.zeros(mem, np.uint8)
        c = np.zeros(mem, np.uint8)
        pr = 0.3 if it < 4 else 0.05
        r[act] = rng.random(len(act)) < pr
        c[act] = rng.random(len(act)) < (0.2 if it < 4 else 0.9)
        r1, c1 = adapt_sanity(act, lev, nbr, mem, minlevel, maxlevel, r, c, xo, yo, DX)
        r2, c2 = cr.sanity(act, lev, nbr, minlevel, maxlevel, xo, yo, DX, r, c)
        assert np.array_equal(r1, r2) and np.array_equal(c1, c2), it
        assert not (r1 & c1).any()
        free_before = sorted(set(range(mem)) - set(act.tolist()))
        nref = int(r1[act].sum())
        act2, lev2, nbr2, x2, y2, ch, sb = adapt_tables(act, lev, nbr, xo, yo, mem, DX, 0, r1, c1)
        _check_mesh(act2, lev2, nbr2, x2, y2, area)
        # quads: parents one level up, origins moved by the reference's rule, siblings gone
        parents = [ib for ib in act if c1[ib]]
        for p in parents:
            assert lev2[p] == lev[p] - 1
            d = np.float32(cr.calcres(DX, int(lev[p]) + 1))
            assert x2[p] == np.float32(np.float32(xo[p]) + d) and y2[p] == np.float32(np.float32(yo[p]) + d)
            assert set(sb[p]) == {nbr[p, cr.RB], nbr[p, cr.TL], nbr[nbr[p, cr.RB], cr.TL]}
            assert not set(sb[p]) & set(act2.tolist())
        # active order: survivors in order, then children of refined blocks in order,
        # taking ids that were free before the pass, ascending
        gone = set(sb[parents].ravel().tolist()) if parents else set()
        keep = [ib for ib in act if ib not in gone]
        kids = [int(k) for ib in keep if r1[ib] for k in ch[ib]]
        assert act2.tolist() == keep + kids
        assert kids == free_before[: 3 * nref]
        merged += len(parents)
        refined += nref
        act, lev, nbr, xo, yo = act2, lev2, nbr2, x2, y2
    assert merged > 0 and refined > 0


def test_malformed_quad_flags_are_rejected():
    mem = 64
    act, lev, nbr, xo, yo = _tables(4, 4, mem)
    r = np.zeros(mem, np.uint8)
    r[act] = 1
    act1, lev1, nbr1, x1, y1, _ = refine_tables(act, lev, nbr, xo, yo, mem, DX, 0, r)
    c = np.zeros(mem, np.uint8)
    c[int(nbr1[0, cr.RB])] = 1  # the right block of a quad is not its parent
    with pytest.raises(RuntimeError):
        adapt_tables(act1, lev1, nbr1, x1, y1, mem, DX, 0, np.zeros(mem, np.uint8), c)
    c[:] = 0
    c[0] = 1
    r2 = np.zeros(mem, np.uint8)
    r2[0] = 1  # refining and coarsening the same block
    with pytest.raises(RuntimeError):
        adapt_tables(act1, lev1, nbr1, x1, y1, mem, DX, 0, r2, c)
