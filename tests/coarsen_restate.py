"""CPU restatement of the coarsening extension of the refinement pass (test
infrastructure, compared with the library in tests/test_adapt_coarsen.py and
tests/test_gpu_adapt_coarsen.py).

The reference's refinesanitycheck (src/Adaptation.cu:157-296) and
checkneighbourrefine (:298-312) are restated without the line that cancels every
coarsening flag (:173-175); coarsen (:677-1015) merges each flagged quad into its
lower-left block.  The depth-or-slope criterion has no counterpart in the reference;
it is restated from the library's documented definition.  Neighbour tables are
checked against a brute-force search over block extents, a method independent of
the library's lookup by quadtree coordinates."""
from __future__ import annotations

import numpy as np

LB, LT, RB, RT, BL, BR, TL, TR = range(8)


def calcres(dx: float, level: int) -> float:
    return dx / (1 << level) if level >= 0 else dx * (1 << -level)


def hgrad_flags(h, zs, level, active, dx, eps, hthr, gthr, dtype=np.float32):
    """Refine / coarsen-candidate flag per block id from interior cells h, zs
    (nblkmem, 16, 16) indexed [block, y, x]."""
    T = dtype
    nb = len(level)
    refine = np.zeros(nb, np.uint8)
    coarsen = np.zeros(nb, np.uint8)
    epsT, h1, g1 = T(eps), T(hthr), T(gthr)
    hh, gh = h1 * T(0.5), g1 * T(0.5)
    for ib in active:
        hb = np.asarray(h[ib], T)
        z = np.asarray(zs[ib], T)
        dxl = T(calcres(dx, int(level[ib])))
        wet = hb > epsT

        def slope(axis):
            g = np.zeros((16, 16), T)
            for y in range(16):
                for x in range(16):
                    if not wet[y, x]:
                        continue
                    if axis == 0:
                        okm = x > 0 and wet[y, x - 1]
                        okp = x < 15 and wet[y, x + 1]
                        zm = z[y, x - 1] if x > 0 else T(0)
                        zp = z[y, x + 1] if x < 15 else T(0)
                    else:
                        okm = y > 0 and wet[y - 1, x]
                        okp = y < 15 and wet[y + 1, x]
                        zm = z[y - 1, x] if y > 0 else T(0)
                        zp = z[y + 1, x] if y < 15 else T(0)
                    if okm and okp:
                        g[y, x] = (zp - zm) / (T(2) * dxl)
                    elif okp:
                        g[y, x] = (zp - z[y, x]) / dxl
                    elif okm:
                        g[y, x] = (z[y, x] - zm) / dxl
            return g

        gx, gy = slope(0), slope(1)
        g2 = gx * gx + gy * gy
        refine[ib] = 1 if np.any((hb > h1) | (g2 > g1 * g1)) else 0
        coarsen[ib] = 0 if np.any((hb > hh) | (g2 > gh * gh)) else 1
    return refine, coarsen


def sanity(active, level, nbr, minlevel, maxlevel, xo, yo, dx, refine, coarsen, allow_coarsen=True):
    """refinesanitycheck with coarsening kept; nbr is (nblkmem, 8)."""
    r = np.array(refine, np.uint8)
    c = np.array(coarsen, np.uint8)
    for ib in active:
        if r[ib] and level[ib] == maxlevel:
            r[ib] = 0
        if c[ib] and level[ib] == minlevel:
            c[ib] = 0
        if not allow_coarsen or r[ib]:
            c[ib] = 0
    if allow_coarsen:
        for ib in active:
            if r[ib]:
                c[nbr[ib]] = 0
        for ib in active:
            lv = level[ib]
            if c[ib] and any(lv < level[nbr[ib, k]] for k in (LB, RB, TL, BL)):
                c[ib] = 0
    changed = True
    while changed:
        changed = False
        for ib in active:
            if not r[ib]:
                continue
            for k in (TL, BL, LB, RB):
                nb = nbr[ib, k]
                if not r[nb] and level[nb] < level[ib]:
                    r[nb] = 1
                    c[nb] = 0
                    changed = True
                if level[nb] == level[ib]:
                    c[nb] = 0
    if not allow_coarsen:
        return r, c
    for ib in active:
        if not c[ib]:
            continue
        dxl = calcres(dx, int(level[ib]))
        ix, iy = int(xo[ib] / dxl / 16.0), int(yo[ib] / dxl / 16.0)
        rr, t = nbr[ib, RB], nbr[ib, TL]
        tr = nbr[nbr[ib, TR], RB]
        lv = level[ib]
        corner = ix % 2 == 0 and iy % 2 == 0 and rr != ib and t != ib and tr != nbr[ib, TR]
        if not (corner and level[rr] == lv and level[t] == lv and level[tr] == lv and c[rr] and c[t] and c[tr]):
            c[ib] = 0
    return r, c


def block_xy(xo, yo, level, dx, ib):
    dxl = calcres(dx, int(level[ib]))
    return int(np.floor((xo[ib] / dxl - 0.5) / 16.0 + 0.5)), int(np.floor((yo[ib] / dxl - 0.5) / 16.0 + 0.5))


def brute_neighbours(active, level, xo, yo, dx, nbr_shape):
    """Neighbour tables by a search over block extents: a side touching one block
    of its own or a coarser level names it twice, two finer blocks name the lower /
    left one then the upper / right one, no block names the block itself."""
    act = list(active)
    top = max(int(level[ib]) for ib in act) + 1
    ext = {}
    for ib in act:
        bx, by = block_xy(xo, yo, level, dx, ib)
        s = 1 << (top - int(level[ib]))
        ext[ib] = (bx * s, (bx + 1) * s, by * s, (by + 1) * s)
    out = np.zeros(nbr_shape, np.int32)
    for ib in act:
        x0, x1, y0, y1 = ext[ib]
        sides = [[], [], [], []]
        for jb in act:
            if jb == ib:
                continue
            a0, a1, b0, b1 = ext[jb]
            yov = b0 < y1 and b1 > y0
            xov = a0 < x1 and a1 > x0
            if a1 == x0 and yov:
                sides[0].append((b0, jb))
            if a0 == x1 and yov:
                sides[1].append((b0, jb))
            if b1 == y0 and xov:
                sides[2].append((a0, jb))
            if b0 == y1 and xov:
                sides[3].append((a0, jb))
        for s in range(4):
            lst = sorted(sides[s])
            if not lst:
                lo = hi = ib
            elif len(lst) == 1:
                lo = hi = lst[0][1]
            else:
                assert len(lst) == 2, (ib, s, lst)
                lo, hi = lst[0][1], lst[1][1]
            out[ib, 2 * s] = lo
            out[ib, 2 * s + 1] = hi
    return out


def balanced(active, level, nbr) -> bool:
    """Every side neighbour within one level (the reference's checkBUQsanity intent)."""
    return all(abs(int(level[nbr[ib, k]]) - int(level[ib])) <= 1 for ib in active for k in range(8))


def covered_area(active, level, dx) -> float:
    return float(sum((16 * calcres(dx, int(level[ib]))) ** 2 for ib in active))


def merged_cells(old, quads, dtype=np.float32):
    """coarsen, step 1: the parent's cells from the old interior values `old`
    (nblkmem, 16, 16) [block, y, x] of its quad; quads is a list of
    (parent, right, top, top-right)."""
    T = dtype
    out = {}
    for q in quads:
        p = np.zeros((16, 16), T)
        for iy in range(16):
            for ix in range(16):
                src = q[(1 if ix >= 8 else 0) + (2 if iy >= 8 else 0)]
                cx, cy = 2 * (ix & 7), 2 * (iy & 7)
                a = old[src]
                p[iy, ix] = T(0.25) * (((T(a[cy, cx]) + T(a[cy, cx + 1])) + T(a[cy + 1, cx])) + T(a[cy + 1, cx + 1]))
        out[q[0]] = p
    return out
