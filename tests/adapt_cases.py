"""Reference-side drivers for the refinement-pass tests (test infrastructure):
a reference model whose bathymetry forcing is the case's own bed on the level-0
cell centres, so that Adaptation() re-interpolates a real bed."""
from __future__ import annotations

import numpy as np

import cases
from bg_flood_b200.adapt import parse_criterion
from oracle.pyoracle import Reference

MEM = 4096  # block slots of the host tables in the table tests

ADAPT_CASES = {
    "island64_e1_l2": lambda: cases.amr_island(64, 1, 2, 0.5),
    "hump64_e1_l2": lambda: cases.amr_hump(64, 1, 2, 0.3),
    "dam64_e1_l3": lambda: cases.amr_dambreak(64, 1, 3),
    "island128_e2_l3": lambda: cases.amr_island(128, 2, 3, 0.4),
}


def level0_grids(case):
    n0 = case.n0
    ii = (np.arange(n0) + 0.5) * case.dx
    X, Y = np.meshgrid(case.xo + ii, case.yo + ii)
    zb0 = case.zb_fn(X, Y).astype(np.float32)
    eta0 = case.adapt_eta_fn if case.adapt_eta_fn is not None else case.eta_fn
    h0 = np.maximum(eta0(X, Y) - zb0, 0).astype(np.float32)
    return zb0, h0


def reference_with_bathy(case) -> Reference:
    zb0, h0 = level0_grids(case)
    z0 = np.zeros_like(zb0)
    r = Reference(case.paramtext, case.n0, case.n0, case.dx, case.xo, case.yo, zb0, h0, z0, z0, None,
                  case.nextoutputtime)
    r.set_bathy(case.xo + 0.5 * case.dx, case.yo + 0.5 * case.dx, case.dx, zb0)
    return r


def criterion_of(case):
    line = [ln for ln in case.paramtext.splitlines() if ln.startswith("Adaptation")][0]
    return parse_criterion(line.split("=", 1)[1])


def id_tables(r: Reference, mem: int = MEM):
    """The reference's current tables indexed by block id: (active, level, nbr8, xo, yo)."""
    act = r.active()
    lev_a, nb_a, xo_a, yo_a = r.blocks()
    level = np.zeros(mem, np.int32)
    nbr = np.zeros((mem, 8), np.int32)
    xo = np.zeros(mem)
    yo = np.zeros(mem)
    level[act] = lev_a
    nbr[act] = nb_a
    xo[act] = xo_a
    yo[act] = yo_a
    return act, level, nbr, xo, yo


# ---------------------------------------------------------------- Targetlevel criterion

def target_case():
    """The hump case with the Targetlevel criterion (maps added separately)."""
    case = cases.amr_hump(64, 1, 2, 0.3)
    case.paramtext = "\n".join("Adaptation = Targetlevel" if ln.startswith("Adaptation") else ln
                               for ln in case.paramtext.splitlines()) + "\n"
    return case


def target_maps(case):
    """Two target-level maps of 17 x 17 nodes over the level-0 domain, as
    (xo, yo, dx, levels (ny, nx) int32).  The first asks for level 2 everywhere and
    is overridden by the second (the reference applies the maps in turn and the
    last decides): level 2 in a disc, 1 in a band around it and along the south
    edge, 0 elsewhere."""
    ext = case.n0 * case.dx
    dxm = ext / 16.0
    xs = case.xo + dxm * np.arange(17)
    ys = case.yo + dxm * np.arange(17)
    X, Y = np.meshgrid(xs, ys)
    r = np.hypot(X - (case.xo + 0.3 * ext), Y - (case.yo + 0.6 * ext))
    second = np.where(r < 0.2 * ext, 2, np.where(r < 0.3 * ext, 1, 0))
    second[Y < case.yo + 0.15 * ext] = 1
    first = np.full((17, 17), 2)
    return [(case.xo, case.yo, dxm, first.astype(np.int32)), (case.xo, case.yo, dxm, second.astype(np.int32))]
