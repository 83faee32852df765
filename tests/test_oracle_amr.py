"""The CPU oracle against the reference on meshes refined by the reference's own
InitialAdaptation(): cross-level halo fills (restriction, barycentric prolongation,
wet/dry restriction and prolongation), bed-gradient halos, flux restriction at
coarse/fine faces and the substituted source terms, all bit-identical (float).

The reference-marked test runs the reference built from its sources next to the
oracle; the fixture test replays the committed block tables and reference
results (tests/golden/amr*.npz, written by tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import cases
from runners import interior, make_amr_pair, make_oracle_amr

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")

CASES = [
    # (case, steps, expected level histogram)
    (lambda: cases.amr_hump(64, 1, 1, 0.3), 30, [12, 16]),
    (lambda: cases.amr_hump(64, 2, 2, 0.3), 30, [8, 23, 36]),
    (lambda: cases.amr_dambreak(64, 1, 2), 40, [0, 40, 96]),
    (lambda: cases.amr_dambreak(64, 2, 2), 40, [0, 40, 96]),
    (lambda: cases.amr_dambreak(64, 1, 3), 20, [0, 32, 32, 384]),
]

FIXTURES = {
    "amrhump64_e1_l1": lambda: cases.amr_hump(64, 1, 1, 0.3),
    "amrhump64_e2_l2": lambda: cases.amr_hump(64, 2, 2, 0.3),
    "amrdam64_e1_l2": lambda: cases.amr_dambreak(64, 1, 2),
    "amrdam64_e2_l2": lambda: cases.amr_dambreak(64, 2, 2),
    "amrdam64_e1_l3": lambda: cases.amr_dambreak(64, 1, 3),
}


def load_tables(name):
    g = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return g, (g["level"], g["nbr"], g["xo"], g["yo"])


@pytest.mark.reference
@pytest.mark.parametrize("mk,nsteps,hist", CASES, ids=["hump_l1_e1", "hump_l2_e2", "dam_l2_e1", "dam_l2_e2", "dam_l3_e1"])
def test_oracle_matches_reference_on_adapted_mesh(have_reference, mk, nsteps, hist):
    case = mk()
    ref, orc, (lev, nbr, xo, yo) = make_amr_pair(case)
    assert list(np.bincount(lev, minlength=len(hist))) == hist
    # the level interfaces really exist: some neighbour is on another level
    assert any(lev[nbr[b, k]] != lev[b] for b in range(len(lev)) for k in range(8))
    dr = ref.step(nsteps)
    do = orc.step(nsteps)
    assert np.array_equal(dr, do), (dr[:5], do[:5])
    for name in ("h", "u", "v", "zs"):
        a, b = interior(ref.get(name)), interior(orc.get(name))
        assert np.array_equal(a, b), (name, float(np.abs(a - b).max()))


@pytest.mark.parametrize("name", list(FIXTURES))
def test_oracle_matches_reference_fixture_on_adapted_mesh(name):
    g, tables = load_tables(name)
    o = make_oracle_amr(FIXTURES[name](), tables)
    dts = o.step(int(g["nsteps"]))
    assert np.array_equal(dts, g["dts"])
    for k in ("h", "u", "v"):
        assert np.array_equal(interior(o.get(k)).astype(np.float32), g[k]), k
