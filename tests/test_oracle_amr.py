"""The CPU oracle against the reference on meshes refined by the reference's own
InitialAdaptation(): cross-level halo fills (restriction, barycentric prolongation,
wet/dry restriction and prolongation), bed-gradient halos, flux restriction at
coarse/fine faces and the substituted source terms, all bit-identical (float)."""
import numpy as np
import pytest

import cases
from runners import interior, make_amr_pair

pytestmark = pytest.mark.reference

CASES = [
    # (case, steps, expected level histogram)
    (lambda: cases.amr_hump(64, 1, 1, 0.3), 30, [12, 16]),
    (lambda: cases.amr_hump(64, 2, 2, 0.3), 30, [8, 23, 36]),
    (lambda: cases.amr_dambreak(64, 1, 2), 40, [0, 40, 96]),
    (lambda: cases.amr_dambreak(64, 2, 2), 40, [0, 40, 96]),
]


@pytest.mark.parametrize("mk,nsteps,hist", CASES, ids=["hump_l1_e1", "hump_l2_e2", "dam_l2_e1", "dam_l2_e2"])
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
