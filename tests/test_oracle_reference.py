"""The CPU oracle against the reference BG_Flood compiled from its own sources:
bit-identical block tables, bed gradients, dt sequences and fields (float)."""
import numpy as np
import pytest

import cases
from runners import interior, make_oracle, make_reference

pytestmark = pytest.mark.reference

CASES = [
    (lambda: cases.gauss(48, engine=1, aoibnd=3), 40),
    (lambda: cases.gauss(48, engine=2, aoibnd=3), 40),
    (lambda: cases.gauss(32, engine=1, aoibnd=0), 30),
    (lambda: cases.hump_walls(64, engine=2), 30),
    (lambda: cases.hump_walls(48, engine=1), 30),
    (lambda: cases.conical_island(64, engine=1), 40),
    (lambda: cases.conical_island(48, engine=2), 40),
    (lambda: cases.dam_break(48, engine=1), 40),
    (lambda: cases.dam_break(32, engine=2), 40),
    (lambda: cases.rain_on_terrain(48, engine=1), 30),
]


@pytest.mark.parametrize("mk,nsteps", CASES, ids=[f"case{i}" for i in range(len(CASES))])
def test_oracle_matches_reference_bitwise(have_reference, mk, nsteps):
    case = mk()
    ref = make_reference(case)
    orc, mesh = make_oracle(case)
    lev, nbr, xo, yo = ref.blocks()
    # neighbour tables and levels of the product mesh builder == the reference InitMesh
    assert np.array_equal(lev, mesh.level)
    assert np.array_equal(nbr, mesh.nbr)
    assert np.array_equal(xo.astype(np.float32), mesh.xo.astype(np.float32))
    assert np.array_equal(yo.astype(np.float32), mesh.yo.astype(np.float32))
    # bed, bed halo and bed gradients (corner halo cells are never written by either)
    # (x-gradients exist on the interior and the left/right halo columns, y-gradients
    # on the interior and the bottom/top halo rows; the other halo cells are never written)
    sel = {"zb": (slice(None), slice(1, 17), slice(0, 18)), "dzbdx": (slice(None), slice(1, 17), slice(0, 18)),
           "dzbdy": (slice(None), slice(0, 18), slice(1, 17))}
    for name, s in sel.items():
        a, b = ref.get(name)[s], orc.get(name)[s]
        assert np.array_equal(a, b), name
    dr = ref.step(nsteps)
    do = orc.step(nsteps)
    assert np.array_equal(dr, do), (dr[:5], do[:5])
    for name in ("h", "u", "v", "zs"):
        a, b = interior(ref.get(name)), interior(orc.get(name))
        assert np.array_equal(a, b), (name, float(np.abs(a - b).max()))
