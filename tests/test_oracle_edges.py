"""Edge meshes on the CPU: the oracle against the reference's FlowCPU (built from
its sources) on a single block, one-block-wide strips and an all-dry domain."""
import numpy as np
import pytest

from oracle.pyoracle import ref_available
from runners import interior, make_oracle, make_reference
from test_gpu_edges import _case

pytestmark = pytest.mark.skipif(not ref_available(), reason="reference build (oracle/_ref) not present")


@pytest.mark.parametrize("nx,ny,kind,engine", [
    (16, 16, "hump", 1), (16, 16, "dam", 2), (128, 16, "dam", 1), (16, 128, "dam", 2), (48, 32, "dry", 1),
])
def test_edge_meshes_oracle_matches_reference(nx, ny, kind, engine):
    c = _case(nx, ny, kind, engine)
    r = make_reference(c)
    o, _ = make_oracle(c)
    assert np.array_equal(r.step(15), o.step(15))
    for name in ("h", "u", "v", "zs"):
        assert np.array_equal(interior(r.get(name)), interior(o.get(name))), name
