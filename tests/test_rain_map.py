"""Gridded rain on the CPU: the oracle against the reference's own rain-map path
(a two-frame DynForcingP installed in the reference harness; its netCDF reader is
not part of this build), bit for bit over the steps of the case."""
import os

import numpy as np
import pytest

from oracle.pyoracle import ref_available
from rainmap_case import MAP, NSTEPS, rainmap_case
from runners import interior, make_oracle, make_reference

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rainmap48_e1.npz")


def _oracle():
    c, before, after = rainmap_case()
    o, _ = make_oracle(c)
    o.set_rain_map(MAP["xo"], MAP["yo"], MAP["dx"], MAP["dy"], MAP["to"], MAP["dt"], np.stack([before, after]))
    return o


def test_rain_map_oracle_matches_reference_golden():
    g = np.load(GOLD)
    o = _oracle()
    dts = o.step(NSTEPS)
    assert np.array_equal(dts, g["dts"])
    for k in ("h", "u", "v"):
        assert np.array_equal(interior(o.get(k)).astype(np.float32), g[k]), k
    assert float(interior(o.get("h")).sum()) > 0.0  # it rained on the dry terrain


@pytest.mark.skipif(not ref_available(), reason="reference build (oracle/_ref) not present")
def test_rain_map_oracle_matches_reference_live():
    c, before, after = rainmap_case()
    r = make_reference(c)
    r.set_rain_map(MAP["xo"], MAP["yo"], MAP["dx"], MAP["dy"], MAP["to"], MAP["dt"], before, after)
    o = _oracle()
    assert np.array_equal(r.step(NSTEPS), o.step(NSTEPS))
    for k in ("h", "u", "v", "zs"):
        assert np.array_equal(interior(r.get(k)), interior(o.get(k))), k
