"""Scenarios from BG_param.txt + ESRI ASCII bathymetry, on the CPU.

The host set-up (bg_flood_b200.model_setup, readforcing and the native readers)
is compared with the reference's own start-up from the same files
(tests/golden/setup_<case>.npz, made by make_golden.py from Readparamfile,
readforcing, checkparamsanity, InitMesh, InitialConditions, InitialAdaptation),
and the oracle run from these inputs with the reference's FlowCPU run.  All
comparisons are bit-exact.
"""
import math
import os

import numpy as np
import pytest

from bg_flood_b200.model_setup import inputs_on_mesh, prepare_model, read_param_file
from bg_flood_b200.readforcing import read_asc, read_asc_header, read_uniform_series, readinputtimetxt
from oracle.pyoracle import REF_PARAM_NAMES, Reference, ref_available, ref_read_asc
from runners import make_oracle_inputs, normalise_reference_surface
from setup_cases import ASC_VARIANTS, CASES, RUN_CASES, asc_text, write_asc_variant, write_case

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SETUP_STEPS = 20
I = (slice(None), slice(1, 17), slice(1, 17))
needs_ref = pytest.mark.skipif(not ref_available(), reason="reference build (oracle/_ref) not present")


def golden(name):
    return np.load(os.path.join(GOLD, f"setup_{name}.npz"))


def interior(a):
    return np.asarray(a)[I]


# ------------------------------------------------------------------ .asc reader

@pytest.mark.parametrize("name", [v[0] for v in ASC_VARIANTS])
def test_asc_reader_matches_reference_golden(tmp_path, name):
    g = np.load(os.path.join(GOLD, "asc_variants.npz"))
    path = write_asc_variant(name, str(tmp_path))
    head = read_asc_header(path)
    assert np.array_equal(np.array(head, np.float64), g[f"{name}_head"])
    grid = read_asc(path)
    assert grid.val.dtype == np.float32 and np.array_equal(grid.val, g[f"{name}_val"])
    assert grid.dy == grid.dx


@needs_ref
@pytest.mark.parametrize("name", [v[0] for v in ASC_VARIANTS])
def test_asc_reader_matches_reference_live(tmp_path, name):
    path = write_asc_variant(name, str(tmp_path))
    head, val = ref_read_asc(path)
    assert read_asc_header(path) == head
    assert np.array_equal(read_asc(path).val, val)


def test_asc_header_registration(tmp_path):
    z = np.zeros((3, 4), np.float32)
    for reg, shift in (("corner", 0.5), ("center", 0.5), ("mixed", 0.0)):
        p = tmp_path / f"{reg}.asc"
        p.write_text(asc_text(z, 2.0, 10.0, 20.0, reg))
        nx, ny, dx, xo, yo, ga = read_asc_header(str(p))
        # yllcenter or xllcorner moves both origins by half a cell, as in the reference
        assert (nx, ny, dx, ga) == (4, 3, 2.0, 0.0)
        assert (xo, yo) == (10.0 + shift * 2.0, 20.0 + shift * 2.0)


def test_asc_errors(tmp_path):
    z = np.arange(12, dtype=np.float32).reshape(3, 4)
    good = asc_text(z, 1.0, 0.0, 0.0)
    with pytest.raises(ValueError, match="could not be opened"):
        read_asc(str(tmp_path / "missing.asc"))
    short = tmp_path / "short.asc"
    short.write_text("\n".join(good.splitlines()[:4]) + "\n")
    with pytest.raises(ValueError, match="header"):
        read_asc_header(str(short))
    nocols = tmp_path / "nocols.asc"
    nocols.write_text(good.replace("ncols", "NCOLS"))
    with pytest.raises(ValueError, match="ncols"):
        read_asc_header(str(nocols))
    trunc = tmp_path / "trunc.asc"
    trunc.write_text("\n".join(good.splitlines()[:8]) + "\n")
    with pytest.raises(ValueError, match="data"):
        read_asc(str(trunc))
    bad = tmp_path / "bad.asc"
    bad.write_text(good.replace(" 5 ", " nan "))
    with pytest.raises(ValueError):
        read_asc(str(bad))


def test_uniform_series(tmp_path):
    p = tmp_path / "s.txt"
    p.write_text("# header\n0\t1.5\n10 2.5\n20,3.5\n\n")
    t, v = read_uniform_series(str(p))
    assert list(t) == [0.0, 10.0, 20.0] and list(v) == [1.5, 2.5, 3.5]
    ref = [""]
    assert readinputtimetxt("2020-01-01T00:00:00", ref) == 0.0 and ref[0] == "2020-01-01T00:00:00"
    assert readinputtimetxt("2020-01-01T01:00:30", ref) == 3630.0
    bad = tmp_path / "b.txt"
    bad.write_text("1\n")
    with pytest.raises(ValueError):
        read_uniform_series(str(bad))


def test_param_file_keys(tmp_path):
    pf = write_case("offset", str(tmp_path))
    p = read_param_file(pf)
    assert p.bathy == ["bathy.asc"] and p.zsoffset == 0.05
    assert len(p.segments) == 1 and p.segments[0].side == "bot" and p.segments[0].type == 3
    assert p.segments[0].file == "bnd.txt"
    (tmp_path / "BG_param.txt").write_text("bathy = bathy.asc\nwindfiles = w.txt\n")
    with pytest.raises(ValueError, match="not supported"):
        read_param_file(str(tmp_path / "BG_param.txt"))
    (tmp_path / "BG_param.txt").write_text("bathy = bathy.asc\nriver = r.txt,1,2,3\n")
    with pytest.raises(ValueError, match="5 comma-separated"):
        read_param_file(str(tmp_path / "BG_param.txt"))
    (tmp_path / "BG_param.txt").write_text("bathy = bathy.asc\nriver = r.txt, 1,2,3,4\n")
    assert read_param_file(str(tmp_path / "BG_param.txt")).rivers == [("r.txt", 1.0, 2.0, 3.0, 4.0)]
    (tmp_path / "BG_param.txt").write_text("bathy = bathy.asc\ncf = 1e-3\n")
    assert read_param_file(str(tmp_path / "BG_param.txt")).cf == 1e-3
    (tmp_path / "BG_param.txt").write_text("bathy = bathy.asc\ncf = manning.nc\n")
    with pytest.raises(ValueError, match="roughness map"):
        read_param_file(str(tmp_path / "BG_param.txt"))
    (tmp_path / "BG_param.txt").write_text("bathy = bathy.nc?z\n")
    with pytest.raises(ValueError, match="not supported"):
        prepare_model(str(tmp_path / "BG_param.txt"))


# ------------------------------------------------------------------ set-up

def _check_params(p, inp, prm):
    mine = dict(xo=p.xo, yo=p.yo, xmax=p.xmax, ymax=p.ymax, dx=p.dx, nblk=inp.mesh.nblk,
                doubleprecision=p.doubleprecision, zsoffset=p.zsoffset, endtime=p.endtime, totaltime=p.totaltime,
                nextoutputtime=inp.nextoutputtime, initlevel=p.initlevel, minlevel=p.minlevel, maxlevel=p.maxlevel,
                mask=p.mask, CFL=p.CFL, engine=p.engine)
    for k, v in mine.items():
        assert float(v) == prm[k], k


@pytest.mark.parametrize("name", [c for c in CASES if c != "adapt"])
def test_setup_matches_reference(tmp_path, name):
    g = golden(name)
    prm = dict(zip(REF_PARAM_NAMES, g["params"]))
    inp = prepare_model(write_case(name, str(tmp_path)))
    _check_params(inp.param, inp, prm)
    m = inp.mesh
    assert np.array_equal(m.level, g["level"]) and np.array_equal(m.nbr, g["nbr"])
    assert np.array_equal(m.xo, g["xo"]) and np.array_equal(m.yo, g["yo"])
    for k in ("zb", "h", "zs", "u", "v"):
        assert np.array_equal(interior(getattr(inp, k)), g[k]), k
    ac = np.ones_like(g["active_cell"]) if inp.active_cell is None else interior(inp.active_cell)
    assert np.array_equal(ac, g["active_cell"])
    if inp.rain is None:
        assert len(g["rain_t"]) == 0
    else:
        assert np.array_equal(inp.rain[0], g["rain_t"]) and np.array_equal(inp.rain[1], g["rain_r"])
    assert len(inp.segments) == int(prm["nseg"])
    for s, (typ, times, levels, _) in enumerate(inp.segments):
        assert typ == int(g[f"seg{s}_type"])
        assert np.array_equal(np.asarray(times, np.float64), g[f"seg{s}_t"])
        assert np.array_equal(np.asarray(levels, np.float64), g[f"seg{s}_w"])


def test_setup_masked_blocks(tmp_path):
    # the "cold" case drops the blocks whose cells all lie above mask
    inp = prepare_model(write_case("cold", str(tmp_path)))
    assert inp.mesh.nblk == 6 and inp.mesh.nbx * inp.mesh.nby == 9
    assert (interior(inp.h) > 0).any() and (interior(inp.h) == 0).any()


def test_setup_adapted_mesh_initial_conditions(tmp_path):
    # InitialConditions on the reference's refined tables (two levels)
    g = golden("adapt")
    base = prepare_model(write_case("adapt", str(tmp_path)))
    inp = inputs_on_mesh(base, g["level"], g["nbr"], g["xo"], g["yo"])
    assert set(np.unique(inp.mesh.level)) == {0, 1}
    for k in ("zb", "h", "zs", "u", "v"):
        assert np.array_equal(interior(getattr(inp, k)), g[k]), k


def _inputs(name, d):
    inp = prepare_model(write_case(name, d))
    if name == "adapt":
        g = golden(name)
        inp = inputs_on_mesh(inp, g["level"], g["nbr"], g["xo"], g["yo"])
    return inp


@pytest.mark.parametrize("name", RUN_CASES)
def test_oracle_run_from_files_matches_reference(tmp_path, name):
    g = golden(name)
    o = make_oracle_inputs(_inputs(name, str(tmp_path)))
    dts = o.step(SETUP_STEPS)
    assert np.array_equal(dts, g["dts"])
    for k in ("h", "zs", "u", "v"):
        assert np.array_equal(interior(o.get(k)), g[f"run_{k}"]), k


@needs_ref
@pytest.mark.parametrize("name", ["cold", "rain"])
def test_setup_matches_reference_live(tmp_path, name, monkeypatch):
    pf = write_case(name, str(tmp_path))
    monkeypatch.chdir(tmp_path)
    r = Reference.from_file("BG_param.txt")
    inp = prepare_model(pf)
    lev, nbr, xo, yo = r.mesh_active_order()
    assert np.array_equal(nbr, inp.mesh.nbr) and np.array_equal(xo, inp.mesh.xo)
    for k in ("zb", "h", "zs"):
        assert np.array_equal(interior(r.get(k)), interior(getattr(inp, k))), k
    # the unmodified reference (dy = 0 for .asc grids) gives a bed of inf or nan
    r0 = Reference.from_file("BG_param.txt", fix_asc_dy=False)
    assert not np.isfinite(interior(r0.get("zb"))).any()
    normalise_reference_surface(r, bool(inp.param.doubleprecision))
    o = make_oracle_inputs(inp)
    assert np.array_equal(r.step(5), o.step(5))
    assert not math.isnan(float(interior(o.get("h")).sum()))
