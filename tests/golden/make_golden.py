"""Regenerates the golden fixtures of tests/golden from the reference BG_Flood
built from its own sources (oracle/_ref/libbgf_ref.so).

    python tests/golden/make_golden.py

For each small case of tests/cases.py it runs the reference FlowCPU for a fixed
number of steps and stores the dt sequence and the interior h, u, v, zs (float32)
in <case>.npz.  zs_verif_buttinger.json holds the reference's own known-answer
values of the Gaussian-hump test (src/Testing.cu:436, checked at src/Testing.cu:645-670).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "tests")]

import cases  # noqa: E402
from runners import interior, make_amr_pair, make_reference  # noqa: E402

GOLDEN_CASES = {
    "gauss48_e1_b3": (lambda: cases.gauss(48, 1, 3), 40),
    "gauss48_e2_b3": (lambda: cases.gauss(48, 2, 3), 40),
    "hump64_e2": (lambda: cases.hump_walls(64, 2), 30),
    "island64_e1": (lambda: cases.conical_island(64, 1), 40),
    "dam48_e1": (lambda: cases.dam_break(48, 1), 40),
    "rain48_e1": (lambda: cases.rain_on_terrain(48, 1), 30),
}

# Meshes refined by the reference's own InitialAdaptation(): the block tables in
# active order are stored with the reference's dt sequence and fields, so the
# oracle and the GPU library can be run on the same tables without the reference.
AMR_GOLDEN_CASES = {
    "amrhump64_e1_l1": (lambda: cases.amr_hump(64, 1, 1, 0.3), 30),
    "amrhump64_e2_l2": (lambda: cases.amr_hump(64, 2, 2, 0.3), 30),
    "amrdam64_e1_l2": (lambda: cases.amr_dambreak(64, 1, 2), 40),
    "amrdam64_e2_l2": (lambda: cases.amr_dambreak(64, 2, 2), 40),
    "amrdam64_e1_l3": (lambda: cases.amr_dambreak(64, 1, 3), 40),
}


def main_amr():
    for name, (mk, nsteps) in AMR_GOLDEN_CASES.items():
        case = mk()
        ref, _, (lev, nbr, xo, yo) = make_amr_pair(case)
        dts = ref.step(nsteps)
        out = {k: interior(ref.get(k)).astype(np.float32) for k in ("h", "u", "v")}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), dts=dts, nsteps=nsteps, level=lev, nbr=nbr, xo=xo,
                            yo=yo, **out)
        print(name, nsteps, np.bincount(lev), dts[:3])


def main_adapt_tables():
    """Iterations of the reference's Adaptation() with the pre-sanity criterion flags
    and the tables before and after each iteration (tests/test_adapt_tables.py)."""
    from adapt_cases import ADAPT_CASES, criterion_of, id_tables, reference_with_bathy
    out = {}
    for name in ("island64_e1_l2", "hump64_e1_l2", "dam64_e1_l3"):
        case = ADAPT_CASES[name]()
        crit = criterion_of(case)
        r = reference_with_bathy(case)
        for it in range(8):
            act, level, nbr, xo, yo = id_tables(r)
            stem = f"{name}_it{it}"
            out[f"{stem}_pre"] = crit.flags(r.get(crit.var)[:, 1:17, 1:17])
            out[f"{stem}_act"], out[f"{stem}_level"], out[f"{stem}_nbr"] = act, level, nbr
            out[f"{stem}_xo"], out[f"{stem}_yo"] = xo, yo
            rf, _ = r.flags()
            out[f"{stem}_refine"] = rf
            act_r, level_r, nbr_r, xo_r, yo_r = id_tables(r)
            out[f"{stem}_act_out"], out[f"{stem}_level_out"], out[f"{stem}_nbr_out"] = act_r, level_r[act_r], nbr_r[act_r]
            out[f"{stem}_xo_out"], out[f"{stem}_yo_out"] = xo_r[act_r], yo_r[act_r]
            print(stem, len(act), "->", len(act_r))
            if len(act_r) == len(act):
                break
    np.savez_compressed(os.path.join(HERE, "adapt_tables.npz"), **out)


def main_adapt_full():
    """The reference's whole Adaptation() from a uniform level-0 mesh: final tables
    and interior h, zs, u, v, zb in active order (tests/test_gpu_adapt.py)."""
    from adapt_cases import ADAPT_CASES, id_tables, reference_with_bathy
    for name in ("island64_e1_l2", "hump64_e1_l2", "dam64_e1_l3"):
        case = ADAPT_CASES[name]()
        r = reference_with_bathy(case)
        r.adaptation()
        act, level, nbr, xo, yo = id_tables(r)
        out = {k: interior(r.get(k)).astype(np.float32) for k in ("h", "zs", "u", "v", "zb")}
        np.savez_compressed(os.path.join(HERE, f"adapt_{name}.npz"), act=act, level=level[act], nbr=nbr[act],
                            xo=xo[act], yo=yo[act], **out)
        print("adapt", name, len(act))
    # adaptation in the middle of a run: 20 flow steps first, so u and v are not zero
    for name in ("hump64_e1_l2", "island64_e1_l2"):
        case = ADAPT_CASES[name]()
        r = reference_with_bathy(case)
        r.step(20)
        r.adaptation()
        act, level, nbr, xo, yo = id_tables(r)
        out = {k: interior(r.get(k)).astype(np.float32) for k in ("h", "zs", "u", "v", "zb")}
        np.savez_compressed(os.path.join(HERE, f"adapt_{name}_t20.npz"), act=act, level=level[act], nbr=nbr[act],
                            xo=xo[act], yo=yo[act], **out)
        print("adapt after 20 steps", name, len(act))


def main():
    for name, (mk, nsteps) in GOLDEN_CASES.items():
        case = mk()
        ref = make_reference(case)
        dts = ref.step(nsteps)
        out = {k: interior(ref.get(k)).astype(np.float32) for k in ("h", "u", "v", "zs")}
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), dts=dts, nsteps=nsteps, **out)
        print(name, nsteps, dts[:3])


SETUP_STEPS = 20


def main_setup():
    """Scenarios set up by the reference's own start-up from BG_param.txt files
    (tests/setup_cases.py; ref_create_from_file, with dy = dx for the .asc grid):
    scalars, tables in active order, interior bed and initial state, rain mask,
    series; then, with the initial zs set to zb + h, SETUP_STEPS steps of its
    FlowCPU (cases of RUN_CASES).  Also the reference's .asc reader on the reader
    variants.  Written to setup_<case>.npz and asc_variants.npz."""
    import tempfile

    from oracle.pyoracle import REF_PARAM_NAMES, Reference, ref_read_asc
    from runners import normalise_reference_surface
    from setup_cases import ASC_VARIANTS, CASES, RUN_CASES, write_asc_variant, write_case
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as tmp:
        for name in CASES:
            d = os.path.join(tmp, name)
            write_case(name, d)
            os.chdir(d)
            try:
                r = Reference.from_file("BG_param.txt")
                prm = r.params()
                lev, nbr, xo, yo = r.mesh_active_order()
                out = dict(params=np.array([prm[k] for k in REF_PARAM_NAMES]), level=lev, nbr=nbr, xo=xo, yo=yo)
                for k in ("zb", "h", "zs", "u", "v"):
                    out[k] = interior(r.get(k))
                out["active_cell"] = interior(r.active_cell()).astype(np.int8)
                out["rain_t"], out["rain_r"] = r.rain()
                for s in range(int(prm["nseg"])):
                    typ, t, w = r.segment(s)
                    out[f"seg{s}_type"], out[f"seg{s}_t"], out[f"seg{s}_w"] = np.int32(typ), t, w
                if name in RUN_CASES:
                    normalise_reference_surface(r, bool(prm["doubleprecision"]))
                    out["dts"] = r.step(SETUP_STEPS)
                    for k in ("h", "zs", "u", "v"):
                        out[f"run_{k}"] = interior(r.get(k))
                np.savez_compressed(os.path.join(HERE, f"setup_{name}.npz"), **out)
                print("setup", name, r.nblk, prm["doubleprecision"])
            finally:
                os.chdir(cwd)
        out = {}
        for name, _ in ASC_VARIANTS:
            path = write_asc_variant(name, tmp)
            head, val = ref_read_asc(path)
            out[f"{name}_head"] = np.array(head, np.float64)
            out[f"{name}_val"] = val
        np.savez_compressed(os.path.join(HERE, "asc_variants.npz"), **out)


def main_rainmap():
    """The reference's FlowCPU with a two-frame rain map (tests/rainmap_case.py)."""
    from rainmap_case import MAP, NSTEPS, rainmap_case
    c, before, after = rainmap_case()
    r = make_reference(c)
    r.set_rain_map(MAP["xo"], MAP["yo"], MAP["dx"], MAP["dy"], MAP["to"], MAP["dt"], before, after)
    dts = r.step(NSTEPS)
    out = {k: interior(r.get(k)).astype(np.float32) for k in ("h", "u", "v", "zs")}
    np.savez_compressed(os.path.join(HERE, "rainmap48_e1.npz"), dts=dts, nsteps=NSTEPS, **out)
    print("rainmap48_e1", NSTEPS, dts[:3])


def main_adapt_target():
    """The reference's Adaptation() with the Targetlevel criterion and two target-level
    maps (the last decides): final tables and interior fields (tests/test_gpu_adapt.py)."""
    from adapt_cases import id_tables, reference_with_bathy, target_case, target_maps
    case = target_case()
    r = reference_with_bathy(case)
    for xo, yo, dx, lv in target_maps(case):
        r.add_target_map(xo, yo, dx, lv)
    r.adaptation()
    act, level, nbr, xo, yo = id_tables(r)
    out = {k: interior(r.get(k)).astype(np.float32) for k in ("h", "zs", "u", "v", "zb")}
    np.savez_compressed(os.path.join(HERE, "adapt_target_hump64.npz"), act=act, level=level[act], nbr=nbr[act],
                        xo=xo[act], yo=yo[act], **out)
    print("adapt Targetlevel", len(act), np.bincount(level[act]))


if __name__ == "__main__":
    if sys.argv[1:] == ["target"]:
        main_adapt_target()
        sys.exit(0)
    if sys.argv[1:] == ["setup"]:
        main_setup()
        sys.exit(0)
    if sys.argv[1:] == ["rainmap"]:
        main_rainmap()
        sys.exit(0)
    main()
    main_amr()
    main_adapt_tables()
    main_adapt_full()
