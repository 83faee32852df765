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


if __name__ == "__main__":
    main()
    main_amr()
    main_adapt_tables()
    main_adapt_full()
