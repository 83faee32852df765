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
from runners import interior, make_reference  # noqa: E402

GOLDEN_CASES = {
    "gauss48_e1_b3": (lambda: cases.gauss(48, 1, 3), 40),
    "gauss48_e2_b3": (lambda: cases.gauss(48, 2, 3), 40),
    "hump64_e2": (lambda: cases.hump_walls(64, 2), 30),
    "island64_e1": (lambda: cases.conical_island(64, 1), 40),
    "dam48_e1": (lambda: cases.dam_break(48, 1), 40),
    "rain48_e1": (lambda: cases.rain_on_terrain(48, 1), 30),
}


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
