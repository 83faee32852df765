"""Gridded rain case shared by the CPU and GPU tests and the fixture script: rain
on the seeded fractal terrain of cases.rain_on_terrain, the rate a coarse
two-frame grid (not square, partly outside the model domain) interpolated in
time and space."""
import numpy as np

import cases

NSTEPS = 30
MAP = dict(xo=-20.0, yo=-30.0, dx=90.0, dy=95.0, to=0.0, dt=600.0)


def rainmap_case():
    c = cases.rain_on_terrain(48, 1)
    c.rain = None
    rng = np.random.default_rng(11)
    before = rng.uniform(0.0, 100.0, (6, 7)).astype(np.float32)
    after = rng.uniform(0.0, 150.0, (6, 7)).astype(np.float32)
    return c, before, after
