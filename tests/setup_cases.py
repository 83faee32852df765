"""Seeded scenario directories for the BG_param.txt / .asc set-up tests.

Each case writes a small BG_Flood input set (BG_param.txt, an ESRI ASCII
bathymetry, optional rain and boundary series) into a directory.  The files are
synthetic: sloping, wavy beds with a wet/dry front, sized so the reference's
own start-up and a few steps run in well under a second on one core.
"""
from __future__ import annotations

import os

import numpy as np

# name -> description; every case is built by write_case(name, dir)
CASES = ("cold", "rain", "warm", "coarse", "offset", "adapt", "river")
# cases whose run the reference's CPU step can pin: with zsoffset != 0 its CPU
# boundary loop adds the offset once per boundary cell visited, cumulatively
# (src/Boundary.cu:646-648, zsbnd is the loop's own variable), where its GPU
# kernel adds it once (src/Boundary.cu:460); this library follows the GPU kernel.
RUN_CASES = ("cold", "rain", "warm", "coarse", "adapt", "river")


def asc_text(z: np.ndarray, cellsize: float, x0: float, y0: float, reg: str = "corner", sep: str = " ",
             eol: str = "\n", nodata: bool = True, fmt: str = "{:.6g}") -> str:
    """An ESRI ASCII grid of z (ny, nx; row 0 south).  reg: "corner" (xllcorner /
    yllcorner), "center" (xllcenter / yllcenter) or "mixed" (xllcenter / yllcorner)."""
    ny, nx = z.shape
    keys = {"corner": ("xllcorner", "yllcorner"), "center": ("xllcenter", "yllcenter"),
            "mixed": ("xllcenter", "yllcorner")}[reg]
    head = [f"ncols{sep}{nx}", f"nrows{sep}{ny}", f"{keys[0]}{sep}{x0!r}", f"{keys[1]}{sep}{y0!r}",
            f"cellsize{sep}{cellsize!r}"]
    head.append(f"NODATA_value{sep}-9999" if nodata else f"nodata_value{sep}-9999")
    rows = [sep.join(fmt.format(float(v)) for v in z[j]) for j in range(ny - 1, -1, -1)]
    return eol.join(head + rows) + eol


def bed(nx: int, ny: int, seed: int, slope: float = 0.06, base: float = -0.5, amp: float = 0.08) -> np.ndarray:
    rng = np.random.default_rng(seed)
    i = np.arange(nx)[None, :]
    j = np.arange(ny)[:, None]
    ph = rng.uniform(0, 2 * np.pi, 2)
    z = base + slope * i + amp * np.sin(j / 4.0 + ph[0]) * np.cos(i / 6.0 + ph[1])
    return z.astype(np.float32)


def write_case(name: str, d: str) -> str:
    """Writes case `name` into directory d; returns the BG_param.txt path."""
    os.makedirs(d, exist_ok=True)
    w = lambda fn, txt: open(os.path.join(d, fn), "w", newline="").write(txt)
    if name == "cold":
        # float model, corner registration, the right third above mask (blocks dropped)
        z = bed(48, 48, 1)
        w("bathy.asc", asc_text(z, 0.5, 100.0, 200.0, "corner"))
        w("BG_param.txt", "# cold start\nbathy = bathy.asc\nzsinit = 0.3\nmask = 1.0;\n"
                          "endtime = 20\noutputtimestep = 5\ncf = 0.001\nfrictionmodel = 0\n")
    elif name == "rain":
        # rain file (forces double), partial rain mask, centre registration, tabs, CRLF
        z = bed(40, 36, 2, slope=0.03, base=-0.2)
        w("topo.asc", asc_text(z, 0.25, 0.0, 0.0, "center", sep="\t", eol="\r\n"))
        w("rain.txt", "# t mm/h\n0\t360\n30\t720\n60\t0\n")
        w("BG_param.txt", "bathy = topo.asc\nrainfile = rain.txt\nmask = 0.6\nzsinit = -0.5\n"
                          "eps = 0.000001\ncf = 0.000004\nfrictionmodel = 1\nendtime = 50\noutputtimestep = 10\n")
    elif name == "warm":
        # positive-down file, warm start from a left boundary series, start time
        z = bed(48, 32, 3, slope=0.02, base=-0.4)
        w("depth.asc", asc_text(-z, 0.5, 10.0, 20.0, "mixed"))
        w("left.txt", "0 0.2\n100 0.4\n200 0.1\n")
        w("BG_param.txt", "bathy = depth.asc\nposdown = 1\nleft = 2,left.txt\n"
                          "totaltime = 10\nendtime = 150\noutputtimestep = 25\n")
    elif name == "offset":
        # water-level offset: absent from the warm start, added to the boundary level
        z = bed(32, 48, 6, slope=0.02, base=-0.4)
        w("bathy.asc", asc_text(z, 0.5, 0.0, 0.0, "corner"))
        w("bnd.txt", "0,0.1\n50,0.3\n")
        w("BG_param.txt", "bathy = bathy.asc\nbot = bnd.txt,3\nzsoffset = 0.05\nendtime = 40\n"
                          "outputtimestep = 10\n")
    elif name == "coarse":
        # model cells twice the grid spacing: the bed is the mean of the grid nodes in a cell
        z = bed(66, 66, 4, slope=0.015, base=-0.3, amp=0.2)
        w("dem.asc", asc_text(z, 0.25, 5.0, 5.0, "corner"))
        w("BG_param.txt", "DEM = dem.asc\ndx = 0.5\nzsinit = 0.1\nendtime = 30\noutputtimestep = 10\n")
    elif name == "adapt":
        # initial refinement of the wet blocks, one level
        z = bed(64, 48, 5, slope=0.03, base=-0.6)
        w("bathy.asc", asc_text(z, 1.0, 0.0, 0.0, "corner"))
        w("BG_param.txt", "bathy = bathy.asc\nzsinit = 0.2\ninitlevel = 0\nmaxlevel = 1\nminlevel = 0\n"
                          "Adaptation = Threshold,0.3,h\nendtime = 30\noutputtimestep = 10\n")
    elif name == "river":
        # two rivers into a dry valley (one box straddling two blocks), one box
        # outside the domain (dropped); the run's end time comes from the flow files
        z = bed(48, 48, 7, slope=0.0, base=0.2, amp=0.1)
        yy = np.arange(48)[:, None]
        z = (z + 0.02 * np.abs(yy - 24)).astype(np.float32)
        w("bathy.asc", asc_text(z, 1.0, 0.0, 0.0, "corner"))
        w("q1.txt", "0 0.0\n10 2.5\n60 4.0\n")
        w("q2.txt", "# t q\n0,1.0\n80,0.5\n")
        w("q3.txt", "0 1.0\n100 1.0\n")
        w("BG_param.txt", "bathy = bathy.asc\nzsinit = -1\nriver = q1.txt,3.2,5.9,22.1,26.8\n"
                          "river = q2.txt,15.5,16.6,10.0,12.0\nriver = q3.txt,100,110,100,110\n"
                          "outputtimestep = 10\nfrictionmodel = 0\ncf = 0.001\n")
    else:
        raise KeyError(name)
    return os.path.join(d, "BG_param.txt")


# .asc header / data variants for the reader tests: (name, kwargs for asc_text)
ASC_VARIANTS = (
    ("corner_space", dict(reg="corner")),
    ("center_tab", dict(reg="center", sep="\t")),
    ("mixed_crlf", dict(reg="mixed", eol="\r\n")),
    ("lower_nodata", dict(reg="corner", nodata=False, fmt="{:.8e}")),
)


def write_asc_variant(name: str, d: str) -> str:
    kw = dict(ASC_VARIANTS)[name]
    rng = np.random.default_rng(sum(name.encode()))
    z = (rng.standard_normal((19, 23)) * 3.0).astype(np.float32)
    z[4, 5] = -9999.0
    path = os.path.join(d, name + ".asc")
    with open(path, "w", newline="") as fh:
        fh.write(asc_text(z, 0.125, 1234.5, -56.25, **kw))
    return path
