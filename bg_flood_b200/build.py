"""Builds the native library of the package in-tree (bg_flood_b200/_lib).

The CUDA sources are compiled for sm_100a only.  ``--fmad=false`` keeps every
floating-point operation separately rounded, which is what lets the kernels
reproduce the reference CPU build bit for bit in single precision.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "_lib")
LIBNAME = "libbgflood_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O2",
           "-Xcompiler", "-ffp-contract=off"]
# (source, object name, extra flags): the flow kernels are built twice
SOURCES = [
    ("bgf_flow.cu", "bgf_flow_exact.o", ["-DBGF_VARIANT=exact", "--fmad=false"]),
    ("bgf_flow.cu", "bgf_flow_fast.o", ["-DBGF_VARIANT=fast", "-DBGF_FAST=1", "--fmad=true", "-prec-div=false", "-prec-sqrt=false",
                                        "-ftz=true"]),
    ("bgf_amr.cu", "bgf_amr_exact.o", ["-DBGF_VARIANT=exact", "--fmad=false"]),
    ("bgf_amr.cu", "bgf_amr_fast.o", ["-DBGF_VARIANT=fast", "-DBGF_FAST=1", "--fmad=true", "-prec-div=false", "-prec-sqrt=false",
                                      "-ftz=true"]),
    ("bgf_adapt.cu", "bgf_adapt.o", ["--fmad=false"]),
    ("bgf_capi.cu", "bgf_capi.o", ["--fmad=false"]),
    ("bgf_noalloc.cu", "bgf_noalloc.o", ["--fmad=false"]),
    ("bgf_host.cpp", "bgf_host.o", ["-x", "cu", "--fmad=false"]),
    ("bgf_adapt_host.cpp", "bgf_adapt_host.o", ["-x", "cu", "--fmad=false"]),
    ("bgf_io.cpp", "bgf_io.o", ["-x", "cu", "--fmad=false"]),
    ("bgf_layout.cu", "bgf_layout.o", ["--fmad=false"]),
    ("bgf_gauge.cu", "bgf_gauge.o", ["--fmad=false"]),
    ("bgf_adapt_dev.cu", "bgf_adapt_dev.o", ["--fmad=false"]),
]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    """Compiles the CUDA kernels and the C ABI into bg_flood_b200/_lib and returns the .so path."""
    os.makedirs(LIBDIR, exist_ok=True)
    out = os.path.join(LIBDIR, LIBNAME)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(ROOT, "include", "bg_flood_b200.h")]
    if not force and not _stale(out, deps):
        return out
    objs = []
    for src, oname, extra in SOURCES:
        obj = os.path.join(LIBDIR, oname)
        # later flags override the defaults (--fmad, -prec-div, ...)
        cmd = [nvcc(), *ARCH, *NVFLAGS, *extra, "-c", os.path.join(CSRC, src), "-o", obj]
        if ptxas_info:
            cmd.insert(1, "-Xptxas=-v")
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [nvcc(), *ARCH, "-shared", *objs, "-o", out, "-lcudart"]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True)
    return out


def build_oracle(force: bool = False) -> str:
    """Compiles the CPU oracle (test infrastructure) into oracle/liboracle.so."""
    odir = os.path.join(ROOT, "oracle")
    out = os.path.join(odir, "liboracle.so")
    deps = [os.path.join(odir, f) for f in ("bgf_oracle.c", "bgf_oracle.h", "bgf_oracle_impl.inc")]
    if force or _stale(out, deps):
        subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                        "-o", out, os.path.join(odir, "bgf_oracle.c"), "-lm"], check=True)
    return out


def build_reference_oracle(refsrc: str | None = None, faithful: bool = False) -> str | None:
    """Builds the reference sources into oracle/_ref/libbgf_ref.so (test infrastructure and
    the CPU baseline).  ``refsrc`` is the reference's src directory, else the environment
    variable BG_FLOOD_REFERENCE_SRC; without either nothing is built.  ``faithful`` builds
    oracle/_ref/faithful/libbgf_ref.so with the reference Makefile's host flags (no -O)."""
    refsrc = refsrc or os.environ.get("BG_FLOOD_REFERENCE_SRC")
    if not refsrc or not os.path.isdir(refsrc):
        return None
    out = os.path.join(ROOT, "oracle", "_ref", "faithful") if faithful else os.path.join(ROOT, "oracle", "_ref")
    cmd = ["make", "-C", os.path.join(ROOT, "oracle", "ref"), f"REFSRC={refsrc}", f"OUT={out}", "-j8"]
    if faithful:
        cmd.append("HOSTOPT=-O0")
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL)
    return os.path.join(out, "libbgf_ref.so")


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv))
