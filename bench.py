#!/usr/bin/env python
"""Flow-step benchmark: cell-updates/s of the B200 library on the wet/dry run-up
workload (1024x1024 cells of 16x16 blocks, dx = 0.05 m, conical island, Manning
n = 0.01, solitary wave entering from the west), one JSON line on stdout.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

A step is one full flow step (predictor + corrector) of the whole grid.
* value:   device time of K steps (CUDA events around the two kernels on the
           library's stream), L2 flushed before every step, max over ranks.
* e2e:     the same K steps through the C ABI with host buffers: state upload
           from page-locked host arrays, K bgf_flow_step calls (each returns dt
           to the host), state download into page-locked arrays; wall clock.
* roofline: the dominant kernel's algorithmic bytes per launch / its mean event
           time, against the measured HBM copy bandwidth.
* cpu_baseline: the reference BG_Flood FlowCPU (built from its sources,
           oracle/_ref) on a 256x256 window of the same workload.
With N > 1 (torchrun) every rank runs its own replica of the scenario: the path
has no exchange step between independent scenarios (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, os.path.join(ROOT, "tests")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "cell-updates/s"
UNIT = "cell-updates/s"
WORKLOAD = "wet/dry run-up 1024x1024 cells (16x16 blocks), dx=0.05 m, conical island, solitary wave, Manning n=0.01"
ALG_BYTES_FLUX = 28    # h,u,v,zb read + dh,dhu,dhv written (FP32)
ALG_BYTES_UPDATE = 40  # h,u,v,dh,dhu,dhv,zb read + h,u,v written (FP32)
REF_WINDOW = 256       # the reference's FlowCPU is timed on a window of this many cells per side


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=1024, help="grid cells per side")
    ap.add_argument("--engine", type=int, default=1)
    ap.add_argument("--fastmath", type=int, default=1, help="1: fast-math kernels, 0: bit-exact kernels")
    ap.add_argument("--layout", type=int, default=2, help="thread layout of the single-level kernels (profiling runs)")
    ap.add_argument("--no-extra", action="store_true", help="skip the secondary measurements")
    ap.add_argument("--only", choices=["amr", "ensemble", "ensemble_small", "serve"], default=None,
                    help="run one secondary measurement alone and print it (profiling runs)")
    ap.add_argument("--amr", type=int, default=2048, help="level-0 cells per side of the AMR measurement (0: skip)")
    ap.add_argument("--ensemble", type=int, default=64, help="members of the batched-ensemble measurement (0: skip)")
    ap.add_argument("--ens-max-blocks", type=int, default=16384)
    ap.add_argument("--serve", type=int, default=48, help="requests of the serving measurement (0: skip)")
    ap.add_argument("--serve-rate", type=float, default=200.0, help="Poisson arrival rate, requests/s")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="run this many flow steps of the workload and exit (for ncu captures of the stage kernels)")
    ap.add_argument("--cpu-sample", choices=["O2", "makefile"], default=None,
                    help="internal: time the reference FlowCPU build in this process and print one JSON line")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def host_cpu() -> dict:
    """The host the CPU baseline ran on: CPU model, logical CPUs and the cores this
    process may use."""
    model = ""
    try:
        with open("/proc/cpuinfo") as fh:
            for ln in fh:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        allowed = len(os.sched_getaffinity(0))
    except AttributeError:
        allowed = os.cpu_count() or 1
    return {"cpu_model": model, "nproc": os.cpu_count() or 1, "affinity_cores": allowed}


def measured_peak_hbm():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clock and throttle reasons with NVML while the timed region runs."""

    def __init__(self, dev: int):
        self.samples, self.reasons = [], set()
        self.stop_ev = threading.Event()
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(dev)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nv = None

    def _run(self):
        nv = self.nv
        names = {}
        for attr in ("HW_SLOWDOWN", "HW_THERMAL_SLOWDOWN", "SW_THERMAL_SLOWDOWN", "SW_POWER_CAP", "HW_POWER_BRAKE_SLOWDOWN"):
            v = getattr(nv, "nvmlClocksEventReason" + "".join(w.title() for w in attr.split("_")), None) or \
                getattr(nv, "nvmlClocksThrottleReason" + "".join(w.title() for w in attr.split("_")), None)
            if v is not None:
                names[attr.lower()] = v
        while not self.stop_ev.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                try:
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except Exception:
                    r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                for n, bit in names.items():
                    if r & bit:
                        self.reasons.add(n)
            except Exception:
                pass
            time.sleep(0.005)  # the timed region can be tens of milliseconds

    def __enter__(self):
        if self.nv:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.nv:
            self.stop_ev.set()
            self.t.join()

    def summary(self):
        med = float(np.median(self.samples)) if self.samples else None
        return {"sm_mhz": med, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


def workload_case(n: int, engine: int, dev: int, fastmath: int = 1):
    import cases
    case = cases.conical_island(n, engine=engine, dx=0.05 * 1024 / n if n != 1024 else 0.05)
    case.param.GPUDEVICE = dev
    case.param.fastmath = fastmath
    return case


def flushed_steps(f, loop, steps, flush):
    """K flow steps, L2 flushed before each; returns (flux_ms, update_ms) summed."""
    import torch
    f.set_profiling(True)
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        loop.totaltime += f.flow_step(loop)
    a, b, n = f.kernel_timing()
    f.set_profiling(False)
    return a, b


def _cpu_sample_here(build: str, steps: int, warmup: int, engine: int) -> dict:
    """The reference FlowCPU (built from its sources: "O2" host optimisation, or
    "makefile", the reference Makefile's own host flags without -O) on a
    REF_WINDOW x REF_WINDOW window of the workload, in this process.  Records the
    wall time, the CPU time (user + system) and the largest number of threads the
    process ran, so the parallelism is measured, not assumed."""
    import resource
    import cases
    from oracle.pyoracle import REF_LIB, REF_LIB_FAITHFUL, ref_available
    case = cases.conical_island(REF_WINDOW, engine=engine, dx=0.05)
    ncell = REF_WINDOW * REF_WINDOW
    faithful = build == "makefile"
    if ref_available(faithful):
        from runners import make_reference
        r = make_reference(case, lib_path=REF_LIB_FAITHFUL if faithful else REF_LIB)
        kind, run = "reference", r.step
    else:
        from runners import make_oracle
        r, _ = make_oracle(case)
        kind, run = "port", r.step
    run(warmup)

    def nthreads() -> int:
        try:
            with open("/proc/self/status") as fh:
                for ln in fh:
                    if ln.startswith("Threads:"):
                        return int(ln.split()[1])
        except OSError:
            pass
        return 0
    idle = nthreads()  # the interpreter's own (and any idle library pool) threads
    peak = [idle]
    stop = threading.Event()

    def watch():
        while not stop.is_set():
            peak[0] = max(peak[0], nthreads() - 1)  # less this watcher
            time.sleep(0.005)
    th = threading.Thread(target=watch, daemon=True)
    th.start()
    ru0 = resource.getrusage(resource.RUSAGE_SELF)
    t0 = time.perf_counter()
    run(steps)
    wall = time.perf_counter() - t0
    ru1 = resource.getrusage(resource.RUSAGE_SELF)
    stop.set()
    th.join()
    cpu = (ru1.ru_utime - ru0.ru_utime) + (ru1.ru_stime - ru0.ru_stime)
    return {"value": ncell * steps / wall, "kind": kind, "build": build, "wall_s": wall, "steps": steps,
            "cpu_s": cpu, "parallelism": cpu / wall, "threads_max": 1 + peak[0] - idle}


def cpu_reference_sample(steps: int, warmup: int, engine: int, build: str = "O2") -> dict:
    """_cpu_sample_here in a child process (the two reference builds export the same
    symbols, so each is loaded alone)."""
    import subprocess
    cmd = [sys.executable, os.path.abspath(__file__), "--cpu-sample", build, "--steps", str(steps), "--warmup",
           str(warmup), "--engine", str(engine)]
    out = subprocess.run(cmd, check=True, capture_output=True, text=True).stdout
    return json.loads(out.strip().splitlines()[-1])


def cpu_baseline_entry(r: dict) -> dict:
    hc = host_cpu()
    return {"value": r["value"], "unit": UNIT, "cores": r["threads_max"], "kind": r["kind"],
            "sample": f"{r['steps']} FlowCPU steps on a {REF_WINDOW}x{REF_WINDOW} window of the workload "
                      f"({r['wall_s']:.1f} s), reference host build {r['build']}",
            "measured_parallelism": round(r["parallelism"], 2),
            "cores_meaning": "largest number of threads the reference ran at once (its per-variable std::threads plus "
                             "the calling thread); measured_parallelism = CPU time / wall time",
            "host": hc, "taskset_cores": sorted(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else None}


def reference_gpu_baseline(n: int, engine: int, steps: int) -> dict:
    """The reference's own FlowGPU (its CUDA sources compiled for sm_100a by
    oracle/ref/Makefile) on the same workload and GPU, through the oracle harness:
    wall clock of `steps` steps after 3 untimed ones (each reference step reads its dt
    back to the host, so the clock covers its work), and its distance from FlowCPU."""
    import torch
    from runners import interior, make_oracle, make_reference
    case = workload_case(n, engine, 0, 0)
    case.paramtext = case.paramtext.replace("gpudevice = -1", "gpudevice = 0")
    r = make_reference(case)
    r.step(3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    r.step(steps)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    o, _ = make_oracle(workload_case(n, engine, 0, 0))
    o.step(3 + steps)
    diff = float(np.abs(interior(r.get("zs")) - interior(o.get("zs"))).max())
    del r
    return {"value": n * n * steps / wall, "unit": UNIT, "ms_per_step": wall / steps * 1e3,
            "sample": f"{steps} FlowGPU steps of the {n}x{n} workload after 3 untimed ones, wall clock",
            "build": "reference sources compiled for sm_100a (nvcc defaults: FMA contraction)",
            "max_abs_zs_vs_flowcpu_m": diff}


def accuracy_full_run(n: int, engine: int, dev: int, fastmath: int, endtime: float = 20.0) -> dict:
    """The whole simulated run of the workload (as the configuration states it) in the
    headline build against the reference's own FP64 FlowGPU (its CUDA sources built
    for sm_100a) over the same simulated time, both on this GPU: max |eta|, |hu|,
    |hv| over all cells at the end, and the step counts."""
    import torch
    from runners import interior, make_gpu, make_reference
    case = workload_case(n, engine, dev, fastmath)
    case.nextoutputtime = endtime
    f, mesh, loop = make_gpu(case)
    nsteps = f.run(loop, endtime=endtime)
    zs, h, u, v = f.get_state()
    def reference_run(use_double):
        rc = workload_case(n, engine, dev, fastmath)
        rc.nextoutputtime = endtime
        rc.paramtext = rc.paramtext.replace("gpudevice = -1", "gpudevice = 0")
        r = make_reference(rc, use_double=use_double)
        rsteps, rtime = 0, 0.0
        t0 = time.perf_counter()
        while rtime < endtime - 1e-12 and rsteps < 200000:
            rtime += float(r.step(1)[0])  # the harness adds dt to its FP64 time the same way
            rsteps += 1
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        fields = [interior(r.get(k)).astype(np.float64) for k in ("zs", "h", "u", "v")]
        del r
        return fields, rtime, rsteps, wall

    def errors(a, b):
        (za, ha, ua, va), (zb, hb, ub, vb) = a, b
        return {"max_abs_eta_m": float(np.abs(za - zb).max()), "max_abs_hu_m2s": float(np.abs(ha * ua - hb * ub).max()),
                "max_abs_hv_m2s": float(np.abs(ha * va - hb * vb).max())}

    r64, rtime, rsteps, wall64 = reference_run(True)
    r32, _, rsteps32, _ = reference_run(False)
    ours = [interior(a).astype(np.float64) for a in (zs, h, u, v)]
    out = {"vs": "reference FlowGPU, FP64 build, same GPU", "simulated_s": loop.totaltime,
           "reference_simulated_s": rtime, "steps": nsteps, "reference_steps": rsteps,
           "reference_fp64_wall_s": wall64, **errors(ours, r64),
           "reference_fp32": {"steps": rsteps32, **errors(r32, r64)},
           "reference_fp32_meaning": "the reference's own FP32 FlowGPU against its FP64 build over the same run",
           "target_eta_m": 1e-3}
    return out


def accuracy_vs_fp64(n: int, engine: int, dev: int, fastmath: int, steps: int = 20) -> dict:
    """The headline build from the workload's start against the FP64 oracle over the
    same number of steps: max |eta| and max |h u| differences over all cells."""
    from runners import make_gpu, make_oracle
    case = workload_case(n, engine, dev, fastmath)
    f, mesh, loop = make_gpu(case)
    for _ in range(steps):
        loop.totaltime += f.flow_step(loop)
    zs, h, u, v = f.get_state()
    o, _ = make_oracle(workload_case(n, engine, dev, fastmath), use_double=True)
    o.step(steps)
    it = (slice(None), slice(1, 17), slice(1, 17))
    eta_err = float(np.abs(zs[it].astype(np.float64) - o.get("zs")[it]).max())
    hu_err = float(np.abs((h[it].astype(np.float64) * u[it]) - o.get("h")[it] * o.get("u")[it]).max())
    hv_err = float(np.abs((h[it].astype(np.float64) * v[it]) - o.get("h")[it] * o.get("v")[it]).max())
    return {"vs": "FP64 oracle (CPU restatement of FlowCPU, pinned to the reference)", "steps": steps,
            "simulated_s": loop.totaltime, "max_abs_eta_m": eta_err, "max_abs_hu_m2s": hu_err, "max_abs_hv_m2s": hv_err,
            "target_eta_m": 1e-3}


ACC_T = 300.0       # simulated seconds of the ensemble accuracy runs
ACC_MAX_BLOCKS = 1024


def _oracle_member(args):
    """The FP64 or FP32 oracle on ensemble member k to ACC_T; (zs, hu) interiors."""
    k, seed, min_blocks, use_double = args
    import cases
    from runners import interior, make_oracle
    c = cases.ensemble_member(k, seed, min_blocks, ACC_MAX_BLOCKS)
    c.nextoutputtime = ACC_T
    o, _ = make_oracle(c, use_double=use_double)
    while o.totaltime < ACC_T:
        o.step(1)
    zs, h, u = (interior(o.get(n)) for n in ("zs", "h", "u"))
    return zs, h * u


def ensemble_accuracy(seed: int, min_blocks: int, dev: int, fastmath: int, members=(0, 1, 3, 7)) -> dict:
    """Split-precision FP32 members (two rain, two tsunami; block counts capped at
    ACC_MAX_BLOCKS) after ACC_T simulated seconds against the FP64 oracle, with the
    reference's own FP32 arithmetic (the oracle's FP32 build) against the same FP64
    oracle beside it.  The oracle runs in spawned processes while the GPU runs."""
    import multiprocessing as mp
    import cases
    from runners import interior, make_gpu
    ctx = mp.get_context("spawn")
    jobs = [(k, seed, min_blocks, dbl) for k in members for dbl in (True, False)]
    with ctx.Pool(min(len(jobs), max(1, (os.cpu_count() or 2) - 1))) as pool:
        pending = pool.map_async(_oracle_member, jobs)
        gpu = {}
        for k in members:
            c = cases.ensemble_member(k, seed, min_blocks, ACC_MAX_BLOCKS)
            c.param.GPUDEVICE = dev
            c.param.fastmath = fastmath
            c.param.splitprecision = 1
            c.nextoutputtime = ACC_T
            f, _, lp = make_gpu(c)
            f.run(lp, endtime=ACC_T)
            zs, h, u, v = f.get_state()
            gpu[k] = (c.name, interior(zs).astype(np.float64), (interior(h).astype(np.float64) * interior(u)))
            del f
        ora = dict(zip(jobs, pending.get()))
    acc = {}
    for k in members:
        name, zs, hu = gpu[k]
        z64, q64 = ora[(k, seed, min_blocks, True)]
        z32, q32 = ora[(k, seed, min_blocks, False)]
        acc[name] = {"kind": "tsunami" if k % 4 == 3 else "rain", "simulated_s": ACC_T,
                     "max_eta_err_m": float(np.abs(zs - z64).max()), "max_hu_err_m2s": float(np.abs(hu - q64).max()),
                     "reference_fp32_eta_err_m": float(np.abs(z32 - z64).max()),
                     "reference_fp32_hu_err_m2s": float(np.abs(q32 - q64).max())}
    return {"vs": "FP64 oracle (CPU restatement of FlowCPU, pinned to the reference)",
            "reference_fp32": "the oracle's FP32 build against the same FP64 oracle: the error of evaluating the "
                              "reference's algorithm in FP32", "members": acc}


def _member_levels(k: int, seed: int, amr: bool) -> int:
    """Refinement levels above level 0 of ensemble member k: 0, 1 or 2 (seeded) for
    rain members when the ensemble has AMR members, 0 for tsunamis (split precision
    runs on single-level meshes)."""
    if not amr or k % 4 == 3:
        return 0
    return int(np.random.default_rng([seed, k, 7]).integers(0, 3))


def _build_member(c, levels: int):
    """The handle of an ensemble member: single-level (make_gpu) or refined to
    `levels` levels above level 0 where the bed lies in the lowest 10 % of the
    member's relief (Inrange criterion on zb), from its own bathymetry grid."""
    from runners import make_gpu
    if levels == 0:
        f, mesh, lp = make_gpu(c)
        return f, lp
    from bg_flood_b200.adapt import Criterion, INRANGE
    from bg_flood_b200.flow import FlowB200, Loop
    from bg_flood_b200.mesh import boundary_segments, grid_to_buq, uniform_mesh
    c.param.maxlevel, c.param.minlevel, c.param.initlevel = levels, 0, 0
    mesh = uniform_mesh(c.nx, c.ny, c.dx)
    lo = float(c.zb.min())
    hi = lo + 0.1 * (float(c.zb.max()) - lo)
    mem = 3 * mesh.nblk
    while True:
        f = FlowB200(c.param, mem)
        pad = lambda a: np.concatenate([a, np.zeros((mem - len(a), 18, 18), a.dtype)])
        f.set_blocks(mesh.active, mesh.level, mesh.nbr, mesh.xo, mesh.yo)
        f.set_bed(pad(grid_to_buq(c.zb, mesh, np.float32)))
        for typ, times, lv, sides in boundary_segments(mesh, c.param.segments, c.param.aoibnd, 0.0, 0.0):
            f.add_segment(typ, times, lv, sides)
        if c.rain is not None:
            f.set_rain(*c.rain)
        f.set_state(*(pad(grid_to_buq(a, mesh, np.float32)) for a in (c.h, c.u, c.v)))
        f.set_bathy(0.5 * c.dx, 0.5 * c.dx, c.dx, c.zb)
        try:
            f.adapt(Criterion(INRANGE, "zb", lo, hi), maxiteration=levels + 1)
            break
        except RuntimeError:
            f.close()
            if mem >= mesh.nblk * 4 ** levels:
                raise
            mem *= 2
    lp = Loop(totaltime=0.0, dt=0.0, dtmax=0.0, nextoutputtime=c.nextoutputtime)
    f.init_dt(lp)
    return f, lp


def ensemble_bench(nscen: int, seed: int, min_blocks: int, max_blocks: int, steps: int, dev: int, fastmath: int,
                   accuracy: bool = True, peak_rate: float | None = None, amr: bool = True):
    """Batched ensemble against the plain one-scenario-at-a-time loop on the same
    seeded members (level-0 block counts log-uniform in [min_blocks, max_blocks];
    rain on fractal terrain, with 0-2 refinement levels when amr, in FP32; and
    deep-water tsunamis in split precision), each member advanced by `steps` steps.
    The batched form runs two pools (split and FP32 members), one after the other.
    Device time of the steps (CUDA events around the graphs) and wall clock
    including the host set-up of every member."""
    import cases
    from bg_flood_b200.pool import ScenarioPool
    members = [cases.ensemble_member(k, seed, min_blocks, max_blocks) for k in range(nscen)]
    levels = [_member_levels(k, seed, amr) for k in range(nscen)]
    for k, c in enumerate(members):
        c.param.GPUDEVICE = dev
        c.param.fastmath = fastmath
        c.param.splitprecision = 1 if k % 4 == 3 else 0   # tsunamis: FP32 deviations from FP64 block datums
    build = lambda k: _build_member(members[k], levels[k])
    # warm-up of both paths on the smallest member
    small = int(np.argmin([(c.nx // 16) * (c.ny // 16) for c in members]))
    f, lp = build(small)
    f.run(lp, endtime=1e30, maxsteps=4)
    del f
    plain_ms, t0 = 0.0, time.perf_counter()
    member_ms, blocks = [], []
    for k in range(nscen):
        f, lp = build(k)
        blocks.append(f.nblk)
        f.run(lp, endtime=1e30, maxsteps=steps)
        member_ms.append(f.last_run_timing()[0])
        plain_ms += member_ms[-1]
        del f
    plain_wall = time.perf_counter() - t0
    # the reference's loop structure: one host call per step, the step's dt read back
    # before the next (Mainloop); wall clock of the steps alone, set-up excluded
    step_loop_s = 0.0
    for k in range(nscen):
        f, lp = build(k)
        lp.totaltime += f.flow_step(lp)
        ts = time.perf_counter()
        for _ in range(steps):
            lp.totaltime += f.flow_step(lp)
        step_loop_s += time.perf_counter() - ts
        del f
    cells = [256 * b for b in blocks]
    best_member_rate = max(cl * steps / (ms / 1e3) for cl, ms in zip(cells, member_ms))
    t0 = time.perf_counter()
    groups = [[k for k in range(nscen) if members[k].param.splitprecision == sp] for sp in (1, 0)]
    groups = [g for g in groups if g]
    pools = [ScenarioPool(members[g[0]].param, sum(blocks[k] for k in g), len(g)) for g in groups]
    t1 = time.perf_counter()
    # the members' host set-up in four threads (numpy and the C ABI release the
    # interpreter lock); the plain loop above prepares one member at a time
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(4) as ex:
        built = list(ex.map(build, range(nscen)))
    t2 = time.perf_counter()
    for g, pool in zip(groups, pools):
        for k in g:
            f, lp = built[k]
            pool.admit(f, lp, 1e30, maxsteps=steps)
    t3 = time.perf_counter()
    batched_ms = 0.0
    for pool in pools:
        assert pool.run(steps + 2) == 0
        batched_ms += pool.timing()[0]
    batched_wall = time.perf_counter() - t0
    phases = {"pool_create_s": t1 - t0, "build_s": t2 - t1, "admit_s": t3 - t2, "run_s": time.perf_counter() - t3}
    del pools, built
    batched_rate = sum(blocks) * 256 * steps / (batched_ms / 1e3)
    acc = ensemble_accuracy(seed, min_blocks, dev, fastmath) if accuracy else None
    return {"scenarios": nscen, "precision": "tsunamis FP32 split (deviations from FP64 block datums), rain FP32",
            "members_per_level_count": {str(n + 1): int(sum(1 for x in levels if x == n)) for n in range(3)},
            "accuracy_vs_fp64": acc, "blocks_total": int(sum(blocks)), "blocks_min": int(min(blocks)),
            "blocks_max": int(max(blocks)), "steps_per_scenario": steps,
            "plain_device_ms": plain_ms, "batched_device_ms": batched_ms,
            "plain_scenarios_per_s": nscen / (plain_ms / 1e3), "batched_scenarios_per_s": nscen / (batched_ms / 1e3),
            "speedup_device": plain_ms / batched_ms,
            "best_member_cell_rate": best_member_rate,
            "speedup_device_bound": plain_ms / (sum(cells) * steps / max(best_member_rate, batched_rate) * 1e3),
            "speedup_device_bound_at_peak": None if peak_rate is None else
            plain_ms / (sum(cells) * steps / max(peak_rate, best_member_rate, batched_rate) * 1e3),
            "speedup_bound_meaning": "plain device time / (all members' cell-updates at the best cell rate measured: "
                                     "the best single member, the batched run or, at_peak, the large single-grid "
                                     "device loop): what batching could gain at most if every member ran that fast",
            "plain_per_step_loop_s": step_loop_s,
            "speedup_vs_per_step_loop": step_loop_s / (batched_ms / 1e3),
            "per_step_loop_meaning": "one bgf_flow_step call per step with its dt read back (the reference's "
                                     "Mainloop structure), wall clock of the steps, against the batched device time",
            "plain_wall_s": plain_wall, "batched_wall_s": batched_wall,
            "speedup_wall": plain_wall / batched_wall, "batched_phases": phases,
            "cell_updates_per_s_batched": sum(blocks) * 256 * steps / (batched_ms / 1e3)}


def amr_bench(n0: int, maxlevel: int, steps: int, dev: int, fastmath: int, readapt_every: int = 50,
              mem_factor: int = 16):
    """Quadtree rain-on-grid: seeded fractal terrain (0-300 m relief, carved valley) on
    an n0 x n0 level-0 grid (dx = 10 m), rain of 50 mm/h, Manning n = 0.035, a lake
    filling the lowest 3 % of the terrain at the start.  The mesh follows the
    depth-or-slope criterion (refine where h > 0.01 m or |grad eta| > 1e-3, coarsen
    below half of both; coarsening is an extension, the reference cancels it) up to
    maxlevel: adapted at the start and again every readapt_every steps while the
    device loop runs.  Reports the device loop's cell-updates/s over all levels, the
    adaptation passes' wall time and the rate with that time included."""
    import cases
    from bg_flood_b200.adapt import depth_or_slope
    from bg_flood_b200.flow import FlowB200, Loop
    from bg_flood_b200.mesh import boundary_segments, grid_to_buq, uniform_mesh
    case = cases.rain_on_terrain(n0, engine=1, dx=10.0, seed=11)
    case.param.GPUDEVICE = dev
    case.param.fastmath = fastmath
    case.param.maxlevel, case.param.minlevel, case.param.initlevel = maxlevel, 0, 0
    zfill = float(np.quantile(case.zb, 0.03))
    h0 = np.maximum(np.float32(zfill) - case.zb, 0.0).astype(np.float32)
    mesh = uniform_mesh(n0, n0, case.dx)
    mem = mesh.nblk * mem_factor
    f = FlowB200(case.param, mem)
    f.set_blocks(mesh.active, mesh.level, mesh.nbr, mesh.xo, mesh.yo)
    pad = lambda a: np.concatenate([a, np.zeros((mem - len(a), 18, 18), a.dtype)])
    f.set_bed(pad(grid_to_buq(case.zb, mesh, np.float32)))
    for typ, times, levels, sides in boundary_segments(mesh, case.param.segments, case.param.aoibnd, 0.0, 0.0):
        f.add_segment(typ, times, levels, sides)
    f.set_rain(*case.rain)
    z = np.zeros_like(case.zb)
    f.set_state(*(pad(grid_to_buq(a, mesh, np.float32)) for a in (h0, z, z)))
    f.set_bathy(0.5 * case.dx, 0.5 * case.dx, case.dx, case.zb)
    crit = depth_or_slope(0.01, 1e-3)
    t0 = time.perf_counter()
    nblk, it = f.adapt(crit, maxiteration=maxlevel + 1, allow_coarsen=True)
    adapt0_s = time.perf_counter() - t0

    def mesh_stats():
        act, lev, nbr, _, _ = f.get_blocks()
        act = act[: f.nblk]
        hist = np.bincount(lev[act], minlength=maxlevel + 1).tolist()
        cross = int(np.count_nonzero((lev[nbr[act]] != lev[act][:, None]).any(axis=1)))
        return hist, cross

    hist0, cross0 = mesh_stats()
    loop = Loop(totaltime=0.0, dt=0.0, dtmax=0.0, nextoutputtime=1e30)
    f.init_dt(loop)
    f.run(loop, endtime=1e30, maxsteps=10)
    ms_total, cells_total, launches, passes = 0.0, 0, 0, []
    done = 0
    while done < steps:
        k = min(readapt_every, steps - done)
        n = f.nblk
        f.run(loop, endtime=1e30, maxsteps=k)
        ms, nl = f.last_run_timing()
        ms_total += ms
        launches += nl
        cells_total += n * 256 * k
        done += k
        if done < steps:
            t0 = time.perf_counter()
            n2, it2 = f.adapt(crit, maxiteration=maxlevel + 1, allow_coarsen=True)
            passes.append({"after_step": done, "s": time.perf_counter() - t0, "blocks_before": n, "blocks_after": n2,
                           "passes": it2})
    hist1, cross1 = mesh_stats()
    adapt_total = sum(p["s"] for p in passes)
    return {"level0_cells": n0 * n0, "maxlevel": maxlevel, "nblkmem": mem,
            "criterion": "h > 0.01 m or |grad eta| > 1e-3, coarsen below half (extension)",
            "blocks_start": int(nblk), "blocks_per_level_start": hist0, "adapt_passes_start": it,
            "adapt_start_s": adapt0_s, "blocks_multilevel_chain_start": cross0,
            "blocks_end": int(f.nblk), "blocks_per_level_end": hist1, "blocks_multilevel_chain_end": cross1,
            "steps": steps, "readapt_every": readapt_every, "readaptations": passes,
            "simulated_s": loop.totaltime, "ms": ms_total, "launches_per_step": launches / steps,
            "cell_updates_per_s": cells_total / (ms_total / 1e3),
            "cell_updates_per_s_with_adaptation": cells_total / (ms_total / 1e3 + adapt_total)}


def serving_bench(nreq: int, seed: int, rate: float, dev: int, fastmath: int, budget_gb: float = 150.0,
                  rates=None):
    """Poisson streams of flood scenarios (blocks log-uniform in [16, 2048], 100-400
    steps each) at each arrival rate of `rates` (default: rate, 5x rate and all at
    once), served by the continuous-batching server under an HBM budget and by the
    plain loop (one at a time, arrival order).  Time-to-solution percentiles and
    completed scenarios per second of wall clock per rate; the headline keys are
    those of the first rate."""
    rates = list(rates) if rates is not None else [rate, 5.0 * rate, math.inf]
    out = {}
    srv = None
    for k, lam in enumerate(rates):
        r, srv = _serving_at_rate(nreq, seed, lam, dev, fastmath, budget_gb, srv)
        if k == 0:
            out.update(r)
        out.setdefault("sweep", []).append({"rate_per_s": lam if math.isfinite(lam) else "all_at_once",
                                           "served_host_s": r["served"]["host_s"],
                                           "served_gpu_ms": r["served"]["gpu_ms"],
                                           "served_per_s": r["served"]["scenarios_per_s"],
                                           "plain_per_s": r["plain"]["scenarios_per_s"],
                                           "served_p50_s": r["served"]["p50_s"], "served_p99_s": r["served"]["p99_s"],
                                           "plain_p50_s": r["plain"]["p50_s"], "plain_p99_s": r["plain"]["p99_s"]})
    srv.pool.close()
    return out


def _serving_at_rate(nreq: int, seed: int, rate: float, dev: int, fastmath: int, budget_gb: float, srv):
    import cases
    from bg_flood_b200.serve import FloodServer, Request, serve_sequential
    from runners import make_gpu
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, nreq)) if math.isfinite(rate) else np.zeros(nreq)
    reqs = []
    for k in range(nreq):
        case = cases.ensemble_member(k, seed, 16, 2048)
        case.param.GPUDEVICE = dev
        case.param.fastmath = fastmath

        def build(case=case):
            f, mesh, loop = make_gpu(case)
            return f, loop
        reqs.append(Request(k, float(arrivals[k]), (case.nx // 16) * (case.ny // 16), build,
                            maxsteps=int(rng.integers(100, 400))))
    param = cases.ensemble_member(0, seed, 16, 2048).param
    param.GPUDEVICE = dev
    param.fastmath = fastmath
    out = {}
    # the server is long-lived: its start-up (the HBM budget's block slots) is timed
    # separately, not charged to the stream
    ts = time.perf_counter()
    if srv is None:
        srv = FloodServer(param, budget_gb * 1e9, max_scenarios=64, chunk_steps=64, keep_fields=True)
        # short untimed streams of other scenarios over the same size range prime what
        # a long-lived process has warm (kernel modules, the memory pool, page-locked
        # staging of each size class), for both paths
        prime = []
        for k in range(16):
            pc = cases.ensemble_member(k, seed + 1000, 16, 2048)
            pc.param.GPUDEVICE = dev
            pc.param.fastmath = fastmath

            def pbuild(case=pc):
                f, mesh, loop = make_gpu(case)
                return f, loop
            prime.append(Request(1000 + k, 0.0, (pc.nx // 16) * (pc.ny // 16), pbuild, maxsteps=20))
        srv.serve(prime, realtime=False)
        serve_sequential(prime[:4], realtime=False)
    startup_s = time.perf_counter() - ts
    for name, fn in (("served", None), ("plain", serve_sequential)):
        t0 = time.perf_counter()
        if fn is None:
            res = srv.serve(reqs, realtime=True)
        else:
            res = fn(reqs, realtime=True)
        wall = time.perf_counter() - t0
        tts = np.array([r.time_to_solution for r in res])
        out[name] = {"p50_s": float(np.percentile(tts, 50)), "p99_s": float(np.percentile(tts, 99)),
                     "scenarios_per_s": nreq / wall, "wall_s": wall}
        if fn is None:
            out[name]["host_s"] = dict(srv.host_s)
            out[name]["gpu_ms"] = srv.gpu_ms
            out[name]["pool_blocks"] = srv.nblk_pool
            out[name]["startup_s"] = startup_s
    out["rate_per_s"] = rate if math.isfinite(rate) else "all_at_once"
    out["requests"] = nreq
    return out, srv


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    steps = max(1, args.steps if args.steps <= 20 else 10)
    r = cpu_reference_sample(steps, min(args.warmup, 3), args.engine, "O2")
    cb = cpu_baseline_entry(r)
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": steps, "warmup": min(args.warmup, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "engine": args.engine,
                   "sample": f"{REF_WINDOW}x{REF_WINDOW} window of the workload (the reference's FlowCPU takes about "
                             f"a second per step on it; the full 1024x1024 grid is 16x that per step)"},
        "cpu_baseline": cb,
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.cpu_sample:
        print(json.dumps(_cpu_sample_here(args.cpu_sample, args.steps, args.warmup, args.engine)), flush=True)
        return
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return

    import torch
    import torch.distributed as dist
    from runners import make_gpu

    torch.cuda.set_device(local)
    if args.only:
        # one secondary measurement alone, for profiling its launches
        if args.only == "amr":
            r = amr_bench(args.amr, 3, args.steps, local, args.fastmath)
        elif args.only == "ensemble":
            r = ensemble_bench(args.ensemble, 2024, 64, args.ens_max_blocks, args.steps, local, args.fastmath)
        elif args.only == "ensemble_small":
            r = ensemble_bench(args.ensemble, 2025, 40, 512, args.steps, local, args.fastmath, accuracy=False, amr=False)
        else:
            r = serving_bench(args.serve, 7, args.serve_rate, local, args.fastmath)
        print(json.dumps({"measurement": args.only, **r}))
        return
    if args.profile_steps:
        f, mesh, loop = make_gpu(workload_case(args.n, args.engine, local, args.fastmath))
        f.set_kernel_layout(args.layout)
        for _ in range(args.profile_steps):
            loop.totaltime += f.flow_step(loop)
        print(json.dumps({"profile_steps": args.profile_steps, "totaltime": loop.totaltime}))
        return
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))

    case = workload_case(args.n, args.engine, local, args.fastmath)
    f, mesh, loop = make_gpu(case)
    ncell = mesh.nblk * 256
    # launch shape from the autotuner (state restored afterwards)
    tuned_grid, tuned_ms = f.autotune(loop, 20)

    for _ in range(args.warmup):
        loop.totaltime += f.flow_step(loop)

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    f.set_profiling(True)
    launches0 = f.kernel_launches()
    clocks = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with clocks:
        for _ in range(args.steps):
            flush.zero_()                 # L2 (126 MB) flushed before every timed step
            torch.cuda.synchronize()
            loop.totaltime += f.flow_step(loop)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    flux_ms, update_ms, nprof = f.kernel_timing()
    launches = f.kernel_launches() - launches0
    f.set_profiling(False)
    step_ms = (flux_ms + update_ms) / max(nprof, 1)
    from bg_flood_b200.replicas import replica_throughput
    value, tmax_ms = replica_throughput(ncell * args.steps, flux_ms + update_ms, dist if world > 1 else None,
                                        device=f"cuda:{local}")

    # dominant kernel roofline
    peak, peak_kind = measured_peak_hbm()
    # the handle runs the two-cells-per-thread stage kernels (its default layout)
    kern = {"flux2_kernel": (flux_ms / nprof, ALG_BYTES_FLUX), "update2_kernel": (update_ms / nprof, ALG_BYTES_UPDATE)}
    dom = max(kern, key=lambda k: kern[k][0])
    dom_ms, dom_b = kern[dom]
    achieved = dom_b * ncell / (dom_ms / 1e3) / 1e9
    # both stage kernels (their times are within a few per cent of each other, so the
    # one named dominant can change from run to run)
    per_kernel = {k: {"us_per_launch": ms * 1e3, "alg_bytes_per_cell": b,
                      "achieved": b * ncell / (ms / 1e3) / 1e9} for k, (ms, b) in kern.items()}
    traffic = None
    variant = "fastmath" if args.fastmath else "exact"
    tfile = os.path.join(ROOT, "profiles", f"{dom}_runup{args.n}_{variant}.md")
    if os.path.exists(tfile):
        for ln in open(tfile):
            if ln.startswith("dram_bytes_per_cell:"):
                traffic = float(ln.split(":")[1]) * ncell

    # end to end through the C ABI with host buffers
    # the step inputs and results live in page-locked host buffers, allocated once as
    # a caller that streams states would hold them
    zs, h, u, v = f.get_state()
    keep = [torch.empty(a.shape, dtype=torch.float64 if a.dtype == np.float64 else torch.float32, pin_memory=True)
            for a in (zs, h, u, v, h, u, v)]
    outs = [t.numpy() for t in keep[:4]]
    h, u, v = [t.numpy() for t in keep[4:]]
    f.get_state(out=outs)
    h[...], u[...], v[...] = outs[1], outs[2], outs[3]
    e2e_loop = type(loop)(totaltime=0.0, dt=0.0, dtmax=0.0, nextoutputtime=case.nextoutputtime)
    f.init_dt(e2e_loop)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f.set_state(h, u, v)
    for _ in range(args.steps):
        e2e_loop.totaltime += f.flow_step(e2e_loop)
    f.get_state(out=outs)
    e2e_s = time.perf_counter() - t0
    # bytes that crossed the host link: whole 18x18 tiles of h, u, v up and of zs, h,
    # u, v down (page-locked arrays go by DMA), and per step the time state up (80 B)
    # with the dt seed (8 B), the time state (80 B) and the error word (4 B) down
    tslot = 80
    es = outs[0].itemsize
    h2d = (3 * f.nblkmem * 324 * es + args.steps * (tslot + 8)) / args.steps
    d2h = (4 * f.nblkmem * 324 * es + args.steps * (tslot + 4)) / args.steps
    e2e_val = world * ncell * args.steps / e2e_s

    extra = {}
    if not args.no_extra and rank == 0:
        # the other kernel variant on the same workload, same protocol
        other = workload_case(args.n, args.engine, local, 1 - args.fastmath)
        fo, _, lo = make_gpu(other)
        for _ in range(3):
            lo.totaltime += fo.flow_step(lo)
        a, b = flushed_steps(fo, lo, min(args.steps, 50), flush)
        extra["bitexact_kernels" if args.fastmath else "fastmath_kernels"] = {
            "value": ncell * min(args.steps, 50) / ((a + b) / 1e3), "flux_ms": a / min(args.steps, 50),
            "update_ms": b / min(args.steps, 50)}
        del fo
        # production mode: the device-resident loop (CUDA graphs), L2-warm, same workload
        l2 = type(loop)(totaltime=0.0, dt=0.0, dtmax=0.0, nextoutputtime=1e30)
        f.init_dt(l2)
        f.run(l2, endtime=1e30, maxsteps=20)
        f.run(l2, endtime=1e30, maxsteps=400)
        ms, nl = f.last_run_timing()
        extra["device_loop_L2_resident"] = {"value": ncell * 400 / (ms / 1e3), "steps": 400, "ms": ms}
        del f
        # the whole simulated run of the workload (20 s) in the device loop, from a
        # fresh start: late steps read the far end of the boundary series
        fr, mr, lr = make_gpu(workload_case(args.n, args.engine, local, args.fastmath))
        lr.nextoutputtime = 1e30
        t0 = time.perf_counter()
        nfull = fr.run(lr, endtime=20.0)
        wall_full = time.perf_counter() - t0
        msf, _ = fr.last_run_timing()
        extra["full_run_20s"] = {"value": mr.nblk * 256 * nfull / (msf / 1e3), "steps": nfull, "ms": msf,
                                 "wall_s": wall_full, "simulated_s": lr.totaltime}
        del fr
        # a grid well above L2 (4096^2 cells, ~1 GB of state): HBM-bound device loop
        big = workload_case(4096, args.engine, local, args.fastmath)
        fb, mb, lb = make_gpu(big)
        fb.run(lb, endtime=1e30, maxsteps=10)
        fb.run(lb, endtime=1e30, maxsteps=100)
        msb, _ = fb.last_run_timing()
        extra["device_loop_4096x4096"] = {"value": mb.nblk * 256 * 100 / (msb / 1e3), "steps": 100, "ms": msb}
        del fb
        if args.amr > 0:
            extra["amr_rain_on_grid"] = amr_bench(args.amr, 3, 200, local, args.fastmath)
        if args.ensemble > 0:
            grid_rate = extra["device_loop_4096x4096"]["value"]
            extra["ensemble"] = ensemble_bench(args.ensemble, 2024, 64, args.ens_max_blocks, 100, local,
                                               args.fastmath, peak_rate=grid_rate)
            # the small end of the stated member sizes (1e4 to 1.3e5 cells), where one
            # member alone cannot fill the GPU
            extra["ensemble_small_members"] = ensemble_bench(args.ensemble, 2025, 40, 512, 100, local,
                                                             args.fastmath, accuracy=False, peak_rate=grid_rate,
                                                             amr=False)
        if args.serve > 0:
            extra["serving"] = serving_bench(args.serve, 7, args.serve_rate, local, args.fastmath)

    cpu = None
    if rank == 0 and world == 1:
        # the reference's FlowCPU on the host cores: the -O2 build is the baseline, the
        # Makefile-flags build (no host optimisation, as the reference ships) beside it
        cpu = cpu_baseline_entry(cpu_reference_sample(8, 1, args.engine, "O2"))
        if not args.no_extra:
            extra["cpu_baseline_makefile_flags"] = cpu_baseline_entry(
                cpu_reference_sample(2, 0, args.engine, "makefile"))
        extra["accuracy"] = accuracy_vs_fp64(args.n, args.engine, local, args.fastmath)
        if not args.no_extra:
            extra["reference_flowgpu_b200"] = reference_gpu_baseline(args.n, args.engine, 20)
            extra["accuracy_full_run"] = accuracy_full_run(args.n, args.engine, local, args.fastmath)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "cells": ncell, "blocks": mesh.nblk, "engine": args.engine,
                       "kernels": "fast-math (tolerance parity)" if args.fastmath else "bit-exact",
                       "launch_grid": {"grid": tuned_grid, "tuned_ms_per_step": tuned_ms,
                                       "meaning": "CTAs of the fused kernels, 0 = one per block (autotuned)"},
                       "l2": "flushed (256 MB write) before every timed step",
                       "reference_arm_sample": f"{REF_WINDOW}x{REF_WINDOW} window of the workload",
                       "kernel_layout": "two cells per thread (bgf_set_kernel_layout 2)", "parallelism":
                       f"replicas x{world}" if world > 1 else "single GPU"},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                         "alg_bytes_per_cell": dom_b,
                         "kernels": {k: {**v, "frac": v["achieved"] / peak} for k, v in per_kernel.items()},
                         "step": {"alg_bytes_per_cell_update": ALG_BYTES_FLUX + ALG_BYTES_UPDATE,
                                  "achieved": (ALG_BYTES_FLUX + ALG_BYTES_UPDATE) * value / world / 1e9,
                                  "frac": (ALG_BYTES_FLUX + ALG_BYTES_UPDATE) * value / world / 1e9 / peak}},
            "accuracy": extra.pop("accuracy", None),
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "cpu_baseline": cpu,
            "gpu_launches": int(launches),
            "clocks": clocks.summary(),
            "kernels_ms_per_step": {"flux2_kernel": flux_ms / nprof, "update2_kernel": update_ms / nprof},
            "extra": extra,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
