"""Batched scenario pool: many independent scenarios advanced together on one GPU
(the C ABI's bgf_pool_*).  No counterpart in the reference, which runs one
scenario per process.

A scenario is prepared in its own ``FlowB200`` handle (tables, bed, state,
boundaries, rain), then admitted into the pool's block slots; every pool step is
one launch pair over all admitted scenarios, each with its own dt and clock.
Retiring copies the state back into the scenario's handle."""
from __future__ import annotations

import ctypes

import numpy as np

from ._native import lib
from .flow import BGFError, CLoop, FlowB200, Loop, _check

__all__ = ["ScenarioPool"]


class ScenarioPool:
    def __init__(self, param, nblk_pool: int, max_scenarios: int, track_hmax: bool = False, stream: int | None = None):
        self.param = param
        self.dtype = np.float64 if param.doubleprecision else np.float32  # device precision
        self._cparam = param.to_c()
        h = ctypes.c_void_p()
        _check(lib().bgf_pool_create(ctypes.byref(self._cparam), int(nblk_pool), int(max_scenarios),
                                     1 if track_hmax else 0, ctypes.c_void_p(stream) if stream else None,
                                     ctypes.byref(h)), "bgf_pool_create")
        self.handle = h
        self.nblk_pool = int(nblk_pool)
        self.members: dict[int, FlowB200] = {}

    def close(self):
        if self.handle:
            lib().bgf_pool_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def admit(self, f: FlowB200, loop: Loop, endtime: float, outputtimestep: float = 0.0,
              maxsteps: int = 2**31 - 1) -> int:
        c = loop.to_c()
        slot = ctypes.c_int(-1)
        _check(lib().bgf_pool_admit(self.handle, f.handle, ctypes.byref(c), float(endtime), float(outputtimestep),
                                    int(maxsteps), ctypes.byref(slot)), "bgf_pool_admit")
        self.members[slot.value] = f
        return slot.value

    def try_admit(self, f: FlowB200, loop: Loop, endtime: float, **kw) -> int | None:
        """admit, or None when the pool has no room (BGF_EBUDGET)."""
        try:
            return self.admit(f, loop, endtime, **kw)
        except BGFError as e:
            if e.status == 7:
                return None
            raise

    def run(self, maxsteps: int) -> int:
        """Pool steps until all scenarios finished or maxsteps ran; returns the number still running."""
        n = ctypes.c_int(0)
        _check(lib().bgf_pool_run(self.handle, int(maxsteps), ctypes.byref(n)), "bgf_pool_run")
        return n.value

    def run_async(self, maxsteps: int) -> None:
        """Enqueues maxsteps (<= 512) pool steps and returns at once; wait() completes them."""
        _check(lib().bgf_pool_run_async(self.handle, int(maxsteps)), "bgf_pool_run_async")

    def prepare(self) -> None:
        """While a run_async run is in flight: applies the admissions and retirements
        made since it started to the tables now (uploads queued behind the run), so the
        next run_async launches at once (bgf_pool_prepare)."""
        _check(lib().bgf_pool_prepare(self.handle), "bgf_pool_prepare")

    def wait(self) -> int:
        """Waits for the steps run_async enqueued; returns the number still running."""
        n = ctypes.c_int(0)
        _check(lib().bgf_pool_wait(self.handle, ctypes.byref(n)), "bgf_pool_wait")
        return n.value

    def finish(self, slots, nblks, with_max: bool = False):
        """Retires finished scenarios for their fields only (bgf_pool_finish): returns,
        per slot, (FlowB200, h (nblk, 16, 16), hmax or None, Loop, nsteps, status).
        The scenarios' handles are not updated; may overlap steps from run_async."""
        n = len(slots)
        if n == 0:
            return []
        hs = [np.zeros((nb, 16, 16), self.dtype) for nb in nblks]
        hm = [np.zeros((nb, 16, 16), self.dtype) for nb in nblks] if with_max else None
        ptrs = (ctypes.c_void_p * n)(*[a.ctypes.data for a in hs])
        mptrs = (ctypes.c_void_p * n)(*[a.ctypes.data for a in hm]) if with_max else None
        loops = (CLoop * n)()
        steps = (ctypes.c_int64 * n)()
        status = (ctypes.c_int * n)()
        sl = (ctypes.c_int * n)(*[int(x) for x in slots])
        _check(lib().bgf_pool_finish(self.handle, n, sl, ptrs, mptrs, loops, steps, status), "bgf_pool_finish")
        out = []
        for k, slot in enumerate(slots):
            lp = Loop()
            lp.from_c(loops[k])
            f = self.members.pop(slot)
            ng = getattr(self, "_ngauges", {}).pop(slot, 0)
            if ng:
                f._ngauges = ng
            out.append((f, hs[k], hm[k] if with_max else None, lp, int(steps[k]), int(status[k])))
        return out

    def query(self, slot: int):
        """(Loop, status, nsteps); status 0 running, 1 finished, 2 dt underflow,
        3 non-finite state."""
        c = Loop().to_c()
        st = ctypes.c_int(0)
        n = ctypes.c_int64(0)
        _check(lib().bgf_pool_query(self.handle, int(slot), ctypes.byref(c), ctypes.byref(st), ctypes.byref(n)),
               "bgf_pool_query")
        loop = Loop()
        loop.from_c(c)
        return loop, st.value, n.value

    def retire(self, slot: int):
        """Copies the scenario back into its handle; returns (FlowB200, Loop, nsteps)."""
        c = Loop().to_c()
        n = ctypes.c_int(0)
        _check(lib().bgf_pool_retire(self.handle, int(slot), ctypes.byref(c), ctypes.byref(n)), "bgf_pool_retire")
        loop = Loop()
        loop.from_c(c)
        f = self.members.pop(slot)
        ng = getattr(self, "_ngauges", {}).pop(slot, 0)
        if ng:
            f._ngauges = ng  # its unread gauge samples came with it
        return f, loop, n.value

    def depth(self, slot: int, nblk: int, with_max: bool = False):
        """Interior depth (nblk, 16, 16) of a scenario in its active order, and its
        running maximum when the pool tracks it."""
        h = np.zeros((nblk, 16, 16), self.dtype)
        hm = np.zeros((nblk, 16, 16), self.dtype) if with_max else None
        _check(lib().bgf_pool_get_depth(self.handle, int(slot), h.ctypes.data_as(ctypes.c_void_p),
                                        None if hm is None else hm.ctypes.data_as(ctypes.c_void_p)),
               "bgf_pool_get_depth")
        return (h, hm) if with_max else h

    def set_gauges(self, slot: int, gauges) -> None:
        """Gauges of a scenario: (block index in its active order, i, j)."""
        g = np.asarray(list(gauges), np.int32).reshape(-1, 3)
        cols = [np.ascontiguousarray(g[:, k]) for k in range(3)]
        _check(lib().bgf_pool_set_gauges(self.handle, int(slot), len(g),
                                         *[c.ctypes.data_as(ctypes.c_void_p) for c in cols]), "bgf_pool_set_gauges")
        self._ngauges = getattr(self, "_ngauges", {})
        self._ngauges[slot] = len(g)

    def read_gauges(self, slot: int, max_samples: int = 1 << 16):
        """(times (s, n), values (s, n, 4) as h, zs, u, v) of a scenario's samples
        since the last read."""
        n = max(getattr(self, "_ngauges", {}).get(slot, 0), 1)
        t = np.zeros((max_samples, n))
        v = np.zeros((max_samples, n, 4))
        ns = ctypes.c_int(0)
        _check(lib().bgf_pool_read_gauges(self.handle, int(slot), int(max_samples),
                                          t.ctypes.data_as(ctypes.c_void_p), v.ctypes.data_as(ctypes.c_void_p),
                                          ctypes.byref(ns)), "bgf_pool_read_gauges")
        return t[:ns.value], v[:ns.value]

    def timing(self):
        """(gpu_ms, steps) of the last run() and the free block slots."""
        ms = ctypes.c_double(0)
        st = ctypes.c_int64(0)
        fb = ctypes.c_int(0)
        _check(lib().bgf_pool_timing(self.handle, ctypes.byref(ms), ctypes.byref(st), ctypes.byref(fb)),
               "bgf_pool_timing")
        return ms.value, st.value, fb.value

    def set_grid(self, grid: int) -> None:
        _check(lib().bgf_pool_set_grid(self.handle, int(grid)), "bgf_pool_set_grid")

    def set_kernel_layout(self, layout: int) -> None:
        """Thread layout of the single-level kernels (1, 2 or 3), as FlowB200.set_kernel_layout."""
        _check(lib().bgf_pool_set_kernel_layout(self.handle, int(layout)), "bgf_pool_set_kernel_layout")

    def autotune(self, steps: int = 20) -> tuple:
        """Times the pool step for each launch shape over the live scenarios and keeps
        the fastest; their state is unchanged afterwards.  Returns (grid, ms_per_step)."""
        g = ctypes.c_int(0)
        ms = ctypes.c_double(0.0)
        _check(lib().bgf_pool_autotune(self.handle, int(steps), ctypes.byref(g), ctypes.byref(ms)),
               "bgf_pool_autotune")
        return g.value, ms.value
