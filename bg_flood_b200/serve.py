"""Serving loop: flood scenarios arrive over time and are run together on one GPU
(continuous batching over the scenario pool).  No counterpart in the reference.

A request carries a builder that prepares the scenario in its own handle (host
set-up and upload), its block count and its run length.  The server admits
requests in arrival order while the pool's block slots -- sized from an HBM
budget -- and scenario slots allow, keeps admitted scenarios resident, advances
all of them together in chunks of pool steps, and retires each one as soon as it
finishes, copying its final depth and maximum-depth map back to the host.  Its
gauges are recorded on the device after every step (the reference's time-series
output) and the server collects them once per chunk.  Time-to-solution is measured
from arrival to retirement."""
from __future__ import annotations

import sys
import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from .flow import FlowB200, Loop
from .pool import ScenarioPool

__all__ = ["Request", "Result", "FloodServer", "bytes_per_block_slot", "serve_sequential"]


def bytes_per_block_slot(doubleprecision: bool = False, track_hmax: bool = True) -> int:
    """Device bytes one block slot of a pool holds: state (two buffers of h, u, v),
    step scratch, bed and bed gradients with halos, friction, rain mask, boundary
    means, maximum depth and the block tables."""
    e = 8 if doubleprecision else 4
    cells = 256 * (6 + 3 + 1 + (1 if track_hmax else 0)) * e + 324 * 3 * e
    return cells + 256 + 64 * 4 + 128


@dataclass
class Request:
    rid: int
    arrival: float             # seconds after the start of the stream
    nblk: int
    build: object              # () -> (FlowB200, Loop)
    endtime: float = 1e30
    maxsteps: int = 2**31 - 1
    gauges: list = field(default_factory=list)  # (block index in active order, cell j*16+i)


@dataclass
class Result:
    rid: int
    arrival: float
    admitted: float
    finished: float
    nsteps: int
    totaltime: float
    h: np.ndarray | None = None
    hmax: np.ndarray | None = None
    gauge_series: list = field(default_factory=list)  # per step: (simulated time, [h at each gauge])
    status: int = 1            # as ScenarioPool.query: 1 finished, 2 dt underflow, 3 non-finite state

    @property
    def time_to_solution(self) -> float:
        return self.finished - self.arrival


class FloodServer:
    def __init__(self, param, hbm_budget_bytes: float, max_scenarios: int = 64, chunk_steps: int = 64,
                 track_hmax: bool = True, keep_fields: bool = True):
        per = bytes_per_block_slot(bool(param.doubleprecision), track_hmax)
        self.nblk_pool = max(1, int(hbm_budget_bytes // per))
        self.pool = ScenarioPool(param, self.nblk_pool, max_scenarios, track_hmax=track_hmax)
        self.chunk = int(chunk_steps)
        self.track_hmax = track_hmax
        self.keep_fields = keep_fields
        self.gpu_ms = 0.0
        self.host_s = {"admit": 0.0, "enqueue": 0.0, "run": 0.0, "query": 0.0, "retire": 0.0, "fields": 0.0}

    def serve(self, requests: list[Request], realtime: bool = True, prefetch: int = 16,
              builders: int = 4) -> list[Result]:
        """Runs the stream to completion.  With realtime, a request becomes visible at
        its arrival time on the wall clock; otherwise all are queued at t = 0.
        Arrived requests are prepared (host set-up and upload into their own handle)
        by `builders` background threads while the pool computes, at most `prefetch`
        ahead; they are admitted in the order they become ready.  Each chunk of pool
        steps is enqueued before the host retires the scenarios that finished in
        the previous chunk (their fields gathered on the pool's copy stream),
        admits ready requests (queued behind the chunk) and builds the next chunk's
        tables (their uploads also queued behind the chunk), so all of it overlaps
        the device work and the next chunk launches as soon as this one ends."""
        self.gpu_ms = 0.0
        self.host_s = {k: 0.0 for k in self.host_s}
        pending = sorted(requests, key=lambda r: r.arrival)
        ready: list[tuple[Request, object]] = []   # (request, (FlowB200, Loop))
        lock = threading.Condition()
        stop = [False]
        nexti = [0]
        errors: list = []
        t0 = time.perf_counter()
        now = lambda: time.perf_counter() - t0

        def builder():
            try:
                while True:
                    with lock:
                        while len(ready) >= prefetch and not stop[0]:
                            lock.wait(0.01)
                        if stop[0] or nexti[0] >= len(pending):
                            return
                        r = pending[nexti[0]]
                        nexti[0] += 1
                    if realtime and r.arrival > now():
                        time.sleep(r.arrival - now())
                    if r.nblk > self.nblk_pool:
                        raise ValueError(f"request {r.rid} needs {r.nblk} blocks, the pool holds {self.nblk_pool}")
                    built = r.build()
                    with lock:
                        ready.append((r, built))
                        lock.notify_all()
            except Exception as e:  # reported by the serving loop
                with lock:
                    errors.append(e)
                    lock.notify_all()

        # retired handles are released by a closer thread: their destruction (stream,
        # events, memory back to the pool) stays off the loop that feeds the device
        closeq: queue.Queue = queue.Queue()

        def closer():
            while True:
                f = closeq.get()
                if f is None:
                    return
                f.close()

        ths = [threading.Thread(target=builder, daemon=True) for _ in range(max(1, builders))]
        reaper = threading.Thread(target=closer, daemon=True)
        reaper.start()
        # the serving loop makes many short calls; a short interpreter switch interval
        # keeps the preparing threads from holding it off the GPU for milliseconds
        switch = sys.getswitchinterval()
        sys.setswitchinterval(min(switch, 0.0002))
        for th in ths:
            th.start()
        live: dict[int, tuple[Request, FlowB200, float, list]] = {}
        out: list[Result] = []
        finished: list[int] = []  # slots that finished in the last chunk, retired during the next one
        nreq = len(pending)

        def retire(slots):
            ta = time.perf_counter()
            res = self.pool.finish(slots, [live[s][0].nblk for s in slots], with_max=self.track_hmax)
            tb = time.perf_counter()
            self.host_s["fields"] += tb - ta
            for slot, (f, h, hmax, loop, n, status) in zip(slots, res):
                r, _, t_adm, series = live.pop(slot)
                closeq.put(f)
                out.append(Result(r.rid, r.arrival, t_adm, now(), n, loop.totaltime,
                                  h if self.keep_fields else None, hmax if self.keep_fields else None, series, status))
            self.host_s["retire"] += time.perf_counter() - tb

        def admit_ready():
            # arrival order while block and scenario slots allow; with a chunk in
            # flight the admission is queued behind it and joins the next chunk
            with lock:
                while ready:
                    r, (f, loop) = ready[0]
                    ta = time.perf_counter()
                    slot = self.pool.try_admit(f, loop, r.endtime, maxsteps=r.maxsteps)
                    self.host_s["admit"] += time.perf_counter() - ta
                    if slot is None:
                        break
                    ready.pop(0)
                    if r.gauges:
                        self.pool.set_gauges(slot, [(b, c % 16, c // 16) for b, c in r.gauges])
                    live[slot] = (r, f, now(), [])
                    lock.notify_all()
                if errors:
                    raise RuntimeError(f"request preparation failed: {errors[0]}") from errors[0]

        try:
            while len(out) < nreq:
                running = len(live) > len(finished)
                if running:
                    # the next chunk runs on the device while the host retires the
                    # scenarios that finished in the last one (their state is frozen)
                    # and admits the requests that became ready
                    # (enqueue: the table rebuild after admissions and retirements, then
                    # the chunk's graph launches; run: the wait for the chunk)
                    ta = time.perf_counter()
                    self.pool.run_async(self.chunk)
                    self.host_s["enqueue"] += time.perf_counter() - ta
                if finished:
                    retire(finished)
                    finished = []
                admit_ready()
                if running:
                    # the next chunk's tables, built while this chunk runs
                    ta = time.perf_counter()
                    self.pool.prepare()
                    self.host_s["enqueue"] += time.perf_counter() - ta
                if not running:
                    if not live and len(out) < nreq:
                        with lock:
                            if not any(th.is_alive() for th in ths) and not ready:
                                raise RuntimeError("request preparation stopped before the stream ended")
                            lock.wait(0.01)
                    continue
                ta = time.perf_counter()
                self.pool.wait()
                self.host_s["run"] += time.perf_counter() - ta
                self.gpu_ms += self.pool.timing()[0]
                for slot in list(live):
                    r, f, t_adm, series = live[slot]
                    ta = time.perf_counter()
                    loop, status, n = self.pool.query(slot)
                    self.host_s["query"] += time.perf_counter() - ta
                    if r.gauges:
                        t, v = self.pool.read_gauges(slot)
                        series.extend((float(tk), [float(x) for x in vk[:, 0]]) for tk, vk in zip(t[:, 0], v))
                    if status != 0:
                        finished.append(slot)
        finally:
            with lock:
                stop[0] = True
                lock.notify_all()
            for th in ths:
                th.join(timeout=10)
            closeq.put(None)
            reaper.join(timeout=60)
            sys.setswitchinterval(switch)
        return sorted(out, key=lambda x: x.rid)


def serve_sequential(requests: list[Request], realtime: bool = True) -> list[Result]:
    """The plain loop: one scenario at a time in arrival order, each run alone to
    completion with the device-resident loop (bgf_run)."""
    out = []
    t0 = time.perf_counter()
    now = lambda: time.perf_counter() - t0
    for r in sorted(requests, key=lambda r: r.arrival):
        if realtime and r.arrival > now():
            time.sleep(r.arrival - now())
        t_adm = now()
        f, loop = r.build()
        n = f.run(loop, endtime=r.endtime, maxsteps=r.maxsteps)
        zs, h, u, v = f.get_state()
        f.close()
        out.append(Result(r.rid, r.arrival, t_adm, now(), n, loop.totaltime, None, None))
    return out
