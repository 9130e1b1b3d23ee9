"""Serving: a request loop that keeps simulations resident in a ``Pool``.

Continuous batching for simulation requests (no counterpart in the
reference, whose callers run one ``Simulation`` per task): requests arrive
over time with their own bodies, parameters, seed and horizon; the loop
admits them, in arrival order, whenever the pool has a free slot and room for
their bodies and grid cells (the pool is sized from an HBM budget,
``Pool.for_budget``); all admitted simulations advance together in the packed
step kernel, chunk by chunk; a simulation that reaches its horizon is read
back (state and shape index) and retired at the end of that chunk, which
frees its room for the requests still waiting.  Each result equals the one of
the same request run alone with the same kernel variant, bit for bit.
A request can be cancelled (``Server.cancel``, from the result callback or
another thread): at the next chunk boundary it leaves the queue, or the pool
with its state so far, and is reported with ``cancelled = True``.
"""

from __future__ import annotations

import threading
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from .model import ArgumentError, Bodies, DeviceError, PeriodicBox
from .pool import grid_cells, padded


@dataclass
class Request:
    """One simulation request: ``Simulation(bodies, box; kw...)`` run for ``horizon`` steps."""
    bodies: Bodies
    box: PeriodicBox
    kw: dict
    horizon: int
    arrival: float = 0.0  # seconds after the stream starts
    id: int = 0

    @property
    def work(self) -> int:
        return self.bodies.n * self.horizon


@dataclass
class Result:
    id: int
    n: int
    horizon: int
    arrival: float
    admitted: float
    finished: float
    bodies: Bodies = field(repr=False)
    shape_index_mean: float = float("nan")
    cancelled: bool = False  # left before its horizon (bodies: the state it reached, or None if never admitted)
    steps: int = -1          # steps taken (the horizon unless cancelled)

    @property
    def latency(self) -> float:
        """Time to result: arrival to the result on the host."""
        return self.finished - self.arrival


class Server:
    """Continuous-batching loop over a pool.

    ``chunk`` caps the steps between two admission/retirement points; the loop
    shortens a chunk to the fewest steps any admitted simulation has left, so a
    finished simulation leaves (and frees its room) at once.  ``policy``:
    "fifo" admits in arrival order (a request that does not fit yet blocks the
    ones behind it); "sjf" admits the waiting requests with the least work
    (bodies × horizon) first and fills the room with any that fit (lower
    median time to result under overload; large requests wait longer);
    "evict" is "sjf" that also makes room for a waiting request by evicting
    the running one with the most work left, if that is at least
    ``evict_ratio`` times the waiting one's: the evicted request keeps its
    state and clock and is re-admitted later where it stopped (the pool's
    admission at a clock), so its result is still that of its solo run."""

    def __init__(self, pool, chunk=512, min_chunk=32, T=np.float32, clock=time.perf_counter, sleep=time.sleep,
                 policy="fifo", evict_ratio=4.0):
        if policy not in ("fifo", "sjf", "evict"):
            raise ArgumentError("policy must be 'fifo', 'sjf' or 'evict'")
        if not float(evict_ratio) > 1.0:  # a ratio above 1 rules out two requests evicting each other in turn
            raise ArgumentError("evict_ratio must be > 1")
        self.policy = policy
        self.evict_ratio = float(evict_ratio)
        self.evictions = 0
        self.pool = pool
        self.chunk = int(chunk)
        self.min_chunk = int(min_chunk)
        self.T = T
        self.clock = clock
        self.sleep = sleep
        self.chunks = 0
        self.device_ms = 0.0  # device time of the pool's runs (pools that report it)
        self._cancel = set()
        self._cancel_lock = threading.Lock()

    def cancel(self, request):
        """Withdraw a request: at the next chunk boundary it leaves the queue
        or the pool (safe to call from the result callback or another thread).
        ``request`` is the ``Request`` itself, or an id, which withdraws every
        request of the stream that carries that id (ids need not be unique)."""
        with self._cancel_lock:
            self._cancel.add(("obj", id(request)) if isinstance(request, Request) else ("id", int(request)))

    def _take_cancelled(self):
        with self._cancel_lock:
            ids, self._cancel = self._cancel, set()
        return ids

    def _fits_empty(self, r: Request) -> bool:
        u = self.pool.usage()
        cells = grid_cells(r.box, r.bodies.R0, r.kw.get("skin", 0.3), self.T)
        return padded(r.bodies.n) <= u["max_bodies"] and cells <= u["max_cells"]

    def serve(self, requests, on_result=None):
        """Run the stream; returns the results in completion order."""
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        for r in pending:
            if not self._fits_empty(r):
                raise ArgumentError(f"request {r.id} ({r.bodies.n} bodies) does not fit in an empty pool")
        waiting = deque()
        active = {}  # slot -> (request, first admitted)
        results = []
        resume = {}  # id(request) -> (state, clock, time) of an evicted request
        first = {}   # id(request) -> first admission time (keyed by object: ids need not be unique)
        t0 = self.clock()
        now = lambda: self.clock() - t0

        def left_of(q):  # body-steps a waiting request has left
            return q.bodies.n * (q.horizon - (resume[id(q)][1] if id(q) in resume else 0))

        steps_now = {}  # slot -> steps done, read once per admission pass (steps change only in runs)

        def admit(q):
            b, c, tq = resume.get(id(q), (q.bodies, 0, 0.0))
            if c:
                slot = self.pool.try_add(b, q.box, horizon=q.horizon, clock=c, t=tq, **q.kw)
            else:
                slot = self.pool.try_add(b, q.box, horizon=q.horizon, **q.kw)
            if slot is not None:
                steps_now[slot] = c
                resume.pop(id(q), None)
                first.setdefault(id(q), now())
                active[slot] = (q, first[id(q)])
            return slot

        while pending or waiting or active:
            marks = self._take_cancelled()
            if marks:
                hit = lambda q: ("obj", id(q)) in marks or ("id", q.id) in marks
                for q in [q for q in list(waiting) + list(pending) if hit(q)]:  # not running
                    b, c, _ = resume.pop(id(q), (None, 0, 0.0))
                    results.append(Result(q.id, q.bodies.n, q.horizon, q.arrival, first.get(id(q), float("nan")),
                                          now(), b, cancelled=True, steps=c))
                waiting = deque(q for q in waiting if not hit(q))
                pending = deque(q for q in pending if not hit(q))
                for s in [s for s, (r, _) in active.items() if hit(r)]:
                    r, adm = active.pop(s)
                    steps = self.pool.slot(s)[1]
                    b = self.pool.bodies(s)
                    self.pool.remove(s)
                    results.append(Result(r.id, r.bodies.n, r.horizon, r.arrival, adm, now(), b, cancelled=True,
                                          steps=steps))
            t = now()
            while pending and pending[0].arrival <= t:
                waiting.append(pending.popleft())
            if self.policy == "fifo":
                while waiting:  # admission in arrival order, as slots and memory free up
                    if admit(waiting[0]) is None:
                        break
                    waiting.popleft()
            else:  # least work left first; every waiting request that fits is admitted
                admitted, evicted = set(), []
                if self.policy == "evict" and waiting:
                    steps_now.clear()
                    steps_now.update((s, self.pool.slot(s)[1]) for s in active)
                for r in sorted(waiting, key=lambda q: (left_of(q), q.arrival)):
                    slot = admit(r)
                    while slot is None and self.policy == "evict" and active:
                        work_left = {s: v.bodies.n * (v.horizon - steps_now[s]) for s, (v, _) in active.items()}
                        s = max(work_left, key=work_left.get)
                        if work_left[s] < self.evict_ratio * left_of(r):
                            break
                        v, _ = active.pop(s)
                        b, _, tv, _ = self.pool.state(s)
                        resume[id(v)] = (b, steps_now.pop(s), tv)
                        self.pool.remove(s)
                        self.evictions += 1
                        evicted.append(v)
                        slot = admit(r)
                    if slot is not None:
                        admitted.add(id(r))
                if admitted:
                    waiting = deque(q for q in waiting if id(q) not in admitted)
                waiting.extend(evicted)
            if not active:
                if pending:
                    self.sleep(max(0.0, pending[0].arrival - now()))
                continue
            before = {s: self.pool.slot(s)[1] for s in active}
            left = min(r.horizon - before[s] for s, (r, _) in active.items())
            self.pool.run(max(min(self.chunk, left), min(self.min_chunk, self.chunk)))
            self.chunks += 1
            if all(self.pool.slot(s)[1] == before[s] and not self.pool.done(s) for s in active):
                raise DeviceError("serving: a pool round advanced no simulation and none is done")
            timing = getattr(self.pool, "last_timing", None)
            if timing is not None:
                self.device_ms += timing()[0]
            for s in [s for s in active if self.pool.done(s)]:
                r, adm = active.pop(s)
                b = self.pool.bodies(s)
                si = self.pool.shape_index(s)
                self.pool.remove(s)
                res = Result(r.id, r.bodies.n, r.horizon, r.arrival, adm, now(), b,
                             float(np.mean(si)) if len(si) else float("nan"), steps=r.horizon)
                results.append(res)
                if on_result:
                    on_result(res)
        return results


def summary(results, makespan=None):
    """p50/p99 time to result and body-steps/s of a served stream (completed
    requests; cancelled ones are counted apart, with the steps they took)."""
    done = [r for r in results if not r.cancelled]
    lat = np.array([r.latency for r in done]) if done else np.array([float("nan")])
    work = sum(r.n * r.horizon for r in done) + sum(r.n * max(r.steps, 0) for r in results if r.cancelled)
    span = makespan if makespan is not None else max(r.finished for r in results) - min(r.arrival for r in results)
    return {"requests": len(done), "cancelled": len(results) - len(done), "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "mean_s": float(lat.mean()), "body_steps": int(work),
            "makespan_s": float(span), "body_steps_per_s": work / span if span > 0 else float("nan")}


def sequential_latencies(arrivals, durations):
    """Times to result of a loop that runs requests one at a time in arrival
    order (start = max(arrival, previous finish))."""
    t, out = 0.0, []
    for a, d in zip(arrivals, durations):
        t = max(t, a) + d
        out.append(t - a)
    return np.array(out)
