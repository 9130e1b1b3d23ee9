"""Host logic of the serving loop (continuous batching) on CPU, with a fake
pool and a fake clock: admission in arrival order as slots and memory free
up, admission while other requests are running, retirement at the end of
the chunk a request finishes in, rejection of requests that never fit, and
the p50/p99 statistics.  The GPU pool itself is covered by test_gpu_pool.py
and test_gpu_serving.py."""

import numpy as np
import pytest

from conftest import fcc

serving = fcc.serving


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(0.0, dt)


class FakePool:
    """The Pool interface the server uses; a step of all admitted bodies
    costs bodies / rate seconds of the fake clock."""

    def __init__(self, clock, max_bodies=256, max_cells=10_000, max_sims=4, rate=1e6):
        self.clock, self.rate = clock, rate
        self.cap = dict(max_bodies=max_bodies, max_cells=max_cells, max_sims=max_sims)
        self.sims, self.next, self.log = {}, 0, []

    def usage(self):
        return dict(bodies=sum(serving.padded(s["n"]) for s in self.sims.values()),
                    cells=sum(s["cells"] for s in self.sims.values()), sims=len(self.sims), **self.cap)

    def try_add(self, bodies, box, horizon, clock=0, **kw):
        u = self.usage()
        cells = serving.grid_cells(box, bodies.R0, kw.get("skin", 0.3), np.float32)
        if (u["sims"] >= u["max_sims"] or u["bodies"] + serving.padded(bodies.n) > u["max_bodies"]
                or u["cells"] + cells > u["max_cells"]):
            return None
        slot = min(set(range(self.cap["max_sims"])) - set(self.sims))
        self.sims[slot] = dict(n=bodies.n, cells=cells, horizon=horizon, steps=clock, seed=kw["seed"], bodies=bodies)
        self.log.append(("add", kw["seed"], self.clock.t))
        return slot

    def run(self, n):
        self.log.append(("run", n, sorted(s["seed"] for s in self.sims.values())))
        busy = sum(s["n"] for s in self.sims.values() if s["steps"] < s["horizon"])
        for s in self.sims.values():
            s["steps"] += min(n, s["horizon"] - s["steps"])
        self.clock.t += n * busy / self.rate

    def slot(self, s):
        x = self.sims[s]
        return True, x["steps"], x["horizon"]

    def done(self, s):
        x = self.sims[s]
        return x["steps"] >= x["horizon"]

    def bodies(self, s):
        return self.sims[s]["bodies"]

    def state(self, s):
        x = self.sims[s]
        return x["bodies"], x["steps"], 0.005 * x["steps"], x["steps"]

    def shape_index(self, s):
        return np.full(self.sims[s]["n"], 3.6)

    def remove(self, s):
        self.log.append(("remove", self.sims[s]["seed"], self.clock.t))
        del self.sims[s]


def req(i, nx, ny, horizon, arrival):
    b, box = fcc.hexagonal_monolayer(nx, ny, packing=0.95, maxmode=10, rng=i)
    return fcc.Request(b, box, dict(types=(fcc.BodyType(),), energies=(fcc.Tension(0.01),), seed=i), horizon,
                       arrival, i)


def test_continuous_batching_admits_while_others_run():
    clk = FakeClock()
    pool = FakePool(clk, max_bodies=160, max_sims=4)
    # r0: 96 bodies, long; r1: 48 bodies, short; r2 arrives while both run and
    # fits only once r1 has left; r3 arrives later and fits beside r0 and r2
    reqs = [req(0, 8, 12, 5000, 0.0), req(1, 8, 6, 300, 0.0), req(2, 8, 6, 400, 0.01), req(3, 2, 4, 200, 0.4)]
    srv = fcc.Server(pool, chunk=256, min_chunk=1, clock=clk, sleep=clk.sleep)
    res = srv.serve(reqs)
    order = [r.id for r in res]
    assert order.index(1) < order.index(2) < order.index(0)
    adds = [e for e in pool.log if e[0] == "add"]
    rem1 = next(e for e in pool.log if e[0] == "remove" and e[1] == 1)
    add2 = next(e for e in adds if e[1] == 2)
    assert add2[2] == rem1[2]            # r2 enters at the boundary r1 leaves
    runs_with_0_and_2 = [e for e in pool.log if e[0] == "run" and 0 in e[2] and 2 in e[2]]
    assert runs_with_0_and_2             # and shares the device with r0 (continuous batching)
    # the chunk is cut to the fewest remaining steps: r1 leaves after exactly 300 steps
    first_runs = [e[1] for e in pool.log if e[0] == "run"][:2]
    assert first_runs == [256, 44]
    assert all(r.latency >= 0 and r.admitted >= r.arrival for r in res)


def test_fifo_admission_without_overtaking():
    clk = FakeClock()
    pool = FakePool(clk, max_bodies=128, max_sims=8)
    reqs = [req(0, 8, 12, 1000, 0.0), req(1, 8, 8, 100, 0.01), req(2, 2, 2, 100, 0.02)]
    fcc.Server(pool, chunk=128, clock=clk, sleep=clk.sleep).serve(reqs)
    adds = [e[1] for e in pool.log if e[0] == "add"]
    assert adds == [0, 1, 2]  # r2 would fit beside r0 but waits behind r1


def test_idle_server_sleeps_until_arrival_and_rejects_oversized():
    clk = FakeClock()
    pool = FakePool(clk, max_bodies=64, max_sims=2)
    res = fcc.Server(pool, clock=clk, sleep=clk.sleep).serve([req(0, 4, 4, 10, 5.0)])
    assert res[0].admitted >= 5.0 and res[0].arrival == 5.0
    with pytest.raises(fcc.ArgumentError):
        fcc.Server(FakePool(FakeClock(), max_bodies=64), clock=clk, sleep=clk.sleep).serve([req(1, 10, 10, 10, 0)])


def test_summary_and_sequential_latencies():
    rs = [serving.Result(i, 10, 100, 0.1 * i, 0.1 * i, 0.1 * i + 1.0 + (i == 9) * 9, None) for i in range(10)]
    s = serving.summary(rs)
    assert s["requests"] == 10 and s["p50_s"] == pytest.approx(1.0) and s["p99_s"] > 9
    assert s["body_steps"] == 10_000
    lat = serving.sequential_latencies([0.0, 0.0, 5.0], [1.0, 2.0, 1.0])
    assert np.allclose(lat, [1.0, 3.0, 1.0])


def test_sjf_admits_small_work_first_and_backfills():
    clk = FakeClock()
    pool = FakePool(clk, max_bodies=128, max_sims=8)
    # all waiting at t = 0: r0 is big, r1 small, r2 medium; r0 does not fit
    # beside r2 + r1, so sjf runs r1 and r2 first and r0 after they leave
    reqs = [req(0, 8, 12, 1000, 0.0), req(1, 2, 2, 100, 0.0), req(2, 4, 4, 300, 0.0)]
    res = fcc.Server(pool, chunk=128, clock=clk, sleep=clk.sleep, policy="sjf").serve(reqs)
    adds = [e[1] for e in pool.log if e[0] == "add"]
    assert adds[:2] == [1, 2] and adds[2] == 0
    assert [r.id for r in res][-1] == 0
    with pytest.raises(fcc.ArgumentError):
        fcc.Server(pool, policy="lifo")


def test_cancelled_requests_leave_the_queue_and_the_pool():
    """A request cancelled while it runs leaves the pool with the state it
    reached; one cancelled while it waits never runs; the others are
    unaffected (a cancelled request is a fault injected on the host)."""
    clk = FakeClock()
    pool = FakePool(clk, max_bodies=160, max_sims=4)
    # r0 long and running, r1 short and running, r2 waits for room
    reqs = [req(0, 8, 12, 5000, 0.0), req(1, 8, 6, 300, 0.0), req(2, 8, 12, 400, 0.01), req(3, 2, 4, 200, 0.02)]
    srv = fcc.Server(pool, chunk=256, min_chunk=1, clock=clk, sleep=clk.sleep)

    def on_result(res):
        if res.id == 1:  # when r1 finishes: cancel r0 (running) and r2 (still waiting)
            srv.cancel(0)
            srv.cancel(2)

    res = {r.id: r for r in srv.serve(reqs, on_result=on_result)}
    assert set(res) == {0, 1, 2, 3}
    assert res[0].cancelled and 0 < res[0].steps < 5000 and res[0].bodies is not None
    assert res[2].cancelled and res[2].steps == 0 and res[2].bodies is None
    assert not res[1].cancelled and res[1].steps == 300
    assert not res[3].cancelled and res[3].steps == 200
    assert not any(e[0] == "add" and e[1] == 2 for e in pool.log)  # r2 never entered the pool
    assert ("remove", 0) in [(e[0], e[1]) for e in pool.log]
    assert pool.usage()["sims"] == 0
    s = serving.summary(list(res.values()))
    assert s["requests"] == 2 and s["cancelled"] == 2


def test_evict_policy_makes_room_and_resumes_where_it_stopped():
    """A short request that does not fit evicts the running request with the
    most work left; the evicted one is re-admitted at the clock it reached
    (its state saved) and still ends at its horizon."""
    clk = FakeClock()
    pool = FakePool(clk, max_bodies=128, max_sims=8)
    # r0 (96 bodies, long) runs alone; r1 (64 bodies, short) arrives and does not fit beside it
    reqs = [req(0, 8, 12, 4000, 0.0), req(1, 8, 8, 200, 0.001)]
    srv = fcc.Server(pool, chunk=128, min_chunk=1, clock=clk, sleep=clk.sleep, policy="evict")
    res = {r.id: r for r in srv.serve(reqs)}
    assert srv.evictions >= 1
    adds = [e for e in pool.log if e[0] == "add"]
    assert [e[1] for e in adds][:3] == [0, 1, 0]        # r0, r1 in r0's place, r0 again
    assert res[1].finished < res[0].finished
    assert not res[0].cancelled and res[0].steps == 4000
    with pytest.raises(fcc.ArgumentError):
        fcc.Server(pool, policy="lru")
    with pytest.raises(fcc.ArgumentError):
        fcc.Server(pool, policy="evict", evict_ratio=1.0)


def test_a_round_without_progress_raises_instead_of_looping():
    """A pool whose step counts stop moving short of the horizon (a slot
    held by mistake) makes the loop raise DeviceError instead of spinning."""
    clk = FakeClock()

    class StuckPool(FakePool):
        def run(self, n):
            self.clock.t += 1e-3

    pool = StuckPool(clk)
    srv = fcc.Server(pool, chunk=64, min_chunk=1, clock=clk, sleep=clk.sleep)
    with pytest.raises(fcc.DeviceError):
        srv.serve([req(0, 4, 4, 100, 0.0)])
    assert srv.chunks == 1


def test_evict_stream_neither_loses_nor_repeats_steps():
    """A random overloaded stream under "evict": every request ends at its
    horizon and the pool advanced each one by exactly its horizon in total
    (an evicted request resumes where it stopped; no step is run twice)."""
    clk = FakeClock()

    class CountingPool(FakePool):
        advanced = {}

        def run(self, n):
            for s in self.sims.values():
                self.advanced[s["seed"]] = self.advanced.get(s["seed"], 0) + min(n, s["horizon"] - s["steps"])
            super().run(n)

    rng = np.random.default_rng(3)
    reqs = [req(i, int(rng.integers(2, 9)), 2 * int(rng.integers(1, 5)), int(rng.integers(20, 3000)),
                float(rng.uniform(0.0, 0.05))) for i in range(24)]
    pool = CountingPool(clk, max_bodies=160, max_sims=3)
    srv = fcc.Server(pool, chunk=64, min_chunk=1, clock=clk, sleep=clk.sleep, policy="evict")
    res = srv.serve(reqs)
    assert srv.evictions >= 1
    assert sorted(r.id for r in res) == list(range(len(reqs)))
    assert all(not r.cancelled and r.steps == r.horizon for r in res)
    for q in reqs:
        assert pool.advanced[q.kw["seed"]] == q.horizon, q.id


def test_cancelling_an_evicted_request_reports_the_state_it_reached():
    """An evicted request cancelled while it waits to be re-admitted is
    reported with the state and clock it had reached, not as never run."""
    clk = FakeClock()
    pool = FakePool(clk, max_bodies=128, max_sims=8)
    reqs = [req(0, 8, 12, 4000, 0.0), req(1, 8, 8, 200, 0.001)]
    srv = fcc.Server(pool, chunk=128, min_chunk=1, clock=clk, sleep=clk.sleep, policy="evict")
    res = {r.id: r for r in srv.serve(reqs, on_result=lambda r: srv.cancel(0) if r.id == 1 else None)}
    assert srv.evictions == 1
    assert not res[1].cancelled and res[1].steps == 200
    assert res[0].cancelled and 0 < res[0].steps < 4000 and res[0].bodies is not None
    assert res[0].admitted == 0.0
    assert [e[1] for e in pool.log if e[0] == "add"] == [0, 1]  # never re-admitted


def test_requests_without_distinct_ids_keep_their_own_admission_times():
    """Request ids default to 0; the loop's bookkeeping is per request, so
    a stream that leaves them all at 0 still gets each admission time right."""
    clk = FakeClock()
    pool = FakePool(clk, max_bodies=256, max_sims=1)
    reqs = [fcc.Request(q.bodies, q.box, q.kw, q.horizon, q.arrival) for q in
            (req(0, 4, 4, 100, 0.0), req(1, 4, 4, 100, 0.0), req(2, 4, 4, 100, 0.0))]
    res = fcc.Server(pool, chunk=64, min_chunk=1, clock=clk, sleep=clk.sleep, policy="sjf").serve(reqs)
    adm = sorted(r.admitted for r in res)
    assert len(res) == 3 and adm[0] < adm[1] < adm[2]
    assert all(r.admitted < r.finished for r in res)


def test_cancel_by_request_object_leaves_equal_ids_alone():
    """Requests that share an id (the default 0) are cancelled one by one by
    passing the Request itself; cancelling by id withdraws all that carry it."""
    clk = FakeClock()
    pool = FakePool(clk, max_bodies=256, max_sims=1)
    reqs = [fcc.Request(q.bodies, q.box, q.kw, q.horizon, q.arrival) for q in
            (req(0, 4, 4, 100, 0.0), req(1, 4, 4, 100, 0.0), req(2, 4, 4, 100, 0.0))]
    srv = fcc.Server(pool, chunk=64, min_chunk=1, clock=clk, sleep=clk.sleep)
    srv.cancel(reqs[1])  # still waiting when the loop starts: never admitted
    res = srv.serve(reqs)
    by_seed = {r.bodies is None: r for r in res}
    assert len(res) == 3 and sum(r.cancelled for r in res) == 1
    assert by_seed[True].cancelled and by_seed[True].steps == 0
    assert sum(1 for e in pool.log if e[0] == "add") == 2
    srv = fcc.Server(fcc_pool := FakePool(clk, max_bodies=256, max_sims=1), chunk=64, min_chunk=1, clock=clk,
                     sleep=clk.sleep)
    srv.cancel(0)
    res = srv.serve(reqs)
    assert len(res) == 3 and all(r.cancelled for r in res)
    assert not any(e[0] == "add" for e in fcc_pool.log)


def test_evicted_request_resumes_with_its_own_time():
    """Eviction saves the state, clock and time the pool reports and
    re-admits with all three (a resumed time is not recomputed as clock * dt)."""
    clk = FakeClock()
    pool = FakePool(clk, max_bodies=128, max_sims=8)
    seen = []
    orig = pool.try_add

    def try_add(bodies, box, horizon, clock=0, **kw):
        seen.append((clock, kw.get("t")))
        return orig(bodies, box, horizon, clock=clock, **kw)

    pool.try_add = try_add
    reqs = [req(0, 8, 12, 4000, 0.0), req(1, 8, 8, 200, 0.001)]
    fcc.Server(pool, chunk=128, min_chunk=1, clock=clk, sleep=clk.sleep, policy="evict").serve(reqs)
    resumed = [(c, t) for c, t in seen if c]
    assert resumed and all(t == pytest.approx(0.005 * c) for c, t in resumed)
