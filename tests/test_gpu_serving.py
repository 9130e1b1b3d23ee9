"""Serving on the GPU (marked ``gpu``): a stream of requests of uneven N,
parameters and horizons through the continuous-batching loop on a pool too
small to hold them all at once.  Every result must equal the same request
run alone (tolerance: bitwise equality of the final state), and requests
must have shared the device (admitted while others were running)."""

import numpy as np
import pytest

from conftest import fcc

pytestmark = pytest.mark.gpu


def stream(count=10, seed=5):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        nx, ny = int(rng.integers(3, 10)), 2 * int(rng.integers(2, 5))
        b, box = fcc.polydisperse_monolayer(nx, ny, packing=0.95, maxmode=10, seed=100 + i)
        kw = dict(types=(fcc.BodyType(v0=float(rng.uniform(0.02, 0.2)), Dr=float(rng.uniform(0.005, 0.05)), μab=0.1),),
                  energies=(fcc.Tension(float(rng.uniform(0.001, 0.1))), fcc.Overlap(1.0)), dt=0.005, seed=100 + i)
        reqs.append(fcc.Request(b, box, kw, int(rng.integers(50, 400)), 0.0 if i < 6 else 0.002 * i, i))
    return reqs


def test_served_results_equal_alone_and_overlap():
    reqs = stream()
    pool = fcc.Pool(T=np.float32, max_bodies=160, max_cells=4096, max_sims=3)
    srv = fcc.Server(pool, chunk=64)
    res = srv.serve(reqs)
    assert sorted(r.id for r in res) == list(range(len(reqs)))
    # continuous batching: some request was admitted while another was running
    assert any(a.admitted < b.admitted < a.finished for a in res for b in res if a is not b)
    # and some request had to wait for room
    assert any(r.admitted > r.arrival + 1e-3 for r in res)
    for r in res:
        q = reqs[r.id]
        sim = fcc.Simulation(q.bodies, q.box, T=np.float32, **q.kw)
        sim.run(q.horizon)
        a = sim.bodies
        for f in ("x", "y", "θ", "coef", "imgx", "imgy"):
            assert np.array_equal(getattr(a, f), getattr(r.bodies, f)), (r.id, f)
        assert r.shape_index_mean == pytest.approx(float(np.mean(sim.shape_index())), rel=0, abs=0)
    assert pool.usage()["sims"] == 0


def test_evicted_requests_resume_exactly():
    """With the "evict" policy a short request that does not fit evicts the
    long one running; the long one is re-admitted at the clock it reached and
    its result still equals its solo run, bit for bit, time included."""
    rng = np.random.default_rng(9)
    reqs = []
    for i, (nx, ny, horizon, arrival) in enumerate([(10, 8, 900, 0.0), (9, 6, 120, 0.05), (5, 4, 80, 0.1)]):
        b, box = fcc.polydisperse_monolayer(nx, ny, packing=0.95, maxmode=10, seed=300 + i)
        kw = dict(types=(fcc.BodyType(v0=float(rng.uniform(0.05, 0.2)), Dr=0.02, μab=0.1),),
                  energies=(fcc.Tension(0.01), fcc.Overlap(1.0)), dt=0.005, seed=300 + i)
        reqs.append(fcc.Request(b, box, kw, horizon, arrival, i))
    pool = fcc.Pool(T=np.float32, max_bodies=128, max_cells=4096, max_sims=3)
    # virtual time: 10 ms per chunk of 64 steps, so r1 arrives while r0 runs
    t = {"idle": 0.0}
    srv = fcc.Server(pool, chunk=64, policy="evict", clock=lambda: t["idle"] + 0.01 * srv.chunks,
                     sleep=lambda dt: t.__setitem__("idle", t["idle"] + max(dt, 0.0)))
    res = {r.id: r for r in srv.serve(reqs)}
    assert srv.evictions >= 1
    assert sorted(res) == [0, 1, 2] and not any(r.cancelled for r in res.values())
    for q in reqs:
        sim = fcc.Simulation(q.bodies, q.box, T=np.float32, **q.kw)
        sim.run(q.horizon)
        a = sim.bodies
        for f in ("x", "y", "θ", "coef", "imgx", "imgy"):
            assert np.array_equal(getattr(a, f), getattr(res[q.id].bodies, f)), (q.id, f)
    assert pool.usage()["sims"] == 0


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_pool_resume_after_a_dt_change_keeps_state_and_time(T):
    """A simulation whose dt changed before its checkpoint, re-admitted to a
    pool at its clock with its time, continues bit for bit: state, clock and
    time equal those of the uninterrupted simulation (the time is carried,
    not recomputed as clock * dt, which would be off after the change)."""
    b, box = fcc.polydisperse_monolayer(6, 6, packing=0.95, maxmode=10, seed=41)
    kw = dict(types=(fcc.BodyType(v0=0.1, Dr=0.02, μab=0.1),), energies=(fcc.Tension(0.02), fcc.Overlap(1.0)),
              seed=41)
    a = fcc.Simulation(b, box, T=T, dt=0.005, **kw)
    a.run(60)
    a.dt = 0.004
    a.run(40)
    ckpt, clock, t_ckpt = a.bodies, a.clock, a.t
    assert clock == 100 and abs(t_ckpt - 100 * 0.004) > 1e-3  # clock * dt would be wrong here
    pool = fcc.Pool(T=T, max_bodies=64, max_cells=1024, max_sims=2)
    s = pool.add(ckpt, box, dt=0.004, horizon=180, clock=clock, t=t_ckpt, **kw)
    pool.run(1000)
    got, c2, t2, steps = pool.state(s)
    a.run(80)
    ref = a.bodies
    for f in ("x", "y", "θ", "coef", "imgx", "imgy"):
        assert np.array_equal(getattr(ref, f), getattr(got, f)), f
    assert c2 == a.clock == 180 and steps == 180
    assert t2 == a.t
