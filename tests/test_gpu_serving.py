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
