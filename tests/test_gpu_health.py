"""Failure detection on the GPU without a GPU fault (marked ``gpu``).

Faults are made on the host: a non-finite shape coefficient written with
set_state (the reference has no NaN detection; the library flags the state),
and a grid barrier one of whose blocks never arrives (the self-test kernel),
whose wait runs out after a fixed number of polls and reports an error status
instead of hanging; the device stays usable afterwards.  No test traps,
faults or hangs a GPU."""

import numpy as np
import pytest

from conftest import fcc

pytestmark = pytest.mark.gpu


def small(seed=3):
    b, box = fcc.polydisperse_monolayer(8, 8, packing=0.95, maxmode=10, seed=seed)
    kw = dict(types=(fcc.BodyType(v0=0.1, Dr=0.01, μab=0.1),), energies=(fcc.Tension(0.01), fcc.Overlap(1.0)),
              dt=0.005, seed=seed)
    return b, box, kw


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_nonfinite_state_is_flagged_and_cleared_by_set_state(T):
    b, box, kw = small()
    s = fcc.Simulation(b, box, T=T, **kw)
    s.run(5)
    assert s.health() == {"nonfinite": False, "barrier_error": False}
    bad = s.bodies
    bad.coef[3, 7] = np.nan  # one mode amplitude of body 8
    s.set_state(bad)
    s.run(2)
    assert s.health() == {"nonfinite": True, "barrier_error": False}
    assert np.isnan(s.bodies.x[7])
    assert np.isfinite(np.delete(s.bodies.x, 7)).all()  # the others keep stepping: no contact with a NaN contour
    s.set_state(b)  # a finite state clears the flag
    s.run(3)
    assert s.health() == {"nonfinite": False, "barrier_error": False}


def test_barrier_wait_runs_out_with_an_error_status():
    err, ms = fcc.barrier_selftest(1)  # one block waits for no one
    assert err == 0
    err, ms = fcc.barrier_selftest(4)  # the last block never arrives: both kinds of wait run out
    assert err == 1 and 0 < ms < 10_000
    b, box, kw = small(5)  # the device is still usable
    s = fcc.Simulation(b, box, T=np.float32, **kw)
    s.run(20)
    assert np.isfinite(s.bodies.x).all()
    assert s.health() == {"nonfinite": False, "barrier_error": False}


def test_state_outside_the_box_matches_the_oracle():
    """Positions written from the host outside [0, L) (a host-injected fault:
    the reference would index its cell grid out of bounds) are clamped into
    the grid for the cell list and wrapped by the first update, with image
    counters; FP64 against the oracle after 30 steps (rtol 1e-8)."""
    from conftest import oracle
    b, box, kw = small(9)
    bad = b.copy()
    bad.x[:5] += box.Lx
    bad.y[5:10] -= 2 * box.Ly
    g = fcc.Simulation(bad, box, T=np.float64, **kw)
    g.run(30)
    o = oracle.OracleSimulation(bad, box, T=np.float64, **kw)
    o.step(30)
    a, c = g.bodies, o.bodies
    assert np.allclose(a.x, c.x, rtol=1e-8) and np.allclose(a.y, c.y, rtol=1e-8)
    assert np.allclose(a.coef, c.coef, rtol=1e-8, atol=1e-12)
    assert np.array_equal(a.imgx, c.imgx) and np.array_equal(a.imgy, c.imgy)
    assert (a.x >= 0).all() and (a.x < box.Lx).all() and (a.y >= 0).all() and (a.y < box.Ly).all()
    assert g.health() == {"nonfinite": False, "barrier_error": False}


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_checkpoint_and_resume_continue_the_trajectory(T):
    """Checkpoint = the body state and the clock (the Philox draw index);
    resume = a new simulation given both with set_state.  The resumed run
    takes the same steps as the uninterrupted one, bit for bit (Overlap
    pressures are sums of J = 1, so the rebuilt lists' neighbour order does
    not enter the results)."""
    b, box, kw = small(11)
    a = fcc.Simulation(b, box, T=T, **kw)
    a.run(150)
    state, clock = a.bodies, a.clock
    a.run(150)
    r = fcc.Simulation(state, box, T=T, **kw)
    r.set_state(state, clock=clock)
    r.run(150)
    x, y = a.bodies, r.bodies
    assert r.clock == a.clock
    for f in ("x", "y", "θ", "coef", "imgx", "imgy"):
        assert np.array_equal(getattr(x, f), getattr(y, f)), f
