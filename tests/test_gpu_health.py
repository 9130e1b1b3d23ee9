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
    assert not err
    err, ms = fcc.barrier_selftest(4)  # the last block never arrives
    assert err and 0 < ms < 10_000
    b, box, kw = small(5)  # the device is still usable
    s = fcc.Simulation(b, box, T=np.float32, **kw)
    s.run(20)
    assert np.isfinite(s.bodies.x).all()
    assert s.health() == {"nonfinite": False, "barrier_error": False}
