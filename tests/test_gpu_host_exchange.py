"""The host side of the boundary on the GPU (marked ``gpu``): fcc_set_state
and fcc_get_state copy the caller's arrays as they are and convert on the
device.  Pinned (fcc_host_alloc) and ordinary arrays, and arrays that the
Python mirror has to re-lay out first (coef in C order), all give the same
bits; get_state(out=...) writes in place what sim.bodies returns."""

import numpy as np
import pytest

from conftest import fcc

pytestmark = pytest.mark.gpu

FIELDS = ("x", "y", "θ", "imgx", "imgy", "coef", "R0", "type", "parent")


def deformed(T):
    cells, box = fcc.hexagonal_monolayer(6, 6, packing=0.95, maxmode=6, rng=3)
    b = fcc.with_nuclei(cells, ratio=0.5)
    b.coef[1:] = 0.04 * np.random.default_rng(4).standard_normal((b.ncoef - 1, b.n))
    b.imgx[:] = np.arange(b.n) % 3 - 1
    kw = dict(types=(fcc.BodyType(v0=0.1, Dr=0.05), fcc.BodyType(drag="parent")),
              energies=(fcc.Tension(0.05), fcc.Overlap(1.0)), T=T, seed=8)
    return b, box, kw


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_pinned_and_pageable_exchange_give_the_same_bits(T):
    b, box, kw = deformed(T)
    sim = fcc.Simulation(b, box, **kw)
    sim.run(25)
    ref = sim.bodies
    out = fcc.pinned_bodies(b.n, b.ncoef)
    assert out.coef.flags.f_contiguous and fcc.abi.direct_host(out, writable=True) is not None
    sim.get_state(out=out)
    for f in FIELDS:
        assert np.array_equal(getattr(out, f), getattr(ref, f)), f
    # the same state loaded three ways continues identically
    c_order = ref.copy()
    c_order.coef = np.ascontiguousarray(ref.coef)  # not the ABI's layout: re-laid out by the mirror
    assert fcc.abi.direct_host(c_order) is None
    runs = []
    for src in (fcc.pinned_copy(ref), ref, c_order):
        s2 = fcc.Simulation(b, box, **kw)
        s2.set_state(src, clock=sim.clock)
        s2.run(15)
        runs.append(s2.bodies)
    sim.set_state(ref, clock=sim.clock)
    sim.run(15)
    last = sim.bodies
    for r in runs:
        for f in FIELDS:
            assert np.array_equal(getattr(r, f), getattr(last, f)), f


def test_get_state_rejects_buffers_of_another_layout():
    b, box, kw = deformed(np.float32)
    sim = fcc.Simulation(b, box, **kw)
    bad = fcc.pinned_bodies(b.n, b.ncoef)
    bad.coef = np.ascontiguousarray(bad.coef)
    with pytest.raises(fcc.ArgumentError):
        sim.get_state(out=bad)
    with pytest.raises(fcc.ArgumentError):
        sim.get_state(out=fcc.pinned_bodies(b.n + 1, b.ncoef))
