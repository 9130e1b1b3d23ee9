"""The packed multi-simulation engine (``Pool``) against simulations run alone
and against the oracle (marked ``gpu``).

The property a pool promises: a simulation packed with others, admitted and
retired around it, produces the trajectory it produces alone with the same
kernel variant, bit for bit (tolerance: equality of every state array, the
clock, t and the rebuild count).  FP64 pools are also checked against the
CPU oracle (30 noisy steps, rtol 1e-8, test/test_cuda.jl:123-131).
"""

import numpy as np
import pytest

from conftest import fcc, oracle

pytestmark = pytest.mark.gpu


def monolayer(nx, ny, seed, v0=0.06, eta=0.01, perimeter=False, T=np.float32, fast=False):
    """A small polydisperse monolayer with its own parameters (a batch member)."""
    bodies, box = fcc.polydisperse_monolayer(nx, ny, packing=0.95, maxmode=10, seed=seed)
    rng = np.random.default_rng(seed + 100)
    bodies.coef[1:] = 0.03 * (2 * rng.random((bodies.ncoef - 1, bodies.n)) - 1)
    energies = [fcc.Tension(eta), fcc.Overlap(1.0)]
    if perimeter:
        energies.append(fcc.PerimeterElasticity(0.1, 3.7))
    kw = dict(types=(fcc.BodyType(v0=2.0 if fast else v0, Dr=0.01, μab=0.1),), energies=tuple(energies), dt=0.005,
              seed=seed, skin=0.05 if fast else 0.3)
    return bodies, box, kw


MEMBERS = [(5, 6, 11, 0.06, 0.01, False), (7, 4, 12, 0.2, 0.001, True), (9, 8, 13, 0.02, 0.1, False),
           (11, 6, 14, 0.1, 0.03, True)]


def members(T, fast=False):
    return [monolayer(nx, ny, seed, v0, eta, per, T, fast) for nx, ny, seed, v0, eta, per in MEMBERS]


def alone(bodies, box, kw, T, steps, **extra):
    s = fcc.Simulation(bodies, box, T=T, **kw, **extra)
    s.run(steps)
    return s


def assert_same(pool, slot, sim):
    b, clk, t, steps = pool.state(slot)
    a = sim.bodies
    for f in ("x", "y", "θ", "coef", "imgx", "imgy"):
        assert np.array_equal(getattr(b, f), getattr(a, f)), f
    assert clk == sim.clock and steps == sim.nsteps and t == sim.t
    assert pool.builds(slot) == sim.builds


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_pool_equals_alone_bitwise(T):
    ms = members(T, fast=True)
    pool = fcc.Pool(T=T, max_bodies=4096, max_cells=4096, max_sims=8)
    slots = [pool.add(b, box, horizon=300, **kw) for b, box, kw in ms]
    pool.run(300)
    for s, (b, box, kw) in zip(slots, ms):
        ref = alone(b, box, kw, T, 300)
        assert ref.builds > 5
        assert_same(pool, s, ref)
    # the members differ from each other (independent streams and parameters)
    assert not np.array_equal(pool.bodies(slots[0]).x[:10], pool.bodies(slots[1]).x[:10])


def test_long_lone_run_equals_pool_bitwise():
    """A lone FP32 simulation of 10000 bodies over 20000 steps (40 launches of
    512 steps, warps taking groups dynamically) repeats bit for bit and equals
    its pool run: the block-local noise clock every warp reads is ticked
    before the step's closing block barrier."""
    bodies, box, kw = monolayer(100, 100, 21, v0=0.1, eta=0.01, perimeter=True)
    steps = 20000
    first, second = alone(bodies, box, kw, np.float32, steps), alone(bodies, box, kw, np.float32, steps)
    pool = fcc.Pool(T=np.float32, max_bodies=16384, max_cells=16384, max_sims=2)
    slot = pool.add(bodies, box, horizon=steps, **kw)
    pool.run(steps)
    for f in ("x", "y", "θ", "coef", "imgx", "imgy"):
        assert np.array_equal(getattr(first.bodies, f), getattr(second.bodies, f)), f
    assert_same(pool, slot, first)


@pytest.mark.parametrize("variant", [0, 3])
def test_pool_with_many_slots_takes_the_full_scan_rebuild(variant, monkeypatch):
    """A rebuild visits the bodies and cells of the rebuilding simulations
    through a work list in shared memory; with more slots than that list can
    hold (4000 here) every phase scans the whole arena instead.  Both give
    the trajectory of the simulation alone with the same launch variant, bit
    for bit."""
    ms = members(np.float32, fast=True)
    pool = fcc.Pool(T=np.float32, max_bodies=4096, max_cells=4096, max_sims=4000)
    pool.config(variant=variant)
    slots = [pool.add(b, box, horizon=200, **kw) for b, box, kw in ms]
    pool.run(200)
    assert pool.variant()["variant"] == variant
    monkeypatch.setenv("FCC_VARIANT", str(variant))
    for s, (b, box, kw) in zip(slots, ms):
        ref = alone(b, box, kw, np.float32, 200)
        assert ref.builds > 3
        assert_same(pool, s, ref)


def test_pool_admission_retirement_and_horizons():
    """Retire one simulation mid-run, admit another while the rest keep their
    state; every simulation stops at its own horizon."""
    T = np.float32
    ms = members(T, fast=True)
    pool = fcc.Pool(T=T, max_bodies=4096, max_cells=4096, max_sims=8)
    hz = [400, 57, 400, 173]
    slots = [pool.add(b, box, horizon=h, **kw) for (b, box, kw), h in zip(ms, hz)]
    pool.run(150)
    assert [pool.slot(s)[1] for s in slots] == [150, 57, 150, 150]
    pool.remove(slots[1])
    extra = monolayer(6, 6, 21, 0.15, 0.02, True, T, fast=True)
    s_new = pool.add(extra[0], extra[1], horizon=200, **extra[2])
    pool.run(10_000)
    assert [pool.slot(s)[1] for s in (slots[0], slots[2], slots[3], s_new)] == [400, 400, 173, 200]
    for s, (b, box, kw), h in ((slots[0], ms[0], 400), (slots[2], ms[2], 400), (slots[3], ms[3], 173),
                               (s_new, extra, 200)):
        assert_same(pool, s, alone(b, box, kw, T, h))
    u = pool.usage()
    assert u["sims"] == 4 and u["bodies"] % 8 == 0


def test_pool_neighbor_overflow_regrows_keeping_other_lists():
    T = np.float32
    ms = members(T, fast=True)
    pool = fcc.Pool(T=T, max_bodies=4096, max_cells=4096, max_sims=8, nl_capacity=2)
    slots = [pool.add(b, box, horizon=120, **kw) for b, box, kw in ms]
    pool.run(120)
    for s, (b, box, kw) in zip(slots, ms):
        assert_same(pool, s, alone(b, box, kw, T, 120))


def test_pool_full_and_limits():
    T = np.float32
    b, box, kw = monolayer(9, 8, 5, T=T)
    pool = fcc.Pool(T=T, max_bodies=160, max_cells=4096, max_sims=2)
    s0 = pool.add(b, box, horizon=10, **kw)            # 72 bodies
    s1 = pool.add(b, box, horizon=10, **kw)            # 144 of 160
    with pytest.raises(fcc.PoolFull):
        pool.add(b, box, horizon=10, **kw)
    pool.remove(s0)
    s2 = pool.add(b, box, horizon=10, **kw)
    assert s2 == s0
    pool.run(10)
    assert np.array_equal(pool.bodies(s1).x, pool.bodies(s2).x)  # same inputs, same seed: same result
    with pytest.raises(fcc.ArgumentError):
        pool.remove(7)
    with pytest.raises(fcc.DimensionMismatch):  # every member of a pool shares its nθ
        _add_with_ntheta(fcc.Pool(T=T, nθ=40, max_bodies=256, max_cells=256, max_sims=2), b, box, kw, 64)


def _add_with_ntheta(pool, bodies, box, kw, nθ):
    import ctypes as C
    params = fcc.abi.ParamsBuffer(box, kw["types"], kw["energies"], (), kw["dt"], nθ, np.float32, kw["seed"], 0.3, 32)
    buf = fcc.abi.BodiesBuffer.from_bodies(bodies)
    slot = C.c_int32()
    pool._call("pool_add", pool._h, C.byref(params.p), C.byref(buf.s), 10, C.byref(slot))


def test_pool_fp64_matches_oracle():
    """Two FP64 members against the oracle: 30 noisy steps, rtol 1e-8, equal builds."""
    T = np.float64
    ms = members(T)[:2]
    pool = fcc.Pool(T=T, max_bodies=1024, max_cells=1024, max_sims=4)
    slots = [pool.add(b, box, horizon=30, **kw) for b, box, kw in ms]
    pool.run(30)
    for s, (b, box, kw) in zip(slots, ms):
        o = oracle.OracleSimulation(b, box, T=T, **kw)
        o.step(30)
        bg, bo = pool.bodies(s), o.bodies
        assert np.allclose(bg.x, bo.x, rtol=1e-8)
        assert np.allclose(bg.θ, bo.θ, rtol=1e-8)
        assert np.allclose(bg.coef, bo.coef, rtol=1e-8, atol=1e-12)
        assert pool.builds(s) == o.builds
        assert np.allclose(pool.shape_index(s), o.shape_index(), rtol=1e-12)


def test_pool_typed_bodies_with_parent_drag():
    """Cells with nuclei (parent drag, bonds: the split step) packed with a
    second such simulation equal their runs alone."""
    T = np.float32
    out = []
    for seed in (3, 4):
        cells, box = fcc.hexagonal_monolayer(4, 4, packing=0.9, maxmode=6, rng=seed)
        nb = fcc.with_nuclei(cells, ratio=0.5)
        kw = dict(types=(fcc.BodyType(v0=0.3, Dr=0.05, μab=0.1), fcc.BodyType(drag="parent", μab=0.1)),
                  energies=(fcc.OnTypes(fcc.Tension(0.01), 1), fcc.OnTypes(fcc.Tension(0.05), 2), fcc.Overlap(1.0),
                            fcc.HarmonicBond(0.5)), bonds=tuple(fcc.parent_bonds(nb)), dt=0.005, seed=seed)
        out.append((nb, box, kw))
    pool = fcc.Pool(T=T, max_bodies=1024, max_cells=1024, max_sims=4)
    slots = [pool.add(b, box, horizon=80, **kw) for b, box, kw in out]
    pool.run(80)
    for s, (b, box, kw) in zip(slots, out):
        assert_same(pool, s, alone(b, box, kw, T, 80))


def test_pool_graph_replay_equals_direct_launches():
    """Rounds replayed from a recorded CUDA graph equal direct launches."""
    T = np.float32
    ms = members(T, fast=True)
    pools = [fcc.Pool(T=T, max_bodies=4096, max_cells=4096, max_sims=8) for _ in range(2)]
    pools[1].graph(False)
    slots = [[p.add(b, box, horizon=10**6, **kw) for b, box, kw in ms] for p in pools]
    for p in pools:
        for _ in range(4):
            p.run(64)  # equal rounds: recorded once, then replayed
    active, replays = pools[0].graph()
    assert pools[1].graph() == (False, 0)
    if active:
        assert replays >= 4
    for s0, s1 in zip(*slots):
        a, b = pools[0].bodies(s0), pools[1].bodies(s1)
        for f in ("x", "y", "θ", "coef", "imgx", "imgy"):
            assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_pool_tune_leaves_no_trace():
    """The autotuner times variants from a snapshot and restores it: a tuned
    pool continues exactly like an untuned one (result-invariant candidates)."""
    T = np.float32
    ms = members(T, fast=True)
    pa = fcc.Pool(T=T, max_bodies=4096, max_cells=4096, max_sims=8)
    pb = fcc.Pool(T=T, max_bodies=4096, max_cells=4096, max_sims=8)
    sa = [pa.add(b, box, horizon=400, **kw) for b, box, kw in ms]
    sb = [pb.add(b, box, horizon=400, **kw) for b, box, kw in ms]
    pa.run(100)
    pb.run(100)
    v, us = pa.tune(32)
    assert v >= 0 and us > 0               # a variant sharing 8 lanes x 5 node slots
    assert pa.variant()["lanes"] == 8 and pa.variant()["slots"] == 5
    pa.run(300)
    pb.run(300)
    for x, y in zip(sa, sb):
        a, b = pa.state(x), pb.state(y)
        assert a[1:] == b[1:]
        for f in ("x", "y", "θ", "coef", "imgx", "imgy"):
            assert np.array_equal(getattr(a[0], f), getattr(b[0], f)), f
        assert pa.builds(x) == pb.builds(y)


@pytest.mark.parametrize("family,T", [((0, 5), np.float32), ((2, 4), np.float32), ((0, 5), np.float64)])
def test_variant_families_give_identical_bits(family, T, monkeypatch):
    """Launch variants the library groups into one family (same lanes x node
    slots, other block size / register budget) produce bit-identical
    trajectories: the property the autotuner's default candidate set and a
    single simulation's choice of launch shape rely on."""
    b, box, kw = monolayer(24, 24, 31, 0.2, 0.01, True, T, fast=True)
    out = []
    for v in family:
        monkeypatch.setenv("FCC_VARIANT", str(v))
        s = fcc.Simulation(b, box, T=T, **kw)
        s.run(300)
        out.append((s.bodies, s.builds))
    (a, ba), (c, bc) = out
    assert ba == bc and ba > 5
    for f in ("x", "y", "θ", "coef", "imgx", "imgy"):
        assert np.array_equal(getattr(a, f), getattr(c, f)), f


def test_pool_edge_cases():
    """Empty pools, empty simulations, run(0), retiring everything, a slot
    that is gone, and an FP64 pool with graph replay and tuning."""
    T = np.float32
    pool = fcc.Pool(T=T, max_bodies=1024, max_cells=4096, max_sims=4)
    pool.run(10)                       # nothing admitted: a no-op
    assert pool.last_timing()[2] == 0
    b, box, kw = monolayer(5, 6, 41, T=T)
    empty = fcc.Bodies.new([], [], [], np.zeros((19, 0)), [])
    s0 = pool.add(empty, box, horizon=5, **kw)   # no bodies: only the clock moves
    s1 = pool.add(b, box, horizon=7, **kw)
    pool.run(0)
    assert pool.slot(s1)[1] == 0
    pool.run(100)
    assert pool.slot(s0)[1:] == (5, 5) and pool.slot(s1)[1:] == (7, 7)
    assert pool.state(s0)[0].n == 0
    assert_same(pool, s1, alone(b, box, kw, T, 7))
    pool.remove(s0)
    pool.remove(s1)
    assert pool.usage()["sims"] == 0 and pool.usage()["bodies"] == 0
    with pytest.raises(fcc.ArgumentError):
        pool.state(s1)
    s2 = pool.add(b, box, horizon=7, **kw)      # the arena is reusable after it emptied
    pool.run(7)
    assert_same(pool, s2, alone(b, box, kw, T, 7))
    # FP64: graph replay and the autotuner keep the trajectories of a lone run
    T = np.float64
    ms = members(T, fast=True)[:2]
    pool = fcc.Pool(T=T, max_bodies=2048, max_cells=2048, max_sims=4)
    slots = [pool.add(b, box, horizon=192, **kw) for b, box, kw in ms]
    v, us = pool.tune(16)
    assert v in (0, 5)  # the FP64 builds: 256- and 224-thread blocks, one family
    for _ in range(3):
        pool.run(64)
    assert pool.graph()[0] in (True, False)
    for sl, (b, box, kw) in zip(slots, ms):
        assert_same(pool, sl, alone(b, box, kw, T, 192))
