"""Parity on the configured workloads themselves (marked ``gpu``), each
against the CPU oracle with a stated tolerance:

- the plain N = 1024 FP64 monolayer (hexagonal_monolayer(32, 32; packing
  0.95), modes 2..10, Tension(0.01) + Overlap(1.0), v0 0.06, Dr 0.01, μab 0.1,
  dt 0.005, Philox seed 1234): 200 noisy steps, rtol 1e-8 and equal rebuild
  counts, as test/test_cuda.jl:31-39 does for 30 steps; forces of the final
  state at 1e-12 of each field's scale;
- the cells-with-nuclei workload (4096 cells of R0 = 1 plus 4096 nuclei of
  R0 = 0.5 in a 64 x 64 packing at 0.9, OnTypes tensions 0.01 / 0.05, Overlap
  for every pair, nuclei without self-propulsion): forces on a deformed state,
  FP64 at 1e-12, FP32 against the FP64 oracle at 1e-5 with Heaviside flips
  excluded and counted, and one FP64 step at 1e-12 — with every mode on both
  types (the reference's shared modes), and with the nuclei held to modes
  2..6 (BodyType maxmode, against the oracle with the same limit; 30 noisy
  FP64 steps at rtol 1e-8 and equal rebuild counts, and the nuclei's modes
  7..10 exactly zero after an FP32 run);
- the N = 65536 and 262144 polydisperse monolayers (256 x 256, 512 x 512):
  one evaluation of the forces of a deformed FP32 state against the FP64
  oracle at 1e-5, flips excluded and counted.

A Heaviside flip is a contour node whose Overlap pressure g = J H(d) differs
between the two evaluations by at least J/2: FP32 rounding of the depth d
(about 1e-5 at coordinates of 250) decides the side of a near-tie, and the
body's force then moves by O(J).  At most 1% of the bodies may be excluded.
"""

import math

import numpy as np
import pytest

from conftest import fcc, oracle

pytestmark = pytest.mark.gpu

G = fcc.Simulation
O = oracle.OracleSimulation
FIELDS = ("gx", "gy", "gθ", "gcoef", "Ebody")


def relerr(a, b, keep=None):
    a, b = np.asarray(a, float), np.asarray(b, float)
    scale = max(float(np.abs(b).max()), 1e-300)
    if keep is not None:
        a, b = a[..., keep], b[..., keep]
    return float(np.abs(a - b).max() / scale) if a.size else 0.0


def as_f32(b):
    b = b.copy()
    for f in ("x", "y", "θ", "coef", "R0"):
        setattr(b, f, np.asfortranarray(np.asarray(getattr(b, f), np.float32).astype(np.float64)))
    return b


def flips(g, o, J=1.0):
    """Bodies with a node whose contact pressure differs by at least J/2."""
    return np.abs(np.asarray(g.grad.P) - np.asarray(o.grad.P)).max(axis=0) >= 0.5 * J


# ------------------------------------------------------------------ plain
def plain_config():
    bodies, box = fcc.hexagonal_monolayer(32, 32, packing=0.95, maxmode=10, rng=1234)
    kw = dict(types=(fcc.BodyType(v0=0.06, Dr=0.01, μab=0.1),), energies=(fcc.Tension(0.01), fcc.Overlap(1.0)),
              dt=0.005, seed=1234, T=np.float64)
    return bodies, box, kw


def test_plain_n1024_fp64_trajectory_matches_oracle():
    bodies, box, kw = plain_config()
    assert bodies.n == 1024
    g, o = G(bodies, box, **kw), O(bodies, box, **kw)
    assert g.neighbor_dims()[:2] == (15, 13)  # the 15 x 13 cell grid of the workload
    g.run(200)
    o.step(200)
    bg, bo = g.bodies, o.bodies
    assert np.allclose(bg.x, bo.x, rtol=1e-8, atol=0)
    assert np.allclose(bg.y, bo.y, rtol=1e-8, atol=0)
    assert np.allclose(bg.θ, bo.θ, rtol=1e-8, atol=0)
    assert np.allclose(bg.coef, bo.coef, rtol=1e-8, atol=1e-12)
    assert np.array_equal(bg.imgx, bo.imgx) and np.array_equal(bg.imgy, bo.imgy)
    assert g.builds == o.builds and g.nsteps == o.nsteps == 200
    # the shapes did deform, so the comparison is not of circles
    assert np.abs(bo.coef[1:]).max() > 1e-4
    g.refresh()
    o.set_state(bg, clock=o.clock)
    o.refresh()
    for f in FIELDS:
        assert relerr(getattr(g.grad, f), getattr(o.grad, f)) < 1e-12, f


# ------------------------------------------------------------ cells + nuclei
def nuclei_config(T, drag="substrate", nucleus_maxmode=0, side=64):
    cells, box = fcc.hexagonal_monolayer(side, side, packing=0.9, maxmode=10, rng=1234)
    bodies = fcc.with_nuclei(cells, ratio=0.5)
    kw = dict(types=(fcc.BodyType(v0=0.06, Dr=0.01, μab=0.1),
                     fcc.BodyType(v0=0.0, drag=drag, μab=0.1, maxmode=nucleus_maxmode)),
              energies=(fcc.OnTypes(fcc.Tension(0.01), 1), fcc.OnTypes(fcc.Tension(0.05), 2), fcc.Overlap(1.0)),
              dt=0.005, seed=1234, T=T)
    return bodies, box, kw


@pytest.fixture(scope="module")
def nuclei_state():
    """The 8192-body state after 200 FP32 steps of the workload (deformed
    shapes, nuclei pushed off their cells' centres), FP32-representable."""
    bodies, box, kw = nuclei_config(np.float32)
    sim = G(bodies, box, **kw)
    sim.run(200)
    return as_f32(sim.bodies), box


def test_nuclei_forces_fp64_match_oracle(nuclei_state):
    state, box = nuclei_state
    _, _, kw = nuclei_config(np.float64)
    g, o = G(state, box, **kw).refresh(), O(state, box, **kw).refresh()
    assert state.n == 8192
    for f in FIELDS:
        assert relerr(getattr(g.grad, f), getattr(o.grad, f)) < 1e-12, f
    assert np.array_equal(g.neighbors.count, o.neighbors.count)


def test_nuclei_forces_fp32_vs_fp64_oracle(nuclei_state):
    state, box = nuclei_state
    _, _, k64 = nuclei_config(np.float64)
    _, _, k32 = nuclei_config(np.float32)
    g, o = G(state, box, **k32).refresh(), O(state, box, **k64).refresh()
    flip = flips(g, o)
    assert flip.mean() <= 0.01
    for f in FIELDS:
        assert relerr(getattr(g.grad, f), getattr(o.grad, f), ~flip) < 1e-5, f


@pytest.mark.parametrize("drag", ["parent", "substrate"])
def test_nuclei_one_step_fp64_matches_oracle(nuclei_state, drag):
    state, box = nuclei_state
    _, _, kw = nuclei_config(np.float64, drag)
    g, o = G(state, box, **kw), O(state, box, **kw)
    g.step(1)
    o.step(1)
    bg, bo = g.bodies, o.bodies
    for f, scale in (("x", 1e-12), ("y", 1e-12), ("θ", 1e-12)):
        d = np.abs(getattr(bg, f) - getattr(state, f))  # the increment's scale
        assert np.abs(getattr(bg, f) - getattr(bo, f)).max() <= scale * max(d.max(), 1e-300) + 1e-13, f
    dc = np.abs(bo.coef - state.coef).max()
    assert np.abs(bg.coef - bo.coef).max() <= 1e-12 * dc + 1e-15


# ------------------------------------------------ N = 65536 and 262144 FP32
@pytest.mark.parametrize("side", [256, 512])
def test_large_fp32_forces_vs_oracle(side):
    bodies, box = fcc.polydisperse_monolayer(side, side, packing=0.95, maxmode=10, seed=1234)
    kw = dict(types=(fcc.BodyType(v0=0.06, Dr=0.01, μab=0.1),),
              energies=(fcc.Tension(0.01), fcc.Overlap(1.0), fcc.PerimeterElasticity(0.1, 3.7)), dt=0.005, seed=1234)
    g = G(bodies, box, T=np.float32, **kw)
    g.run(100)
    state = as_f32(g.bodies)
    g.set_state(state)
    g.refresh()
    o = O(state, box, T=np.float64, **kw).refresh()
    assert state.n == side * side
    flip = flips(g, o)
    assert flip.mean() <= 0.01
    for f in FIELDS:
        assert relerr(getattr(g.grad, f), getattr(o.grad, f), ~flip) < 1e-5, f
    assert math.isfinite(float(np.asarray(g.grad.Ebody).sum()))


# --------------------------------------------- nuclei held to modes 2..6
def test_nuclei_modes_2_to_6_match_the_masked_oracle(nuclei_state):
    state, box = nuclei_state
    _, _, kw = nuclei_config(np.float64, nucleus_maxmode=6)
    g, o = G(state, box, **kw).refresh(), O(state, box, **kw).refresh()
    for f in FIELDS:
        assert relerr(getattr(g.grad, f), getattr(o.grad, f)) < 1e-12, f
    # the loaded state already has the nuclei's modes 7..10 at zero
    nuc = state.type == 2
    assert np.abs(g.bodies.coef[6:10][:, nuc]).max() == 0 and np.abs(g.bodies.coef[15:19][:, nuc]).max() == 0


def test_nuclei_modes_2_to_6_short_trajectory_fp64():
    bodies, box, kw = nuclei_config(np.float64, nucleus_maxmode=6, side=16)
    bodies.coef[1:] = 0.03 * np.random.default_rng(12).standard_normal((bodies.ncoef - 1, bodies.n))
    g, o = G(bodies, box, **kw), O(bodies, box, **kw)
    g.run(30)
    o.step(30)
    bg, bo = g.bodies, o.bodies
    assert np.allclose(bg.x, bo.x, rtol=1e-8) and np.allclose(bg.θ, bo.θ, rtol=1e-8)
    assert np.allclose(bg.coef, bo.coef, rtol=1e-8, atol=1e-12)
    assert g.builds == o.builds
    nuc = bodies.type == 2
    for b in (bg, bo):
        assert np.abs(b.coef[6:10][:, nuc]).max() == 0 and np.abs(b.coef[15:19][:, nuc]).max() == 0
        assert np.abs(b.coef[6:10][:, ~nuc]).max() > 0  # the cells keep every mode


def test_nuclei_modes_2_to_6_stay_zero_in_fp32():
    bodies, box, kw = nuclei_config(np.float32, nucleus_maxmode=6)
    sim = G(bodies, box, **kw)
    sim.run(200)
    b = sim.bodies
    nuc = b.type == 2
    assert np.isfinite(b.coef).all()
    assert np.abs(b.coef[6:10][:, nuc]).max() == 0 and np.abs(b.coef[15:19][:, nuc]).max() == 0
    assert np.abs(b.coef[1:6][:, nuc]).max() > 0
    assert np.allclose(fcc.areas(sim), math.pi * np.asarray(bodies.R0, np.float32).astype(float) ** 2, rtol=2e-5)
