"""The CPU oracle pinned against the reference's own known answers.

Each test restates one of the reference's tests (file:line cited) against the
oracle, so that the oracle is trusted before it judges the CUDA path:
Philox KATs, the golden N = 64 trajectory of the original C++ code, and the
analytic / finite-difference / brute-force checks of the reference suite.
"""

import json
import math
import os

import numpy as np
import pytest

from conftest import GOLDEN, deformed_coef, fcc, oracle

O = oracle.OracleSimulation


def test_philox_known_answers():
    """test/test_random.jl:4-11 (Random123 Philox4x32-10 KATs), bit-exact."""
    kat = json.load(open(os.path.join(GOLDEN, "philox_kat.json")))["vectors"]
    for v in kat:
        assert oracle.philox4x32(v["ctr"], v["key"]) == tuple(v["out"])


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_philox_noise_statistics(T):
    """test/test_random.jl:13-34: moments and independence of the normals."""
    ξ = oracle.philox_noise(42, 7, 100_000, T)
    for r in range(3):
        assert abs(ξ[r].mean()) < 0.015
        assert abs(ξ[r].var() - 1) < 0.02
        assert abs((ξ[r] ** 4).mean() - 3) < 0.1
    assert abs(np.corrcoef(ξ[0], ξ[1])[0, 1]) < 0.015
    assert abs(np.corrcoef(ξ[0], ξ[2])[0, 1]) < 0.015
    ξ8 = oracle.philox_noise(42, 8, 100_000, T)
    assert abs(np.corrcoef(ξ.ravel(), ξ8.ravel())[0, 1]) < 0.01
    assert np.array_equal(oracle.philox_noise(42, 7, 10, T), ξ[:, :10])
    assert not np.array_equal(oracle.philox_noise(43, 7, 10, T), ξ[:, :10])
    assert np.isfinite(ξ).all()
    # draw index uses all 64 bits (test/test_random.jl:46-49)
    assert not np.array_equal(oracle.philox_noise(1, 1, 1, T), oracle.philox_noise(1, 1 + (1 << 32), 1, T))


def n64_sim(init, T=np.float64):
    """The regression set-up of test/test_dynamics.jl:53-64."""
    N = init.shape[1]
    Ls = math.sqrt(N * math.pi / (0.95 * 2 * math.sqrt(3)))
    coef = np.zeros((11, N))
    coef[0] = 1.0
    bodies = fcc.Bodies.new(init[0], init[1], init[2], coef, np.ones(N))
    box = fcc.PeriodicBox(2 * Ls, math.sqrt(3) * Ls)
    types = (fcc.BodyType(v0=0.06, Dr=0.0, μab=0.1),)
    return bodies, box, dict(types=types, energies=(fcc.Tension(0.01), fcc.Overlap(1.0)), dt=0.005, T=T)


def compare_n64(sim, ref, atol):
    b = sim.bodies
    pos = np.vstack([b.x + b.imgx * sim.box.Lx, b.y + b.imgy * sim.box.Ly])
    err = max(np.abs(pos[0] - ref[3]).max(), np.abs(pos[1] - ref[4]).max(), np.abs(b.θ - ref[2]).max(),
              np.abs(b.coef[1:] - ref[5:15]).max())
    assert err <= atol, err
    return err


def test_reference_n64_trajectory(ref_n64):
    """test/test_dynamics.jl:53-70: the original C++ code's N = 64 run
    (Dr = 0, deterministic) after 1001 and 4001 steps, atol 1e-10."""
    init, snaps = ref_n64
    bodies, box, kw = n64_sim(init)
    sim = O(bodies, box, **kw)
    errs = {}
    for n in sorted(snaps):
        sim.step(n - sim.nsteps)
        errs[n] = compare_n64(sim, snaps[n], 1e-10)
    assert sim.nsteps == 4001


def test_geometry_synthesis():
    """test/test_geometry.jl:23-47: synthesis vs direct evaluation, FD R', R''."""
    coef = np.zeros((11, 1))
    coef[1:6, 0] = [0.1, -0.05, 0.03, 0.0, 0.02]
    coef[6:11, 0] = [0.02, 0.04, 0.0, -0.01, 0.01]
    coef[0, 0] = math.sqrt(1 - np.sum(coef[1:, 0] ** 2) / 2)
    θ, R0 = 0.7, 1.3
    sim = O(fcc.Bodies.new([0.0], [0.0], [θ], coef, [R0]), fcc.PeriodicBox(10.0, 10.0), types=(fcc.BodyType(),))
    g = sim.geom

    def Rdirect(φ):
        return R0 * (coef[0, 0] + sum(coef[n - 1, 0] * np.cos(n * (φ - θ)) + coef[4 + n, 0] * np.sin(n * (φ - θ))
                                      for n in range(2, 7)))

    φs = np.arange(40) * (2 * math.pi / 40)
    assert np.allclose(g.R[:, 0], Rdirect(φs), rtol=1e-12)
    h = 1e-6
    assert np.allclose(g.dR[:, 0], (Rdirect(φs + h) - Rdirect(φs - h)) / (2 * h), rtol=1e-7, atol=1e-9)
    assert np.allclose(g.ddR[:, 0], (Rdirect(φs + h) - 2 * Rdirect(φs) + Rdirect(φs - h)) / h**2, rtol=1e-3, atol=1e-3)
    assert g.rmax[0] >= Rdirect(np.linspace(0, 2 * math.pi, 1000)).max()


def single_body(terms, θ=0.4, R0=1.2, nθ=40, type=1, ntypes=1, T=np.float64):
    """test/test_energies.jl:28-35."""
    coef = deformed_coef().reshape(-1, 1)
    bodies = fcc.Bodies.new([1.0], [2.0], [θ], coef, [R0], type=type)
    sim = O(bodies, fcc.PeriodicBox(20.0, 20.0), types=tuple(fcc.BodyType() for _ in range(ntypes)),
            energies=terms, nθ=nθ, T=T)
    return sim, coef


def test_circle_energies():
    """test/test_energies.jl:65-71."""
    coef = np.zeros((11, 1))
    coef[0] = 1
    sim = O(fcc.Bodies.new([1.0], [2.0], [0.4], coef, [1.0]), fcc.PeriodicBox(20.0, 20.0),
            types=(fcc.BodyType(),), energies=(fcc.Tension(0.1),), nθ=64)
    sim.refresh()
    assert math.isclose(sim.body_energy(), 0.1 * 2 * math.pi, rel_tol=1e-12)
    assert math.isclose(sim.shape_index()[0], 2 * math.sqrt(math.pi), rel_tol=1e-12)


def fd_shape_gradient(sim, coef, h=1e-6):
    """test/test_energies.jl:37-53."""
    g = np.zeros(coef.shape[0] - 1)
    b = sim.bodies
    for r in range(1, coef.shape[0]):
        E = []
        for δ in (h, -h):
            c = coef.copy()
            c[r] += δ
            b.coef[:] = c
            sim.set_state(b)
            sim.refresh()
            E.append(sim.body_energy())
        g[r - 1] = (E[0] - E[1]) / (2 * h)
    b.coef[:] = coef
    sim.set_state(b)
    sim.refresh()
    return g


@pytest.mark.parametrize("term", [fcc.Tension(0.37), fcc.PerimeterElasticity(0.5, 3.9)], ids=["Tension", "PerimeterElasticity"])
def test_fd_shape_gradient(term):
    """test/test_energies.jl:73-85: rtol 1e-6; no force or torque from body terms."""
    sim, coef = single_body((term,))
    sim.refresh()
    g = sim.grad
    assert np.allclose(g.gcoef[1:, 0], fd_shape_gradient(sim, coef), rtol=1e-6, atol=1e-9)
    assert g.gx[0] == 0 and g.gy[0] == 0 and g.gθ[0] == 0


def test_on_types_restricts_terms():
    """test/test_energies.jl:96-103."""
    for type, active in ((1, False), (2, True)):
        sim, _ = single_body((fcc.OnTypes(fcc.Tension(1.0), 2),), type=type, ntypes=2)
        sim.refresh()
        assert (sim.body_energy() > 0) == active
        assert bool(np.any(sim.grad.gcoef != 0)) == active


def brute_force_pressure(sim):
    """test/test_contact.jl:4-21: O(N²) contact pressure on the host."""
    b, g = sim.bodies, sim.geom
    N, nθ = sim.N, sim.nθ
    K = (sim.ncoef - 1) // 2
    n = np.arange(2, K + 2)
    P = np.zeros((nθ, N))
    φ = np.arange(nθ) * (2 * math.pi / nθ)
    for i in range(N):
        ux = b.x[i] + g.R[:, i] * np.cos(φ)
        uy = b.y[i] + g.R[:, i] * np.sin(φ)
        for j in range(N):
            if j == i:
                continue
            dx = fcc.minimum_image(ux - b.x[j], sim.box.Lx)
            dy = fcc.minimum_image(uy - b.y[j], sim.box.Ly)
            ψ = np.arctan2(dy, dx)
            lab = g.lab[:, j]
            Rj = b.R0[j] * (lab[0] + (lab[1:K + 1, None] * np.cos(np.outer(n, ψ))).sum(0)
                            + (lab[K + 1:, None] * np.sin(np.outer(n, ψ))).sum(0))
            d = Rj - np.hypot(dx, dy)
            for term in sim.energies:
                t = term.term if isinstance(term, fcc.OnTypes) else term
                if isinstance(term, fcc.OnTypes) and b.type[i] not in term.types:
                    continue
                if isinstance(t, (fcc.Overlap, fcc.LinearRepulsion)):
                    P[:, i] += [t.pressure(dd, b.type[i], b.type[j], b.parent[i] == b.parent[j]) for dd in d]
                elif isinstance(t, fcc.Adhesion):  # the compiled functor's g(d), restated
                    P[:, i] += [-t.a if -t.b < dd < 0 else 0.0 for dd in d]
    return P


def jittered_monolayer(seed=2):
    """test/test_contact.jl:69-79 (jittered, deformed 8 x 8 monolayer)."""
    bodies, box = fcc.hexagonal_monolayer(8, 8, packing=0.98, rng=seed)
    rng = np.random.default_rng(3)
    bodies.x[:] = np.mod(bodies.x + 0.4 * rng.standard_normal(64), box.Lx)
    bodies.y[:] = np.mod(bodies.y + 0.4 * rng.standard_normal(64), box.Ly)
    bodies.coef[1:, :] = 0.05 * np.random.default_rng(5).standard_normal((10, 64))
    return bodies, box


def test_cell_list_matches_brute_force():
    """test/test_contact.jl:69-86, including capacity growth."""
    bodies, box = jittered_monolayer()
    sim = O(bodies, box, types=(fcc.BodyType(),), energies=(fcc.Overlap(1.0), fcc.LinearRepulsion(0.3)))
    sim.refresh()
    nb = sim.neighbors
    assert nb.ncx >= 3 and nb.ncy >= 3
    P = sim.grad.P
    assert (P > 0).sum() > 100
    assert np.allclose(P, brute_force_pressure(sim), rtol=1e-12, atol=1e-12)
    small = O(bodies, box, types=(fcc.BodyType(),), energies=(fcc.Overlap(1.0), fcc.LinearRepulsion(0.3)),
              nl_capacity=2)
    small.refresh()
    nb2 = small.neighbors
    assert nb2.cap >= nb2.count.max() > 2
    assert np.allclose(small.grad.P, P, rtol=0, atol=0)


def two_body(terms, d=1.5, R0=(1.0, 1.0), nθ=40, deformed=False, θ=(0.3, -1.1), type=(1, 1), parent=(1, 2), ntypes=1):
    """test/test_contact.jl:24-35."""
    coef = np.zeros((11, 2))
    coef[0] = 1
    if deformed:
        coef[:, 0] = deformed_coef(5)
        coef[:, 1] = deformed_coef(6)
    bodies = fcc.Bodies.new([5.0, 5.0 + d], [5.0, 5.0], θ, coef, R0, type=type, parent=parent)
    sim = O(bodies, fcc.PeriodicBox(10.0, 10.0), types=tuple(fcc.BodyType() for _ in range(ntypes)),
            energies=terms, nθ=nθ)
    sim.refresh()
    return sim


def test_two_discs_overlap_force():
    """test/test_contact.jl:88-96: dA/dd = -√(4 - d²), rtol 1e-3 at nθ = 8000."""
    d = 1.5
    g = two_body((fcc.Overlap(1.0),), d=d, nθ=8000).grad
    assert math.isclose(g.gx[0], math.sqrt(4 - d * d), rel_tol=1e-3)
    assert math.isclose(g.gx[1], -math.sqrt(4 - d * d), rel_tol=1e-3)
    assert abs(g.gy[0]) < 1e-6


def test_nucleus_attraction_to_own_cell():
    """test/test_contact.jl:122-133 (related coupling sign)."""
    terms = (fcc.Overlap([[1.0, 1.0], [1.0, 1.0]], related=[[0.0, -2.0], [-2.0, 0.0]]),)
    partial = two_body(terms, d=0.9, R0=(1.0, 0.4), type=(1, 2), parent=(1, 1), ntypes=2, nθ=400)
    assert partial.grad.gx[1] > 0.1
    assert partial.grad.gx[0] < -0.1
    inside = two_body(terms, d=0.3, R0=(1.0, 0.4), type=(1, 2), parent=(1, 1), ntypes=2, nθ=400)
    assert abs(inside.grad.gx[1]) < 1e-10 and abs(inside.grad.gx[0]) < 1e-10


def skin_sim(skin, v0=1.0):
    """test/test_contact.jl:135-141."""
    bodies, box = fcc.hexagonal_monolayer(6, 6, packing=0.97, rng=2)
    return O(bodies, box, types=(fcc.BodyType(v0=v0, Dr=1.0, Dt=0.01, μab=1.0),),
             energies=(fcc.Tension(0.1), fcc.Overlap(1.0), fcc.LinearRepulsion(0.3)), dt=0.01, skin=skin, seed=3)


def test_verlet_skin():
    """test/test_contact.jl:135-161."""
    with pytest.raises(fcc.ArgumentError):
        skin_sim(-0.1)
    sim = skin_sim(0.2)
    exact = True
    for _ in range(60):
        sim.step(1)
        sim.update_neighbors()
        sim.compute_gradients()
        exact &= np.allclose(sim.grad.P, brute_force_pressure(sim), rtol=1e-12, atol=1e-12)
    assert exact
    assert 3 < sim.builds < 50
    assert skin_sim(0.0).step(10).builds == 10
    a, b = skin_sim(0.0, v0=0.3).step(100), skin_sim(0.5, v0=0.3).step(100)
    assert b.builds < a.builds
    assert np.allclose(b.bodies.x, a.bodies.x, rtol=1e-10)
    assert np.allclose(b.bodies.coef, a.bodies.coef, rtol=1e-10)


def test_hard_area_constraint():
    """test/test_dynamics.jl:23-31."""
    bodies, box = fcc.hexagonal_monolayer(2, 2)
    bodies.coef[1:, :] = (0.05 * np.arange(1, 11))[:, None]
    sim = O(bodies, box, types=(fcc.BodyType(),), nθ=64)
    c = sim.bodies.coef
    assert np.all(np.hypot(c[1:6], c[6:11]).sum(0) <= math.sqrt(2 / 3) + 1e-12)
    assert np.allclose(sim.areas(), math.pi, rtol=1e-12)


def test_isolated_cell_self_propels():
    """test/test_dynamics.jl:33-43: crosses the periodic boundary."""
    coef = np.zeros((11, 1))
    coef[0] = 1
    sim = O(fcc.Bodies.new([1.0], [1.0], [0.3], coef, [1.0]), fcc.PeriodicBox(5.0, 5.0),
            types=(fcc.BodyType(v0=0.5),), energies=(fcc.Tension(0.1), fcc.Overlap(1.0)), dt=0.01)
    sim.step(3000)
    b = sim.bodies
    X = np.array([b.x[0] + b.imgx[0] * 5.0, b.y[0] + b.imgy[0] * 5.0])
    assert np.allclose(X, [1 + 15 * math.cos(0.3), 1 + 15 * math.sin(0.3)], rtol=1e-8)
    assert 0 <= b.x[0] < 5 and 0 <= b.y[0] < 5
    assert math.isclose(b.θ[0], 0.3, rel_tol=1e-12)
    assert np.abs(b.coef[1:, 0]).max() < 1e-14
    assert math.isclose(sim.t, 30, rel_tol=1e-9)


def test_rotational_diffusion():
    """test/test_dynamics.jl:45-51: var θ = 2 Dr t, rtol 0.1."""
    N = 4000
    rng = np.random.default_rng(1)
    coef = np.zeros((11, N))
    coef[0] = 1
    sim = O(fcc.Bodies.new(rng.random(N), rng.random(N), np.zeros(N), coef, np.ones(N)), fcc.PeriodicBox(1.0, 1.0),
            types=(fcc.BodyType(Dr=0.1),), dt=0.01, seed=7)
    sim.step(500)
    θ = sim.bodies.θ
    assert abs(np.mean(θ**2) / (2 * 0.1 * sim.t) - 1) < 0.1


def cell_nucleus(nucleus=None, cell=None, dt=0.01, energies=(), bonds=(), x2=5.0):
    """test/test_parents.jl:10-16."""
    coef = np.zeros((11, 3))
    coef[0] = 1
    bodies = fcc.Bodies.new([5.0, x2, 1.0], [5.0, 5.0, 1.0], [0.3, -1.0, 2.0], coef, [1.0, 0.5, 1.0],
                            type=[1, 2, 1], parent=[1, 1, 3])
    return O(bodies, fcc.PeriodicBox(10.0, 10.0), types=(cell or fcc.BodyType(), nucleus or fcc.BodyType(drag="parent")),
             energies=energies, bonds=bonds, dt=dt)


def test_nucleus_is_carried_along():
    """test/test_parents.jl:67-74."""
    sim = cell_nucleus(cell=fcc.BodyType(v0=0.5))
    sim.step(2000)
    b = sim.bodies
    X = np.vstack([b.x + b.imgx * 10.0, b.y + b.imgy * 10.0])
    assert np.allclose(X[:, 0], [5 + 10 * math.cos(0.3), 5 + 10 * math.sin(0.3)], rtol=1e-8)
    assert np.allclose(X[:, 1], X[:, 0], rtol=1e-12)


def test_bonded_nucleus_relaxes():
    """test/test_parents.jl:121-132: δ(n) = δ0 (1 - μ k dt)^n, rtol 1e-12."""
    μ, k, δ0, n = 2.0, 0.5, 0.2, 300
    coef = np.zeros((11, 3))
    coef[0] = 1
    bodies = fcc.Bodies.new([5.0, 5.0 + δ0, 1.0], [5.0, 5.0, 1.0], [0.3, -1.0, 2.0], coef, [1.0, 0.5, 1.0],
                            type=[1, 2, 1], parent=[1, 1, 3])
    sim = O(bodies, fcc.PeriodicBox(10.0, 10.0), types=(fcc.BodyType(), fcc.BodyType(μr=μ, drag="parent")),
            energies=(fcc.HarmonicBond(k),), bonds=fcc.parent_bonds(bodies), dt=0.01)
    sim.step(n)
    b = sim.bodies
    assert b.x[0] == 5.0 and b.y[0] == 5.0
    assert math.isclose(b.x[1] - 5.0, δ0 * (1 - μ * k * 0.01) ** n, rel_tol=1e-12)


def test_bond_forces():
    """test/test_parents.jl:99-119: bonded pair across the periodic boundary."""
    coef = np.zeros((11, 3))
    coef[0] = 1
    bodies = fcc.Bodies.new([9.8, 0.4, 5.0], [3.0, 3.5, 5.0], np.zeros(3), coef, np.ones(3), type=[1, 2, 1])
    box = fcc.PeriodicBox(10.0, 10.0)
    Δ = np.array([9.8 - 0.4 - 10, 3.0 - 3.5])
    for terms, k in (((fcc.HarmonicBond(0.7),), 0.7), ((fcc.OnTypes(fcc.HarmonicBond(0.7), 1, 2),), 0.7),
                     ((fcc.OnTypes(fcc.HarmonicBond(0.7), 1),), 0.0), ((fcc.HarmonicBond(0.7), fcc.HarmonicBond(0.3)), 1.0)):
        sim = O(bodies, box, types=(fcc.BodyType(), fcc.BodyType()), energies=terms, bonds=[(1, 2)])
        sim.compute_gradients()
        g = sim.grad
        assert np.allclose([g.gx[0], g.gy[0]], k * Δ, atol=1e-14)
        assert np.allclose([g.gx[1], g.gy[1]], -k * Δ, atol=1e-14)
        assert g.gx[2] == 0 and g.gy[2] == 0


def test_argument_errors():
    """Validation where the reference throws (src/simulation.jl:108-118,
    src/basis.jl:36-38, src/energies/bonds.jl:56-59)."""
    coef = np.zeros((11, 2))
    coef[0] = 1
    box = fcc.PeriodicBox(10.0, 10.0)
    child = fcc.BodyType(drag="parent")
    with pytest.raises(fcc.ArgumentError):
        fcc.BodyType(drag="cytoplasm")
    with pytest.raises(fcc.ArgumentError):  # parent drag without a parent
        O(fcc.Bodies.new([1.0, 2.0], [1.0, 2.0], np.zeros(2), coef, np.ones(2), type=[1, 2]), box,
          types=(fcc.BodyType(), child))
    with pytest.raises(fcc.ArgumentError):  # parent with parent drag itself
        O(fcc.Bodies.new([1.0, 2.0], [1.0, 2.0], np.zeros(2), coef, np.ones(2), type=[2, 2], parent=[2, 1]), box,
          types=(fcc.BodyType(), child))
    with pytest.raises(fcc.ArgumentError):  # parent out of range
        O(fcc.Bodies.new([1.0, 2.0], [1.0, 2.0], np.zeros(2), coef, np.ones(2), parent=[1, 3]), box,
          types=(fcc.BodyType(),))
    with pytest.raises(fcc.ArgumentError):  # nθ ≤ 2 maxmode
        O(fcc.Bodies.new([1.0, 2.0], [1.0, 2.0], np.zeros(2), coef, np.ones(2)), box, types=(fcc.BodyType(),), nθ=12)
    with pytest.raises(fcc.DimensionMismatch):  # even coefficient rows
        O(fcc.Bodies.new([1.0, 2.0], [1.0, 2.0], np.zeros(2), np.zeros((10, 2)), np.ones(2)), box, types=(fcc.BodyType(),))
    for bonds in ([(1, 1)], [(1, 2), (2, 1)], [(1, 4)]):
        with pytest.raises(fcc.ArgumentError):
            O(fcc.Bodies.new([1.0, 2.0, 3.0], [1.0, 2.0, 3.0], np.zeros(3), np.hstack([coef, coef[:, :1]]), np.ones(3)),
              box, types=(fcc.BodyType(),), energies=(fcc.HarmonicBond(1.0),), bonds=bonds)


def test_type_maxmode_equals_a_simulation_with_fewer_modes():
    """A body type limited to modes 2..6 inside a modes-2..10 simulation is
    the same dynamics as a modes-2..6 simulation: the masked modes enter as
    zero (even when given) and stay zero.  Every type limited here, so the
    two runs are comparable body for body (FP64, 40 noisy steps, 1e-12)."""
    cells, box = fcc.hexagonal_monolayer(4, 4, packing=0.95, maxmode=10, rng=5)
    b10 = fcc.with_nuclei(cells, ratio=0.5)
    b10.coef[1:] = 0.03 * np.random.default_rng(6).standard_normal((18, b10.n))
    b6 = b10.copy()
    b6.coef = np.asfortranarray(np.vstack([b10.coef[:1], b10.coef[1:6], b10.coef[10:15]]))
    def kw(mm):
        return dict(types=(fcc.BodyType(v0=0.1, Dr=0.05, μab=0.2, maxmode=mm),
                           fcc.BodyType(drag="parent", μab=0.2, maxmode=mm)),
                    energies=(fcc.Tension(0.05), fcc.Overlap(1.0)), seed=4)
    a = oracle.OracleSimulation(b10, box, **kw(6)).step(40)
    c = oracle.OracleSimulation(b6, box, **kw(0)).step(40)
    ba, bc = a.bodies, c.bodies
    assert np.abs(ba.coef[6:10]).max() == 0 and np.abs(ba.coef[15:19]).max() == 0
    for f in ("x", "y", "θ"):
        assert np.allclose(getattr(ba, f), getattr(bc, f), rtol=1e-12, atol=1e-12), f
    assert np.allclose(np.vstack([ba.coef[:6], ba.coef[10:15]]), bc.coef, rtol=1e-12, atol=1e-14)
    with pytest.raises(fcc.ArgumentError):
        oracle.OracleSimulation(b6, box, **kw(7))
    with pytest.raises(fcc.ArgumentError):
        fcc.BodyType(maxmode=-1)


# ------------------------------------------------------- compiled user terms
@pytest.mark.parametrize("term", [fcc.Bending(0.3), fcc.ShapeIndexElasticity(0.7, 3.9)], ids=["Bending", "ShapeIndexElasticity"])
def test_user_body_term_fd_shape_gradient(term):
    """A compiled user BodyTerm (include/fcc_user_terms.h) through the same
    finite-difference check as the built-ins (test/test_energies.jl:73-85,
    rtol 1e-6); Bending needs R'' and its pullback (GDD)."""
    sim, coef = single_body((term,))
    sim.refresh()
    g = sim.grad
    assert np.abs(g.GDD).max() > 0 if isinstance(term, fcc.Bending) else np.abs(g.GDD).max() == 0
    assert np.allclose(g.gcoef[1:, 0], fd_shape_gradient(sim, coef), rtol=1e-6, atol=1e-9)
    assert g.gx[0] == 0 and g.gy[0] == 0 and g.gθ[0] == 0


def test_user_bending_of_a_circle():
    """∮ c² ds of a circle of radius R0 is 2π / R0."""
    coef = np.zeros((11, 1))
    coef[0] = 1
    sim = O(fcc.Bodies.new([1.0], [2.0], [0.4], coef, [1.3]), fcc.PeriodicBox(20.0, 20.0),
            types=(fcc.BodyType(),), energies=(fcc.Bending(0.25),), nθ=64).refresh()
    assert math.isclose(sim.body_energy(), 0.25 * 2 * math.pi / 1.3, rel_tol=1e-12)


def test_user_contact_term_matches_brute_force_and_widens_the_lists():
    """A compiled user ContactTerm with an interaction range (Adhesion): the
    node pressures equal the O(N²) restatement, and the range widens the
    neighbour lists (contact_range, src/energies/contact.jl:54)."""
    bodies, box = jittered_monolayer()
    terms = (fcc.Overlap(1.0), fcc.Adhesion(0.4, 0.15))
    sim = O(bodies, box, types=(fcc.BodyType(),), energies=terms).refresh()
    P = sim.grad.P
    assert (P < 0).sum() > 20  # nodes in the adhesion band
    assert np.allclose(P, brute_force_pressure(sim), rtol=1e-12, atol=1e-12)
    plain = O(bodies, box, types=(fcc.BodyType(),), energies=terms[:1]).refresh()
    assert sim.neighbors.count.sum() > plain.neighbors.count.sum()


def test_user_contact_two_discs_attract():
    """Two discs a little apart, inside the adhesion band: the energy falls as
    they approach (gradient towards the other body)."""
    g = two_body((fcc.Adhesion(1.0, 0.2),), d=2.1, nθ=400).grad
    assert g.gx[0] < -1e-3 and g.gx[1] > 1e-3
    assert abs(g.gy[0]) < 1e-9


def test_user_bond_term_gradient():
    """A compiled user BondTerm (QuarticBond): dE/dΔ = k |Δ|² Δ on each centre."""
    coef = np.zeros((11, 2))
    coef[0] = 1
    bodies = fcc.Bodies.new([5.0, 6.3], [5.0, 5.4], [0.1, 0.2], coef, [1.0, 1.0])
    sim = O(bodies, fcc.PeriodicBox(20.0, 20.0), types=(fcc.BodyType(),), energies=(fcc.QuarticBond(0.7),),
            bonds=[(1, 2)]).refresh()
    dx, dy = 5.0 - 6.3, 5.0 - 5.4
    r2 = dx * dx + dy * dy
    assert np.allclose([sim.grad.gx[0], sim.grad.gy[0]], [0.7 * r2 * dx, 0.7 * r2 * dy], rtol=1e-12)
    assert np.allclose([sim.grad.gx[1], sim.grad.gy[1]], [-0.7 * r2 * dx, -0.7 * r2 * dy], rtol=1e-12)


def test_unknown_user_term_is_an_argument_error():
    sim_args = dict(types=(fcc.BodyType(),), energies=(fcc.UserBodyTerm(1.0, 0.0, index=99),))
    with pytest.raises(fcc.ArgumentError):
        single_body(sim_args["energies"])
