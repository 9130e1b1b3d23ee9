"""Parity of the CUDA path against the CPU oracle (marked ``gpu``).

Inputs are identical for both sides; tolerances are stated per test:
- Philox normals: rtol 4 eps (test/test_cuda.jl:22-29); the uniforms use 52
  bits of two words in FP64, so any word difference would show;
- cell and neighbour lists: bit-exact at equal precision on equal inputs;
- forces/gradients and one-step updates: max error / max magnitude per field
  <= 1e-12 in FP64, <= 1e-5 in FP32 (FP32 compared against the FP64 oracle on
  FP32-representable inputs, bodies at an Overlap near-tie excluded and
  counted: the Heaviside g = J H(d) flips there; a one-step θ also carries
  the difference between the Float32 and Float64 rotational noise draws);
- trajectories: the reference's golden N = 64 run at atol 1e-10
  (test/test_dynamics.jl:53-70), 30 noisy FP64 steps at rtol 1e-8 with equal
  rebuild counts (test/test_cuda.jl:123-131);
- run (persistent multi-step launches) == step (one launch per step),
  bit for bit (test/test_cuda.jl:133-185).
"""

import math
import threading

import numpy as np
import pytest

from conftest import deformed_coef, fcc, oracle
from test_oracle import brute_force_pressure, jittered_monolayer, n64_sim

pytestmark = pytest.mark.gpu

G = fcc.Simulation
O = oracle.OracleSimulation


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def as_f32_bodies(b):
    b = b.copy()
    for f in ("x", "y", "θ", "coef", "R0"):
        setattr(b, f, f32(getattr(b, f)))
    return b


def relerr(a, b, mask=None):
    a, b = np.asarray(a, float), np.asarray(b, float)
    scale = max(np.abs(b).max(), 1e-300) if b.size else 1.0
    if mask is not None:
        a, b = a[..., mask], b[..., mask]
    return float(np.abs(a - b).max() / scale) if a.size else 0.0


LAYOUT_ENERGIES = (fcc.Tension(0.1), fcc.OnTypes(fcc.PerimeterElasticity(0.2, 3.7), 2),
                   fcc.Overlap([[1.0, 1.0], [1.0, 1.0]], related=[[1.0, -2.0], [-2.0, 1.0]]),
                   fcc.LinearRepulsion(0.5), fcc.HarmonicBond(0.2))


def layout_bodies(maxmode=6):
    """Nucleated soft fluid with deformed shapes (test/test_layout.jl:21-29)."""
    cells, box = fcc.hexagonal_monolayer(5, 4, packing=0.97, maxmode=maxmode, rng=2)
    bodies = fcc.with_nuclei(cells)
    bodies.coef[1:, :] = 0.04 * np.random.default_rng(5).standard_normal((bodies.ncoef - 1, bodies.n))
    return bodies, box


def layout_kw(T=np.float64, nθ=40, v0=0.2, skin=0.3, seed=7, energies=LAYOUT_ENERGIES, drag="parent", **kw):
    types = (fcc.BodyType(v0=v0, Dr=0.1), fcc.BodyType(Dr=0.1, drag=drag))
    return dict(types=types, energies=energies, nθ=nθ, T=T, skin=skin, seed=seed, **kw)


def pair(bodies, box, bonds=(), **kw):
    return G(bodies, box, bonds=bonds, **kw), O(bodies, box, bonds=bonds, **kw)


# ------------------------------------------------------------------ Philox
@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_philox_noise_matches_oracle(T):
    g = fcc.philox_noise(9, 12, 1000, T)
    c = oracle.philox_noise(9, 12, 1000, T)
    eps = np.finfo(T).eps
    assert np.allclose(g, c, rtol=4 * eps, atol=0)
    # 64-bit draw index and per-body independence of N
    assert np.array_equal(fcc.philox_noise(9, 1 << 33, 10, T), fcc.philox_noise(9, 1 << 33, 20, T)[:, :10])
    assert not np.array_equal(fcc.philox_noise(9, 1, 10, T), fcc.philox_noise(9, 1 + (1 << 32), 10, T))


# ---------------------------------------------------- cell / neighbour lists
@pytest.mark.parametrize("T", [np.float32, np.float64])
@pytest.mark.parametrize("case", ["grid", "collapsed", "overflow", "ragged"])
def test_neighbor_build_bit_exact(T, case):
    """update_celllist! + neighbour kernel, bit-exact against the oracle."""
    rng = np.random.default_rng(11)
    if case == "collapsed":
        n, Lx, Ly = 60, 9.0, 30.0  # ncx = 2 -> 1 cell column, minimum image over the whole row
    elif case == "ragged":
        n, Lx, Ly = 333, 31.0, 17.5
    else:
        n, Lx, Ly = 2000, 90.0, 70.0
    x = rng.random(n) * Lx
    y = rng.random(n) * Ly
    rmax = 0.8 + 0.6 * rng.random(n)
    if T == np.float32:
        x, y, rmax = f32(x), f32(y), f32(rmax)
    cutoff = 2 * 1.4 * (1 + math.sqrt(2 / 3)) + 0.3
    cap = 2 if case == "overflow" else 48
    a = fcc.build_neighbors(x, y, rmax, Lx, Ly, cutoff, 0.3, cap, T)
    b = oracle.build_neighbors(x, y, rmax, Lx, Ly, cutoff, 0.3, cap, T)
    for u, v in zip(a[:4], b[:4]):
        assert np.array_equal(u, v)
    cnt = b[5]
    assert np.array_equal(a[5], cnt)
    assert cnt.max() > 0
    if case == "overflow":
        assert cnt.max() > cap
    for i in range(n):
        k = min(cnt[i], cap)
        assert np.array_equal(a[4][:k, i], b[4][:k, i])


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_step_kernel_rebuild_equals_standalone_build(T):
    """The list rebuild inside the persistent step kernel (single simulation:
    descriptor in shared memory, cell scan and sort from registers, 8 lanes
    per body) gives, on the same state, the lists of the stand-alone build
    kernels that test_neighbor_build_bit_exact pins to the oracle."""
    b, box = fcc.polydisperse_monolayer(40, 40, packing=0.95, maxmode=10, seed=3)
    b.coef[1:] = 0.03 * (2 * np.random.default_rng(3).random((b.ncoef - 1, b.n)) - 1)
    kw = dict(types=(fcc.BodyType(v0=0.1, Dr=0.01, μab=0.1),), energies=(fcc.Tension(0.01), fcc.Overlap(1.0)),
              dt=0.005, seed=3, skin=0.0, T=T)
    a = G(b, box, **kw)
    a.run(1)  # skin 0: the step's prologue builds the lists from the initial state
    c = G(b, box, **kw)
    c.update_neighbors(force=True)
    na, nc = a.neighbors, c.neighbors
    for f in ("cellid", "perm", "start", "stop", "count"):
        assert np.array_equal(getattr(na, f), getattr(nc, f)), f
    assert na.count.max() > 0
    for i in range(b.n):
        k = min(nc.count[i], nc.cap)
        assert np.array_equal(na.idx[:k, i], nc.idx[:k, i])


def test_neighbor_build_empty_and_single():
    for n in (1, 2):
        x, y, r = np.full(n, 1.0), np.linspace(1, 2, n), np.ones(n)
        a = fcc.build_neighbors(x, y, r, 10.0, 10.0, 3.93, 0.3, 4)
        b = oracle.build_neighbors(x, y, r, 10.0, 10.0, 3.93, 0.3, 4)
        for u, v in zip(a, b):
            assert np.array_equal(u, v)


# ---------------------------------------------------------------- geometry
@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_geometry_matches_oracle(T):
    bodies, box = layout_bodies()
    if T == np.float32:
        bodies = as_f32_bodies(bodies)
    g, o = pair(bodies, box, **layout_kw(T=T))
    tol = 1e-13 if T == np.float64 else 2e-6
    og = o.geom
    gg = g.geom
    for f in ("lab", "labR0", "R", "dR", "ddR", "rmax"):
        assert relerr(getattr(gg, f), getattr(og, f)) < tol, f
    # the GPU's shape constraints (FP64 sums) reproduce the oracle's coefficients
    assert relerr(g.bodies.coef, o.bodies.coef) < tol


# ---------------------------------------------------------------- gradients
FIELDS = ("GR", "GD", "GDD", "P", "gx", "gy", "gθ", "glab", "gcoef", "Ebody")


@pytest.mark.parametrize("nθ", [40, 37, 64])
def test_gradients_match_oracle_fp64(nθ):
    """test/test_cuda.jl:10-20 (there rtol 1e-10); here 1e-12 of each field's scale."""
    bodies, box = layout_bodies()
    g, o = pair(bodies, box, bonds=fcc.parent_bonds(bodies), **layout_kw(nθ=nθ))
    g.refresh()
    o.refresh()
    assert (o.grad.P > 0).sum() > 100
    nb_g, nb_o = g.neighbors, o.neighbors
    assert np.array_equal(nb_g.count, nb_o.count)
    for f in FIELDS:
        assert relerr(getattr(g.grad, f), getattr(o.grad, f)) < 1e-12, f


def near_ties(o, thr=3e-6):
    """Bodies with a node whose penetration depth |d| into a neighbour is
    below `thr`: FP32 computes d to ~1e-6, so the Heaviside g = J H(d) may
    legitimately flip there."""
    _, _, md = o.contact_counters()
    return md < thr


@pytest.mark.parametrize("nθ", [40, 64])
def test_gradients_fp32_vs_fp64_oracle(nθ):
    """FP32 bulk against the FP64 oracle: 1e-5 of each field's scale, excluding
    (and counting) bodies at an Overlap near-tie."""
    bodies, box = layout_bodies()
    bodies = as_f32_bodies(bodies)
    kw = layout_kw(nθ=nθ)
    g = G(bodies, box, bonds=fcc.parent_bonds(bodies), **{**kw, "T": np.float32})
    o = O(bodies, box, bonds=fcc.parent_bonds(bodies), **kw)
    g.refresh()
    o.refresh()
    tie = near_ties(o)
    keep = ~tie
    assert tie.sum() <= max(2, bodies.n // 10)
    for f in FIELDS:
        assert relerr(getattr(g.grad, f), getattr(o.grad, f), keep) < 1e-5, f


def test_single_body_fd_gradient_on_gpu():
    """test/test_energies.jl:73-85 on the GPU: FD rtol 1e-6, no force/torque."""
    from test_oracle import single_body
    for term in (fcc.Tension(0.37), fcc.PerimeterElasticity(0.5, 3.9)):
        coef = deformed_coef().reshape(-1, 1)
        mk = lambda c: G(fcc.Bodies.new([1.0], [2.0], [0.4], c, [1.2]), fcc.PeriodicBox(20.0, 20.0),
                         types=(fcc.BodyType(),), energies=(term,))
        sim = mk(coef).refresh()
        g = sim.grad
        assert g.gx[0] == 0 and g.gy[0] == 0 and g.gθ[0] == 0
        fd = np.zeros(10)
        h = 1e-6
        for r in range(1, 11):
            E = []
            for δ in (h, -h):
                c = coef.copy()
                c[r] += δ
                E.append(mk(c).refresh().body_energy())
            fd[r - 1] = (E[0] - E[1]) / (2 * h)
        assert np.allclose(g.gcoef[1:, 0], fd, rtol=1e-6, atol=1e-9)
        o, _ = single_body((term,))
        o.refresh()
        assert relerr(g.gcoef, o.grad.gcoef) < 1e-12


def test_cell_list_pressure_matches_brute_force():
    """test/test_contact.jl:69-86 on the GPU, including capacity regrowth."""
    bodies, box = jittered_monolayer()
    kw = dict(types=(fcc.BodyType(),), energies=(fcc.Overlap(1.0), fcc.LinearRepulsion(0.3)))
    sim = G(bodies, box, **kw).refresh()
    assert np.allclose(sim.grad.P, brute_force_pressure(sim), rtol=1e-12, atol=1e-12)
    small = G(bodies, box, nl_capacity=2, **kw).refresh()
    nb = small.neighbors
    assert nb.cap >= nb.count.max() > 2
    assert np.array_equal(small.grad.P, sim.grad.P)
    o = O(bodies, box, **kw).refresh()
    no, ng = o.neighbors, sim.neighbors
    for f in ("cellid", "perm", "start", "stop", "count"):
        assert np.array_equal(getattr(ng, f), getattr(no, f)), f
    for i in range(bodies.n):
        assert np.array_equal(ng.idx[:ng.count[i], i], no.idx[:no.count[i], i])


def test_two_discs_overlap_force_chunked():
    """test/test_contact.jl:88-96 at nθ = 8000 (multi-chunk node loop)."""
    from test_oracle import two_body
    d = 1.5
    coef = np.zeros((11, 2))
    coef[0] = 1
    bodies = fcc.Bodies.new([5.0, 5.0 + d], [5.0, 5.0], [0.3, -1.1], coef, [1.0, 1.0])
    g = G(bodies, fcc.PeriodicBox(10.0, 10.0), types=(fcc.BodyType(),), energies=(fcc.Overlap(1.0),), nθ=8000)
    gr = g.refresh().grad
    assert math.isclose(gr.gx[0], math.sqrt(4 - d * d), rel_tol=1e-3)
    assert math.isclose(gr.gx[1], -math.sqrt(4 - d * d), rel_tol=1e-3)
    assert abs(gr.gy[0]) < 1e-6
    o = two_body((fcc.Overlap(1.0),), d=d, nθ=8000)
    F = np.abs(o.grad.gx).max()  # gy and the torque vanish by symmetry: measure them on the force scale
    for f in ("gx", "gy", "gθ"):
        assert np.abs(getattr(gr, f) - getattr(o.grad, f)).max() < 1e-12 * F, f
    for f in ("gcoef", "P", "GR"):
        assert relerr(getattr(gr, f), getattr(o.grad, f)) < 1e-12, f


def test_nucleus_attraction_on_gpu():
    """test/test_contact.jl:122-133."""
    terms = (fcc.Overlap([[1.0, 1.0], [1.0, 1.0]], related=[[0.0, -2.0], [-2.0, 0.0]]),)

    def sim(d):
        coef = np.zeros((11, 2))
        coef[0] = 1
        b = fcc.Bodies.new([5.0, 5.0 + d], [5.0, 5.0], [0.3, -1.1], coef, [1.0, 0.4], type=[1, 2], parent=[1, 1])
        return G(b, fcc.PeriodicBox(10.0, 10.0), types=(fcc.BodyType(), fcc.BodyType()), energies=terms, nθ=400).refresh()

    p = sim(0.9).grad
    assert p.gx[1] > 0.1 and p.gx[0] < -0.1
    q = sim(0.3).grad
    assert abs(q.gx[1]) < 1e-10 and abs(q.gx[0]) < 1e-10


# ------------------------------------------------------------ one-step update
@pytest.mark.parametrize("drag", ["parent", "substrate"])
def test_one_step_matches_oracle_fp64(drag):
    """One Euler-Maruyama step (noise, parent drag, bonds, constraints):
    state increments within 1e-12 of their scale."""
    bodies, box = layout_bodies()
    kw = layout_kw(drag=drag)
    g, o = pair(bodies, box, bonds=fcc.parent_bonds(bodies), **kw)
    b0 = o.bodies
    g.step(1)
    o.step(1)
    bg, bo = g.bodies, o.bodies
    for f in ("x", "y", "θ", "coef"):
        dg = getattr(bg, f) - getattr(b0, f)
        do = getattr(bo, f) - getattr(b0, f)
        assert relerr(dg, do) < 1e-12, f
    assert np.array_equal(bg.imgx, bo.imgx) and np.array_equal(bg.imgy, bo.imgy)
    assert g.nsteps == o.nsteps == 1 and g.clock == 1
    assert math.isclose(g.t, o.t, rel_tol=0, abs_tol=1e-15)
    assert g.builds == o.builds == 1


def test_one_step_fp32_vs_fp64_oracle():
    bodies, box = layout_bodies()
    bodies = as_f32_bodies(bodies)
    kw = layout_kw(drag="substrate", energies=LAYOUT_ENERGIES[:4])
    g = G(bodies, box, **{**kw, "T": np.float32})
    o = O(bodies, box, **kw)
    o.refresh()
    keep = ~near_ties(o)
    b0 = o.bodies
    g.step(1)
    o.step(1)
    bg, bo = g.bodies, o.bodies
    for f in ("x", "y", "θ", "coef"):
        # the FP32 state resolves an increment only to the FP32 spacing of the
        # state itself: 1e-5 of the increments' scale plus 2 ulp of the state
        sg, so, s0 = getattr(bg, f), getattr(bo, f), getattr(b0, f)
        dg, do = sg - s0, so - s0
        tol = 1e-5 * np.abs(do).max() + 2 * np.spacing(np.abs(so).astype(np.float32)).astype(np.float64)
        assert (np.abs(dg - do)[..., keep] <= tol[..., keep]).all(), f


# ------------------------------------------------------------ trajectories
def test_short_fp32_trajectory_vs_fp64_oracle():
    """Five FP32 steps of a 64 x 64 monolayer against the FP64 oracle, same
    initial state and Philox stream.  Stated tolerance: 95% of the bodies
    within 4 FP32 ulps of their coordinates in position (~3e-5 in a box of
    side ~120) and 1e-6 in every shape coefficient, all within 2e-3: a node
    at an Overlap near-tie can flip its Heaviside contact in FP32 (a force
    jump J dphi R) and move its body by up to ~1e-3 within a few steps; the
    rest differ at FP32 rounding of the state."""
    bodies, box = fcc.hexagonal_monolayer(64, 64, packing=0.95, maxmode=10, rng=7)
    rng = np.random.default_rng(7)
    bodies.coef[1:] = 0.02 * (2 * rng.random((bodies.ncoef - 1, bodies.n)) - 1)
    bodies = as_f32_bodies(bodies)
    kw = dict(types=(fcc.BodyType(v0=0.06, Dr=0.01, μab=0.1),), energies=(fcc.Tension(0.01), fcc.Overlap(1.0)),
              dt=0.005, seed=7)
    g = G(bodies, box, T=np.float32, **kw).step(5)
    o = O(bodies, box, T=np.float64, **kw).step(5)
    bg, bo = g.bodies, o.bodies
    dr = np.hypot(bg.x + bg.imgx * box.Lx - bo.x - bo.imgx * box.Lx, bg.y + bg.imgy * box.Ly - bo.y - bo.imgy * box.Ly)
    dc = np.abs(bg.coef - bo.coef).max(axis=0)
    ulp = np.spacing(np.maximum(np.abs(bo.x), np.abs(bo.y)).astype(np.float32)).astype(np.float64)
    assert np.mean((dr < 4 * ulp) & (dc < 1e-6)) >= 0.95
    assert dr.max() < 2e-3 and dc.max() < 2e-3
    assert g.builds == o.builds


@pytest.mark.parametrize("mode", ["step", "run"])
def test_reference_n64_golden_on_gpu(ref_n64, mode):
    """The original C++ code's N = 64 trajectory (test/test_dynamics.jl:53-70)
    on the GPU in FP64, atol 1e-10 after 1001 and 4001 steps."""
    from test_oracle import compare_n64
    init, snaps = ref_n64
    bodies, box, kw = n64_sim(init)
    sim = G(bodies, box, **kw)
    for n in sorted(snaps):
        k = n - sim.nsteps
        sim.step(k) if mode == "step" else sim.run(k)
        compare_n64(sim, snaps[n], 1e-10)
    assert sim.nsteps == 4001


def test_short_trajectory_matches_oracle():
    """test/test_cuda.jl:123-131: 30 noisy FP64 steps, rtol 1e-8, equal builds."""
    bodies, box = layout_bodies()
    g, o = pair(bodies, box, bonds=fcc.parent_bonds(bodies), **layout_kw())
    g.step(30)
    o.step(30)
    bg, bo = g.bodies, o.bodies
    assert np.allclose(bg.x, bo.x, rtol=1e-8)
    assert np.allclose(bg.θ, bo.θ, rtol=1e-8)
    assert np.allclose(bg.coef, bo.coef, rtol=1e-8, atol=1e-12)
    assert g.builds == o.builds


def fast(**kw):
    """Fast cells and a thin skin: many rebuilds (test/test_cuda.jl:138-139)."""
    bodies, box = layout_bodies()
    return G(bodies, box, bonds=fcc.parent_bonds(bodies), **layout_kw(v0=2.0, skin=0.05, **kw))


def state(s):
    b = s.bodies
    return (b.x, b.y, b.θ, b.coef, b.imgx, b.imgy)


def same(a, b):
    return (all(np.array_equal(u, v) for u, v in zip(state(a), state(b))) and a.t == b.t and a.nsteps == b.nsteps
            and a.builds == b.builds)


def test_run_equals_step_bitwise():
    """Persistent multi-step launches == one launch per step, incl. many
    rebuilds, callbacks, a dt change and capacity regrowth
    (test/test_cuda.jl:133-185)."""
    a, b = fast(), fast()
    a.step(200)
    b.run(200)
    assert a.builds > 10
    assert same(a, b)
    a, b = fast(), fast()
    seen = []
    a.step(100)
    b.run(100, every=7, callback=lambda s: seen.append(s.nsteps))
    assert seen == list(range(7, 99, 7)) + [100]
    assert same(a, b)
    a.dt = b.dt = 0.004
    a.step(30)
    b.run(30)
    assert same(a, b)
    c, d = fast(nl_capacity=1), fast()
    c.run(60)
    d.step(60)
    assert same(c, d)
    assert c.neighbors.cap > 1
    e = fast()
    e.run(20, graph=False)
    f = fast()
    f.step(20)
    assert same(e, f)


def test_fp32_monolayer_overflow_regrows_inside_runs():
    """The FP32 step kernel of a lone monolayer (no parent drag: the fused
    step and its own rebuild phases) with a neighbour capacity of 1: lists
    overflow inside multi-step launches, the launch stops stepping, the host
    regrows and reruns the missing steps; the result equals step-by-step
    launches and a run with room from the start, bit for bit
    (src/neighbors.jl:226-233, test/test_cuda.jl:133-185)."""
    bodies, box = fcc.hexagonal_monolayer(12, 12, packing=0.97, maxmode=10, rng=3)
    bodies.coef[1:, :] = 0.03 * np.random.default_rng(8).standard_normal((bodies.ncoef - 1, bodies.n))
    kw = dict(types=(fcc.BodyType(v0=1.0, Dr=0.5, μab=0.1),), energies=(fcc.Tension(0.01), fcc.Overlap(1.0)),
              dt=0.005, seed=11, skin=0.05, T=np.float32)
    a = G(bodies, box, nl_capacity=1, **kw).run(120)
    b = G(bodies, box, nl_capacity=1, **kw).step(120)
    c = G(bodies, box, **kw).run(120)
    assert a.neighbors.cap > 1 and a.builds > 5
    assert same(a, b)
    assert all(np.array_equal(u, v) for u, v in zip(state(a), state(c)))


def test_skin_zero_rebuilds_every_step_and_agrees():
    """test/test_contact.jl:155-160: skin 0 vs 0.5 agree to 1e-10."""
    bodies, box = fcc.hexagonal_monolayer(6, 6, packing=0.97, rng=2)
    mk = lambda skin: G(bodies, box, types=(fcc.BodyType(v0=0.3, Dr=1.0, Dt=0.01, μab=1.0),),
                        energies=(fcc.Tension(0.1), fcc.Overlap(1.0), fcc.LinearRepulsion(0.3)), dt=0.01, skin=skin, seed=3)
    assert mk(0.0).step(10).builds == 10
    a, b = mk(0.0).step(100), mk(0.5).step(100)
    assert b.builds < a.builds
    assert np.allclose(b.bodies.x, a.bodies.x, rtol=1e-10)
    assert np.allclose(b.bodies.coef, a.bodies.coef, rtol=1e-10, atol=1e-14)


def test_concurrent_simulations_equal_sequential():
    """test/test_cuda.jl:187-196: one host thread (and stream) per simulation."""
    seq = [fast(seed=s).run(150) for s in (1, 2, 3)]
    par = [fast(seed=s) for s in (1, 2, 3)]
    ths = [threading.Thread(target=s.run, args=(150,)) for s in par]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    for a, b in zip(seq, par):
        assert np.array_equal(a.bodies.x, b.bodies.x) and np.array_equal(a.bodies.coef, b.bodies.coef)
    assert not np.array_equal(par[0].bodies.x, par[1].bodies.x)


def test_float32_runs():
    sim = fast(T=np.float32).step(50)
    b = sim.bodies
    assert np.isfinite(b.coef).all() and np.isfinite(b.x).all()


# ------------------------------------------------------------ dynamics cases
def test_isolated_cell_self_propels_gpu():
    """test/test_dynamics.jl:33-43 (one body, collapsed grid, boundary crossing)."""
    coef = np.zeros((11, 1))
    coef[0] = 1
    sim = G(fcc.Bodies.new([1.0], [1.0], [0.3], coef, [1.0]), fcc.PeriodicBox(5.0, 5.0),
            types=(fcc.BodyType(v0=0.5),), energies=(fcc.Tension(0.1), fcc.Overlap(1.0)), dt=0.01)
    sim.run(3000)
    X = fcc.unwrapped_positions(sim)[:, 0]
    assert np.allclose(X, [1 + 15 * math.cos(0.3), 1 + 15 * math.sin(0.3)], rtol=1e-8)
    b = sim.bodies
    assert 0 <= b.x[0] < 5 and 0 <= b.y[0] < 5
    assert math.isclose(b.θ[0], 0.3, rel_tol=1e-12)
    assert np.abs(b.coef[1:, 0]).max() < 1e-14
    assert math.isclose(sim.t, 30, rel_tol=1e-9)


def test_rotational_diffusion_gpu():
    """test/test_dynamics.jl:45-51."""
    N = 4000
    rng = np.random.default_rng(1)
    coef = np.zeros((11, N))
    coef[0] = 1
    sim = G(fcc.Bodies.new(rng.random(N), rng.random(N), np.zeros(N), coef, np.ones(N)), fcc.PeriodicBox(1.0, 1.0),
            types=(fcc.BodyType(Dr=0.1),), dt=0.01, seed=7).run(500)
    θ = sim.bodies.θ
    assert abs(np.mean(θ**2) / (2 * 0.1 * sim.t) - 1) < 0.1


def test_parents_on_gpu():
    """test/test_parents.jl:67-74 and :121-132 (carried nucleus, bond relaxation)."""
    coef = np.zeros((11, 3))
    coef[0] = 1
    mk = lambda x2: fcc.Bodies.new([5.0, x2, 1.0], [5.0, 5.0, 1.0], [0.3, -1.0, 2.0], coef, [1.0, 0.5, 1.0],
                                   type=[1, 2, 1], parent=[1, 1, 3])
    sim = G(mk(5.0), fcc.PeriodicBox(10.0, 10.0), types=(fcc.BodyType(v0=0.5), fcc.BodyType(drag="parent")), dt=0.01)
    sim.run(2000)
    X = fcc.unwrapped_positions(sim)
    assert np.allclose(X[:, 0], [5 + 10 * math.cos(0.3), 5 + 10 * math.sin(0.3)], rtol=1e-8)
    assert np.allclose(X[:, 1], X[:, 0], rtol=1e-12)
    μ, k, δ0, n = 2.0, 0.5, 0.2, 300
    b = mk(5.0 + δ0)
    sim = G(b, fcc.PeriodicBox(10.0, 10.0), types=(fcc.BodyType(), fcc.BodyType(μr=μ, drag="parent")),
            energies=(fcc.HarmonicBond(k),), bonds=fcc.parent_bonds(b), dt=0.01)
    sim.step(n)
    s = sim.bodies
    assert s.x[0] == 5.0 and s.y[0] == 5.0
    assert math.isclose(s.x[1] - 5.0, δ0 * (1 - μ * k * 0.01) ** n, rel_tol=1e-12)


def test_observables_on_gpu():
    """test/test_dynamics.jl:23-31, test/test_energies.jl:65-71, test/test_parents.jl:174-189."""
    bodies, box = fcc.hexagonal_monolayer(2, 2)
    bodies.coef[1:, :] = (0.05 * np.arange(1, 11))[:, None]
    sim = G(bodies, box, types=(fcc.BodyType(),), nθ=64)
    c = sim.bodies.coef
    assert np.all(np.hypot(c[1:6], c[6:11]).sum(0) <= math.sqrt(2 / 3) + 1e-12)
    assert np.allclose(fcc.areas(sim), math.pi, rtol=1e-12)
    coef = np.zeros((11, 1))
    coef[0] = 1
    one = G(fcc.Bodies.new([1.0], [2.0], [0.4], coef, [1.0]), fcc.PeriodicBox(20.0, 20.0), types=(fcc.BodyType(),),
            energies=(fcc.Tension(0.1),), nθ=64).refresh()
    assert math.isclose(fcc.body_energy(one), 0.1 * 2 * math.pi, rel_tol=1e-12)
    assert math.isclose(fcc.shape_index(one)[0], 2 * math.sqrt(math.pi), rel_tol=1e-12)
    cells, box = fcc.hexagonal_monolayer(4, 4)
    nb = fcc.with_nuclei(cells, ratio=0.5)
    nb.x[16] += 0.7
    nb.x[17] += 0.2
    sim = G(nb, box, types=(fcc.BodyType(), fcc.BodyType(drag="parent")), nθ=64)
    assert np.allclose(fcc.areas(sim, type=2), math.pi / 4, rtol=1e-12)
    assert np.allclose(fcc.areas(sim, type=1), math.pi, rtol=1e-12)
    assert len(fcc.shape_index(sim, type=2)) == 16
    p = fcc.protrusion(sim)
    assert np.isnan(p[:16]).all()
    assert abs(p[16] - 0.2) < 1e-12 and abs(p[17] + 0.3) < 1e-12


# --------------------------------------------------------- full-size workloads
def c2_bodies(nx=128, seed=1234):
    return fcc.polydisperse_monolayer(nx, nx, packing=0.95, maxmode=10, seed=seed)


C2_ENERGIES = (fcc.Tension(0.01), fcc.Overlap(1.0), fcc.PerimeterElasticity(0.1, 3.7))
C2_TYPES = (fcc.BodyType(v0=0.06, Dr=0.01, μab=0.1),)


def test_n16384_fp32_forces_vs_oracle():
    """The N = 16384 FP32 workload: forces of the whole monolayer (deformed by
    200 steps) against the FP64 oracle on the same FP32 state, 1e-5 of scale,
    near-ties excluded; neighbour lists identical."""
    bodies, box = c2_bodies()
    g = G(bodies, box, types=C2_TYPES, energies=C2_ENERGIES, dt=0.005, T=np.float32, seed=1234)
    g.run(200)
    state = g.bodies
    o = O(state, box, types=C2_TYPES, energies=C2_ENERGIES, dt=0.005, T=np.float64, seed=1234)
    g.set_state(state)
    g.refresh()
    o.refresh()
    keep = ~near_ties(o)
    assert keep.mean() > 0.95
    for f in ("gx", "gy", "gθ", "gcoef", "Ebody"):
        assert relerr(getattr(g.grad, f), getattr(o.grad, f), keep) < 1e-5, f


def test_n16384_fp32_one_step_vs_fp64_oracle():
    """One FP32 step of the N = 16384 workload through the fused step kernel
    (deformed by 200 steps; its own list rebuild and Philox draw) against one
    FP64 oracle step from the same FP32 state and clock: every increment
    within 1e-5 of its field's increment scale plus 2 FP32 ulp of the state,
    bodies at an Overlap near-tie excluded (at most 5%).  The rotational
    noise is the reference's Float32 draw (24-bit uniforms) on one side and
    its Float64 draw on the other: θ is also allowed the difference of the
    two draws times the noise amplitude sqrt(2 Dr dt) (it reaches 2e-5 of
    the increment where the Box-Muller radius uniform is small)."""
    bodies, box = c2_bodies()
    kw = dict(types=C2_TYPES, energies=C2_ENERGIES, dt=0.005, seed=1234)
    g = G(bodies, box, T=np.float32, **kw)
    g.run(200)
    state, clk = g.bodies, g.clock
    o = O(state, box, T=np.float64, **kw)
    o.set_state(state, clock=clk)
    o.refresh()
    keep = ~near_ties(o)
    assert keep.mean() > 0.95
    g.set_state(state, clock=clk)
    g.step(1)
    o.step(1)
    assert g.clock == o.clock == clk + 1
    bg, bo = g.bodies, o.bodies
    z32, z64 = fcc.philox_noise(1234, clk, bodies.n, np.float32), fcc.philox_noise(1234, clk, bodies.n, np.float64)
    noise = {"θ": math.sqrt(2 * C2_TYPES[0].Dr * 0.005) * np.abs(z32[2] - z64[2])}
    for f in ("x", "y", "θ", "coef"):
        sg, so, s0 = getattr(bg, f), getattr(bo, f), getattr(state, f)
        dg, do = sg - s0, so - s0
        tol = 1e-5 * np.abs(do).max() + 2 * np.spacing(np.abs(so).astype(np.float32)).astype(np.float64)
        tol = tol + noise.get(f, 0.0)
        err = np.abs(dg - do)[..., keep]
        assert (err <= tol[..., keep]).all(), (f, float((err / tol[..., keep]).max()))
    assert np.array_equal(bg.imgx, bo.imgx) and np.array_equal(bg.imgy, bo.imgy)


def test_n16384_fp64_forces_and_one_step_match_oracle():
    """The N = 16384 workload in FP64 (deformed by 200 steps on the GPU):
    every gradient field of the state at 1e-12 of its scale, then one step
    from the same state and clock with increments at 1e-12 of their scale
    plus two ulp of the state (positions up to 250: one ulp of the sum
    x + dx is 6e-14); neighbour counts identical."""
    bodies, box = c2_bodies()
    kw = dict(types=C2_TYPES, energies=C2_ENERGIES, dt=0.005, seed=1234, T=np.float64)
    g = G(bodies, box, **kw)
    g.run(200)
    state, clk = g.bodies, g.clock
    o = O(state, box, **kw)
    o.set_state(state, clock=clk)
    g.set_state(state, clock=clk)
    g.refresh()
    o.refresh()
    assert np.array_equal(g.neighbors.count, o.neighbors.count)
    keep = ~near_ties(o, 1e-12)  # FP64 rounding decides a Heaviside only this close to a tie
    assert keep.mean() > 0.999
    for f in ("gx", "gy", "gθ", "gcoef", "Ebody"):
        assert relerr(getattr(g.grad, f), getattr(o.grad, f), keep) < 1e-12, f
    g.set_state(state, clock=clk)
    o.set_state(state, clock=clk)
    g.step(1)
    o.step(1)
    bg, bo = g.bodies, o.bodies
    for f in ("x", "y", "θ", "coef"):
        sg, so, s0 = getattr(bg, f), getattr(bo, f), getattr(state, f)
        dg, do = sg - s0, so - s0
        tol = 1e-12 * np.abs(do).max() + 2 * np.spacing(np.abs(so))
        err = np.abs(dg - do)[..., keep]
        assert (err <= tol[..., keep]).all(), (f, float((err / tol[..., keep]).max()))
    assert np.array_equal(bg.imgx, bo.imgx) and np.array_equal(bg.imgy, bo.imgy)


@pytest.mark.parametrize("nx", [128, 256, 512])
def test_full_size_invariants(nx):
    """N = 16384, 65536, 262144 FP32: finite state, area πR0² kept by the FP64
    a0, shape bound, and every interacting pair inside the neighbour lists."""
    bodies, box = c2_bodies(nx)
    sim = G(bodies, box, types=C2_TYPES, energies=C2_ENERGIES, dt=0.005, T=np.float32, seed=1234)
    sim.run(100)
    b = sim.bodies
    assert np.isfinite(b.x).all() and np.isfinite(b.coef).all()
    A = fcc.areas(sim)
    assert np.allclose(A, math.pi * f32(bodies.R0) ** 2, rtol=2e-5)
    K = 9
    s = np.hypot(b.coef[1:K + 1], b.coef[K + 1:]).sum(0)
    assert (s <= math.sqrt(2 / 3) * (1 + 1e-6)).all()
    sim.update_neighbors(force=True)
    nb = sim.neighbors
    rng = np.random.default_rng(0)
    rmax = f32(bodies.R0) * (b.coef[0] + s)  # R0 (a0 + sum sqrt(a^2 + b^2)), src/geometry.jl:223-225
    for i in rng.choice(b.n, 64, replace=False):
        dx = fcc.minimum_image(b.x - b.x[i], box.Lx)
        dy = fcc.minimum_image(b.y - b.y[i], box.Ly)
        close = np.nonzero(np.hypot(dx, dy) < rmax + rmax[i])[0]
        close = set(close.tolist()) - {i}
        listed = set((nb.idx[:nb.count[i], i] - 1).tolist())
        assert close <= listed


@pytest.mark.parametrize("drag", ["parent", "substrate"])
def test_typed_bodies_full_size(drag):
    """The cells-with-nuclei configuration (4096 cells of R0 = 1 and 4096
    nuclei of R0 = 0.5 at packing 0.9, OnTypes tensions 0.01 / 0.05, Overlap
    for all pairs, nuclei without self-propulsion), FP32, 200 steps: finite
    state, areas pi R0^2 kept, shape bound, every type's shape index >= 2 sqrt(pi)."""
    cells, box = fcc.hexagonal_monolayer(64, 64, packing=0.9, maxmode=10, rng=1234)
    nb = fcc.with_nuclei(cells, ratio=0.5)
    kw = dict(types=(fcc.BodyType(v0=0.06, Dr=0.01, μab=0.1), fcc.BodyType(v0=0.0, drag=drag, μab=0.1)),
              energies=(fcc.OnTypes(fcc.Tension(0.01), 1), fcc.OnTypes(fcc.Tension(0.05), 2), fcc.Overlap(1.0)),
              dt=0.005, seed=1234)
    sim = G(nb, box, T=np.float32, **kw)
    sim.run(200)
    b = sim.bodies
    assert b.n == 8192 and np.isfinite(b.x).all() and np.isfinite(b.coef).all()
    assert np.allclose(fcc.areas(sim), math.pi * f32(nb.R0) ** 2, rtol=2e-5)
    s = np.hypot(b.coef[1:10], b.coef[10:]).sum(0)
    assert (s <= math.sqrt(2 / 3) * (1 + 1e-6)).all()
    for t in (1, 2):
        assert (fcc.shape_index(sim, type=t) >= 2 * math.sqrt(math.pi) * (1 - 1e-6)).all()
    assert sim.nsteps == 200 and sim.builds >= 1
