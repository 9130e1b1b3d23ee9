"""Compiled user terms (include/fcc_user_terms.h) on the GPU (marked ``gpu``),
against the CPU oracle, which compiles the same functors.  The reference's
user terms are Julia methods on new structs (src/energies/interface.jl:27-106,
README.md:103-160); the functors here restate its own examples (Bending of
README.md:118-121 needs R'') and cover each kind: a two-integral body term
(shape-index elasticity), a contact term with an interaction range
(adhesion) and a bond term (quartic bond).

Tolerances as for the built-in terms: forces and every gradient buffer at
1e-12 of each field's scale in FP64; FP32 against the FP64 oracle at 1e-5
with Heaviside flips excluded (at most 10%, a small system); 30 noisy FP64
steps at rtol 1e-8 with equal rebuild counts (test/test_cuda.jl:31-39);
persistent launches equal one launch per step bit for bit."""

import numpy as np
import pytest

from conftest import fcc, oracle

pytestmark = pytest.mark.gpu

G = fcc.Simulation
O = oracle.OracleSimulation
FIELDS = ("GR", "GD", "GDD", "P", "gx", "gy", "gθ", "glab", "gcoef", "Ebody")


def relerr(a, b, keep=None):
    a, b = np.asarray(a, float), np.asarray(b, float)
    scale = max(float(np.abs(b).max()), 1e-300)
    if keep is not None:
        a, b = a[..., keep], b[..., keep]
    return float(np.abs(a - b).max() / scale) if a.size else 0.0


def system(T=np.float64, nθ=40, **kw):
    """Cells with nuclei, deformed, with every user-term kind in play."""
    cells, box = fcc.hexagonal_monolayer(5, 4, packing=0.97, maxmode=6, rng=2)
    bodies = fcc.with_nuclei(cells)
    bodies.coef[1:, :] = 0.04 * np.random.default_rng(5).standard_normal((bodies.ncoef - 1, bodies.n))
    energies = (fcc.Tension(0.1), fcc.Bending(0.02), fcc.OnTypes(fcc.ShapeIndexElasticity(0.05, 3.7), 1),
                fcc.Overlap([[1.0, 1.0], [1.0, 1.0]], related=[[1.0, -2.0], [-2.0, 1.0]]),
                fcc.Adhesion(0.3, 0.12), fcc.HarmonicBond(0.2), fcc.QuarticBond(0.5))
    args = dict(types=(fcc.BodyType(v0=0.2, Dr=0.1), fcc.BodyType(Dr=0.1, drag="parent")), energies=energies,
                bonds=fcc.parent_bonds(bodies), nθ=nθ, T=T, seed=7)
    args.update(kw)
    return bodies, box, args


def test_user_terms_forces_match_oracle_fp64():
    bodies, box, kw = system()
    g, o = G(bodies, box, **kw).refresh(), O(bodies, box, **kw).refresh()
    assert np.abs(o.grad.GDD).max() > 0 and (np.asarray(o.grad.P) < 0).any()  # R'' and the adhesion band act
    for f in FIELDS:
        assert relerr(getattr(g.grad, f), getattr(o.grad, f)) < 1e-12, f
    assert np.array_equal(g.neighbors.count, o.neighbors.count)  # lists widened by the interaction range


def test_user_terms_fp32_vs_fp64_oracle():
    bodies, box, kw = system()
    b32 = bodies.copy()
    for f in ("x", "y", "θ", "coef", "R0"):
        setattr(b32, f, np.asfortranarray(np.asarray(getattr(b32, f), np.float32).astype(np.float64)))
    g = G(b32, box, **{**kw, "T": np.float32}).refresh()
    o = O(b32, box, **kw).refresh()
    flip = np.abs(np.asarray(g.grad.P) - np.asarray(o.grad.P)).max(axis=0) >= 0.15  # smallest jump: 0.3 / 2
    assert flip.mean() <= 0.1
    for f in ("gx", "gy", "gθ", "gcoef", "Ebody"):
        assert relerr(getattr(g.grad, f), getattr(o.grad, f), ~flip) < 1e-5, f


def test_user_terms_short_trajectory_fp64():
    bodies, box, kw = system()
    g, o = G(bodies, box, **kw), O(bodies, box, **kw)
    g.step(30)
    o.step(30)
    bg, bo = g.bodies, o.bodies
    assert np.allclose(bg.x, bo.x, rtol=1e-8)
    assert np.allclose(bg.θ, bo.θ, rtol=1e-8)
    assert np.allclose(bg.coef, bo.coef, rtol=1e-8, atol=1e-12)
    assert g.builds == o.builds


@pytest.mark.parametrize("T", [np.float32, np.float64])
def test_user_terms_run_equals_step(T):
    bodies, box, kw = system(T=T)
    a, b = G(bodies, box, **kw), G(bodies, box, **kw)
    a.step(60)
    b.run(60)
    for f in ("x", "y", "θ", "coef", "imgx", "imgy"):
        assert np.array_equal(getattr(a.bodies, f), getattr(b.bodies, f)), f
    assert a.builds == b.builds


def test_user_terms_limits():
    bodies, box, kw = system(nθ=64)
    with pytest.raises(fcc.DeviceError):  # one contour chunk only
        G(bodies, box, **kw)
    bodies, box, kw = system()
    pool = fcc.Pool(T=np.float64, max_bodies=64, max_cells=1024, max_sims=2)
    with pytest.raises(fcc.DeviceError):  # pools run built-in terms only
        pool.add(bodies, box, horizon=10, **{k: v for k, v in kw.items() if k not in ("nθ", "T")})
