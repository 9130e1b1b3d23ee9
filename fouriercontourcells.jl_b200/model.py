"""Host-side data model mirroring the reference's public types.

Names, argument meanings and validation follow FourierContourCells.jl so that
scripts and tests read like the reference's own:

- ``BodyType``            src/bodies.jl:30-45
- ``Bodies``, ``vcat``    src/bodies.jl:62-102
- ``PeriodicBox``         src/box.jl:6-9
- energy terms            src/energies/body_terms.jl, contact.jl, bonds.jl,
                          interface.jl:278-298 (``OnTypes``)
- ``hexagonal_monolayer``, ``with_nuclei``   src/initial.jl:11-53
- ``parent_bonds``        src/energies/bonds.jl:37

Julia's ``ArgumentError`` and ``DimensionMismatch`` map to the Python
exceptions of the same names below.  Random initial orientations use numpy's
seeded ``Generator`` (the reference's Xoshiro streams need Julia).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


class ArgumentError(ValueError):
    """Raised where the reference throws ``ArgumentError``."""


class DimensionMismatch(ValueError):
    """Raised where the reference throws ``DimensionMismatch``."""


class DeviceError(RuntimeError):
    """CUDA or device-side failure reported by the native library."""


class PoolFull(RuntimeError):
    """A pool has no free slot, bodies or grid cells for a simulation now."""


# --------------------------------------------------------------------- types
@dataclass(frozen=True)
class BodyType:
    """Dynamical parameters of one body type (src/bodies.jl:30-45).

    Accepts the reference's keyword names ``v0, Dr, Dt, μr, μθ, μab, drag``
    (ASCII aliases ``mu_r, mu_theta, mu_ab``).  ``maxmode`` (not in the
    reference, whose types all share the simulation's modes) limits this
    type's shape modes to n = 2..maxmode; 0 keeps every mode."""

    v0: float = 0.0
    Dr: float = 0.0
    Dt: float = 0.0
    mu_r: float = 1.0
    mu_theta: float = 1.0
    mu_ab: float = 0.1
    drag: str = "substrate"
    maxmode: int = 0

    def __init__(self, v0=0.0, Dr=0.0, Dt=0.0, mu_r=None, mu_theta=None, mu_ab=None, drag="substrate", maxmode=0,
                 **kw):
        μr = kw.pop("μr", None)
        μθ = kw.pop("μθ", None)
        μab = kw.pop("μab", None)
        if kw:
            raise TypeError(f"BodyType got unexpected keyword arguments {sorted(kw)}")
        drag = str(drag).lstrip(":")
        if drag not in ("substrate", "parent"):
            raise ArgumentError(f"drag must be :substrate or :parent, got :{drag}")
        object.__setattr__(self, "v0", float(v0))
        object.__setattr__(self, "Dr", float(Dr))
        object.__setattr__(self, "Dt", float(Dt))
        object.__setattr__(self, "mu_r", float(mu_r if mu_r is not None else (μr if μr is not None else 1.0)))
        object.__setattr__(self, "mu_theta", float(mu_theta if mu_theta is not None else (μθ if μθ is not None else 1.0)))
        object.__setattr__(self, "mu_ab", float(mu_ab if mu_ab is not None else (μab if μab is not None else 0.1)))
        object.__setattr__(self, "drag", drag)
        if int(maxmode) != maxmode or maxmode < 0:
            raise ArgumentError(f"maxmode must be a non-negative integer, got {maxmode}")
        object.__setattr__(self, "maxmode", int(maxmode))

    @property
    def parent_drag(self) -> bool:
        return self.drag == "parent"


# ---------------------------------------------------------------- energies
class EnergyTerm:
    """Supertype of the built-in energy terms (src/energies/interface.jl:27)."""

    kind = 0


class BodyTerm(EnergyTerm):
    pass


class ContactTerm(EnergyTerm):
    pass


class BondTerm(EnergyTerm):
    pass


@dataclass(frozen=True)
class Tension(BodyTerm):
    """Line tension η·l (src/energies/body_terms.jl:8-18)."""

    eta: float
    kind = 1

    def __init__(self, η):
        object.__setattr__(self, "eta", float(η))


@dataclass(frozen=True)
class PerimeterElasticity(BodyTerm):
    """λ (l - p0 √(π R0²))² (src/energies/body_terms.jl:28-34)."""

    lam: float
    p0: float
    kind = 2

    def __init__(self, λ, p0):
        object.__setattr__(self, "lam", float(λ))
        object.__setattr__(self, "p0", float(p0))


@dataclass(frozen=True)
class Overlap(ContactTerm):
    """Excluded volume g(d) = J·H(d) with per-type-pair couplings
    (src/energies/contact.jl:12-28).  ``J`` and ``related`` are scalars or
    square ``ntypes × ntypes`` tables indexed ``[type_i - 1, type_j - 1]``."""

    J: tuple
    Jrelated: tuple
    kind = 3

    def __init__(self, J, related=None):
        Jm = np.atleast_2d(np.asarray(J, dtype=np.float64))
        Rm = Jm if related is None else np.atleast_2d(np.asarray(related, dtype=np.float64))
        if Jm.ndim != 2 or Jm.shape[0] != Jm.shape[1] or Rm.shape != Jm.shape:
            raise DimensionMismatch("coupling tables must be square and equal-sized")
        object.__setattr__(self, "J", tuple(map(tuple, Jm)))
        object.__setattr__(self, "Jrelated", tuple(map(tuple, Rm)))

    def pressure(self, d, ti, tj, related):
        """g(d) for 1-based types (src/energies/contact.jl:25-28)."""
        tab = self.Jrelated if related else self.J
        return tab[ti - 1][tj - 1] if d >= 0 else 0.0


@dataclass(frozen=True)
class LinearRepulsion(ContactTerm):
    """g(d) = k·d for d > 0 (src/energies/contact.jl:37-41)."""

    k: float
    kind = 4

    def __init__(self, k):
        object.__setattr__(self, "k", float(k))

    def pressure(self, d, ti, tj, related):
        return self.k * d if d > 0 else 0.0


@dataclass(frozen=True)
class HarmonicBond(BondTerm):
    """(k/2)(|Δ| - r0)² between bonded centres (src/energies/bonds.jl:12-29)."""

    k: float
    r0: float = 0.0
    kind = 5

    def __init__(self, k, r0=0.0):
        object.__setattr__(self, "k", float(k))
        object.__setattr__(self, "r0", float(r0))


class UserTerm(EnergyTerm):
    """A user-defined term compiled into the library (include/fcc_user_terms.h):
    the C++ functor at ``index`` of its kind's table, with parameters ``a``,
    ``b``.  The reference's user terms are Julia structs with methods
    (src/energies/interface.jl:27-106); here they are C++ functors, since a
    Julia closure cannot cross the C ABI."""

    index = 0

    def __init__(self, a=0.0, b=0.0, index=None):
        self.a, self.b = float(a), float(b)
        if index is not None:
            self.index = int(index)

    def __eq__(self, other):
        return type(self) is type(other) and (self.index, self.a, self.b) == (other.index, other.a, other.b)

    def __hash__(self):
        return hash((type(self).__name__, self.index, self.a, self.b))

    def __repr__(self):
        return f"{type(self).__name__}(a={self.a}, b={self.b}, index={self.index})"


class UserBodyTerm(UserTerm, BodyTerm):
    """A compiled user BodyTerm: E = F(Q), Q_j = ∮ q_j(R, R', R'') dφ."""

    kind = 6


class UserContactTerm(UserTerm, ContactTerm):
    """A compiled user ContactTerm: energy density g(d) with an interaction range."""

    kind = 7


class UserBondTerm(UserTerm, BondTerm):
    """A compiled user BondTerm: bond energy gradient dE/dΔ."""

    kind = 8


class Bending(UserBodyTerm):
    """κ ∮ c² ds, the reference README's user-term example (README.md:118-121);
    entry 0 of the compiled body terms."""

    index = 0

    def __init__(self, κ):
        super().__init__(κ, 0.0)


class ShapeIndexElasticity(UserBodyTerm):
    """k (P / √A - p0)² of the perimeter P and area A (two integrals); entry 1
    of the compiled body terms."""

    index = 1

    def __init__(self, k, p0):
        super().__init__(k, p0)


class Adhesion(UserContactTerm):
    """Energy density -ε in a band of width w outside a neighbour's contour
    (interaction range w); entry 0 of the compiled contact terms."""

    index = 0

    def __init__(self, ε, w):
        super().__init__(ε, w)


class QuarticBond(UserBondTerm):
    """k |Δ|⁴ / 4 between bonded centres; entry 0 of the compiled bond terms."""

    index = 0

    def __init__(self, k):
        super().__init__(k, 0.0)


@dataclass(frozen=True)
class OnTypes(EnergyTerm):
    """Restrict ``term`` to bodies whose type is in ``types``
    (src/energies/interface.jl:278-298)."""

    term: EnergyTerm
    types: tuple

    def __init__(self, term, *types):
        if isinstance(term, OnTypes):
            # nested restriction: intersection of the type sets
            types = tuple(t for t in types if t in term.types)
            term = term.term
        object.__setattr__(self, "term", term)
        object.__setattr__(self, "types", tuple(int(t) for t in types))

    @property
    def kind(self):
        return self.term.kind


def is_body_term(t):
    return isinstance(t, BodyTerm) or (isinstance(t, OnTypes) and is_body_term(t.term))


def is_contact_term(t):
    return isinstance(t, ContactTerm) or (isinstance(t, OnTypes) and is_contact_term(t.term))


def is_bond_term(t):
    return isinstance(t, BondTerm) or (isinstance(t, OnTypes) and is_bond_term(t.term))


# ------------------------------------------------------------------- state
@dataclass
class PeriodicBox:
    """Periodic box [0, Lx) × [0, Ly) (src/box.jl:6-9)."""

    Lx: float
    Ly: float


def minimum_image(d, L):
    """d - L·round(d/L), round half to even (src/box.jl:14)."""
    return d - L * np.rint(np.asarray(d) / L)


def wrap(x, L):
    """Map x into [0, L) and return (x', periods) (src/box.jl:21-30)."""
    s = math.floor(x / L)
    xp = x - s * L
    if xp >= L:
        xp = 0.0
        s += 1
    return xp, int(s)


@dataclass
class Bodies:
    """Structure-of-arrays body state (src/bodies.jl:62-86).

    ``coef`` is ``ncoef × N`` (column i = [a0; a2..aM; b2..bM] of body i),
    kept in Fortran (column-major) order as Julia stores it, so that a body's
    coefficients are contiguous; ``type`` and ``parent`` are 1-based ids."""

    x: np.ndarray
    y: np.ndarray
    θ: np.ndarray
    imgx: np.ndarray
    imgy: np.ndarray
    coef: np.ndarray
    R0: np.ndarray
    type: np.ndarray
    parent: np.ndarray

    @classmethod
    def new(cls, x, y, θ, coef, R0, type=1, parent=None):
        """Bodies(x, y, θ, coef, R0; type = 1, parent = 1:N) (src/bodies.jl:79-86)."""
        x = np.array(x, dtype=np.float64).ravel()
        N = len(x)
        y = np.array(y, dtype=np.float64).ravel()
        θ = np.array(θ, dtype=np.float64).ravel()
        R0 = np.array(R0, dtype=np.float64).ravel()
        coef = np.array(coef, dtype=np.float64, order="F")
        if coef.ndim == 1:
            coef = np.asfortranarray(coef.reshape(-1, 1))
        if not (len(y) == len(θ) == len(R0) == N and coef.shape[1] == N):
            raise DimensionMismatch("inconsistent body array lengths")
        typ = np.full(N, int(type), dtype=np.int32) if np.isscalar(type) else np.array(type, dtype=np.int32).ravel()
        par = np.arange(1, N + 1, dtype=np.int32) if parent is None else np.array(parent, dtype=np.int32).ravel()
        if len(typ) != N or len(par) != N:
            raise DimensionMismatch("inconsistent body array lengths")
        return cls(x, y, θ, np.zeros(N, np.int32), np.zeros(N, np.int32), coef, R0, typ, par)

    @property
    def theta(self):
        return self.θ

    @property
    def n(self):
        return len(self.x)

    @property
    def ncoef(self):
        return self.coef.shape[0]

    def copy(self):
        return Bodies(*(np.array(getattr(self, f)) for f in ("x", "y", "θ", "imgx", "imgy", "coef", "R0", "type", "parent")))


def nbodies(b) -> int:
    return b.n if isinstance(b, Bodies) else b.nbodies


def vcat(*bs: Bodies) -> Bodies:
    """Concatenate body sets, shifting parent ids with their set (src/bodies.jl:96-102)."""
    offs = np.cumsum([0] + [b.n for b in bs[:-1]])
    cat = lambda f: np.concatenate([getattr(b, f) for b in bs])
    parent = np.concatenate([b.parent + np.int32(o) for b, o in zip(bs, offs)]).astype(np.int32)
    return Bodies(cat("x"), cat("y"), cat("θ"), cat("imgx").astype(np.int32), cat("imgy").astype(np.int32),
                  np.asfortranarray(np.hstack([b.coef for b in bs])), cat("R0"), cat("type").astype(np.int32), parent)


def _rng(rng, seed):
    if rng is None:
        return np.random.default_rng(seed)
    if isinstance(rng, (int, np.integer)):
        return np.random.default_rng(int(rng))
    return rng


def hexagonal_monolayer(nx, ny, packing=0.95, R0=1.0, maxmode=6, rng=None):
    """Circular cells on a hexagonal lattice at area fraction ``packing``
    (src/initial.jl:11-29); returns ``(bodies, box)``.  Orientations are
    uniform on [0, 2π) from ``rng`` (a numpy Generator or an integer seed;
    default seed 1)."""
    if ny % 2 != 0:
        raise ArgumentError("ny must be even for a periodic hexagonal lattice")
    N = nx * ny
    r = R0 * math.sqrt(math.pi / (2 * math.sqrt(3) * packing))
    box = PeriodicBox(2 * r * nx, math.sqrt(3) * r * ny)
    n = np.arange(N)
    row, col = np.divmod(n, nx)
    x = (2 * col + (row % 2)) * r
    y = math.sqrt(3) * r * row
    θ = 2 * math.pi * _rng(rng, 1).random(N)
    coef = np.zeros((2 * maxmode - 1, N), order="F")
    coef[0, :] = 1.0
    return Bodies.new(x, y, θ, coef, np.full(N, float(R0))), box


def with_nuclei(cells: Bodies, ratio=0.5, type=2, rng=None):
    """Append one round nucleus per body (src/initial.jl:41-53)."""
    N = cells.n
    coef = np.zeros(cells.coef.shape, order="F")
    coef[0, :] = 1.0
    θ = 2 * math.pi * _rng(rng, 2).random(N)
    nuclei = Bodies.new(cells.x.copy(), cells.y.copy(), θ, coef, ratio * cells.R0, type=type)
    nuclei.imgx[:] = cells.imgx
    nuclei.imgy[:] = cells.imgy
    bodies = vcat(cells, nuclei)
    bodies.parent[N:2 * N] = np.arange(1, N + 1, dtype=np.int32)
    return bodies


def parent_bonds(b: Bodies):
    """One bond between every body and its parent (src/energies/bonds.jl:37)."""
    return [(i + 1, int(p)) for i, p in enumerate(b.parent) if p != i + 1]


def polydisperse_monolayer(nx, ny, packing=0.95, maxmode=10, mean=1.0, sd=0.1, lo=0.8, hi=1.2, seed=1234):
    """Hexagonal lattice at unit spacing radius with per-body radius scales
    R0 ~ Normal(mean, sd) clipped to [lo, hi] (the polydisperse monolayer of
    the N = 16384 workload; the lattice spacing stays that of R0 = mean)."""
    rng = np.random.default_rng(seed)
    bodies, box = hexagonal_monolayer(nx, ny, packing=packing, R0=mean, maxmode=maxmode, rng=rng)
    bodies.R0[:] = np.clip(rng.normal(mean, sd, bodies.n), lo, hi)
    return bodies, box
