"""ctypes mirror of include/fcc.h and marshalling between the host model
(``model.py``) and the C ABI.

The structs here are byte-for-byte the ones in fcc.h; ``build_params`` turns
a reference-style ``Simulation(bodies, box; types, energies, ...)`` call into
an ``fcc_params`` (src/simulation.jl:66-105), and ``BodiesBuffer`` holds the
numpy arrays behind an ``fcc_bodies_host``.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from .model import (ArgumentError, DimensionMismatch, DeviceError, PoolFull, BodyType, Bodies, OnTypes, Tension,
                    PerimeterElasticity, Overlap, LinearRepulsion, HarmonicBond, UserTerm, is_body_term,
                    is_contact_term, is_bond_term)

MAX_TYPES = 8
MAX_TERMS = 16
MAX_MODES = 9

(FCC_OK, FCC_ERR_ARGUMENT, FCC_ERR_DIMENSION, FCC_ERR_CUDA, FCC_ERR_UNSUPPORTED, FCC_ERR_DEVICE, FCC_ERR_NOMEM,
 FCC_ERR_FULL) = range(8)
POOL_ALIGN = 8

c_double_p = C.POINTER(C.c_double)
c_int32_p = C.POINTER(C.c_int32)


class FccTerm(C.Structure):
    _fields_ = [("kind", C.c_int32), ("ntypes_on", C.c_int32), ("types_on", C.c_int32 * MAX_TYPES),
                ("a", C.c_double), ("b", C.c_double), ("nJ", C.c_int32),
                ("J", C.c_double * (MAX_TYPES * MAX_TYPES)), ("Jrel", C.c_double * (MAX_TYPES * MAX_TYPES)),
                ("user", C.c_int32)]


class FccBodyType(C.Structure):
    _fields_ = [("v0", C.c_double), ("Dr", C.c_double), ("Dt", C.c_double), ("mu_r", C.c_double),
                ("mu_theta", C.c_double), ("mu_ab", C.c_double), ("parent_drag", C.c_int32),
                ("maxmode", C.c_int32)]


class FccParams(C.Structure):
    _fields_ = [("Lx", C.c_double), ("Ly", C.c_double), ("dt", C.c_double), ("ntheta", C.c_int32),
                ("precision", C.c_int32), ("seed", C.c_uint64), ("skin", C.c_double),
                ("ntypes", C.c_int32), ("types", C.POINTER(FccBodyType)),
                ("nterms", C.c_int32), ("terms", C.POINTER(FccTerm)),
                ("nbonds", C.c_int64), ("bonds", c_int32_p), ("nl_capacity", C.c_int32)]


class FccBodiesHost(C.Structure):
    _fields_ = [("n", C.c_int64), ("ncoef", C.c_int32), ("x", c_double_p), ("y", c_double_p),
                ("theta", c_double_p), ("imgx", c_int32_p), ("imgy", c_int32_p), ("coef", c_double_p),
                ("R0", c_double_p), ("type", c_int32_p), ("parent", c_int32_p)]


class FccGradientsHost(C.Structure):
    _fields_ = [(f, c_double_p) for f in ("GR", "GD", "GDD", "P", "gx", "gy", "gtheta", "glab", "gcoef", "Ebody")]


class FccGeometryHost(C.Structure):
    _fields_ = [(f, c_double_p) for f in ("lab", "labR0", "R", "dR", "ddR", "rmax")]


class FccNeighborsHost(C.Structure):
    _fields_ = [(f, c_int32_p) for f in ("cellid", "perm", "start", "stop", "idx", "count")]


class FccPoolParams(C.Structure):
    _fields_ = [("precision", C.c_int32), ("ntheta", C.c_int32), ("max_bodies", C.c_int64),
                ("max_cells", C.c_int64), ("max_sims", C.c_int32), ("nl_capacity", C.c_int32),
                ("max_children", C.c_int32), ("max_bonds", C.c_int32)]


FCC_CALLBACK = C.CFUNCTYPE(None, C.c_void_p, C.c_void_p)


def dptr(a):
    return None if a is None else a.ctypes.data_as(c_double_p)


def iptr(a):
    return None if a is None else a.ctypes.data_as(c_int32_p)


def precision_bits(T) -> int:
    """T = Float64/Float32 (numpy dtype, type, or name) -> 64/32."""
    if T in (64, 32):
        return int(T)
    name = str(np.dtype(T) if not isinstance(T, str) else T).lower()
    if name in ("float64", "f8", "double"):
        return 64
    if name in ("float32", "f4", "single", "float"):
        return 32
    raise ArgumentError(f"unsupported precision {T!r}: use Float64 or Float32")


def _term_struct(term) -> FccTerm:
    ft = FccTerm()
    inner = term
    if isinstance(term, OnTypes):
        inner = term.term
        if len(term.types) > MAX_TYPES:
            raise ArgumentError("OnTypes: at most 8 types")
        ft.ntypes_on = len(term.types)
        for u, t in enumerate(term.types):
            ft.types_on[u] = int(t)
    ft.kind = inner.kind
    if isinstance(inner, Tension):
        ft.a = inner.eta
    elif isinstance(inner, PerimeterElasticity):
        ft.a, ft.b = inner.lam, inner.p0
    elif isinstance(inner, LinearRepulsion):
        ft.a = inner.k
    elif isinstance(inner, HarmonicBond):
        ft.a, ft.b = inner.k, inner.r0
    elif isinstance(inner, UserTerm):
        ft.a, ft.b, ft.user = inner.a, inner.b, inner.index
    elif isinstance(inner, Overlap):
        J = np.asarray(inner.J, dtype=np.float64)
        R = np.asarray(inner.Jrelated, dtype=np.float64)
        n = J.shape[0]
        if n > MAX_TYPES:
            raise ArgumentError("Overlap: at most 8 types")
        ft.nJ = n
        # column-major (ti, tj) -> (ti-1) + n*(tj-1), like Julia's SMatrix
        for tj in range(n):
            for ti in range(n):
                ft.J[ti + n * tj] = J[ti, tj]
                ft.Jrel[ti + n * tj] = R[ti, tj]
    else:
        raise ArgumentError("energy terms must be BodyTerms, ContactTerms or BondTerms")
    return ft


class ParamsBuffer:
    """An ``fcc_params`` with the arrays it points to kept alive."""

    def __init__(self, box, types, energies, bonds, dt, nθ, T, seed, skin, nl_capacity):
        types = tuple(types)
        for t in types:
            if not isinstance(t, BodyType):
                raise ArgumentError("types must be BodyType entries")
        if not 1 <= len(types) <= MAX_TYPES:
            raise ArgumentError("types must hold 1..8 BodyType entries")
        energies = tuple(energies)
        for e in energies:
            if not (is_body_term(e) or is_contact_term(e) or is_bond_term(e)):
                raise ArgumentError("energy terms must be BodyTerms, ContactTerms or BondTerms")
        if len(energies) > MAX_TERMS:
            raise ArgumentError("at most 16 energy terms")
        self.types = (FccBodyType * len(types))()
        for q, t in enumerate(types):
            self.types[q] = FccBodyType(t.v0, t.Dr, t.Dt, t.mu_r, t.mu_theta, t.mu_ab, 1 if t.parent_drag else 0,
                                        int(t.maxmode))
        self.terms = (FccTerm * max(1, len(energies)))()
        for q, e in enumerate(energies):
            self.terms[q] = _term_struct(e)
        bl = np.asarray(list(bonds), dtype=np.int32).reshape(-1, 2) if len(bonds) else np.zeros((0, 2), np.int32)
        self.bonds = np.ascontiguousarray(bl.ravel())
        self.p = FccParams()
        self.p.Lx, self.p.Ly = float(box.Lx), float(box.Ly)
        self.p.dt = float(dt)
        self.p.ntheta = int(nθ)
        self.p.precision = precision_bits(T)
        self.p.seed = int(seed) & 0xFFFFFFFFFFFFFFFF
        self.p.skin = float(skin)
        self.p.ntypes = len(types)
        self.p.types = self.types
        self.p.nterms = len(energies)
        self.p.terms = self.terms
        self.p.nbonds = len(bl)
        self.p.bonds = iptr(self.bonds)
        self.p.nl_capacity = int(nl_capacity)


class BodiesBuffer:
    """Contiguous numpy arrays behind an ``fcc_bodies_host``.

    ``coef`` is ``ncoef × N`` in Fortran (column-major) order, as Julia
    stores it: one body's coefficients are contiguous, which is the ABI's
    layout, so ``coefT`` (``N × ncoef``, C order) is a view of the same
    memory."""

    def __init__(self, n: int, ncoef: int):
        self.n, self.ncoef = n, ncoef
        self.x = np.zeros(n)
        self.y = np.zeros(n)
        self.theta = np.zeros(n)
        self.imgx = np.zeros(n, np.int32)
        self.imgy = np.zeros(n, np.int32)
        self.coefT = np.zeros((n, ncoef))
        self.R0 = np.zeros(n)
        self.type = np.zeros(n, np.int32)
        self.parent = np.zeros(n, np.int32)
        self.s = FccBodiesHost(n, ncoef, dptr(self.x), dptr(self.y), dptr(self.theta), iptr(self.imgx),
                               iptr(self.imgy), dptr(self.coefT), dptr(self.R0), iptr(self.type), iptr(self.parent))

    @classmethod
    def from_bodies(cls, b: Bodies):
        buf = cls(b.n, b.ncoef)
        buf.fill(b)
        return buf

    def fill(self, b: Bodies):
        self.x[:] = b.x
        self.y[:] = b.y
        self.theta[:] = b.θ
        self.imgx[:] = b.imgx
        self.imgy[:] = b.imgy
        self.coefT[:] = np.asarray(b.coef).T
        self.R0[:] = b.R0
        self.type[:] = b.type
        self.parent[:] = b.parent

    def to_bodies(self) -> Bodies:
        return Bodies(self.x.copy(), self.y.copy(), self.theta.copy(), self.imgx.copy(), self.imgy.copy(),
                      self.coefT.copy().T, self.R0.copy(), self.type.copy(), self.parent.copy())


def _flat(a, dtype, writable):
    """`a` itself if it is a contiguous 1-d array of `dtype` (writable when
    asked), else None."""
    if (isinstance(a, np.ndarray) and a.dtype == dtype and a.ndim == 1 and a.flags.c_contiguous
            and (a.flags.writeable or not writable)):
        return a
    return None


def direct_host(b: Bodies, writable: bool = False):
    """An ``fcc_bodies_host`` over the arrays of `b` themselves, or None when
    one of them is not already in the ABI's layout (contiguous float64 /
    int32 vectors, ``coef`` ``ncoef × N`` in Fortran order).  The library
    then reads (set_state) or writes (get_state) them in place with one copy
    each to or from the device — a DMA when they are pinned."""
    n = b.n
    f = {k: _flat(getattr(b, a), dt, writable) for k, a, dt in (
        ("x", "x", np.float64), ("y", "y", np.float64), ("theta", "θ", np.float64), ("imgx", "imgx", np.int32),
        ("imgy", "imgy", np.int32), ("R0", "R0", np.float64), ("type", "type", np.int32),
        ("parent", "parent", np.int32))}
    c = b.coef
    if (any(v is None or len(v) != n for v in f.values()) or not isinstance(c, np.ndarray) or c.dtype != np.float64
            or c.ndim != 2 or c.shape[1] != n or not c.flags.f_contiguous or (writable and not c.flags.writeable)):
        return None
    return FccBodiesHost(n, c.shape[0], dptr(f["x"]), dptr(f["y"]), dptr(f["theta"]), iptr(f["imgx"]),
                         iptr(f["imgy"]), c.ctypes.data_as(c_double_p), dptr(f["R0"]), iptr(f["type"]),
                         iptr(f["parent"]))


def bodies_over(block: np.ndarray, n: int, ncoef: int) -> Bodies:
    """A ``Bodies`` whose arrays are views into one uint8 `block` of at least
    ``bodies_bytes(n, ncoef)`` bytes, every array 64-byte aligned and in the
    ABI's layout (so ``direct_host`` takes it as it is)."""
    views, off = {}, 0
    base = block.ctypes.data

    def take(name, dtype, count):
        nonlocal off
        off += (-(base + off)) % 64
        nb = count * np.dtype(dtype).itemsize
        views[name] = block[off:off + nb].view(dtype)
        off += nb

    for name, dt in (("x", np.float64), ("y", np.float64), ("θ", np.float64), ("R0", np.float64)):
        take(name, dt, n)
    for name in ("imgx", "imgy", "type", "parent"):
        take(name, np.int32, n)
    take("coef", np.float64, n * ncoef)
    views["coef"] = views["coef"].reshape(n, ncoef).T
    return Bodies(**views)


def bodies_bytes(n: int, ncoef: int) -> int:
    """Bytes ``bodies_over`` needs (with room for the 64-byte alignment)."""
    return 8 * n * (4 + ncoef) + 4 * 4 * n + 9 * 64


def check(status: int, lasterr) -> None:
    """Map an ``fcc_status`` to the reference's exception types."""
    if status == FCC_OK:
        return
    msg = lasterr()
    msg = msg.decode() if isinstance(msg, bytes) else str(msg)
    if status == FCC_ERR_ARGUMENT:
        raise ArgumentError(msg)
    if status == FCC_ERR_DIMENSION:
        raise DimensionMismatch(msg)
    if status == FCC_ERR_FULL:
        raise PoolFull(msg)
    raise DeviceError(f"status {status}: {msg}")


def declare(lib, prefix: str):
    """Declare the argument types of the fcc_/fcco_ entry points on ``lib``."""
    P = C.c_void_p
    sig = {
        "create": [C.POINTER(FccParams), C.POINTER(FccBodiesHost), C.POINTER(P)],
        "destroy": [P],
        "step": [P, C.c_int64],
        "update_neighbors": [P, C.c_int32],
        "compute_gradients": [P],
        "get_state": [P, C.POINTER(FccBodiesHost), C.POINTER(C.c_int64), C.POINTER(C.c_double), C.POINTER(C.c_int64)],
        "set_state": [P, C.POINTER(FccBodiesHost), C.c_int64],
        "set_dt": [P, C.c_double],
        "get_gradients": [P, C.POINTER(FccGradientsHost)],
        "get_geometry": [P, C.POINTER(FccGeometryHost)],
        "neighbor_dims": [P, c_int32_p, c_int32_p, c_int32_p, C.POINTER(C.c_int64), c_int32_p],
        "get_neighbors": [P, C.POINTER(FccNeighborsHost)],
        "perimeters": [P, C.c_int32, c_double_p, C.POINTER(C.c_int64)],
        "areas": [P, C.c_int32, c_double_p, C.POINTER(C.c_int64)],
        "shape_index": [P, C.c_int32, c_double_p, C.POINTER(C.c_int64)],
        "body_energy": [P, c_double_p],
        "philox_noise": [C.c_uint64, C.c_uint64, C.c_int64, C.c_int32, c_double_p],
        "build_neighbors": [C.c_int32, C.c_int64, c_double_p, c_double_p, c_double_p, C.c_double, C.c_double,
                            C.c_double, C.c_double, C.c_int32, c_int32_p, c_int32_p, c_int32_p, c_int32_p,
                            c_int32_p, c_int32_p],
    }
    for name, args in sig.items():
        fn = getattr(lib, prefix + name)
        fn.argtypes = args
        fn.restype = C.c_int32
    le = getattr(lib, prefix + "last_error")
    le.argtypes = []
    le.restype = C.c_char_p
    return le
