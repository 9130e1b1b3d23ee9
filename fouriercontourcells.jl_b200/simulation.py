"""``Simulation`` over the native B200 library (libfcc_b200.so).

Mirrors src/simulation.jl: ``Simulation(bodies, box; types, energies, bonds,
dt, nθ, T, seed, skin)`` (:66-105), ``step!`` (:165-173), ``run!``
(:220-235), ``compute_gradients!`` (:150-158), ``update_neighbors!``
(:132-142), and the fields the reference's tests read (``sim.bodies``,
``sim.grad``, ``sim.geom``, ``sim.neighbors``, ``sim.t``, ``sim.step``).
Julia's ``step!``/``run!`` are ``step``/``run`` here.

``NativeSimulation`` holds the marshalling shared by every implementation of
the fcc C ABI; ``Simulation`` binds it to libfcc_b200.so, the CUDA library,
and fails loudly when that library is missing: there is no CPU fallback.
"""

from __future__ import annotations

import ctypes as C
import os
import weakref
from collections import namedtuple

import numpy as np

from . import abi
from .model import ArgumentError, Bodies, DeviceError, DimensionMismatch

Gradients = namedtuple("Gradients", "GR GD GDD P gx gy gθ glab gcoef Ebody")
Geometry = namedtuple("Geometry", "lab labR0 R dR ddR rmax")
NeighborInfo = namedtuple("NeighborInfo", "idx count cap builds valid cellid perm start stop ncx ncy")

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libfcc_b200.so")
_LIB = None


def native_library():
    """Load libfcc_b200.so (built in-tree by build.py); raise if it is missing."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise DeviceError(f"native library {LIB_PATH} is missing: run the build (__graft_entry__.build())")
        lib = C.CDLL(LIB_PATH)
        lib._lasterr = abi.declare(lib, "fcc_")
        lib.fcc_run.argtypes = [C.c_void_p, C.c_int64, C.c_int64, abi.FCC_CALLBACK, C.c_void_p, C.c_int32]
        lib.fcc_run.restype = C.c_int32
        lib.fcc_last_timing.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        lib.fcc_last_timing.restype = C.c_int32
        lib.fcc_version.argtypes = []
        lib.fcc_version.restype = C.c_char_p
        lib.fcc_health.argtypes = [C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        lib.fcc_health.restype = C.c_int32
        lib.fcc_barrier_selftest.argtypes = [C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        lib.fcc_barrier_selftest.restype = C.c_int32
        lib.fcc_host_alloc.argtypes = [C.c_int64, C.POINTER(C.c_void_p)]
        lib.fcc_host_alloc.restype = C.c_int32
        lib.fcc_host_free.argtypes = [C.c_void_p]
        lib.fcc_host_free.restype = C.c_int32
        _LIB = lib
    return _LIB


def pinned_bodies(n: int, ncoef: int) -> Bodies:
    """A ``Bodies`` of n bodies in page-locked host memory (``fcc_host_alloc``),
    laid out as the C ABI reads and writes it, so ``set_state`` and
    ``get_state(out=...)`` move it to and from the device by DMA with no host
    copy.  The memory is released when the last of its arrays is collected."""
    lib = native_library()
    nbytes = abi.bodies_bytes(n, ncoef)
    ptr = C.c_void_p()
    abi.check(lib.fcc_host_alloc(nbytes, C.byref(ptr)), lib._lasterr)
    block = np.frombuffer((C.c_uint8 * nbytes).from_address(ptr.value), dtype=np.uint8)
    weakref.finalize(block, lib.fcc_host_free, ptr.value)
    return abi.bodies_over(block, n, ncoef)


def pinned_copy(bodies: Bodies) -> Bodies:
    """``bodies`` copied into page-locked host memory (``pinned_bodies``)."""
    out = pinned_bodies(bodies.n, bodies.ncoef)
    for f in ("x", "y", "θ", "imgx", "imgy", "coef", "R0", "type", "parent"):
        getattr(out, f)[...] = getattr(bodies, f)
    return out


class NativeSimulation:
    """Marshalling over one implementation of the fcc C ABI (prefix ``_pfx``)."""

    _pfx = "fcc_"

    def _library(self):  # pragma: no cover - overridden
        raise NotImplementedError

    def __init__(self, bodies: Bodies, box, types, energies=(), bonds=(), dt=0.005, nθ=40, T=np.float64, seed=1,
                 skin=0.3, nl_capacity=32, **kw):
        nθ = kw.pop("ntheta", nθ)
        if kw:
            raise TypeError(f"Simulation got unexpected keyword arguments {sorted(kw)}")
        self._lib = self._library()
        self._fn = lambda name: getattr(self._lib, self._pfx + name)
        self._params = abi.ParamsBuffer(box, types, energies, bonds, dt, nθ, T, seed, skin, nl_capacity)
        self._buf = None  # host arrays in the ABI's layout, reused for inputs that are not
        self._direct = {}  # writable -> (bodies, its arrays, fcc_bodies_host over them)
        h = C.c_void_p()
        self._call("create", C.byref(self._params.p), C.byref(self._host_in(bodies)), C.byref(h))
        self._h = h
        self.N = bodies.n
        self.ncoef = bodies.ncoef
        self.nθ = int(nθ)
        self.box = box
        self.types = tuple(types)
        self.energies = tuple(energies)
        self.T = np.float64 if abi.precision_bits(T) == 64 else np.float32
        self.seed = seed
        self._type = np.array(bodies.type, dtype=np.int32)

    # ---------------------------------------------------------------- calls
    def _call(self, name, *args):
        abi.check(self._fn(name)(*args), self._lib._lasterr)

    def close(self):
        self._direct = {}
        if getattr(self, "_h", None):
            self._fn("destroy")(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------- dynamics
    def step(self, n: int = 1):
        """step!(sim, n) (src/simulation.jl:165-173)."""
        self._call("step", self._h, int(n))
        return self

    def update_neighbors(self, force: bool = False):
        """update_neighbors!(sim; force) (src/simulation.jl:132-142)."""
        self._call("update_neighbors", self._h, 1 if force else 0)
        return self

    def compute_gradients(self):
        """compute_gradients!(sim) (src/simulation.jl:150-158)."""
        self._call("compute_gradients", self._h)
        return self

    def refresh(self):
        """enforce_shape!, update_geometry!, forced neighbour update and
        gradients after host edits (test/runtests.jl:9-15)."""
        self.update_neighbors(force=True)
        return self.compute_gradients()

    # ---------------------------------------------------------------- state
    _FIELDS = ("x", "y", "θ", "imgx", "imgy", "coef", "R0", "type", "parent")

    def _direct_host(self, bodies: Bodies, writable: bool = False):
        """``abi.direct_host(bodies)``, kept for the next call with the same
        ``Bodies`` holding the same array objects (the exchange loop of a
        caller that reuses its page-locked buffers): the check is nine
        identity tests instead of nine layout checks.  The entry holds
        references to the arrays, so none of them is freed (and its address
        reused) while the kept pointers refer to it."""
        c = getattr(self, "_direct", {}).get(writable)
        if (c is not None and c[0] is bodies and all(getattr(bodies, f) is a for f, a in zip(self._FIELDS, c[1]))
                and (not writable or all(a.flags.writeable for a in c[1]))):
            return c[2]
        h = abi.direct_host(bodies, writable=writable)
        if h is not None and hasattr(self, "_direct"):
            self._direct[writable] = (bodies, tuple(getattr(bodies, f) for f in self._FIELDS), h)
        return h

    def _host_in(self, bodies: Bodies):
        """An ``fcc_bodies_host`` over `bodies` itself when its arrays are in
        the ABI's layout, else over a copy in a buffer this object keeps."""
        h = self._direct_host(bodies)
        if h is not None:
            return h
        if self._buf is None or self._buf.n != bodies.n or self._buf.ncoef != bodies.ncoef:
            self._buf = abi.BodiesBuffer(bodies.n, bodies.ncoef)
        self._buf.fill(bodies)
        return self._buf.s

    def _counters(self):
        clock, t, stp = C.c_int64(), C.c_double(), C.c_int64()
        self._call("get_state", self._h, None, C.byref(clock), C.byref(t), C.byref(stp))
        return clock.value, t.value, stp.value

    def get_state(self, out: Bodies = None) -> Bodies:
        """The body state (the fields of sim.bodies) copied to the host: into
        `out` when given (its arrays are written in place, which takes one
        device-to-host copy per array when they are in the ABI's layout, a DMA
        when `out` is ``pinned_bodies``), else into new arrays."""
        if out is not None:
            h = self._direct_host(out, writable=True)
            if h is None or out.n != self.N or out.ncoef != self.ncoef:
                raise ArgumentError("get_state(out=...) needs writable arrays of this simulation's size in the "
                                    "ABI's layout (contiguous vectors, coef in Fortran order): see pinned_bodies")
            self._call("get_state", self._h, C.byref(h), None, None, None)
            return out
        buf = abi.BodiesBuffer(self.N, self.ncoef)
        self._call("get_state", self._h, C.byref(buf.s), None, None, None)
        return Bodies(buf.x, buf.y, buf.theta, buf.imgx, buf.imgy, buf.coefT.T, buf.R0, buf.type, buf.parent)

    @property
    def bodies(self) -> Bodies:
        """Host copy of sim.bodies."""
        return self.get_state()

    @property
    def clock(self) -> int:
        return self._counters()[0]

    @property
    def t(self) -> float:
        return self._counters()[1]

    @property
    def nsteps(self) -> int:
        """sim.step of the reference (steps taken)."""
        return self._counters()[2]

    def set_state(self, bodies: Bodies, clock: int = -1):
        """Overwrite the body state and the clock (``fcc_set_state``); R0,
        type and parent must be the created ones."""
        if bodies.n != self.N or bodies.ncoef != self.ncoef:
            raise DimensionMismatch("state buffers do not match the simulation")
        self._call("set_state", self._h, C.byref(self._host_in(bodies)), int(clock))
        return self

    @property
    def dt(self):
        return self._params.p.dt

    @dt.setter
    def dt(self, value):
        self._call("set_dt", self._h, float(value))
        self._params.p.dt = float(value)

    @property
    def grad(self) -> Gradients:
        N, nθ, nc = self.N, self.nθ, self.ncoef
        a = {f: np.zeros((N, nθ)) for f in ("GR", "GD", "GDD", "P")}
        v = {f: np.zeros(N) for f in ("gx", "gy", "gtheta", "Ebody")}
        m = {f: np.zeros((N, nc)) for f in ("glab", "gcoef")}
        g = abi.FccGradientsHost(*(abi.dptr(x) for x in (a["GR"], a["GD"], a["GDD"], a["P"], v["gx"], v["gy"],
                                                           v["gtheta"], m["glab"], m["gcoef"], v["Ebody"])))
        self._call("get_gradients", self._h, C.byref(g))
        return Gradients(a["GR"].T, a["GD"].T, a["GDD"].T, a["P"].T, v["gx"], v["gy"], v["gtheta"],
                         m["glab"].T, m["gcoef"].T, v["Ebody"])

    @property
    def geom(self) -> Geometry:
        N, nθ, nc = self.N, self.nθ, self.ncoef
        lab, labR0 = np.zeros((N, nc)), np.zeros((N, nc))
        R, dR, ddR = np.zeros((N, nθ)), np.zeros((N, nθ)), np.zeros((N, nθ))
        rmax = np.zeros(N)
        g = abi.FccGeometryHost(*(abi.dptr(x) for x in (lab, labR0, R, dR, ddR, rmax)))
        self._call("get_geometry", self._h, C.byref(g))
        return Geometry(lab.T, labR0.T, R.T, dR.T, ddR.T, rmax)

    def neighbor_dims(self):
        ncx, ncy, cap, valid = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        builds = C.c_int64()
        self._call("neighbor_dims", self._h, C.byref(ncx), C.byref(ncy), C.byref(cap), C.byref(builds), C.byref(valid))
        return ncx.value, ncy.value, cap.value, builds.value, bool(valid.value)

    @property
    def builds(self) -> int:
        """sim.neighbors.builds."""
        return self.neighbor_dims()[3]

    @property
    def neighbors(self) -> NeighborInfo:
        ncx, ncy, cap, builds, valid = self.neighbor_dims()
        N = self.N
        cellid, perm = np.zeros(N, np.int32), np.zeros(N, np.int32)
        start, stop = np.zeros(ncx * ncy, np.int32), np.zeros(ncx * ncy, np.int32)
        idx, count = np.zeros((N, cap), np.int32), np.zeros(N, np.int32)
        h = abi.FccNeighborsHost(*(abi.iptr(x) for x in (cellid, perm, start, stop, idx, count)))
        self._call("get_neighbors", self._h, C.byref(h))
        return NeighborInfo(idx.T, count, cap, builds, valid, cellid, perm, start, stop, ncx, ncy)

    # ---------------------------------------------------------- observables
    def _observable(self, name, type):
        out = np.zeros(self.N)
        cnt = C.c_int64()
        self._call(name, self._h, int(type or 0), abi.dptr(out), C.byref(cnt))
        return out[: cnt.value]

    def perimeters(self, type=None):
        return self._observable("perimeters", type)

    def areas(self, type=None):
        return self._observable("areas", type)

    def shape_index(self, type=None):
        return self._observable("shape_index", type)

    def body_energy(self) -> float:
        out = C.c_double()
        self._call("body_energy", self._h, C.byref(out))
        return out.value

    def __repr__(self):
        return (f"{type(self).__name__}{{{np.dtype(self.T).name}}}(N={self.N}, nθ={self.nθ}, "
                f"box={self.box.Lx}×{self.box.Ly})")


class Simulation(NativeSimulation):
    """``Simulation`` on the B200 (CUDA) library."""

    _pfx = "fcc_"

    def _library(self):
        return native_library()

    def run(self, n: int, every: int = 0, callback=None, graph: bool = True):
        """run!(sim, n; every, callback, graph) (src/simulation.jl:220-235):
        persistent multi-step launches with one host synchronisation per
        callback (graph = True), or eager per-step launches (graph = False)."""
        if callback is None or every <= 0:
            cb, every = abi.FCC_CALLBACK(), 0
        else:
            cb = abi.FCC_CALLBACK(lambda h, u: callback(self))
        self._cb = cb  # keep alive during the call
        self._call("run", self._h, int(n), int(every), cb, None, 1 if graph else 0)
        return self

    def last_timing(self):
        """(device ms, kernel launches, steps) of the last step/run call."""
        ms, launches, steps = C.c_double(), C.c_int64(), C.c_int64()
        self._call("last_timing", self._h, C.byref(ms), C.byref(launches), C.byref(steps))
        return ms.value, launches.value, steps.value

    def health(self):
        """{"nonfinite", "barrier_error"}: a step produced a non-finite
        position, angle or contour extent (until the next set_state), or a
        grid-barrier wait of the step kernel ran out (no counterpart in the
        reference, which checks neither)."""
        nf, be = C.c_int32(), C.c_int32()
        self._call("health", self._h, C.byref(nf), C.byref(be))
        return {"nonfinite": bool(nf.value), "barrier_error": bool(be.value)}


# ------------------------------------------------------------- functions
def step(sim, n: int = 1):
    """step!(sim, n)."""
    return sim.step(n)


def run(sim, n: int, every: int = 0, callback=None, graph: bool = True):
    """run!(sim, n; every, callback, graph)."""
    return sim.run(n, every=every, callback=callback, graph=graph)


def compute_gradients(sim):
    """compute_gradients!(sim)."""
    return sim.compute_gradients()


def update_neighbors(sim, force: bool = False):
    return sim.update_neighbors(force)


def perimeters(sim, type=None):
    """Perimeters ∮ √(R² + R'²) dφ (src/observables.jl:7-8)."""
    return sim.perimeters(type)


def areas(sim, type=None):
    """Areas ½ ∮ R² dφ (src/observables.jl:11-12)."""
    return sim.areas(type)


def shape_index(sim, type=None):
    """Perimeter / √area per body (src/observables.jl:18)."""
    return sim.shape_index(type)


def body_energy(sim) -> float:
    """Sum of single-body energies of the last gradient evaluation (src/observables.jl:47)."""
    return sim.body_energy()


def positions(sim):
    """Wrapped centres as a 2 × N array (src/observables.jl:21)."""
    b = sim.bodies
    return np.vstack([b.x, b.y])


def unwrapped_positions(sim):
    """Unwrapped centres x + imgx·Lx as a 2 × N array (src/observables.jl:24-29)."""
    b = sim.bodies
    return np.vstack([b.x + b.imgx * sim.box.Lx, b.y + b.imgy * sim.box.Ly])


def contours(sim):
    """(X, Y): nθ × N contour node coordinates around the wrapped centres (src/observables.jl:36-44)."""
    b = sim.bodies
    R = sim.geom.R
    φ = np.arange(sim.nθ) * (2 * np.pi / sim.nθ)
    return b.x[None, :] + R * np.cos(φ)[:, None], b.y[None, :] + R * np.sin(φ)[:, None]


def protrusion(sim, type=None):
    """How far each body pokes out of its parent, max over nodes of
    |u - r_c| - R_c(ψ); NaN for self-parented bodies.  A host diagnostic, as in
    the reference (src/observables.jl:59-79)."""
    b = sim.bodies
    g = sim.geom
    K = (sim.ncoef - 1) // 2
    Lx, Ly = sim.box.Lx, sim.box.Ly
    out = np.full(sim.N, np.nan)
    φ = np.arange(sim.nθ) * (2 * np.pi / sim.nθ)
    for i in range(sim.N):
        c = b.parent[i] - 1
        if c == i:
            continue
        dx = b.x[i] + g.R[:, i] * np.cos(φ) - b.x[c]
        dy = b.y[i] + g.R[:, i] * np.sin(φ) - b.y[c]
        dx -= Lx * np.rint(dx / Lx)
        dy -= Ly * np.rint(dy / Ly)
        ψ = np.arctan2(dy, dx)
        n = np.arange(2, K + 2)
        lab = g.lab[:, c]
        Rc = b.R0[c] * (lab[0] + (lab[1:K + 1, None] * np.cos(np.outer(n, ψ))).sum(0)
                        + (lab[K + 1:, None] * np.sin(np.outer(n, ψ))).sum(0))
        out[i] = np.max(np.hypot(dx, dy) - Rc)
    return out if type is None else out[b.type == type]
