"""``Pool``: many simulations advanced by one packed engine.

The reference runs concurrent simulations as independent ``Simulation``s on
separate tasks and streams (README.md:255-262).  A ``Pool`` packs them into one
device arena and advances all of them with one persistent step-kernel launch
(``fcc_pool_*`` in include/fcc.h): each keeps its own box, types, terms, dt,
seed, Philox stream and neighbour-list rebuilds, and its trajectory equals the
one of the same simulation run alone with the same kernel variant, bit for
bit.  Simulations are admitted while others run (``add`` raises ``PoolFull``
when the slot, bodies or cells are not free) and retired with ``remove``;
``run(n)`` advances each by ``min(n, horizon - steps)``.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi
from .model import ArgumentError, Bodies, PoolFull
from .simulation import native_library

_POOL_SIG = {
    "pool_bytes": [C.POINTER(abi.FccPoolParams), C.POINTER(C.c_int64)],
    "pool_create": [C.POINTER(abi.FccPoolParams), C.POINTER(C.c_void_p)],
    "pool_destroy": [C.c_void_p],
    "pool_add": [C.c_void_p, C.POINTER(abi.FccParams), C.POINTER(abi.FccBodiesHost), C.c_int64,
                 C.POINTER(C.c_int32)],
    "pool_add_at": [C.c_void_p, C.POINTER(abi.FccParams), C.POINTER(abi.FccBodiesHost), C.c_int64, C.c_double,
                    C.c_int64, C.POINTER(C.c_int32)],
    "pool_remove": [C.c_void_p, C.c_int32],
    "pool_run": [C.c_void_p, C.c_int64],
    "pool_slot": [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
    "pool_usage": [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                   C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int32)],
    "pool_get_state": [C.c_void_p, C.c_int32, C.POINTER(abi.FccBodiesHost), C.POINTER(C.c_int64),
                       C.POINTER(C.c_double), C.POINTER(C.c_int64)],
    "pool_observable": [C.c_void_p, C.c_int32, C.c_int32, C.c_int32, abi.c_double_p, C.POINTER(C.c_int64)],
    "pool_builds": [C.c_void_p, C.c_int32, C.POINTER(C.c_int64)],
    "pool_config": [C.c_void_p, C.c_int32, C.c_int32],
    "pool_variant": [C.c_void_p] + [C.POINTER(C.c_int32)] * 6,
    "pool_last_timing": [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
    "pool_tune": [C.c_void_p, C.c_int64, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_double)],
    "pool_graph": [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int64)],
}


def _lib():
    lib = native_library()
    if not getattr(lib, "_pool_declared", False):
        for name, args in _POOL_SIG.items():
            fn = getattr(lib, "fcc_" + name)
            fn.argtypes = args
            fn.restype = C.c_int32
        lib._pool_declared = True
    return lib


def _params(T, nθ, max_bodies, max_cells, max_sims, nl_capacity, max_children, max_bonds):
    return abi.FccPoolParams(abi.precision_bits(T), int(nθ), int(max_bodies), int(max_cells), int(max_sims),
                             int(nl_capacity), int(max_children), int(max_bonds))


def padded(n: int) -> int:
    """Arena bodies a simulation of n bodies takes."""
    return (n + abi.POOL_ALIGN - 1) // abi.POOL_ALIGN * abi.POOL_ALIGN


def grid_cells(box, R0, skin=0.3, T=np.float32) -> int:
    """Grid cells of a simulation (CellList with cutoff 2 R0max (1 + sqrt(2/3)) + skin, src/simulation.jl:90)."""
    from .ops import grid_dims
    T = np.float32 if abi.precision_bits(T) == 32 else np.float64
    r0 = float(np.max(np.asarray(R0, dtype=T))) if len(R0) else 0.0
    cutoff = 2 * r0 * (1 + np.sqrt(2.0 / 3.0)) + skin
    ncx, ncy = grid_dims(float(T(box.Lx)), float(T(box.Ly)), cutoff)
    return ncx * ncy


class Pool:
    """Packed multi-simulation engine on one GPU."""

    def __init__(self, T=np.float32, nθ=40, max_bodies=1 << 20, max_cells=1 << 18, max_sims=256, nl_capacity=32,
                 max_children=1, max_bonds=1):
        self._lib = _lib()
        self.T = np.float64 if abi.precision_bits(T) == 64 else np.float32
        self.nθ = int(nθ)
        self._q = _params(T, nθ, max_bodies, max_cells, max_sims, nl_capacity, max_children, max_bonds)
        h = C.c_void_p()
        self._call("pool_create", C.byref(self._q), C.byref(h))
        self._h = h
        self._slots = {}  # slot -> (n, ncoef, type array, box)

    @staticmethod
    def device_bytes(T=np.float32, nθ=40, max_bodies=1 << 20, max_cells=1 << 18, max_sims=256, nl_capacity=32,
                     max_children=1, max_bonds=1) -> int:
        """Device bytes a pool of these limits holds."""
        lib = _lib()
        q = _params(T, nθ, max_bodies, max_cells, max_sims, nl_capacity, max_children, max_bonds)
        out = C.c_int64()
        abi.check(lib.fcc_pool_bytes(C.byref(q), C.byref(out)), lib._lasterr)
        return out.value

    @classmethod
    def for_budget(cls, hbm_bytes: int, T=np.float32, nθ=40, max_sims=256, cells_per_body=0.25, nl_capacity=32,
                   **kw):
        """The largest pool (bodies, with cells_per_body grid cells per body)
        whose device footprint fits in hbm_bytes."""
        lo, hi = 0, 1 << 30
        while lo < hi:
            mid = (lo + hi + 1) // 2
            b = cls.device_bytes(T, nθ, mid, max(1, int(mid * cells_per_body)), max_sims, nl_capacity, **kw)
            if b <= hbm_bytes:
                lo = mid
            else:
                hi = mid - 1
        if lo < abi.POOL_ALIGN:
            raise ArgumentError("HBM budget too small for a pool")
        return cls(T, nθ, lo, max(1, int(lo * cells_per_body)), max_sims, nl_capacity, **kw)

    def _call(self, name, *args):
        abi.check(getattr(self._lib, "fcc_" + name)(*args), self._lib._lasterr)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fcc_pool_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ slots
    def add(self, bodies: Bodies, box, types, energies=(), bonds=(), dt=0.005, seed=1, skin=0.3, horizon=0,
            nl_capacity=32, clock=0, t=None) -> int:
        """Admit a simulation (the arguments of ``Simulation``); raises PoolFull
        when it does not fit now.  ``clock`` > 0 resumes a checkpoint (the
        state, clock and time ``state`` returned): it holds at clock
        ``horizon``; without ``t`` its time restarts at clock * dt."""
        params = abi.ParamsBuffer(box, types, energies, bonds, dt, self.nθ, self.T, seed, skin, nl_capacity)
        host = abi.direct_host(bodies)
        if host is None:
            buf = abi.BodiesBuffer.from_bodies(bodies)
            host = buf.s
        slot = C.c_int32()
        if clock:
            self._call("pool_add_at", self._h, C.byref(params.p), C.byref(host), int(clock),
                       -1.0 if t is None else float(t), int(horizon), C.byref(slot))
        else:
            self._call("pool_add", self._h, C.byref(params.p), C.byref(host), int(horizon), C.byref(slot))
        self._slots[slot.value] = (bodies.n, bodies.ncoef, np.array(bodies.type, dtype=np.int32), box)
        return slot.value

    def try_add(self, *args, **kw):
        """``add`` that returns None instead of raising PoolFull."""
        try:
            return self.add(*args, **kw)
        except PoolFull:
            return None

    def remove(self, slot: int):
        self._call("pool_remove", self._h, int(slot))
        self._slots.pop(slot, None)

    def run(self, n: int):
        """Advance every simulation by min(n, horizon - steps done)."""
        self._call("pool_run", self._h, int(n))
        return self

    def slot(self, slot: int):
        """(active, steps done, horizon)."""
        a, s, h = C.c_int32(), C.c_int64(), C.c_int64()
        self._call("pool_slot", self._h, int(slot), C.byref(a), C.byref(s), C.byref(h))
        return bool(a.value), s.value, h.value

    def done(self, slot: int) -> bool:
        a, s, h = self.slot(slot)
        return a and s >= h

    @property
    def slots(self):
        return sorted(self._slots)

    def usage(self):
        v = [C.c_int64(), C.c_int64(), C.c_int32(), C.c_int64(), C.c_int64(), C.c_int32()]
        self._call("pool_usage", self._h, *(C.byref(x) for x in v))
        keys = ("bodies", "cells", "sims", "max_bodies", "max_cells", "max_sims")
        return dict(zip(keys, (x.value for x in v)))

    def fits(self, n_bodies: int, n_cells: int) -> bool:
        u = self.usage()
        return (u["sims"] < u["max_sims"] and u["bodies"] + padded(n_bodies) <= u["max_bodies"]
                and u["cells"] + n_cells <= u["max_cells"])

    # ------------------------------------------------------------ state
    def state(self, slot: int):
        """(Bodies, clock, t, steps) of one simulation."""
        if slot not in self._slots:
            raise ArgumentError(f"pool: no simulation in slot {slot}")
        n, ncoef, _, _ = self._slots[slot]
        buf = abi.BodiesBuffer(n, ncoef)
        clk, t, stp = C.c_int64(), C.c_double(), C.c_int64()
        self._call("pool_get_state", self._h, int(slot), C.byref(buf.s), C.byref(clk), C.byref(t), C.byref(stp))
        b = Bodies(buf.x, buf.y, buf.theta, buf.imgx, buf.imgy, buf.coefT.T, buf.R0, buf.type, buf.parent)
        return b, clk.value, t.value, stp.value

    def bodies(self, slot: int) -> Bodies:
        return self.state(slot)[0]

    def _observable(self, slot, which, type):
        if slot not in self._slots:
            raise ArgumentError(f"pool: no simulation in slot {slot}")
        n = self._slots[slot][0]
        out = np.zeros(max(1, n))
        cnt = C.c_int64()
        self._call("pool_observable", self._h, int(slot), which, 0 if type is None else int(type), abi.dptr(out),
                   C.byref(cnt))
        return out[:cnt.value].copy()

    def perimeters(self, slot, type=None):
        return self._observable(slot, 0, type)

    def areas(self, slot, type=None):
        return self._observable(slot, 1, type)

    def shape_index(self, slot, type=None):
        return self._observable(slot, 2, type)

    def builds(self, slot) -> int:
        b = C.c_int64()
        self._call("pool_builds", self._h, int(slot), C.byref(b))
        return b.value

    # ----------------------------------------------------------- launch
    def config(self, variant: int = -1, steps_per_launch: int = 0):
        self._call("pool_config", self._h, int(variant), int(steps_per_launch))

    def variant(self):
        v = [C.c_int32() for _ in range(6)]
        self._call("pool_variant", self._h, *(C.byref(x) for x in v))
        return dict(zip(("variant", "lanes", "slots", "block", "min_blocks", "grid"), (x.value for x in v)))

    def tune(self, steps: int = 64, reorder: bool = False):
        """Autotune the launch shape for this pool's size bucket (from a
        snapshot, restored afterwards); returns (variant, µs per step) or
        (-1, 0) when nothing could be tuned yet."""
        v, us = C.c_int32(), C.c_double()
        self._call("pool_tune", self._h, int(steps), 1 if reorder else 0, C.byref(v), C.byref(us))
        return v.value, us.value

    def graph(self, enable=None):
        """CUDA-graph replay of run rounds: switch on/off (None: query).
        Returns (active, replays)."""
        a, r = C.c_int32(), C.c_int64()
        self._call("pool_graph", self._h, -1 if enable is None else int(bool(enable)), C.byref(a), C.byref(r))
        return bool(a.value), r.value

    def last_timing(self):
        """(device ms, kernel launches, body-steps) of the last run."""
        ms, launches, bs = C.c_double(), C.c_int64(), C.c_int64()
        self._call("pool_last_timing", self._h, C.byref(ms), C.byref(launches), C.byref(bs))
        return ms.value, launches.value, bs.value
