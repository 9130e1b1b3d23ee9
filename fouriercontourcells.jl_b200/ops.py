"""Stateless entry points of the C ABI: Philox noise and the neighbour build.

``philox_noise`` mirrors ``philox_noise!`` (src/random.jl:113-130);
``build_neighbors`` runs ``update_celllist!`` plus the neighbour kernel
(src/neighbors.jl:81-92, 148-174) on caller arrays.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import abi
from .simulation import native_library


def philox_noise(seed: int, draw: int, n: int, T=np.float64, lib=None, prefix="fcc_"):
    """3 × n standard normals of draw ``draw`` (bodies 1..n), as
    ``philox_noise!(zeros(T, 3, n), philox_key(seed), draw)``."""
    lib = lib or native_library()
    out = np.zeros((n, 3))
    st = getattr(lib, prefix + "philox_noise")(int(seed) & (2**64 - 1), int(draw) & (2**64 - 1), int(n),
                                              abi.precision_bits(T), abi.dptr(out))
    abi.check(st, lib._lasterr)
    return out.T


def barrier_selftest(blocks: int = 4, lib=None):
    """Run the self-test of the bounded grid-barrier waits: ``blocks`` blocks
    of which one never arrives, waited for at a generation-word barrier and
    then at a flat barrier.  Returns (error, ms): error is 1 when both waits
    ended with the error status (expected for blocks >= 2), 0 when neither
    did, 2 when only one did."""
    lib = lib or native_library()
    err, ms = C.c_int32(), C.c_double()
    abi.check(lib.fcc_barrier_selftest(int(blocks), C.byref(err), C.byref(ms)), lib._lasterr)
    return int(err.value), ms.value


def grid_dims(Lx, Ly, cutoff):
    """CellList grid size (src/neighbors.jl:27-33)."""
    nc = lambda L: (lambda n: n if n >= 3 else 1)(math.floor(L / cutoff))
    return nc(Lx), nc(Ly)


def build_neighbors(x, y, rmax, Lx, Ly, cutoff, range_, cap=32, T=np.float64, lib=None, prefix="fcc_"):
    """Cell list + neighbour list of the given positions and contour bounds.
    Returns (cellid, perm, start, stop, idx (cap × n), count), 1-based."""
    lib = lib or native_library()
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    rmax = np.ascontiguousarray(rmax, dtype=np.float64)
    n = len(x)
    T32 = abi.precision_bits(T) == 32
    Lxt = float(np.float32(Lx)) if T32 else float(Lx)
    Lyt = float(np.float32(Ly)) if T32 else float(Ly)
    ncx, ncy = grid_dims(Lxt, Lyt, cutoff)
    cellid, perm, count = (np.zeros(n, np.int32) for _ in range(3))
    start, stop = np.zeros(ncx * ncy, np.int32), np.zeros(ncx * ncy, np.int32)
    idx = np.zeros((n, cap), np.int32)
    st = getattr(lib, prefix + "build_neighbors")(abi.precision_bits(T), n, abi.dptr(x), abi.dptr(y), abi.dptr(rmax),
                                                 float(Lx), float(Ly), float(cutoff), float(range_), int(cap),
                                                 abi.iptr(cellid), abi.iptr(perm), abi.iptr(start), abi.iptr(stop),
                                                 abi.iptr(idx), abi.iptr(count))
    abi.check(st, lib._lasterr)
    return cellid, perm, start, stop, idx.T, count
