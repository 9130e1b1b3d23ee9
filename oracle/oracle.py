"""ctypes binding of the CPU oracle (oracle/libfcc_oracle.so).

TEST INFRASTRUCTURE ONLY: used by tests/ as the parity checker and by
bench.py's CPU-baseline leg.  It binds the fcco_ restatement of the
reference's CPU path (fcc_oracle.cpp) behind the same marshalling as the
product's ``Simulation`` (fouriercontourcells.jl_b200/simulation.py), so a
parity test builds both from identical inputs.

Load the package first (it is registered as ``fcc_b200``).
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

import fcc_b200
from fcc_b200 import abi
from fcc_b200.simulation import NativeSimulation

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libfcc_oracle.so")
_LIB = None


def build():
    """Compile the oracle with its Makefile (no-op when up to date)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def library():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        lib._lasterr = abi.declare(lib, "fcco_")
        lib.fcco_protrusion.argtypes = [C.c_void_p, C.c_int32, abi.c_double_p, C.POINTER(C.c_int64)]
        lib.fcco_protrusion.restype = C.c_int32
        lib.fcco_contact_counters.argtypes = [C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), abi.c_double_p]
        lib.fcco_contact_counters.restype = C.c_int32
        lib.fcco_philox4x32.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
        lib.fcco_philox4x32.restype = None
        lib.fcco_set_threads.argtypes = [C.c_int32]
        lib.fcco_set_threads.restype = C.c_int32
        _LIB = lib
    return _LIB


def set_threads(n: int = 0) -> int:
    """OpenMP threads of the oracle (0: all cores); returns the count in use."""
    return library().fcco_set_threads(int(n))


class OracleSimulation(NativeSimulation):
    """The reference's CPU step (Float64 or Float32), restated in C++."""

    _pfx = "fcco_"

    def _library(self):
        return library()

    def run(self, n: int, every: int = 0, callback=None, graph: bool = True):
        """run! on the CPU is step! between callbacks (src/simulation.jl:220-235)."""
        if callback is None or every <= 0:
            return self.step(n)
        done = 0
        while done < n:
            k = min(every, n - done)
            self.step(k)
            done += k
            callback(self)
        return self

    def protrusion(self, type=None):
        out = np.zeros(self.N)
        cnt = C.c_int64()
        self._call("protrusion", self._h, int(type or 0), abi.dptr(out), C.byref(cnt))
        return out[: cnt.value]

    def contact_counters(self):
        """(node-neighbour tests, hits, per-body min |d| over hits) of the last gradient evaluation."""
        t, h = C.c_int64(), C.c_int64()
        md = np.zeros(self.N)
        self._call("contact_counters", self._h, C.byref(t), C.byref(h), abi.dptr(md))
        return t.value, h.value, md


def philox4x32(ctr, key):
    lib = library()
    c = (C.c_uint32 * 4)(*[int(v) & 0xFFFFFFFF for v in ctr])
    k = (C.c_uint32 * 2)(*[int(v) & 0xFFFFFFFF for v in key])
    o = (C.c_uint32 * 4)()
    lib.fcco_philox4x32(c, k, o)
    return tuple(o)


def philox_noise(seed, draw, n, T=np.float64):
    return fcc_b200.ops.philox_noise(seed, draw, n, T, lib=library(), prefix="fcco_")


def build_neighbors(x, y, rmax, Lx, Ly, cutoff, range_, cap=32, T=np.float64):
    return fcc_b200.ops.build_neighbors(x, y, rmax, Lx, Ly, cutoff, range_, cap, T, lib=library(), prefix="fcco_")
