"""CPU checks of the boundary: the built library exports every entry point
that include/fcc.h declares, the ctypes mirror matches the header's structs,
and the host model validates like the reference (no GPU calls)."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, fcc, oracle

HEADER = os.path.join(ROOT, "include", "fcc.h")


def declared_functions(path=HEADER):
    text = open(path).read()
    return sorted(set(re.findall(r"^(?:fcc_status|const char\*)\s+(fcc_\w+)\s*\(", text, re.M)))


def test_header_declares_the_reference_boundary():
    names = declared_functions()
    for required in ("fcc_create", "fcc_destroy", "fcc_step", "fcc_run", "fcc_compute_gradients", "fcc_get_state",
                     "fcc_set_state", "fcc_get_gradients", "fcc_shape_index", "fcc_get_neighbors", "fcc_last_error"):
        assert required in names


def test_library_exports_every_declared_symbol():
    path = fcc.simulation.LIB_PATH
    assert os.path.exists(path), "build the library first (__graft_entry__.build())"
    lib = C.CDLL(path)  # loading needs no GPU
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_oracle_exports_mirror():
    lib = oracle.library()
    for n in declared_functions():
        if n in ("fcc_run", "fcc_last_timing", "fcc_version", "fcc_build_neighbors_noalloc", "fcc_health",
                 "fcc_barrier_selftest", "fcc_host_alloc", "fcc_host_free") or n.startswith("fcc_pool_"):
            continue  # device-only entry points (launch timing, caller device arrays, device health, packed
            # pools, page-locked host memory)
        assert hasattr(lib, "fcco_" + n[4:]), n


def test_struct_layouts_match_header():
    """Sizes of the ctypes mirror against a C compile of fcc.h."""
    import subprocess
    import tempfile
    src = '#include <stdio.h>\n#include "fcc.h"\nint main(){printf("%zu %zu %zu %zu %zu %zu %zu %zu\\n",' \
          'sizeof(fcc_term),sizeof(fcc_body_type),sizeof(fcc_params),sizeof(fcc_bodies_host),' \
          'sizeof(fcc_gradients_host),sizeof(fcc_geometry_host),sizeof(fcc_neighbors_host),sizeof(fcc_pool_params));}'
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "s")
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        sizes = list(map(int, subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()))
    a = fcc.abi
    assert sizes == [C.sizeof(a.FccTerm), C.sizeof(a.FccBodyType), C.sizeof(a.FccParams), C.sizeof(a.FccBodiesHost),
                     C.sizeof(a.FccGradientsHost), C.sizeof(a.FccGeometryHost), C.sizeof(a.FccNeighborsHost),
                     C.sizeof(a.FccPoolParams)]


def test_product_fails_loudly_without_library(monkeypatch):
    """No silent CPU fallback: a missing library is an error."""
    monkeypatch.setattr(fcc.simulation, "LIB_PATH", "/nonexistent/libfcc_b200.so")
    monkeypatch.setattr(fcc.simulation, "_LIB", None)
    bodies, box = fcc.hexagonal_monolayer(2, 2)
    with pytest.raises(fcc.DeviceError):
        fcc.Simulation(bodies, box, types=(fcc.BodyType(),))


def test_host_model_validation():
    """src/bodies.jl:41, src/initial.jl:17, src/energies/contact.jl:15."""
    with pytest.raises(fcc.ArgumentError):
        fcc.BodyType(drag="cytoplasm")
    with pytest.raises(fcc.ArgumentError):
        fcc.hexagonal_monolayer(3, 3)
    with pytest.raises(fcc.DimensionMismatch):
        fcc.Overlap([[1.0, 2.0], [2.0, 3.0]], related=[[1.0]])
    with pytest.raises(fcc.DimensionMismatch):
        fcc.Bodies.new([0.0, 1.0], [0.0], [0.0, 0.0], np.zeros((11, 2)), [1.0, 1.0])
    o = fcc.Overlap([[1.0, 2.0], [2.0, 3.0]], related=[[1.0, -0.5], [-0.5, 1.0]])
    assert o.pressure(0.1, 1, 2, False) == 2.0
    assert o.pressure(0.1, 1, 2, True) == -0.5
    assert o.pressure(-0.1, 2, 2, False) == 0.0
    assert fcc.Overlap(1.0).pressure(0.0, 1, 1, False) == 1.0
    assert fcc.LinearRepulsion(2.0).pressure(0.25, 1, 1, False) == 0.5


def test_box_helpers():
    """test/test_geometry.jl:16-21."""
    assert fcc.wrap(-0.5, 2.0) == (1.5, -1)
    assert fcc.wrap(4.5, 2.0) == (0.5, 2)
    assert fcc.wrap(-1e-18, 2.0) == (0.0, 0)
    assert abs(fcc.minimum_image(1.6, 2.0) + 0.4) < 1e-15


def test_initial_conditions():
    """src/initial.jl:11-53 and test/test_parents.jl:151-172."""
    b, box = fcc.hexagonal_monolayer(32, 32, packing=0.95, maxmode=10)
    assert b.n == 1024 and b.ncoef == 19
    r = np.sqrt(np.pi / (2 * np.sqrt(3) * 0.95))
    assert np.isclose(box.Lx, 64 * r) and np.isclose(box.Ly, np.sqrt(3) * r * 32)
    assert np.isclose(1024 * np.pi / (box.Lx * box.Ly), 0.95)
    cells, _ = fcc.hexagonal_monolayer(4, 4)
    nb = fcc.with_nuclei(cells, ratio=0.4)
    assert nb.n == 32
    assert list(nb.parent) == list(range(1, 17)) * 2
    assert list(nb.type) == [1] * 16 + [2] * 16
    assert np.allclose(nb.R0[16:], 0.4)
    assert fcc.parent_bonds(nb) == [(16 + i, i) for i in range(1, 17)]
    c = fcc.vcat(fcc.Bodies.new([1.0, 2.0], [1.0, 2.0], np.zeros(2), np.zeros((11, 2)), np.ones(2), parent=[1, 1]),
                 fcc.Bodies.new([3.0, 4.0], [3.0, 4.0], np.zeros(2), np.zeros((11, 2)), np.ones(2), type=2, parent=[2, 2]))
    assert list(c.parent) == [1, 1, 4, 4] and list(c.type) == [1, 1, 2, 2]


def test_pool_host_helpers():
    """Arena padding and grid-cell counts the pool's admission uses."""
    from conftest import fcc as f
    assert [f.pool.padded(n) for n in (0, 1, 8, 9, 30)] == [0, 8, 8, 16, 32]
    bodies, box = f.polydisperse_monolayer(128, 128, packing=0.95, maxmode=10, seed=1234)
    # cutoff 2 * 1.2 * (1 + sqrt(2/3)) + 0.3 = 4.66: a 53 x 46 grid
    assert f.pool.grid_cells(box, bodies.R0, T=np.float32) == 53 * 46


def test_pool_device_bytes_without_gpu():
    """The footprint query needs no device (admission by HBM budget)."""
    b1 = fcc.Pool.device_bytes(np.float32, 40, 1 << 20, 1 << 18, 256)
    b2 = fcc.Pool.device_bytes(np.float32, 40, 2 << 20, 1 << 18, 256)
    b64 = fcc.Pool.device_bytes(np.float64, 40, 1 << 20, 1 << 18, 256)
    assert 0 < b1 < b2 < 2 * b1 + (1 << 22) and b64 > b1
    per_body = (b2 - b1) / (1 << 20)
    assert 400 < per_body < 2000


def _header_prototypes(path=HEADER):
    """name -> list of parameter declarations, from the prototypes of fcc.h."""
    text = re.sub(r"/\*.*?\*/", " ", open(path).read(), flags=re.S)
    out = {}
    for m in re.finditer(r"^(?:fcc_status|const char\*)\s+(fcc_\w+)\s*\(([^)]*)\)\s*;", text, re.M):
        params = [p.strip() for p in m.group(2).split(",") if p.strip()]
        out[m.group(1)] = [] if params == ["void"] else params
    return out


def _header_kind(decl):
    t = re.sub(r"\b\w+$", "", decl.strip()).replace("const", "").strip()  # drop the parameter name
    if "*" in t or t == "fcc_callback":
        return "ptr"
    return {"int64_t": "i64", "int32_t": "i32", "uint64_t": "u64", "double": "f64", "int": "i32"}[t]


def _ctypes_kind(t):
    if t in (C.c_void_p, C.c_char_p) or hasattr(t, "_type_") and isinstance(t._type_, type) \
            or getattr(t, "_flags_", 0) & C._FUNCFLAG_CDECL:
        return "ptr"
    return {C.c_int64: "i64", C.c_int32: "i32", C.c_uint64: "u64", C.c_double: "f64"}[t]


def test_ctypes_signatures_match_the_header():
    """Every argtypes list the Python mirror declares has the header's arity
    and, parameter by parameter, the same kind (pointer, 32/64-bit integer,
    double): a wrong width would pass values silently truncated."""
    protos = _header_prototypes()
    lib = fcc.simulation.native_library()  # loading and declaring need no GPU
    fcc.pool._lib()
    checked = 0
    for name, params in protos.items():
        args = getattr(lib, name).argtypes
        if args is None:
            continue  # not bound from Python (C and Julia callers only)
        assert [_ctypes_kind(a) for a in args] == [_header_kind(p) for p in params], name
        checked += 1
    assert checked >= 30


def test_host_exchange_struct_is_kept_for_the_same_arrays():
    """set_state / get_state(out) keep the exchange struct of the last Bodies
    passed (the same marshalling serves the oracle): reused while the object
    holds the same arrays, rebuilt when an array is replaced, dropped by
    close(); the exchanged values are the same either way."""
    bodies, box = fcc.hexagonal_monolayer(4, 4, packing=0.9, maxmode=6, rng=3)
    kw = dict(types=(fcc.BodyType(v0=0.1, Dr=0.01),), energies=(fcc.Tension(0.1), fcc.Overlap(1.0)), T=np.float64)
    sim = oracle.OracleSimulation(bodies, box, **kw)
    state = sim.bodies
    state.coef = np.asfortranarray(state.coef)
    h1 = sim._direct_host(state)
    assert h1 is not None and sim._direct_host(state) is h1
    state.x = state.x.copy()  # a replaced array: a new struct over it
    h2 = sim._direct_host(state)
    assert h2 is not h1 and C.cast(h2.x, C.c_void_p).value == state.x.ctypes.data
    sim.set_state(state)
    out = sim.bodies
    out.coef = np.asfortranarray(out.coef)
    sim.get_state(out=out)
    assert np.array_equal(out.x, state.x) and np.array_equal(out.coef, state.coef)
    ro = out.copy()
    ro.coef = np.asfortranarray(ro.coef)
    sim.get_state(out=ro)
    ro.x.flags.writeable = False  # no longer writable: the kept struct is not used
    with pytest.raises(fcc.ArgumentError):
        sim.get_state(out=ro)
    sim.close()
    assert sim._direct == {}
