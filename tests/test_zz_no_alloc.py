"""The neighbour build that allocates no device memory.

fcc_build_neighbors_noalloc exists for callers that cannot call cudaMalloc
(code under a memory pool or allocator it does not own, or with a device
budget fixed up front): they hand it arrays already on the device and it
keeps its scratch in a static device array of the library.  This
test allocates its own device buffers (with torch, on the test's side), calls
the entry point through the C ABI, and checks it against fcc_build_neighbors,
the allocating entry point, on two calls in a row: integer outputs, so the
tolerance is equality.  Collected last so that a stop at the first failure has
run every other test before it.
"""

import ctypes as C

import numpy as np
import pytest

from conftest import fcc

pytestmark = pytest.mark.gpu

MAX_BODIES = 16384


def noalloc_fn():
    lib = fcc.native_library()
    f = lib.fcc_build_neighbors_noalloc
    f.argtypes = [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double,
                  C.c_double, C.c_int32] + [C.c_void_p] * 6 + [C.c_void_p]
    f.restype = C.c_int32
    return lib, f


def case(seed, n, Lx, Ly, T):
    rng = np.random.default_rng(seed)
    x = (rng.random(n) * Lx).astype(T)
    y = (rng.random(n) * Ly).astype(T)
    rmax = (0.8 + 0.6 * rng.random(n)).astype(T)
    return x, y, rmax


def run_noalloc(x, y, rmax, Lx, Ly, cutoff, rng_, cap, T, stream=None):
    import torch
    lib, f = noalloc_fn()
    n = len(x)
    ncx, ncy = fcc.ops.grid_dims(float(np.float32(Lx)) if T == np.float32 else Lx,
                                 float(np.float32(Ly)) if T == np.float32 else Ly, cutoff)
    dev = torch.device("cuda")
    dt = torch.float32 if T == np.float32 else torch.float64
    dx, dy, dr = (torch.tensor(a, dtype=dt, device=dev) for a in (x, y, rmax))
    out = {k: torch.full((m,), -7, dtype=torch.int32, device=dev)
           for k, m in (("cellid", n), ("perm", n), ("start", ncx * ncy), ("stop", ncx * ncy), ("idx", n * cap),
                        ("count", n))}
    if stream is not None:  # the inputs were written on the current stream
        stream.wait_stream(torch.cuda.current_stream())
    st = f(32 if T == np.float32 else 64, n, dx.data_ptr(), dy.data_ptr(), dr.data_ptr(), Lx, Ly, cutoff, rng_, cap,
           *(out[k].data_ptr() for k in ("cellid", "perm", "start", "stop", "idx", "count")),
           None if stream is None else stream.cuda_stream)
    assert st == 0, lib.fcc_last_error()
    torch.cuda.synchronize()
    h = {k: v.cpu().numpy() for k, v in out.items()}
    return h["cellid"], h["perm"], h["start"], h["stop"], h["idx"].reshape(n, cap).T, h["count"]


@pytest.mark.parametrize("T", [np.float64, np.float32])
def test_noalloc_matches_allocating_build_twice(T):
    cutoff = 2 * 1.4 * (1 + np.sqrt(2 / 3)) + 0.3
    # two calls in a row on different inputs: the second must not see the first's scratch
    for seed, n, Lx, Ly, cap in ((3, 4000, 120.0, 95.0, 24), (4, 1500, 70.0, 41.0, 8)):
        x, y, rmax = case(seed, n, Lx, Ly, T)
        a = run_noalloc(x, y, rmax, Lx, Ly, cutoff, 0.3, cap, T)
        b = fcc.build_neighbors(x.astype(np.float64), y.astype(np.float64), rmax.astype(np.float64), Lx, Ly,
                                cutoff, 0.3, cap, T)
        for u, v in zip(a, b):
            assert np.array_equal(u, v)
        assert b[5].max() > 0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    lib, f = noalloc_fn()
    st = f(64, MAX_BODIES + 1, *([None] * 3), 100.0, 100.0, 4.0, 0.3, 8, *([None] * 6), None)
    assert st == fcc.abi.FCC_ERR_ARGUMENT
    assert b"FCC_NOALLOC_MAX_BODIES" in lib.fcc_last_error()


def test_noalloc_on_a_side_stream_with_list_overflow():
    """Queued on a non-default stream, with a capacity below the largest
    neighbour count: counts beyond cap are reported as the allocating build
    reports them, and only the first cap entries are stored."""
    import torch
    T = np.float32
    cutoff = 2 * 1.4 * (1 + np.sqrt(2 / 3)) + 0.3
    x, y, rmax = case(7, 3000, 60.0, 50.0, T)
    side = torch.cuda.Stream()
    cap = 4
    a = run_noalloc(x, y, rmax, 60.0, 50.0, cutoff, 0.3, cap, T, stream=side)
    b = fcc.build_neighbors(x.astype(np.float64), y.astype(np.float64), rmax.astype(np.float64), 60.0, 50.0, cutoff,
                            0.3, cap, T)
    assert b[5].max() > cap  # the overflow case
    for u, v in zip(a, b):
        assert np.array_equal(u, v)


def test_noalloc_rejects_a_cutoff_or_box_that_is_not_finite_positive():
    lib, f = noalloc_fn()
    for Lx, cutoff in ((100.0, 0.0), (100.0, -1.0), (100.0, float("nan")), (100.0, float("inf")),
                       (float("nan"), 4.0), (-5.0, 4.0)):
        st = f(64, 10, *([None] * 3), Lx, 100.0, cutoff, 0.3, 8, *([None] * 6), None)
        assert st == fcc.abi.FCC_ERR_ARGUMENT, (Lx, cutoff)
        assert b"finite positive" in lib.fcc_last_error(), (Lx, cutoff)
    # a tiny cutoff gives a grid far beyond the scratch: rejected before any device work
    st = f(64, 10, *([None] * 3), 100.0, 100.0, 1e-30, 0.3, 8, *([None] * 6), None)
    assert st == fcc.abi.FCC_ERR_ARGUMENT
    assert b"FCC_NOALLOC_MAX_CELLS" in lib.fcc_last_error()
