"""Host logic of bench.py's accuracy check, on CPU: the FP32 oracle stands in
for the CUDA path (both evaluate the reference's FP32 arithmetic), so the
check's definition can be exercised without a GPU.

At a near-tie the Overlap pressure g = J H(d) of a contour node may sit on
the other side of zero in FP32 (rounding of d is about 1e-5 at coordinates
of 100), which moves that body's force by O(J).  The check excludes exactly
those bodies (a node pressure apart by at least J/2) and counts them; every
other body must agree with FP64 to the stated bound of 1e-5 of each
field's scale."""

import importlib.util
import os

import numpy as np

from conftest import ROOT, fcc, oracle


def load_bench():
    spec = importlib.util.spec_from_file_location("fcc_bench_host", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class OracleFP32:
    """The parts of the package namespace force_error uses, with the FP32
    oracle in place of the CUDA simulation."""
    Overlap = fcc.Overlap

    @staticmethod
    def Simulation(bodies, box, T, **kw):
        return oracle.OracleSimulation(bodies, box, T=T, **kw)


def test_overlap_jump_reads_every_overlap_coupling():
    bench = load_bench()
    es = (fcc.Tension(0.01), fcc.OnTypes(fcc.Overlap([[1.0, 0.5], [0.5, 2.0]], related=[[0.0, -2.0], [-2.0, 0.0]]), 1, 2))
    assert bench.overlap_jump(fcc, es) == 0.5
    assert bench.overlap_jump(fcc, (fcc.Tension(0.01), fcc.LinearRepulsion(1.0))) is None


def test_force_error_excludes_only_heaviside_flips():
    bench = load_bench()
    bodies, box = fcc.polydisperse_monolayer(48, 48, packing=0.95, maxmode=10, seed=7)
    kw = dict(types=(fcc.BodyType(v0=0.06, Dr=0.01, μab=0.1),),
              energies=(fcc.Tension(0.01), fcc.Overlap(1.0), fcc.PerimeterElasticity(0.1, 3.7)), dt=0.005, seed=7)
    o = oracle.OracleSimulation(bodies, box, T=np.float64, **kw)
    o.step(1500)  # deformed shapes: many contacts, some near-ties
    err = bench.force_error(OracleFP32, oracle, o.bodies, box, kw)
    assert err["max_rel"] < 1e-5, err
    assert 1 <= err["excluded_flips"] and err["excluded_fraction"] < 0.01, err  # this state holds one flip
