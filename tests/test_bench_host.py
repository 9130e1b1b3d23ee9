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


def _request(bench, side=16):
    sp = dict(bench.serve_stream()[3])
    sp.update(nx=side, ny=side)
    return bench.make_request(fcc, sp)


def test_trajectory_audit_passes_fp32_against_fp64():
    """The serving audit's replay with the FP32 oracle standing in for the
    CUDA path: every body within its flip-charged bound."""
    bench = load_bench()
    res = bench.trajectory_audit(OracleFP32, oracle, _request(bench))
    assert res["pass"] and res["frac_within"] >= 0.95, res
    assert res["max_dr_over_bound"] <= 1.0 and res["max_dcoef_over_bound"] <= 1.0, res


def test_trajectory_audit_charges_a_flip_to_the_two_ring():
    """A flip planted in the probe's pressures at one node of body 101, every
    step: counted once per step, charged to that body, its list neighbours
    and theirs, and to no one else."""
    bench = load_bench()
    made = []

    class Planted(oracle.OracleSimulation):
        @property
        def grad(self):
            gr = super().grad
            if self is made[1]:  # the audit's second simulation is its probe
                P = np.array(gr.P)
                P[3, 100] += 1.0
                gr = gr._replace(P=P)
            return gr

    class NS:
        Overlap = fcc.Overlap

        @staticmethod
        def Simulation(bodies, box, T, **kw):
            made.append(Planted(bodies, box, T=T, **kw))
            return made[-1]

    r = _request(bench)
    res = bench.trajectory_audit(NS, oracle, r)
    assert res["flip_events"] >= bench.AUDIT_STEPS, res
    o = oracle.OracleSimulation(r.bodies, r.box, T=np.float64, **r.kw).refresh()
    nb = o.neighbors
    ring1 = set(int(j) - 1 for j in nb.idx[:nb.count[100], 100])
    ring2 = set(ring1)
    for i in ring1:
        ring2 |= set(int(j) - 1 for j in nb.idx[:nb.count[i], i])
    assert 100 in ring2 and len(ring1) >= 5
    assert res["bodies_charged"] >= len(ring2) - 2 and res["bodies_charged"] <= len(ring2) + 12, (res, len(ring2))
    assert res["pass"], res
