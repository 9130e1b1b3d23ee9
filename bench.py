"""Benchmark of the B200 time step: body-steps/s of the N = 16384 FP32 monolayer.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Workload (the metric's configuration): hexagonal_monolayer(128, 128;
packing = 0.95), R0 ~ Normal(1, 0.1) clipped to [0.8, 1.2], modes 2..10,
nθ = 40, Tension(0.01) + Overlap(1.0) + PerimeterElasticity(0.1, 3.7),
v0 = 0.06, Dr = 0.01, μab = 0.1, dt = 0.005, FP32 (FP64 a0 / projection),
synthetic seeded state (no dataset exists for this model).

A "step" is one time step of the whole monolayer.  `value` is device-timed
(CUDA events on the library's stream around the persistent multi-step
launches), `e2e` the same metric through the C ABI with host buffers
(set_state from host arrays, run, get_state to host arrays) under a wall
clock.  Under torchrun every rank runs an independent replica (different
seed): the path does not shard, so there is no collective in the data path;
the job time is the max over ranks.

`--impl reference` times the reference's CPU path on the host cores: the
C++ restatement of it (the oracle), since the Julia reference cannot run in
this image.
"""

import argparse
import importlib.util
import json
import math
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
N_SIDE = 128
WORKLOAD = "hexagonal_monolayer(128,128) N=16384 FP32, Tension(0.01)+Overlap(1.0)+PerimeterElasticity(0.1,3.7)"
METRIC = "body-steps/s at N=16384 FP32"
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "step_kernel_n16384.json")


def load_package():
    name = "fcc_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = os.path.join(ROOT, "fouriercontourcells.jl_b200")
    spec = importlib.util.spec_from_file_location(name, os.path.join(pkg, "__init__.py"), submodule_search_locations=[pkg])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    """The CPU oracle (bench's CPU-baseline leg only)."""
    name = "fcc_oracle"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "oracle", "oracle.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def workload(fcc, seed=1234):
    bodies, box = fcc.polydisperse_monolayer(N_SIDE, N_SIDE, packing=0.95, maxmode=10, seed=seed)
    kw = dict(types=(fcc.BodyType(v0=0.06, Dr=0.01, μab=0.1),),
              energies=(fcc.Tension(0.01), fcc.Overlap(1.0), fcc.PerimeterElasticity(0.1, 3.7)), dt=0.005, seed=seed)
    return bodies, box, kw


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """SM clocks and throttle reasons of one GPU during the timed region."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown", 0x4: "sw_power_cap",
               0x80: "hw_power_brake_slowdown"}

    def __init__(self, index):
        self.index, self.samples, self.reasons, self.max_mhz = index, [], set(), None
        self._stop = threading.Event()
        self._t = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self.nvml = None

    def _loop(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nvml.nvmlDeviceGetClockInfo(self.h, self.nvml.NVML_CLOCK_SM))
                r = self.nvml.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.reasons.update(n for b, n in self.REASONS.items() if r & b)
            except Exception:
                pass
            self._stop.wait(0.05)

    def __enter__(self):
        if self.nvml:
            self._t = threading.Thread(target=self._loop, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join()

    def summary(self):
        med = float(np.median(self.samples)) if self.samples else None
        return {"sm_mhz": med, "sm_max_mhz": self.max_mhz, "reasons": sorted(self.reasons), "samples": len(self.samples)}


# ------------------------------------------------------------ algorithmic work
def algorithmic_per_body_step(tests_per_body, hits_per_body, nθ=40, ncoef=19, K=9):
    """FP32 flops and compulsory HBM bytes of one body-step (the definitions
    behind the roofline; counts of node-neighbour tests and hits come from the
    oracle on the same state)."""
    flops = (2 * 2 * nθ * ncoef      # synthesis of R, R' (the reference's S*labR0 rows needed)
             + 2 * 2 * nθ * ncoef    # pullback glab = C'GR + D'GD
             + 12 * nθ               # body terms (q, Q, W R/q, W R'/q)
             + 10 * tests_per_body   # minimum image + distance test per node-neighbour pair
             + (8 * K + 8) * hits_per_body  # R_j(psi) recurrence and depth per hit
             + 12 * nθ               # contact gradient, force and torque per node
             + 30 * K + 60)          # body frame, update, constraints, lab frame
    # own record read + next record write (96 B each), coefficients r/w, neighbour
    # list (count + ~6 ids), R0, forces/energy written
    bytes_ = 96 + 96 + 2 * 76 + 4 * (1 + 6) + 4 + 16
    return flops, bytes_


def algorithmic_per_body_step_survey(tests_per_body, hits_per_body, nθ=40, ncoef=19, K=9):
    """The same work counted as the reference's dense formulation does it:
    synthesis of R, R', R'' (3 rows of S) and the pullback of all three,
    16 flops per node-neighbour test and 6K + 12 per hit.  Reported beside
    the minimal count above; R'' and its pullback are zero work for these
    terms, which is why the minimal count leaves them out."""
    return (2 * 3 * nθ * ncoef + 2 * 3 * nθ * ncoef + 12 * nθ + 16 * tests_per_body
            + (6 * K + 12) * hits_per_body + 10 * nθ + 30 * K + 60)


# ------------------------------------------------------------ replicas
def replica_seed(rank):
    """Every rank runs an independent monolayer of its own seed."""
    return 1234 + rank


def max_over_ranks(x, dist=None, device="cpu"):
    """Job time = the slowest rank's time (all ranks take this collective)."""
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, n_bodies, steps, seconds):
    """Body-steps/s of the whole job: every rank's bodies over the slowest time."""
    return world * n_bodies * steps / seconds


def flush_l2():
    import torch
    buf = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    buf.fill_(1.0)
    torch.cuda.synchronize()
    del buf


# ------------------------------------------------------------ batching
BATCH_WORKLOAD = ("256 monolayers, N log-uniform on [64, 4096] (square-ish hexagonal packings at 0.95, "
                  "R0 ~ N(1, 0.1) clipped to [0.8, 1.2]), v0 ~ U[0.02, 0.2], eta log-uniform on [0.001, 0.1], "
                  "Tension(eta) + Overlap(1.0), Dr 0.01, mu_ab 0.1, dt 0.005, 2000 steps each, FP32")


def batch_members(fcc, count=256, nmin=64, nmax=4096, seed=2024):
    """The batching workload: `count` independent monolayers of uneven N."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n_t = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        ny = max(2, 2 * round(math.sqrt(2 * n_t / math.sqrt(3)) / 2))  # Lx ~ Ly
        nx = max(1, round(n_t / ny))
        v0 = float(rng.uniform(0.02, 0.2))
        eta = float(math.exp(rng.uniform(math.log(1e-3), math.log(0.1))))
        sd = int(rng.integers(1, 2**31 - 1))
        bodies, box = fcc.polydisperse_monolayer(nx, ny, packing=0.95, maxmode=10, seed=sd)
        kw = dict(types=(fcc.BodyType(v0=v0, Dr=0.01, μab=0.1),), energies=(fcc.Tension(eta), fcc.Overlap(1.0)),
                  dt=0.005, seed=sd)
        out.append((bodies, box, kw))
    return out


def batched_leg(fcc, steps=2000, warm=3, count=256):
    """Batched (one pool, one persistent launch per 512 steps for all 256
    monolayers) against the plain per-simulation loop (each monolayer run
    alone, one after the other), on the same inputs; device-timed."""
    import torch
    members = batch_members(fcc, count)
    total = sum(b.n for b, _, _ in members)
    cells = sum(fcc.pool.grid_cells(box, b.R0, T=np.float32) for b, box, _ in members)
    pool = fcc.Pool(T=np.float32, max_bodies=sum(fcc.pool.padded(b.n) for b, _, _ in members),
                    max_cells=cells, max_sims=count)
    slots = [pool.add(b, box, horizon=warm + steps, **kw) for b, box, kw in members]
    tuned = pool.tune(64)  # launch shape for this size bucket (snapshot restored)
    pool.run(warm)
    flush_l2()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    pool.run(steps)
    wall_b = time.perf_counter() - t0
    ms_b, launches_b, bsteps = pool.last_timing()
    var = pool.variant()
    var["autotuned"] = {"variant": tuned[0], "us_per_step": tuned[1]}
    var["graph"] = dict(zip(("active", "replays"), pool.graph()))
    # plain loop
    wall_p, equal = 0.0, 0
    plain_ms = []  # device ms of each member alone
    for (b, box, kw), slot in zip(members, slots):
        sim = fcc.Simulation(b, box, T=np.float32, **kw)
        sim.run(warm)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.run(steps)
        wall_p += time.perf_counter() - t0
        plain_ms.append(sim.last_timing()[0])
        a, c = sim.bodies, pool.bodies(slot)
        equal += int(all(np.array_equal(getattr(a, f), getattr(c, f)) for f in ("x", "y", "θ", "coef", "imgx")))
        sim.close()
    pool.close()
    ms_p = float(sum(plain_ms))
    # the plain loop's best kernel per member: 16 lanes per body is faster for
    # small monolayers (results then differ from the pool's at FP32 rounding)
    best_ms, prev = 0.0, os.environ.get("FCC_VARIANT")
    for (b, box, kw), m0 in zip(members, plain_ms):
        os.environ["FCC_VARIANT"] = "4"
        sim = fcc.Simulation(b, box, T=np.float32, **kw)
        sim.run(warm)
        sim.run(steps)
        best_ms += min(m0, sim.last_timing()[0])
        sim.close()
    if prev is None:
        os.environ.pop("FCC_VARIANT", None)
    else:
        os.environ["FCC_VARIANT"] = prev
    vb = total * steps / (ms_b * 1e-3)
    vp = total * steps / (ms_p * 1e-3)
    vpb = total * steps / (best_ms * 1e-3)
    return {"workload": BATCH_WORKLOAD, "sims": count, "bodies": total, "steps": steps,
            "batched": {"value": vb, "unit": "body-steps/s", "ms": ms_b, "launches": launches_b,
                        "wall_value": total * steps / wall_b, "kernel": var},
            "plain": {"value": vp, "unit": "body-steps/s", "ms": ms_p, "wall_value": total * steps / wall_p,
                      "kernel": "same variant as the pool (8 lanes x 5 node slots)"},
            "plain_best": {"value": vpb, "unit": "body-steps/s", "ms": best_ms,
                           "kernel": "per member the faster of 8 x 5 and 16 x 3 lanes x node slots"},
            "batched_over_plain": vb / vp,
            "batched_over_plain_best": vb / vpb,
            "bitwise_equal_to_plain": f"{equal}/{count}"}


# ------------------------------------------------------------ accuracy
def overlap_jump(fcc, energies):
    """Smallest nonzero jump J of the Overlap pressures g = J H(d) among
    `energies` (OnTypes unwrapped), or None without an Overlap term."""
    js = []
    for e in energies:
        t = getattr(e, "term", e)
        if isinstance(t, fcc.Overlap):
            js += [abs(v) for row in t.J + t.Jrelated for v in row if v != 0]
    return min(js) if js else None


def force_error(fcc, oracle, bodies, box, kw):
    """FP32 forces of the CUDA path against the FP64 oracle on the same
    (FP32-representable) state: max |error| / max |oracle value| per field.
    Bodies with a Heaviside flip are excluded and counted: a contour node
    whose contact state differs between the two evaluations (node pressure
    apart by at least J/2, J the smallest Overlap jump), because g = J H(d)
    jumps by J where d crosses zero and FP32 rounding of d (about 1e-5 at
    coordinates of 250) decides the side at a near-tie."""
    b = bodies.copy()
    for f in ("x", "y", "θ", "coef", "R0"):
        setattr(b, f, np.asarray(getattr(b, f), dtype=np.float32).astype(np.float64))
    g = fcc.Simulation(b, box, T=np.float32, **kw)
    g.refresh()  # neighbour lists of this state, then compute_gradients!
    o = oracle.OracleSimulation(b, box, T=np.float64, **kw)
    o.refresh()
    J = overlap_jump(fcc, kw["energies"])
    gg, og = g.grad, o.grad
    if J is None:
        flip = np.zeros(b.n, dtype=bool)
    else:
        flip = np.abs(np.asarray(gg.P, float) - np.asarray(og.P, float)).max(axis=0) >= 0.5 * J
    keep = ~flip
    out = {}
    for f in ("gx", "gy", "gθ", "gcoef", "Ebody"):
        a, r = np.asarray(getattr(gg, f), float), np.asarray(getattr(og, f), float)
        scale = max(float(np.abs(r).max()), 1e-300)
        out[f] = float(np.abs(a[..., keep] - r[..., keep]).max() / scale) if keep.any() else 0.0
    g.close()
    return {"max_rel": max(out.values()), "fields": out, "excluded_flips": int(flip.sum()),
            "excluded_fraction": float(flip.mean()),
            "definition": "max |F32 - F64| / max |F64| per field on the same state; bodies with a node whose "
                          "contact state differs (Heaviside flip at a near-tie, |dP| >= J/2) excluded and counted"}


# ------------------------------------------------------------ serving
SERVE_WORKLOAD = ("Poisson stream (lambda = 20 req/s) of requests: N log-uniform on [256, 65536] (square-ish "
                  "hexagonal packings at 0.95, R0 ~ N(1, 0.1) clipped to [0.8, 1.2]), horizon U[1000, 50000] "
                  "steps, v0 U[0.02, 0.2], eta U[0.001, 0.1], Dr U[0.005, 0.05], Tension(eta) + Overlap(1.0), "
                  "mu_ab 0.1, dt 0.005, per-request Philox seed, FP32 bulk with FP64 a0/projection")


def serve_stream(count=2000, rate=20.0, seed=77):
    """Specs of the serving stream (bodies are made on demand)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += float(rng.exponential(1.0 / rate))
        n_t = math.exp(rng.uniform(math.log(256), math.log(65536)))
        ny = max(2, 2 * round(math.sqrt(2 * n_t / math.sqrt(3)) / 2))
        nx = max(1, round(n_t / ny))
        out.append(dict(id=i, arrival=t, nx=nx, ny=ny, horizon=int(rng.integers(1000, 50001)),
                        v0=float(rng.uniform(0.02, 0.2)), eta=float(rng.uniform(0.001, 0.1)),
                        Dr=float(rng.uniform(0.005, 0.05)), seed=int(rng.integers(1, 2**31 - 1))))
    return out


def make_request(fcc, sp):
    bodies, box = fcc.polydisperse_monolayer(sp["nx"], sp["ny"], packing=0.95, maxmode=10, seed=sp["seed"])
    kw = dict(types=(fcc.BodyType(v0=sp["v0"], Dr=sp["Dr"], μab=0.1),),
              energies=(fcc.Tension(sp["eta"]), fcc.Overlap(1.0)), dt=0.005, seed=sp["seed"])
    return fcc.Request(bodies, box, kw, sp["horizon"], sp["arrival"], sp["id"])


AUDIT_STEPS = 10


def trajectory_audit(fcc, oracle, r, steps=AUDIT_STEPS):
    """The first `steps` steps of request r in FP32 on the GPU (its solo run,
    which the served result equals bit for bit) against the FP64 oracle from
    the same FP32-representable initial state and Philox stream.

    Before each step the contact pressures of both runs are evaluated (the
    GPU's on a separate simulation loaded with its state, so the audited run
    is the plain one); a node whose pressure differs by at least J/2 is a
    Heaviside flip (an Overlap near-tie decided the other way by FP32
    rounding).  One flipped node held for one step moves a body by at most
    dt mu_r J s_max and a shape coefficient by at most dt mu_ab J s_max
    (s_max: the longest contour element R0 |r'(phi)| dphi, |dd/dx| <= 1 and
    |dd/dc| <= 1); the contact partner gets the reaction, and a displaced
    body moves its own neighbours by a further factor dt J (contact length)
    ~ 0.005 per step, so body i is charged every event of its two-ring
    neighbourhood (itself, its list neighbours and theirs).  The events are
    seen through the gradient kernel, whose FP32 rounding at a near-tie may
    differ from the step kernel's, so each body is also allowed one node of
    its contacts flipped through the whole replay unseen (`steps` events).
    Stated tolerance: 95% of the bodies within 4 FP32 ulps of their
    coordinates and 1e-6 in every coefficient; every body within one ulp per
    step (coefficients 1e-6 per step) plus (steps + its charge) dt mu J
    s_max."""
    b = r.bodies.copy()
    for f in ("x", "y", "θ", "coef", "R0"):
        setattr(b, f, np.asfortranarray(np.asarray(getattr(b, f), np.float32).astype(np.float64)))
    (bt,) = r.kw["types"]
    J = float(np.max(next(e for e in r.kw["energies"] if isinstance(e, fcc.Overlap)).J))
    g = fcc.Simulation(b, r.box, T=np.float32, **r.kw)
    probe = fcc.Simulation(b, r.box, T=np.float32, **r.kw)
    o = oracle.OracleSimulation(b, r.box, T=np.float64, **r.kw)
    charged, s_max, events = np.zeros(b.n), 0.0, 0
    nθ = g.nθ
    k = np.concatenate([[0.0], np.arange(2, (b.ncoef - 1) // 2 + 2), np.arange(2, (b.ncoef - 1) // 2 + 2)])
    for _ in range(steps):
        cur = g.bodies
        probe.set_state(cur, clock=g.clock)
        probe.refresh()
        o.refresh()
        own = (np.abs(np.asarray(probe.grad.P) - np.asarray(o.grad.P)) >= 0.5 * J).sum(axis=0).astype(float)
        events += int(own.sum())
        if own.any():
            nb = probe.neighbors
            slot, rows = np.nonzero(np.arange(nb.cap)[:, None] < nb.count[None, :])
            cols = nb.idx[slot, rows] - 1  # the lists are 1-based
            ring = own.copy()
            for _ in range(2):  # two rings of list neighbours (the lists are symmetric)
                nxt = ring.copy()
                np.add.at(nxt, rows, ring[cols])
                ring = nxt
            charged += ring
        # R0 (|R| + |R'|) <= R0 sum_k (1 + k) |c_k| bounds R0 sqrt(R^2 + R'^2)
        rad = np.asarray(cur.R0) * ((1 + k)[:, None] * np.abs(np.asarray(cur.coef))).sum(0)
        s_max = max(s_max, 2 * math.pi / nθ * float(rad.max()))
        g.step(1)
        o.step(1)
    bg, bo = g.bodies, o.bodies
    g.close()
    probe.close()
    Lx, Ly = r.box.Lx, r.box.Ly
    dr = np.hypot(bg.x + bg.imgx * Lx - bo.x - bo.imgx * Lx, bg.y + bg.imgy * Ly - bo.y - bo.imgy * Ly)
    dc = np.abs(bg.coef - bo.coef).max(axis=0)
    ulp = np.spacing(np.maximum(np.abs(bo.x), np.abs(bo.y)).astype(np.float32)).astype(np.float64)
    within = float(np.mean((dr < 4 * ulp) & (dc < 1e-6)))
    dt = float(r.kw.get("dt", 0.005))
    bound_dr = steps * ulp + (steps + charged) * dt * bt.mu_r * J * s_max
    bound_dc = steps * 1e-6 + (steps + charged) * dt * bt.mu_ab * J * s_max
    return {"n": b.n, "max_dr": float(dr.max()), "max_dcoef": float(dc.max()), "frac_within": within,
            "flip_events": events, "bodies_charged": int((charged > 0).sum()),
            "max_dr_over_bound": float((dr / bound_dr).max()), "max_dcoef_over_bound": float((dc / bound_dc).max()),
            "pass": bool(within >= 0.95 and (dr <= bound_dr).all() and (dc <= bound_dc).all())}


def serving_leg(fcc, oracle, work=1.5e10, pool_bodies=1 << 18, policy="fifo", plain=True, check_every=1):
    """The first requests of the serving stream (up to `work` body-steps),
    served by continuous batching on one pool sized from an HBM budget, then
    the same requests run one at a time (the plain loop), each result
    compared bit for bit with the served one.  `plain` False (the whole
    stream): no plain loop; every `check_every`-th request is run alone for
    the bitwise comparison only."""
    import torch
    stream = serve_stream()
    offered = 20.0 * float(np.mean([sp["nx"] * sp["ny"] * sp["horizon"] for sp in stream]))
    sample, acc = [], 0.0
    for sp in stream:
        w = sp["nx"] * sp["ny"] * sp["horizon"]
        if sample and acc + w > work:
            break
        sample.append(sp)
        acc += w
    reqs = [make_request(fcc, sp) for sp in sample]
    budget = fcc.Pool.device_bytes(np.float32, 40, pool_bodies, pool_bodies // 4, 256)
    pool = fcc.Pool.for_budget(budget, T=np.float32, max_sims=256)
    srv = fcc.Server(pool, chunk=512, policy=policy)
    torch.cuda.synchronize()
    res = srv.serve(reqs)
    served = fcc.serving.summary(res)
    by_id = {r.id: r for r in res}
    # the plain loop: each request alone, in arrival order
    durations, equal = [], 0
    solo = reqs if plain else reqs[::check_every]
    for r in solo:
        t0 = time.perf_counter()
        sim = fcc.Simulation(r.bodies, r.box, T=np.float32, **r.kw)
        sim.run(r.horizon)
        b = sim.bodies
        durations.append(time.perf_counter() - t0)
        c = by_id[r.id].bodies
        equal += int(all(np.array_equal(getattr(b, f), getattr(c, f)) for f in ("x", "y", "θ", "coef", "imgx")))
        sim.close()
    plain_stats = None
    if plain:
        lat = fcc.serving.sequential_latencies([r.arrival for r in reqs], durations)
        plain_span = max(a + l for a, l in zip((r.arrival for r in reqs), lat)) - min(r.arrival for r in reqs)
        plain_stats = {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
                       "body_steps_per_s": served["body_steps"] / plain_span}
    # audited requests: at least 20 (or all), spread over the sample; each
    # served result equals its solo run bit for bit (checked above for every
    # request), so the audit checks that solo path against the FP64 oracle:
    # the first steps of its trajectory, and the forces of its final state
    audit = reqs[::max(1, len(reqs) // 20)] if len(reqs) >= 20 else list(reqs)
    errs, traj = {}, {}
    for r in audit:
        errs[r.id] = force_error(fcc, oracle, by_id[r.id].bodies, r.box, r.kw)["max_rel"]
        traj[r.id] = trajectory_audit(fcc, oracle, r)
    u = pool.usage()
    pool.close()
    return {"workload": SERVE_WORKLOAD,
            "sample": f"the first {len(reqs)} requests of the seeded 2000-request stream ({acc:.3g} body-steps)",
            "offered_body_steps_per_s": offered,
            "pool": {"hbm_budget_bytes": budget, "max_bodies": u["max_bodies"], "max_sims": u["max_sims"]},
            "policy": policy, "served": served, "plain": plain_stats,
            "served_over_plain": served["body_steps_per_s"] / plain_stats["body_steps_per_s"] if plain else None,
            "chunks": srv.chunks, "device_busy_fraction": srv.device_ms * 1e-3 / max(served["makespan_s"], 1e-9),
            "bitwise_equal_to_alone": f"{equal}/{len(solo)}",
            "audited": len(audit),
            "audit_force_error_vs_fp64": errs,
            "audit_trajectory_vs_fp64": {
                "steps": AUDIT_STEPS, "passed": f"{sum(t['pass'] for t in traj.values())}/{len(traj)}",
                "worst_max_dr": max(t["max_dr"] for t in traj.values()),
                "worst_max_dcoef": max(t["max_dcoef"] for t in traj.values()),
                "worst_dr_over_bound": max(t["max_dr_over_bound"] for t in traj.values()),
                "worst_dcoef_over_bound": max(t["max_dcoef_over_bound"] for t in traj.values()),
                "min_frac_within": min(t["frac_within"] for t in traj.values()),
                "flip_events": sum(t["flip_events"] for t in traj.values()),
                "tolerance": "95% of bodies within 4 FP32 ulps of their coordinates and 1e-6 in every shape "
                             "coefficient; every body within one ulp (1e-6) per step plus dt mu J s_max per "
                             "Heaviside flip event (node x step with |dP| >= J/2 between the runs) in its "
                             "two-ring neighbourhood, plus one node flipped unseen through the replay",
                "per_request": traj}}


# ------------------------------------------------------------------ arms
def cpu_baseline(fcc, oracle, budget_s=15.0, max_steps=200):
    """The oracle (FP64, OpenMP on all host cores) on the same workload,
    for a bounded number of steps (about `budget_s` seconds)."""
    threads = oracle.set_threads(0)
    bodies, box, kw = workload(fcc)
    sim = oracle.OracleSimulation(bodies, box, T=np.float64, **kw)
    sim.step(1)  # first step builds the neighbour list
    t0 = time.perf_counter()
    sim.step(1)
    one = time.perf_counter() - t0
    steps = int(max(2, min(max_steps, budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    sim.step(steps)
    dt = time.perf_counter() - t0
    v = bodies.n * steps / dt
    return {"value": v, "unit": "body-steps/s", "cores": threads, "kind": "port",
            "sample": f"{steps} FP64 steps of the N={bodies.n} workload on {threads} threads (C++ restatement of the reference CPU path)"}, sim


def reference_arm(args):
    """--impl reference: rank 0 times the reference CPU path (its C++
    restatement) on the bench workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    fcc = load_package()
    oracle = load_oracle()
    budget = float(os.environ.get("FCC_REF_BUDGET_S", "60"))
    per = max(1.0, budget / max(1, args.warmup + args.steps))
    threads = oracle.set_threads(0)
    bodies, box, kw = workload(fcc)
    sim = oracle.OracleSimulation(bodies, box, T=np.float64, **kw)
    sim.step(1)
    t0 = time.perf_counter()
    sim.step(1)
    one = time.perf_counter() - t0
    # every bench step is a bounded sample: as many time steps of the full
    # monolayer as fit into the per-step budget (at least one)
    k = max(1, int(per / max(one, 1e-6)))
    for _ in range(args.warmup):
        sim.step(1)
    nsteps = min(args.steps, max(1, int(budget / max(one * k, 1e-6))))
    t0 = time.perf_counter()
    for _ in range(nsteps):
        sim.step(k)
    dt = time.perf_counter() - t0
    value = bodies.n * k * nsteps / dt
    line = {"metric": METRIC, "value": value, "unit": "body-steps/s", "n_gpus": args.gpus, "steps": nsteps,
            "warmup": args.warmup, "ms_per_step": dt / (k * nsteps) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD.replace("FP32", "FP64 (reference CPU path)"), "n": bodies.n, "nθ": 40},
            "impl": "reference",
            "cpu_baseline": {"value": value, "unit": "body-steps/s", "cores": threads, "kind": "port",
                             "sample": f"{nsteps} samples of {k} FP64 time steps of the N={bodies.n} workload "
                                       f"(C++ restatement of the reference CPU path; Julia is not in the image)"},
            "e2e": {"value": value, "unit": "body-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def gpu_arm(args):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local))
    fcc = load_package()
    bodies, box, kw = workload(fcc, seed=replica_seed(rank))
    sim = fcc.Simulation(bodies, box, T=np.float32, **kw)
    N = bodies.n

    # warm-up (also builds the neighbour list and settles the rebuild cadence)
    sim.run(max(3, args.warmup))
    start, start_clock = sim.bodies, sim.clock  # the e2e runs replay the timed steps from here
    flush_l2()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        sim.run(args.steps)
        torch.cuda.synchronize()
    ms, launches, steps = sim.last_timing()
    if dist:
        dist.barrier()
    ms_max = max_over_ranks(ms, dist, "cuda")
    value = job_throughput(world, N, steps, ms_max * 1e-3)

    # end to end through the C ABI with host buffers (wall clock, max over
    # ranks): the same K steps from the same state and clock (the contact work
    # of a monolayer grows as its shapes deform, so later steps cost more).
    # The input state and the result sit in page-locked host memory
    # (fcc_host_alloc); set_state copies the input to the device and
    # get_state copies the result back into the output arrays, each array in
    # one transfer, converted on the device.
    host = fcc.pinned_copy(start)
    out = fcc.pinned_bodies(N, host.ncoef)
    # bytes that cross PCIe: set_state reads x, y, theta, coef and the image
    # counters; get_state writes the same fields (R0, type and parent are the
    # created ones and come from the library's host mirror)
    moved = ("x", "y", "θ", "imgx", "imgy", "coef")
    h2d = sum(getattr(host, f).nbytes for f in moved)
    d2h = sum(getattr(out, f).nbytes for f in moved)
    # five repetitions, the median reported (a single wall-clock sample
    # carries the host's scheduling noise)
    e2e_runs, phases = [], []
    for _ in range(5):
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sim.set_state(host, clock=start_clock)
        t1 = time.perf_counter()
        sim.run(args.steps)
        t2 = time.perf_counter()
        sim.get_state(out=out)
        t3 = time.perf_counter()
        e2e_runs.append(max_over_ranks(t3 - t0, dist, "cuda"))
        phases.append((t1 - t0, t2 - t1, t3 - t2))
        assert np.isfinite(out.x).all()
    e2e = job_throughput(world, N, args.steps, float(np.median(e2e_runs)))
    e2e_phases = {k: float(np.median([p[q] for p in phases])) * 1e3
                  for q, k in enumerate(("set_state_ms", "run_ms", "get_state_ms"))}

    if rank == 0:
        peaks = {}
        try:
            peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        except Exception:
            pass
        hbm_peak = peaks.get("hbm_gbs", 6650.0)
        peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
        # work counters of the state the timed steps ran on (oracle, same state)
        oracle = load_oracle()
        osim = oracle.OracleSimulation(out, box, T=np.float64, **kw)
        osim.refresh()
        tests, hits, _ = osim.contact_counters()
        flops_b, bytes_b = algorithmic_per_body_step(tests / N, hits / N)
        launch_ms = ms / max(1, launches)
        steps_per_launch = steps / max(1, launches)
        bytes_launch = bytes_b * N * steps_per_launch
        achieved_gbs = bytes_launch / (launch_ms * 1e-3) / 1e9
        # DRAM bytes of one timed launch from the committed ncu capture of this
        # launch shape (exact when its step count was captured, else the
        # steady-state bytes per step scaled to the launch)
        traffic = None
        try:
            prof = json.load(open(PROFILE_SUMMARY))
            by = prof.get("dram_bytes_per_launch_by_steps", {})
            key = str(int(round(steps_per_launch)))
            traffic = float(by[key]) if key in by else prof["dram_bytes_per_step"] * steps_per_launch
        except Exception:
            pass
        cs = clk.summary()
        sm_mhz = cs["sm_mhz"] or 1965.0
        fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
        achieved_tf = flops_b * N * steps_per_launch / (launch_ms * 1e-3) / 1e12
        # the CPU baseline and the batching and serving legs are one-GPU figures:
        # they run at N = 1 only (the other ranks would wait for rank 0 at the
        # closing barrier for minutes)
        single = world == 1
        cpu = cpu_baseline(fcc, oracle)[0] if single else None
        batched = batched_leg(fcc, steps=args.batch_steps) if single and not args.skip_batched else None
        served = serving_leg(fcc, oracle, work=args.serve_work, policy=args.serve_policy,
                             pool_bodies=args.serve_pool_bodies) if single and args.serve_work > 0 else None
        ferr = force_error(fcc, oracle, out, box, kw)
        flops_s = algorithmic_per_body_step_survey(tests / N, hits / N)
        # key order: the bulky leg reports first, the headline figures last (a
        # reader of the line's tail sees the roofline, e2e and clocks)
        line = {
            "metric": METRIC, "value": value, "unit": "body-steps/s", "n_gpus": world, "steps": steps,
            "warmup": args.warmup, "ms_per_step": ms_max / steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n": N, "nθ": 40, "modes": "2..10", "parallelism": f"replicas{world}",
                       "steps_per_launch": steps_per_launch,
                       "l2": "flushed before the timed region; state (3.5 MB) is L2-resident by design and each step "
                             "reads the previous step's output"},
            "batched": batched,
            "serving": served,
            "builds": sim.builds,
            "err_vs_fp64": ferr,
            "cpu_baseline": cpu,
            "gpu_launches": launches * world,
            "clocks": cs,
            "e2e": {"value": e2e, "unit": "body-steps/s", "h2d_bytes_per_step": h2d / args.steps,
                    "d2h_bytes_per_step": d2h / args.steps,
                    "api": "fcc_set_state(pinned host) + fcc_run(K) + fcc_get_state(pinned host), wall clock",
                    "runs_s": e2e_runs, "reported": "median of 5", "phases_ms": e2e_phases},
            "roofline_hbm": {"bound": "hbm", "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
                             "frac": achieved_gbs / hbm_peak, "traffic": traffic,
                             "peak_source": f"{peak_src} hbm_gbs",
                             "note": "compulsory bytes per body-step; the state is L2-resident, so HBM does not bind"},
            "roofline": {"bound": "fp32", "achieved": achieved_tf, "peak": fp32_peak, "unit": "TFLOP/s",
                         "frac": achieved_tf / fp32_peak, "traffic": traffic,
                         "flops_per_body_step": flops_b, "tests_per_body": tests / N, "hits_per_body": hits / N,
                         "frac_survey_count": flops_s * N * steps_per_launch / (launch_ms * 1e-3) / 1e12 / fp32_peak,
                         "peak_source": "nominal FP32 (148 SM x 128 lanes x 2 flop) at the sampled SM clock; "
                                        "no measured FP32 peak exists for this pool"},
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20000)
    ap.add_argument("--warmup", type=int, default=200)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--skip-batched", action="store_true", help="leave out the batching leg")
    ap.add_argument("--serve-work", type=float, default=1.5e10,
                    help="body-steps of the serving sample (0: leave out the serving leg)")
    ap.add_argument("--batch-steps", type=int, default=2000, help="steps of the batching leg")
    ap.add_argument("--serve-policy", default="fifo", choices=["fifo", "sjf"], help="serving admission order")
    ap.add_argument("--serve-pool-bodies", type=int, default=1 << 18,
                    help="bodies the serving pool's HBM budget is sized for")
    ap.add_argument("--serve-no-plain", action="store_true",
                    help="serving leg without the plain loop (the whole stream); see --serve-check-every")
    ap.add_argument("--serve-check-every", type=int, default=1,
                    help="with --serve-no-plain: every k-th request is run alone for the bitwise comparison")
    ap.add_argument("--only", choices=["batched", "serving"],
                    help="run one leg alone and print its JSON (profiling; not the bench line)")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
    elif args.only:
        import torch
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        fcc = load_package()
        out = batched_leg(fcc, steps=args.batch_steps) if args.only == "batched" else \
            serving_leg(fcc, load_oracle(), work=args.serve_work, policy=args.serve_policy,
                        pool_bodies=args.serve_pool_bodies, plain=not args.serve_no_plain,
                        check_every=max(1, args.serve_check_every))
        print(json.dumps({"leg": args.only, **out}, default=str), flush=True)
    else:
        gpu_arm(args)


if __name__ == "__main__":
    main()
