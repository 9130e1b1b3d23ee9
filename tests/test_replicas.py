"""Host logic of the multi-GPU bench on CPU: world_size-2 `gloo` ranks.

The time step does not shard (replicas only), so `bench.py --gpus N`
runs N independent monolayers, one per rank, with no collective in the data
path.  What is multi-rank is the timing: the job time is the max over ranks
and the value counts every rank's bodies.  These tests run that logic over
gloo on CPU, and check that the reference arm prints from rank 0 only.
"""

import datetime
import importlib.util
import json
import os
import socket
import subprocess
import sys

import pytest

from conftest import ROOT


def load_bench():
    spec = importlib.util.spec_from_file_location("fcc_bench", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        bench = load_bench()
        ms = 10.0 + 5.0 * rank  # rank 1 is the slow one
        ms_max = bench.max_over_ranks(ms, dist, "cpu")
        value = bench.job_throughput(world, 16384, 512, ms_max * 1e-3)
        q.put((rank, ms_max, value, bench.replica_seed(rank)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [15.0, 15.0]                       # every rank sees the slowest time
    assert out[0][2] == out[1][2] == pytest.approx(2 * 16384 * 512 / 15e-3)
    assert out[0][3] != out[1][3]                                    # independent replicas


def test_reference_arm_prints_on_rank0_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "2", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


@pytest.mark.slow
def test_reference_arm_line():
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", FCC_REF_BUDGET_S="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
