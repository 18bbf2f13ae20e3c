"""The benchmark's multi-rank plumbing on CPU: two gloo ranks (world size 2)
take the max over ranks and meet at barriers exactly as the NCCL ranks do on
GPUs; the reference arm runs on rank 0 only."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _rank(rank, world, port, q):
    import datetime
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    bench.barrier(world)
    m = bench.max_over_ranks(1.5 + rank, world, device="cpu")
    bench.barrier(world)
    q.put((rank, m, bench.job_rate(world, 1024, m, 4)))
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert [g[1] for g in got] == [2.5, 2.5]  # both ranks see the slowest one
    # weak scaling: 2 squares of 1024^2 shares per 2.5/4 ms step
    assert got[0][2] == pytest.approx(2 * 1024 * 1024 * 512 * 8 / (2.5 / 4 * 1e-3) / 1e9)


def _bench(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], env=env, capture_output=True,
                          text=True, timeout=300)


def test_reference_arm_other_ranks_exit_quietly():
    r = _bench({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--impl", "reference", "--gpus", "2",
               "--side", "64", "--steps", "1", "--warmup", "3", "--ref-step-budget", "0.05")
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line(lib):
    r = _bench({"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"}, "--impl", "reference", "--side", "64",
               "--steps", "2", "--warmup", "3", "--ref-step-budget", "0.05")
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["unit"] == "Gb/s" and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
