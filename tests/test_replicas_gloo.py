"""The multi-GPU path of bench.py is replicas (one independent sweep per
rank); its only exchange is the max over ranks of the timed region.  These
run it with world_size 2 on the gloo backend (CPU, no GPU)."""
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # per-rank "device times": the job's time is the slowest rank's
        t = bench.max_over_ranks(torch, 10.0 + 7.5 * rank, torch.device("cpu"), world)
        out[rank] = (t, bench.aggregate_gbs(world, 2e9, 4, t))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_world2():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == 17.5
    # 2 ranks x 2 GB x 4 steps in 17.5 ms
    assert res[0][1] == pytest.approx(2 * 2e9 * 4 / 0.0175 / 1e9)


def test_single_rank_needs_no_process_group():
    import bench
    assert bench.max_over_ranks(torch, 3.25, torch.device("cpu"), 1) == 3.25


def test_reference_arm_other_ranks_exit_quietly():
    """Under torchrun only rank 0 runs and prints the reference arm."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
