"""The multi-rank plumbing of bench.py on CPU (gloo, world size 2): the
timings every rank reports are reduced to their maximum, and the reference
arm runs on rank 0 only (the other ranks exit at once, printing nothing)."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out[rank] = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 3.0], dist, device="cpu")
    finally:
        dist.destroy_process_group()


def test_timings_reduce_to_the_max_over_ranks():
    import torch.multiprocessing as mp

    world = 2
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1] == [2.0, 10.0, 3.0]


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks([4.0, 5.0]) == [4.0, 5.0]


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and r.stdout.strip() == ""
