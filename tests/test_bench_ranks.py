"""bench.py's multi-rank plumbing on the CPU (gloo, world size 2): every rank
joins the process group, the job's time is the maximum over the ranks, and
the reference arm's non-zero ranks exit 0 without work or output. (A single
system does not shard: `--gpus N` runs N replicas with no collective on the
data path; the maximum over ranks is the only exchange.)"""
from __future__ import annotations

import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import bench
    dist = bench._init_dist(world, backend="gloo")
    try:
        v = bench._max_over_ranks(1.5 + rank, dist, "cpu")
        dist.barrier()
        out[rank] = v
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank_main, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    assert dict(out) == {0: 2.5, 1: 2.5}


def test_single_rank_needs_no_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench._init_dist(1) is None
    assert bench._max_over_ranks(3.0, None, "cpu") == 3.0


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload", "ams40",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
