"""The N > 1 bench path on CPU: two gloo ranks (replicas, no data-path
collective).  The ranks of a step take disjoint consecutive batches of the
pool, the whole-job times are the slowest rank's and the counts are summed,
and a non-zero rank of the reference arm prints nothing and exits 0."""
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_rank_batches_are_disjoint_and_consecutive():
    world, B, n = 2, 100, 400
    for step in range(6):
        got = [bench.batch_indices(step, r, world, B, n) for r in range(world)]
        assert not set(got[0]) & set(got[1])
        start = (step * world * B) % n
        assert got[0] + got[1] == [(start + j) % n for j in range(world * B)]


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, init_method="env://")
    try:
        r = bench.reduce_over_ranks(dist, 1.5 + rank, 2.0 - rank, 10 + rank, 1000 * (rank + 1), rank, 7)
        out[rank] = r
    finally:
        dist.destroy_process_group()


def test_reduce_over_two_gloo_ranks():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
        res = dict(out)
    expect = (2.5, 2.0, 21, 3000, 1, 14)
    assert res[0] == expect and res[1] == expect


@pytest.mark.timeout(120)
def test_reference_arm_non_zero_rank_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1", MASTER_ADDR="127.0.0.1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert p.returncode == 0 and p.stdout.strip() == ""
