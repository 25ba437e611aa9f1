"""The multi-GPU path is replicas only: every rank decrypts its own seeded batch,
the only collectives are a barrier and the max over ranks of each timing, and
the reported rate is the whole job's.  These run the bench's cross-rank steps
with two gloo ranks on the CPU, and check that the reference arm under a
launcher runs on rank 0 alone."""
from __future__ import annotations

import datetime
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank: int, world: int, port: int, q) -> None:
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sys.path.insert(0, REPO)
        import bench
        ms = 10.0 + 5.0 * rank                     # rank 1 is the slow one
        slowest = bench.max_over_ranks(ms, world, device="cpu")
        rate = bench.job_rate(world, 65536 * 4, slowest * 1e-3)
        dist.barrier()
        q.put((rank, slowest, rate, bench.rank_seed(rank)))
    finally:
        dist.destroy_process_group()


def test_two_replicas_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, v0, s0), (r1, m1, v1, s1) = got
    assert m0 == m1 == 15.0                       # max over ranks, identical on both
    assert v0 == v1 == pytest.approx(2 * 65536 * 4 / 0.015)
    assert s0 != s1                               # each replica its own batch


def test_reference_arm_rank_nonzero_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(REPO, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "1"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
