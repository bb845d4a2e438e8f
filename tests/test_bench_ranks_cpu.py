"""The multi-GPU path of bench.py on the CPU: replicas over ``gloo`` with world size 2.

The path shards by whole instances (replicas, no collective on the data path): each rank
builds its own seeded workload, and the step time is the slowest rank's (max over ranks).
Checked here without a GPU: the reduction, the per-rank workloads (same shapes, different
data), and that the reference arm prints from rank 0 only."""
import importlib
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        slowest = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        pkg = importlib.import_module("jax-gcm_b200")
        m = bench.workload_members(pkg, "t31", rank)[0]
        dist.barrier()
        q.put((rank, slowest, m.t.shape, float(m.t.astype(np.float64).sum())))
    finally:
        dist.destroy_process_group()


def test_replicas_over_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[1] for o in out] == [2.5, 2.5]          # every rank sees the slowest time
    assert out[0][2] == out[1][2]                      # same shapes on every replica
    assert out[0][3] != out[1][3]                      # different seeded data


def test_reference_arm_prints_from_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setenv("WORLD_SIZE", "2")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2"])
    args = bench.parse_args()
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args)
    assert buf.getvalue() == ""
