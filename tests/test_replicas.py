"""The multi-process path of the benchmark on the CPU: `bench.py --gpus N`
runs N independent replicas of the exact simulation (the exact path does not
shard: link and collide are Gauss-Seidel passes and one random stream is
shared), one process per GPU, with a process group used only to take the
slowest replica's time. Here two `gloo` ranks each run a replica on the
oracle core: the replicas must agree bit for bit, and every rank must get the
same maximum."""

import hashlib
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import datetime

    import torch.distributed as dist

    import bench
    import helpers as H
    import oracle

    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        core = oracle.load(H.pkg)
        nodes, sim = H.scenarios.setup_exact(H.pkg, core, n=400, m=800, collide_radius=5,
                                             coincident=0.01, near=0.01, pinned=0.01)
        sim.tick(3)
        digest = hashlib.sha256(b"".join(np.ascontiguousarray(a).tobytes()
                                         for a in (nodes.x, nodes.y, nodes.vx, nodes.vy))).hexdigest()
        sim.close()
        digests = [None] * world
        dist.all_gather_object(digests, digest)
        slowest = bench.max_over_ranks(1.0 + rank, world)  # a per-rank "time"
        out.put((rank, digests, slowest))
    finally:
        dist.destroy_process_group()


def test_replicas_agree_and_time_is_max_over_ranks():
    import torch.multiprocessing as mp

    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, digests, slowest in results:
        assert len(set(digests)) == 1, "replicas differ"
        assert slowest == float(world), (rank, slowest)


def test_max_over_ranks_single_process():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.5, 1) == 3.5
