"""Batched fast mode across GPUs on the CPU: graphs are independent, so
`bench.py --gpus N` gives each rank its own share of the graphs (greedy size
balance, batch.shard) with no collective on the data path; a process group
only takes the slowest rank's time. Here two `gloo` ranks each take their
share: together they hold every graph exactly once, the loads are balanced,
and both see the same slowest time."""

import os
import socket
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _batch():
    import importlib
    return importlib.import_module("d3-force-wasm_b200.batch")


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_covers_every_graph_once_and_balances():
    B = _batch()
    rng = np.random.default_rng(0)
    sizes = list(np.exp(rng.uniform(np.log(64), np.log(16384), 2048)).astype(int))
    for world in (1, 2, 3, 8):
        parts = B.shard(sizes, world)
        flat = sorted(g for p in parts for g in p)
        assert flat == list(range(len(sizes)))
        loads = [sum(sizes[g] for g in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)


def test_workload_matches_the_configuration():
    B = _batch()
    graphs = B.batch_workload(2048, seed=1)
    n = np.array([g[0] for g in graphs])
    assert n.min() >= 64 and n.max() <= 16384
    assert 5.0e6 < n.sum() < 7.0e6  # about 6M nodes
    for k, (nk, src, tgt) in enumerate(graphs[:6]):
        assert len(src) == 2 * nk and np.all(src != tgt) and src.max() < nk and tgt.max() < nk


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    B = _batch()
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        sizes = [g[0] for g in B.batch_workload(256, seed=4)]
        mine = B.shard(sizes, world)[rank]
        held = torch.zeros(len(sizes), dtype=torch.int64)
        held[mine] = 1
        dist.all_reduce(held)
        slowest = bench.max_over_ranks(float(sum(sizes[g] for g in mine)), world)
        out.put((rank, held.tolist(), slowest, sum(sizes)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_share_the_graphs():
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
    slow = {r[2] for r in results}
    assert len(slow) == 1
    for rank, held, slowest, total in results:
        assert all(h == 1 for h in held)
        assert total / 2 <= slowest <= total / 2 + 16384
