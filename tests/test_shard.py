"""Member sharding over ranks (wfe_b200.shard): the partition, and the final
statistics gather over a world-size-2 gloo process group on the CPU."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from wfe_b200 import shard

SIZES = [120 * 90 * 45] * 8 + [220 * 150 * 45] * 8 + [300 * 200 * 45] * 8


def test_partition_covers_members_once_and_balances():
    for n in (1, 2, 3, 4, 8):
        parts = shard.partition(SIZES, n)
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(len(SIZES)))
        loads = [sum(SIZES[q] for q in p) for p in parts]
        # LPT: no rank exceeds the mean by more than the largest member
        assert max(loads) - sum(loads) / n <= max(SIZES)
        assert all(p == sorted(p) for p in parts)
    assert shard.partition([5, 1, 1], 2) == [[0], [1, 2]]
    with pytest.raises(ValueError):
        shard.partition([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from datetime import timedelta

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    parts = shard.partition(SIZES, world)
    local = {m: {"w_max": float(m) + 0.5, "dry_mass": 1e12 + m} for m in parts[rank]}
    if rank == 1:  # a key only one rank has
        local[parts[1][0]]["qr_max"] = 0.25
    got = shard.gather_stats(local, world)
    if rank == 0:
        out.put(got)
    dist.barrier()
    dist.destroy_process_group()


def test_gather_stats_two_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert sorted(got) == list(range(len(SIZES)))
    for m, st in got.items():
        assert st["w_max"] == m + 0.5 and st["dry_mass"] == 1e12 + m
    parts = shard.partition(SIZES, 2)
    assert got[parts[1][0]]["qr_max"] == 0.25
    assert all("qr_max" not in got[m] for m in got if m != parts[1][0])


def test_gather_stats_single_rank_is_identity():
    local = {3: {"w_max": 1.0}}
    assert shard.gather_stats(local, 1) == local
    assert np.isclose(shard.gather_stats({}, 1).get(0, {"x": 1})["x"], 1)
