"""Ensemble members sharded over GPUs, one process per GPU.

Members are independent, so the data path has no collective: each rank builds
a batched Ensemble of its own members and steps it.  Members are assigned by
the greedy longest-processing-time rule on their cell counts (largest first,
each to the least-loaded rank), which keeps the per-rank work within the
largest member of the mean.  The only exchange is at the end: per-member
statistics (or whole fields) gathered to one rank with torch.distributed
(NCCL over NVLink between GPUs; gloo for host tensors).
"""

from __future__ import annotations

import heapq

import numpy as np


def partition(sizes, nranks: int) -> list:
    """Member indices per rank (LPT greedy on sizes; ties to the lower rank).
    Every rank's list is in increasing member order."""
    if nranks < 1:
        raise ValueError("nranks must be >= 1")
    heap = [(0, r) for r in range(nranks)]
    out = [[] for _ in range(nranks)]
    for m in sorted(range(len(sizes)), key=lambda q: (-sizes[q], q)):
        load, r = heapq.heappop(heap)
        out[r].append(m)
        heapq.heappush(heap, (load + sizes[m], r))
    return [sorted(x) for x in out]


def member_stats(case) -> dict:
    """Scalar diagnostics of one member (the reference's stdout diagnostics,
    src/main.cpp:441-459, plus the FP64 dry-air mass)."""
    thp = case.field("thp", interior=True)
    st = {
        "w_max": case.field_absmax("w"),
        "thp_min": float(thp.min()),
        "thp_max": float(thp.max()),
        "dry_mass": case.dry_mass(),
    }
    if case.moisture:
        st["qc_max"] = float(case.field("qc", interior=True).max())
        st["qr_max"] = float(case.field("qr", interior=True).max())
        st["rain_max"] = float(case.rain(interior=True).max())
    return st


def gather_stats(local: dict, world: int, device=None) -> dict | None:
    """{member index: stats} of every rank on rank 0 (None elsewhere).  The
    statistics travel as one float64 tensor per rank (device tensors with
    NCCL, host tensors with gloo)."""
    if world == 1:
        return dict(local)
    import torch
    import torch.distributed as dist

    keys = sorted({k for st in local.values() for k in st}) if local else []
    # every rank must agree on the key set: exchange it first (small objects)
    all_keys = [None] * world
    dist.all_gather_object(all_keys, keys)
    keys = sorted({k for ks in all_keys for k in ks})
    rows = [[float(m)] + [float(st.get(k, np.nan)) for k in keys] for m, st in sorted(local.items())]
    n = torch.tensor([len(rows)], dtype=torch.int64, device=device)
    counts = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(counts, n)
    cmax = int(max(int(c.item()) for c in counts))
    width = 1 + len(keys)
    buf = torch.full((max(cmax, 1), width), np.nan, dtype=torch.float64, device=device)
    if rows:
        buf[: len(rows)] = torch.tensor(rows, dtype=torch.float64, device=device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    if dist.get_rank() != 0:
        return None
    out = {}
    for r, p in enumerate(parts):
        for row in p[: int(counts[r].item())].cpu().numpy():
            out[int(row[0])] = {k: float(v) for k, v in zip(keys, row[1:]) if not np.isnan(v)}
    return out
