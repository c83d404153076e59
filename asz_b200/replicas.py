"""Multi-GPU replicas: independent fields (or time steps) sharded over ranks, one process per GPU.

ASZ compresses each field on its own, so the natural multi-GPU form is data-parallel replicas with
no collective on the data path: every rank runs the whole single-GPU pipeline on its share of the
units. The only communication is control: the wall time of the slowest rank and the total bytes
processed, reduced once at the end (MAX and SUM). Works with any torch.distributed backend (NCCL on
the GPU box, gloo in the CPU tests).
"""
from __future__ import annotations

import time
from dataclasses import dataclass
from typing import Callable, Sequence


def assign(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Split units over `world` ranks balancing their byte sizes: largest first, each to the rank with
    the least assigned so far (ties to the lowest rank). Deterministic, so every rank computes the
    same assignment without communicating."""
    loads = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (loads[q], q))
        out[r].append(i)
        loads[r] += sizes[i]
    for lst in out:
        lst.sort()
    return out


@dataclass
class ReplicaResult:
    units: list[int]          # units this rank processed
    results: list             # fn's return value per unit, in `units` order
    local_s: float            # this rank's time
    max_s: float              # slowest rank's time (the job's time)
    total_bytes: int          # bytes processed by all ranks


def run(sizes: Sequence[int], fn: Callable[[int], object], dist=None, timer: Callable[[], float] | None = None,
        barrier: Callable[[], None] | None = None) -> ReplicaResult:
    """Process this rank's share of the units with fn(unit) and reduce the timing over ranks.

    `dist` is torch.distributed (initialised) or None for one process. `timer` returns seconds
    (device-synchronised on the GPU path); `barrier` runs before and after the timed region."""
    import torch
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist else (0, 1)
    mine = assign(sizes, world)[rank]
    timer = timer or time.perf_counter
    if barrier:
        barrier()
    elif dist:
        dist.barrier()
    t0 = timer()
    results = [fn(u) for u in mine]
    if barrier:
        barrier()
    local = timer() - t0
    stats = torch.tensor([local, float(sum(sizes[u] for u in mine))], dtype=torch.float64)
    if dist:
        backend = dist.get_backend()
        dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
        t = stats[:1].to(dev)
        b = stats[1:].to(dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dist.all_reduce(b, op=dist.ReduceOp.SUM)
        stats = torch.cat([t.cpu(), b.cpu()])
    return ReplicaResult(mine, results, local, float(stats[0]), int(stats[1]))
