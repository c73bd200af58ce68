"""Host-side helpers for running one engine per GPU under torch.distributed.

Nets are independent given a board, so ranks partition the nets and never
exchange data on the solve path; the only collectives are the timing
reduction (max over ranks) and the barriers around the timed region.  A rank
that fails between steps is noticed by the others either through the store
(a missing heartbeat) or through the process group's short timeout, never by
a device wait.
"""
from __future__ import annotations

import datetime
import time
from typing import Optional, Tuple


def shard(n: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous [begin, end) of n items for `rank` of `world` (sizes differ by <= 1)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank out of range")
    base, extra = divmod(n, world)
    begin = rank * base + min(rank, extra)
    return begin, begin + base + (1 if rank < extra else 0)


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class RankFailure(RuntimeError):
    """Another rank stopped sending heartbeats."""


class Heartbeat:
    """Per-step liveness through the process group's store: every rank posts
    `step` before launching it and checks that all others have posted the
    previous step within `timeout_s`."""

    def __init__(self, store, rank: int, world: int, timeout_s: float = 10.0, prefix: str = "mrc-hb"):
        self.store, self.rank, self.world = store, rank, world
        self.timeout_s = timeout_s
        self.prefix = prefix

    def beat(self, step: int) -> None:
        self.store.set(f"{self.prefix}/{self.rank}", str(step))

    def check(self, step: int) -> None:
        deadline = time.monotonic() + self.timeout_s
        for r in range(self.world):
            if r == self.rank:
                continue
            while True:
                try:
                    self.store.wait([f"{self.prefix}/{r}"], datetime.timedelta(seconds=max(0.05, deadline -
                                                                                            time.monotonic())))
                    seen = int(self.store.get(f"{self.prefix}/{r}"))
                except Exception as e:  # the store's own timeout
                    raise RankFailure(f"rank {r} sent no heartbeat") from e
                if seen >= step:
                    break
                if time.monotonic() > deadline:
                    raise RankFailure(f"rank {r} stopped at step {seen}, expected {step}")
                time.sleep(0.01)


def init_from_env(backend: str, timeout_s: float = 120.0, device=None) -> Optional[object]:
    """init_process_group from RANK/WORLD_SIZE/MASTER_* when WORLD_SIZE > 1."""
    import os

    import torch.distributed as dist

    if int(os.environ.get("WORLD_SIZE", "1")) <= 1:
        return None
    kw = {"timeout": datetime.timedelta(seconds=timeout_s)}
    if device is not None:
        kw["device_id"] = device
    dist.init_process_group(backend, **kw)
    return dist


def sharded_negotiation_round(shard, all_reduce=None) -> dict:
    """One negotiation round of this rank's shard (Engine.negotiation(...,
    owned=...)): rip-up, exchange, route, exchange, settle.  The exchange sets the
    global occupancy to the sum of every rank's local occupancy; `all_reduce`
    (default: torch.distributed SUM over the process group, NCCL on GPUs) is
    called on the global tensor after the local one is copied into it."""
    import torch.distributed as dist

    if all_reduce is None:
        def all_reduce(t):
            dist.all_reduce(t, op=dist.ReduceOp.SUM)

    local, glob = shard.occupancy()

    def exchange():
        glob.copy_(local)
        all_reduce(glob)

    shard.ripup()
    exchange()
    shard.route()
    exchange()
    return shard.settle()
