"""Host-side sharding of code blocks over GPUs (one process per GPU).

The receive path partitions by code block: every block decodes independently,
so N GPUs need no data-path collective.  This module holds the host logic that
splits work across ranks and combines the per-rank timings:

* ``weak_shard`` / ``strong_shard`` — which global block ids a rank owns
  (fixed per-GPU work vs a fixed total split evenly);
* ``balance_blocks`` — a mixed-size batch split so every rank gets about the
  same decoder work (longest-processing-time greedy over per-block cost
  ``nnz(BG) * Zc``, the number of edge updates per iteration);
* ``max_over_ranks`` / ``sum_over_ranks`` — the step time of a multi-GPU job is
  the slowest rank's; processed units add up.  Both work with any
  ``torch.distributed`` backend (NCCL on GPUs, gloo on CPU) and with no process
  group at all (single process);
* ``torchrun_command`` / ``launch_ranks`` — start one process per GPU of this
  node under ``torch.distributed.run`` (rendezvous on 127.0.0.1), so a script
  asked for N GPUs outside a launcher can start its own ranks.
"""

from __future__ import annotations

import heapq
import os
import socket
import subprocess
import sys
from typing import List, Optional, Sequence, Tuple

BG_NNZ = {1: 316, 2: 197}


def weak_shard(per_rank: int, rank: int) -> Tuple[int, int]:
    """(first global block id, count) of a rank when every rank decodes per_rank blocks."""
    if per_rank < 0 or rank < 0:
        raise ValueError("per_rank and rank must be non-negative")
    return rank * per_rank, per_rank


def strong_shard(total: int, rank: int, world: int) -> Tuple[int, int]:
    """(start, count) of a rank's contiguous slice of `total` blocks; the first
    total % world ranks take one extra block."""
    if world < 1 or not 0 <= rank < world or total < 0:
        raise ValueError("need world >= 1, 0 <= rank < world, total >= 0")
    base, extra = divmod(total, world)
    start = rank * base + min(rank, extra)
    return start, base + (1 if rank < extra else 0)


def block_cost(cfg: Sequence[int], zc: int) -> int:
    """Edge updates per iteration of one block: nnz(BG) * Zc (cfg[0] is the base graph)."""
    return BG_NNZ[int(cfg[0])] * int(zc)


def balance_blocks(costs: Sequence[int], world: int) -> List[List[int]]:
    """Split block indices over `world` ranks with about equal total cost
    (longest-processing-time greedy; deterministic, so every rank computes the
    same partition without communicating).  Each rank's list is sorted."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-int(costs[i]), i))
    heap = [(0, r) for r in range(world)]
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(costs[i]), r))
    return [sorted(p) for p in parts]


def _reduce(value: float, op_name: str, dist=None, device=None) -> float:
    if dist is None or not dist.is_available() or not dist.is_initialized():
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Largest value over all ranks (e.g. a step time in ms)."""
    return _reduce(value, "MAX", dist, device)


def sum_over_ranks(value: float, dist=None, device=None) -> float:
    """Sum over all ranks (e.g. blocks or info bits processed)."""
    return _reduce(value, "SUM", dist, device)


def free_port() -> int:
    """An unused TCP port on 127.0.0.1 for the rendezvous."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def torchrun_command(nproc: int, script: str, argv: Sequence[str], port: int,
                     timeout_s: Optional[int] = None) -> List[str]:
    """Command line that runs `script argv` as `nproc` ranks on this node; with
    `timeout_s` the whole launch is bounded (SIGTERM, then SIGKILL 60 s later)."""
    if nproc < 1:
        raise ValueError("nproc must be >= 1")
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nproc}",
           "--master-addr", "127.0.0.1", "--master-port", str(port), script, *argv]
    if timeout_s:
        cmd = ["timeout", "-k", "60", str(int(timeout_s))] + cmd
    return cmd


def launch_ranks(nproc: int, script: str, argv: Sequence[str], timeout_s: Optional[int] = None,
                 env: Optional[dict] = None) -> int:
    """Run `script` as `nproc` ranks (stdout and stderr pass through); returns the
    launcher's exit code."""
    e = dict(os.environ if env is None else env)
    return subprocess.call(torchrun_command(nproc, script, argv, free_port(), timeout_s), env=e)
