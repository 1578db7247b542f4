"""Multi-GPU sharding of independent molecules (one process per GPU).

Molecules never interact, so a multi-GPU run partitions whole systems across ranks and needs no
collective on the data path: each rank builds and evaluates or minimizes its own synthesis.  The
only cross-rank steps are a barrier around timed regions and a max over ranks of the measured
time (throughput = units on all ranks / slowest rank's time).

* ``partition_lpt``: size-sorted greedy (longest processing time first) assignment of systems to
  ranks, balancing the pair count N(N-1)/2 that dominates the work.
* ``max_over_ranks`` / ``sum_over_ranks``: the timing reductions, over whatever process group
  torch.distributed was initialised with (NCCL on GPUs; gloo works on CPU for tests).
* ``spawn_ranks``: one process per rank without torchrun, with the rendezvous environment
  (RANK, LOCAL_RANK, WORLD_SIZE, MASTER_ADDR = 127.0.0.1, a free MASTER_PORT) set in each.
"""
from __future__ import annotations

import heapq
import os
import socket

import numpy as np


def pair_cost(natoms) -> np.ndarray:
    n = np.asarray(natoms, dtype=np.int64)
    return n * (n - 1) // 2 + n      # pairs, plus a per-atom term for the valence work


def partition_lpt(natoms, world: int) -> list:
    """Indices of the systems assigned to each of `world` ranks, largest first to the least
    loaded rank.  Every system lands on exactly one rank; ties go to the lower rank."""
    if world < 1:
        raise ValueError("world size must be positive")
    cost = pair_cost(natoms)
    order = sorted(range(len(cost)), key=lambda k: (-int(cost[k]), k))
    heap = [(0, r) for r in range(world)]
    shards = [[] for _ in range(world)]
    for k in order:
        load, r = heapq.heappop(heap)
        shards[r].append(k)
        heapq.heappush(heap, (load + int(cost[k]), r))
    return [np.array(sorted(s), dtype=np.int64) for s in shards]


def _reduce(value: float, op, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64,
                     device=device if device is not None else "cpu")
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(value: float, device=None) -> float:
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.MAX, device)


def sum_over_ranks(value: float, device=None) -> float:
    import torch.distributed as dist
    return _reduce(value, dist.ReduceOp.SUM, device)


def _free_port() -> int:
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as sock:
        sock.bind(("127.0.0.1", 0))
        return sock.getsockname()[1]


def _rank_entry(rank, fn, nprocs, port, fn_args):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(nprocs),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    fn(*fn_args)


def spawn_ranks(fn, nprocs: int, *fn_args) -> None:
    """Run fn(*fn_args) in nprocs spawned processes, one per rank, each with the rendezvous
    environment torch.distributed reads; raises if any rank fails.  fn must be importable (a
    module-level function)."""
    import torch.multiprocessing as tmp
    tmp.start_processes(_rank_entry, args=(fn, nprocs, _free_port(), fn_args), nprocs=nprocs,
                        start_method="spawn", join=True)
