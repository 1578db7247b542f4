"""Multi-GPU sharding logic on CPU: LPT partition of systems across ranks, and the timing
reductions run as two gloo ranks (the same calls run over NCCL on GPUs)."""
import os
import socket

import numpy as np
import pytest

from stormm_b200 import sharding, synthetic


def test_partition_covers_every_system_once_and_balances():
    sizes = synthetic.batched_sizes(1024)
    for world in (1, 2, 3, 8):
        shards = sharding.partition_lpt(sizes, world)
        assert len(shards) == world
        allidx = np.concatenate(shards)
        assert np.array_equal(np.sort(allidx), np.arange(len(sizes)))
        cost = sharding.pair_cost(sizes)
        loads = np.array([cost[s].sum() for s in shards])
        assert loads.max() - loads.min() <= cost.max()
    again = sharding.partition_lpt(sizes, 4)
    assert all(np.array_equal(a, b) for a, b in zip(again, sharding.partition_lpt(sizes, 4)))


def test_partition_rejects_empty_world():
    with pytest.raises(ValueError):
        sharding.partition_lpt([10, 20], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        sizes = synthetic.batched_sizes(1024)
        mine = sharding.partition_lpt(sizes, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine.tolist())
        tmax = sharding.max_over_ranks(1.5 + rank)
        tsum = sharding.sum_over_ranks(float(len(mine)))
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{tmax} {tsum} {sum(len(g) for g in gathered)} "
                    f"{len(set(i for g in gathered for i in g))}\n")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    for rank in range(2):
        tmax, tsum, total, unique = open(tmp_path / f"rank{rank}.txt").read().split()
        assert float(tmax) == 2.5
        assert float(tsum) == 1024.0
        assert int(total) == 1024 and int(unique) == 1024
