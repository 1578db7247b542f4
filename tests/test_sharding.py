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


def _spawned_rank_main(out_dir):
    """Run by sharding.spawn_ranks: the bench's own shard selection on one rank, checked across
    ranks with gloo collectives."""
    import torch.distributed as dist
    import bench
    world = int(os.environ["WORLD_SIZE"])
    rank = int(os.environ["RANK"])
    dist.init_process_group("gloo")
    try:
        sizes = synthetic.batched_sizes(world * bench.NSYS, seed=synthetic.SEED_BASE + 1)
        mine = bench._shard(sizes, world, rank)
        gathered = [None] * world
        dist.all_gather_object(gathered, mine.tolist())
        t = sharding.max_over_ranks(float(rank))
        with open(os.path.join(out_dir, f"spawn{rank}.txt"), "w") as f:
            allidx = sorted(i for g in gathered for i in g)
            f.write(f"{world} {t} {len(allidx)} {int(allidx == list(range(world * bench.NSYS)))}\n")
    finally:
        dist.destroy_process_group()


def test_spawned_ranks_take_disjoint_lpt_shards_of_one_workload(tmp_path):
    """bench.py --gpus N without torchrun: sharding.spawn_ranks starts one process per rank with
    the rendezvous environment; the ranks' shards of the N x 1,024-molecule workload are
    disjoint and cover it (two gloo ranks on CPU)."""
    sharding.spawn_ranks(_spawned_rank_main, 2, str(tmp_path))
    for rank in range(2):
        world, tmax, total, covered = open(tmp_path / f"spawn{rank}.txt").read().split()
        assert int(world) == 2 and float(tmax) == 1.0
        assert int(total) == 2048 and int(covered) == 1
