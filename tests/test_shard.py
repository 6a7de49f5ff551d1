"""Multi-rank plumbing on the CPU (gloo, two ranks): the LPT spread of the
batched workload's clouds and the reductions that time a job by its slowest
rank.  These are the only collectives of the multi-GPU paths; the data path
itself exchanges nothing."""
import os
import socket

import numpy as np
import pytest

from gvdb2 import shard


def config3_sizes():
    rng = np.random.default_rng(3)  # the sizes of the batched workload (seed 3, log-uniform in [1e4, 2e6])
    return np.floor(np.exp(rng.uniform(np.log(1e4), np.log(2e6), 64))).astype(np.int64)


def test_lpt_partition_covers_and_balances():
    sizes = config3_sizes()
    for n in (1, 2, 3, 8):
        parts = shard.lpt_partition(sizes, n)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        loads = [int(sizes[p].sum()) if p else 0 for p in parts]
        # greedy LPT: no rank exceeds the mean by more than the largest cloud
        assert max(loads) <= sizes.sum() / n + sizes.max()
    assert shard.lpt_partition([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    assert shard.lpt_partition([], 3) == [[], [], []]
    with pytest.raises(ValueError):
        shard.lpt_partition([1], 0)


def _rank_main(rank, world, port, sizes, out_dir):
    import torch.distributed as dist
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        env = shard.RankEnv.from_env()
        assert (env.rank, env.world) == (rank, world)
        mine = shard.lpt_partition(sizes, world)[rank]
        shares = [None] * world
        dist.all_gather_object(shares, mine)
        assert sorted(i for s in shares for i in s) == list(range(len(sizes)))
        assert all(not set(shares[a]) & set(shares[b]) for a in range(world) for b in range(a + 1, world))
        total = shard.sum_over_ranks(float(sum(sizes[i] for i in mine)))
        slowest = shard.max_over_ranks(1.5 + rank)
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{total} {slowest} {len(mine)}\n")
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    sizes = [int(x) for x in config3_sizes()]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_rank_main, args=(2, port, sizes, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    rows = [open(tmp_path / f"rank{r}.txt").read().split() for r in range(2)]
    for total, slowest, _ in rows:
        assert float(total) == float(sum(sizes))
        assert float(slowest) == 2.5
    assert int(rows[0][2]) + int(rows[1][2]) == len(sizes)


def test_single_process_reductions_are_identity():
    assert shard.max_over_ranks(3.25) == 3.25
    assert shard.sum_over_ranks(7.0) == 7.0
