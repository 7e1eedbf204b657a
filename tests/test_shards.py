"""The multi-GPU (one process per GPU) host path on CPU: two gloo ranks split
a committor run's inputs and a swarm's timing exactly as bench.py --gpus N and
shards.sharded_committor do on NCCL, with a CPU stand-in for the per-rank
shooting (the oracle's magnetisation of each input grid)."""
import os
import socket

import numpy as np
import pytest

from gpu_2dising_b200 import shards

import oracle


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_range_partitions_every_item_once():
    for n in (0, 1, 5, 7, 64, 1000):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                start, count = shards.shard_range(n, world, r)
                seen.extend(range(start, start + count))
                assert count in (n // world, n // world + 1)
            assert seen == list(range(n))
    with pytest.raises(ValueError):
        shards.shard_range(4, 2, 2)


def test_rank_seeds_distinct_and_rank0_unchanged():
    seeds = [shards.rank_seed(20240501, r) for r in range(8)]
    assert seeds[0] == 20240501 and len(set(seeds)) == 8


def _stand_in_shoot(grids, shots):
    """Deterministic per-input value computed on the CPU by the oracle."""
    L = grids.shape[1]
    return 0.5 * (1.0 + oracle.magnetisation_gpu(L, grids).astype(np.float64)) + 1e-3 * shots


def _worker(rank, world, port, inputs, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        pb = shards.sharded_committor(inputs, 64, _stand_in_shoot, dist)
        t = shards.max_over_ranks(1.0 + rank, dist)
        n = shards.sum_over_ranks(shards.shard_range(len(inputs), world, rank)[1], dist)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.concatenate([pb, [t, n]]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_inputs", [7, 2])
def test_two_gloo_ranks_match_one_process(tmp_path, n_inputs):
    import torch.multiprocessing as mp
    rng = np.random.default_rng(n_inputs)
    inputs = np.where(rng.random((n_inputs, 8, 8)) < 0.3, 1, -1).astype(np.int32)
    mp.start_processes(_worker, args=(2, _free_port(), inputs, str(tmp_path)), nprocs=2,
                       join=True, start_method="spawn")
    expected = shards.sharded_committor(inputs, 64, _stand_in_shoot, None)
    assert np.allclose(expected, _stand_in_shoot(inputs, 64))
    for r in range(2):
        got = np.load(tmp_path / f"rank{r}.npy")
        assert np.array_equal(got[:n_inputs], expected)  # every rank holds every input's pB
        assert got[n_inputs] == 2.0                       # max over ranks of 1 + rank
        assert got[n_inputs + 1] == n_inputs              # the shards cover the inputs
