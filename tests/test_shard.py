"""CPU: sharding a circuit batch over ranks (host logic of the multi-GPU
batch path): the LPT partition, and two gloo ranks that each take their
shard and gather every instance's status, as the sharded bench does."""
import os
import socket

import numpy as np
import pytest

from ohmnivore_b200 import circuits as ck
from ohmnivore_b200.shard import gather_status, lpt_partition, shard_loads


def test_partition_covers_every_instance_once():
    w = np.random.default_rng(0).integers(50, 20000, 4096)
    for k in (1, 2, 3, 8):
        shards = lpt_partition(w, k)
        allidx = np.concatenate(shards)
        assert np.array_equal(np.sort(allidx), np.arange(w.size))
        loads = shard_loads(w, shards)
        # LPT bound: the heaviest shard carries at most the mean plus one instance
        assert loads.max() <= w.sum() / k + w.max()
        assert lpt_partition(w, k)[0].tolist() == shards[0].tolist()      # deterministic


def test_partition_edge_cases():
    assert [s.tolist() for s in lpt_partition([], 3)] == [[], [], []]
    assert [s.tolist() for s in lpt_partition([5.0], 2)] == [[0], []]
    assert [s.tolist() for s in lpt_partition([1, 1, 1, 1], 2)] == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        lpt_partition([1.0], 0)


def test_monte_carlo_shards_balance():
    ckts = ck.monte_carlo_batch(256, seed=3, vaf=100.0)
    w = [c.n_components for c in ckts]
    loads = shard_loads(w, lpt_partition(w, 4))
    assert loads.max() / loads.mean() < 1.05


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, weights, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = lpt_partition(weights, world)[rank]
        # a stand-in for each instance's solve status: 0, except instance 7 fails (2)
        status = [2 if i == 7 else 0 for i in mine]
        full = gather_status(status, mine, len(weights))
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), np.stack([full, np.isin(np.arange(len(weights)), mine)]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_gather(tmp_path):
    import torch.multiprocessing as mp
    weights = list(np.random.default_rng(1).integers(10, 1000, 37))
    mp.start_processes(_rank_main, args=(2, _free_port(), weights, str(tmp_path)), nprocs=2, join=True,
                       start_method="spawn")
    r0 = np.load(tmp_path / "rank0.npy")
    r1 = np.load(tmp_path / "rank1.npy")
    expect = np.zeros(37, dtype=np.int64)
    expect[7] = 2
    assert np.array_equal(r0[0], expect) and np.array_equal(r1[0], expect)     # every rank sees every status
    assert not np.any(r0[1] & r1[1]) and np.all(r0[1] | r1[1])                 # disjoint shards covering all


def test_gather_status_single_process():
    """Without a process group the local statuses are the whole batch."""
    full = gather_status([0, 2, 0], [4, 1, 0], 5)
    assert full.tolist() == [0, 2, -1, -1, 0]
