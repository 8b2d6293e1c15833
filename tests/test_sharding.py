"""Multi-rank host logic on CPU: two gloo ranks (world_size 2, 127.0.0.1)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from libatssim_b200 import sharding


class FakeInstance:
    def __init__(self, n):
        self.num_verts = n


class FakeMLP:
    """Stands in for libatssim_b200.MLP: a rank-dependent gradient, plain SGD."""

    def __init__(self, n, rank):
        self.p = np.zeros(n, dtype=np.float32)
        self.rank = rank

    def batch_gradient(self, dataset, batch, seed):
        return float(self.rank + 1), np.full(self.p.shape, self.rank + 1.0, dtype=np.float32)

    def apply_gradient(self, grad, lr):
        self.p -= lr * grad


def test_partition_is_complete_and_balanced():
    rng = np.random.RandomState(0)
    sides = rng.randint(16, 257, 256)
    costs = sides * sides * 50
    for world in (1, 2, 4, 8):
        parts = sharding.partition(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [costs[p].sum() for p in parts]
        assert max(loads) - min(loads) <= costs.max()


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        insts = [FakeInstance(n) for n in (100, 400, 900, 1600, 2500, 3600, 4900)]
        mine, idx = sharding.shard(insts, iterations=50)
        everyone = [None] * world
        dist.all_gather_object(everyone, idx)
        s = sharding.allreduce_stats([rank + 1.0, 10.0 * rank])
        mx = sharding.allreduce_stats([rank + 1.0, -rank], op="max")
        gres = sharding.global_residual(np.array([3.0, 4.0]) * (rank + 1))
        mlp = FakeMLP(5, rank)
        loss = sharding.data_parallel_train(mlp, None, steps=3, lr=0.5)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), everyone=np.array(everyone, dtype=object), s=s, mx=mx,
                 gres=gres, p=mlp.p, loss=loss, n=len(mine))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks(tmp_path):
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r = [np.load(tmp_path / f"r{k}.npz", allow_pickle=True) for k in range(2)]
    parts = list(r[0]["everyone"])
    assert sorted(parts[0] + parts[1]) == list(range(7)) and not set(parts[0]) & set(parts[1])
    assert r[0]["n"] + r[1]["n"] == 7
    for k in range(2):
        assert np.allclose(r[k]["s"], [3.0, 10.0])
        assert np.allclose(r[k]["mx"], [2.0, 0.0])
        # sqrt(sum over ranks of (3^2 + 4^2) (k+1)^2) = 5 sqrt(5)
        assert abs(r[k]["gres"] - 5.0 * np.sqrt(5.0)) < 1e-12
        # averaged gradient 1.5 for 3 steps of lr 0.5: every rank holds the same parameters
        assert np.allclose(r[k]["p"], -2.25)
        assert abs(r[k]["loss"] - 1.5) < 1e-12
