"""Sharding a sweep of independent nozzles over ranks (mach2d_b200.sweep),
checked with two gloo processes on the CPU: the assignment is balanced by
cell count and covers every instance once, and the result gather returns
every instance's tuple, in the sweep's order, on every rank."""
import os
import socket

import pytest

from mach2d_b200.sweep import gather_results, shard_indices

HERE = os.path.dirname(os.path.abspath(__file__))


def test_shards_cover_every_instance_once_and_balance_the_cells():
    import numpy as np
    rng = np.random.default_rng(3)
    sizes = [int(rng.integers(64, 513)) * int(rng.integers(32, 129)) for _ in range(256)]
    for world in (1, 2, 3, 4, 8):
        parts = shard_indices(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(256))
        loads = [sum(sizes[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)      # LPT bound
    assert shard_indices([5, 5, 5], 2) == [[0, 2], [1]]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sizes = [100 + 37 * i % 211 for i in range(23)]
        mine = shard_indices(sizes, world)[rank]
        local = {i: (float(i), 2.0 * i, float(rank)) for i in mine}
        res = gather_results(local, len(sizes))
        assert [r[0] for r in res] == [float(i) for i in range(len(sizes))]
        owners = [int(r[2]) for r in res]
        parts = shard_indices(sizes, world)
        assert all(owners[i] == q for q in range(world) for i in parts[q])
        with open(os.path.join(out_dir, f"ok{rank}"), "w") as fh:
            fh.write("ok")
    finally:
        dist.destroy_process_group()


def test_gather_over_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp
    os.environ["PYTHONPATH"] = os.pathsep.join([HERE, os.path.dirname(HERE), os.environ.get("PYTHONPATH", "")])
    mp.spawn(_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, join=True)
    assert sorted(os.listdir(tmp_path)) == ["ok0", "ok1"]


def test_gather_without_a_process_group_is_the_identity():
    assert gather_results({1: (1.0,), 0: (0.0,)}, 2) == [(0.0,), (1.0,)]
    with pytest.raises(KeyError):
        gather_results({0: (0.0,)}, 2)
