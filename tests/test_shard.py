"""The replica path across ranks (mojo_poissonrecon_b200/shard.py) with
world_size 2 over gloo on the CPU; the GPU reconstruction is replaced by a
fake runner, so no device is needed."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from mojo_poissonrecon_b200 import shard


def test_partition_is_greedy_and_complete():
    fp = [5, 1, 9, 3, 3, 7, 2]
    shares = shard.partition(fp, 2)
    assert sorted(i for s in shares for i in s) == list(range(len(fp)))
    loads = [sum(fp[i] for i in s) for s in shares]
    assert abs(loads[0] - loads[1]) <= max(fp)
    assert shard.partition(fp, 2) == shares  # deterministic
    assert shard.partition([], 3) == [[], [], []]
    assert shard.partition(fp, 1) == [list(range(len(fp)))]
    with pytest.raises(ValueError):
        shard.partition(fp, 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, results):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(0)
        clouds = [(rng.random((int(k), 3)), rng.random((int(k), 3)), 5 + (int(k) % 3)) for k in
                  rng.integers(10, 200, size=9)]
        seen = []

        def runner(local):
            seen.extend(len(p) for p, _, _ in local)
            return [(len(p), d, rank) for p, _, d in local]

        out = shard.reconstruct_sharded(clouds, runner=runner)
        t = shard.max_over_ranks(float(rank + 1))
        results[rank] = {"out": out, "seen": seen, "max": t,
                         "expect": [(len(p), d) for p, _, d in clouds]}
    finally:
        dist.destroy_process_group()


def test_two_ranks_over_gloo():
    world = 2
    manager = mp.get_context("spawn").Manager()
    results = manager.dict()
    mp.start_processes(_worker, args=(world, _free_port(), results), nprocs=world, start_method="spawn", join=True)
    r0, r1 = results[0], results[1]
    assert r1["out"] is None
    out = r0["out"]
    assert [(n, d) for n, d, _ in out] == r0["expect"]  # every cloud once, in input order
    assert {rank for _, _, rank in out} == {0, 1}  # both ranks did work
    assert sorted(r0["seen"] + r1["seen"]) == sorted(n for n, _ in r0["expect"])
    assert r0["max"] == r1["max"] == 2.0
