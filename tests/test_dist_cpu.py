"""Iteration sharding across ranks (gloo, world size 2, CPU): the shards
partition the iteration range and the reduced average equals the average of
all iterations rendered on one rank.  Per-iteration images come from the
reference oracle on the CPU (same seeds on every rank)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gpuupbp_b200.dist import combine, shard_iterations


def test_shards_partition_the_range():
    for world in (1, 2, 3, 8):
        got = sorted(i for r in range(world) for i in shard_iterations(r, world, 17, start=3))
        assert got == list(range(3, 20))
    with pytest.raises(ValueError):
        shard_iterations(2, 2, 4)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _image(it):
    # deterministic stand-in for an iteration image (the oracle path is below)
    rng = np.random.default_rng(1000 + it)
    return rng.random((8, 8, 3))


def _worker(rank, world, port, total, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    its = shard_iterations(rank, world, total)
    acc = sum((_image(i) for i in its), np.zeros((8, 8, 3)))
    avg = combine(acc, len(its))
    out[rank] = avg
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_reduction_equals_single_rank():
    world, total = 2, 7
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_worker, args=(world, port, total, out), nprocs=world, start_method="spawn", join=True)
    ref = sum((_image(i) for i in range(total)), np.zeros((8, 8, 3))) / total
    for r in range(world):
        assert np.allclose(out[r], ref, rtol=1e-12)
