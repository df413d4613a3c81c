"""Iteration sharding across ranks (gloo, world size 2, CPU): the shards
partition the iteration range, and two ranks that each render their shard
of a small parity case with the reference's render loop compiled for the
CPU (oracle/_ref), then reduce with gpuupbp_b200.dist.combine, produce the
same average image as one rank rendering every iteration.  The renderer
behind the ranks is the oracle, because this machine has no GPU; the
sharding and the reduction are the B200 path's own (bench.py drives the
GPU renderer through the same two functions)."""
import os
import socket
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from gpuupbp_b200.dist import combine, shard_iterations

CASE = "box_tiny_all"
TOTAL = 5


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


def _render(iterations, scene_dir):
    """Sum of the oracle's images of the given iterations of the parity case."""
    import ref_cpu
    from cases import prepare
    r = ref_cpu.RefRenderer(prepare(CASE, scene_dir), threads=1)
    acc = None
    for it in iterations:
        img = r.run_iteration(it).astype(np.float64)
        acc = img if acc is None else acc + img
    r.close()
    return acc


def _worker(rank, world, port, scene_dir, out, paths):
    import sys
    for p in paths:
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    its = shard_iterations(rank, world, TOTAL)
    out[rank] = (its, combine(_render(its, scene_dir), len(its)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_render_equals_single_rank(oracle_available):
    if not oracle_available:
        pytest.skip("oracle/_ref not built")
    import sys
    world = 2
    with tempfile.TemporaryDirectory() as scene_dir:
        from cases import prepare
        prepare(CASE, scene_dir)  # the scene files exist before the ranks start
        mgr = mp.get_context("spawn").Manager()
        out = mgr.dict()
        mp.start_processes(_worker, args=(world, _free_port(), scene_dir, out, list(sys.path)), nprocs=world,
                           start_method="spawn", join=True)
        ref = _render(range(TOTAL), scene_dir) / TOTAL
    assert sorted(out[0][0] + out[1][0]) == list(range(TOTAL))
    assert ref.max() > 0
    for r in range(world):
        # every rank holds the reduced average of all iterations; the sum order
        # of the reduction differs from one rank's sequential sum
        assert np.allclose(out[r][1], ref, rtol=1e-9, atol=1e-12)
