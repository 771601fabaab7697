"""Multi-rank sharding on CPU ranks (gloo, world size 2).

Scenes are independent, so ranks step disjoint scene ranges with no
collective in the step; these tests check the sharding and the reductions
with the CPU oracle standing in for each rank's GPU, and that a rank which
dies before a collective makes the survivor fail with an error instead of
hanging."""
import datetime
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_shard(rank, world, port, q):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import torch.distributed as dist

    import pyoracle
    from seevr_b200 import Data
    from seevr_b200.shard import reduce_timing, scene_shards

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        full = Data.batch(num_scenes=10, min_bodies=8, max_bodies=40, seed_base=5)
        s0, s1 = scene_shards(full.scene_body_offset(), world)[rank]
        mine = Data.batch(num_scenes=s1 - s0, min_bodies=8, max_bodies=40, seed_base=5 + s0)
        out = pyoracle.run(mine.arrays(), frames=4, substeps=10, pgs_iterations=8)
        parts = [None] * world
        dist.all_gather_object(parts, (s0, s1, out["pos"], out["vel"]))
        ms, work = reduce_timing(10.0 + rank, float(mine.num_dynamic))
        if rank == 0:
            ref = pyoracle.run(full.arrays(), frames=4, substeps=10, pgs_iterations=8)
            pos = np.concatenate([p[2] for p in parts])
            vel = np.concatenate([p[3] for p in parts])
            q.put(("ok", bool(np.array_equal(pos, ref["pos"]) and np.array_equal(vel, ref["vel"])),
                   [(p[0], p[1]) for p in parts], ms, work, full.num_dynamic))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reproduce_the_whole_batch():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_shard, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = q.get(timeout=300)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    tag, equal, shards, ms, work, ndyn = res
    assert tag == "ok" and equal
    assert shards[0][0] == 0 and shards[0][1] == shards[1][0] and shards[1][1] == 10
    assert ms == 11.0          # max over ranks
    assert work == ndyn        # sum over ranks


def test_scene_shards_balance_bodies():
    from seevr_b200.shard import scene_shards

    off = np.concatenate([[0], np.cumsum(np.full(100, 10))])
    sh = scene_shards(off, 4)
    assert sh == [(0, 25), (25, 50), (50, 75), (75, 100)]
    assert scene_shards(off, 1) == [(0, 100)]
    # more ranks than scenes: empty ranges, still a partition
    sh = scene_shards(off[:4], 8)
    assert sh[0][0] == 0 and sh[-1][1] == 3
    assert all(a <= b for a, b in sh)


def _rank_dies(rank, world, port, q):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=5))
    if rank == 1:
        os._exit(3)  # leaves between steps, before the reduction
    try:
        t = torch.ones(1)
        dist.all_reduce(t)
        q.put("no error")
    except Exception as e:  # the survivor learns of the loss from the collective
        q.put("error: " + type(e).__name__)


def test_dead_rank_surfaces_as_error_not_hang():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_dies, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    msg = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert msg.startswith("error")
