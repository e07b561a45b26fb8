"""Multi-process sharding of a view batch (gloo, world size 2, CPU only)."""

import os
import socket

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from numericdream_b200 import abi, shard


def _views():
    vs = []
    for i, (w, h) in enumerate([(64, 64), (1024, 1024), (300, 200), (2048, 1024), (17, 5), (512, 512)]):
        vs.append(abi.make_view(i % 4, w, h, (0.0, 0.0, -3.0)))
    return vs


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    views = _views()
    mine = shard.shard_views(views, world, rank, max_rays_per_item=1 << 19)
    rays = torch.tensor([sum(abi.rays_of(v) for v in mine)], dtype=torch.int64)
    gathered = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(gathered, rays)
    # pixel coverage: every (view, x, y) exactly once across ranks
    cover = torch.zeros(sum(v.width * v.height for v in views), dtype=torch.int32)
    base = {}
    off = 0
    for i, v in enumerate(views):
        base[(v.width, v.height, v.formula)] = off
        off += v.width * v.height
    for t in mine:
        b = base[(t.width, t.height, t.formula)]
        for y in range(t.tile_y, t.tile_y + t.tile_h):
            cover[b + y * t.width + t.tile_x: b + y * t.width + t.tile_x + t.tile_w] += 1
    dist.all_reduce(cover)
    if rank == 0:
        q.put(([int(g.item()) for g in gathered], int(cover.min()), int(cover.max())))
    dist.barrier()
    dist.destroy_process_group()


def test_partition_is_balanced_and_covers_every_pixel_once():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    loads, lo, hi = q.get(timeout=10)
    total = sum(abi.rays_of(v) for v in _views())
    assert sum(loads) == total
    assert lo == 1 and hi == 1
    assert max(loads) <= 0.6 * total


def test_split_tiles_keeps_the_frame():
    v = abi.make_view(0, 100, 60, (0.0, 0.0, -3.0))
    tiles = shard.split_tiles(v, 3, 2)
    assert len(tiles) == 6
    assert sum(abi.rays_of(t) for t in tiles) == 6000
    assert all(t.width == 100 and t.height == 60 for t in tiles)


def test_partition_lpt():
    parts = shard.partition([5, 4, 3, 3, 3], 2)
    loads = [sum([5, 4, 3, 3, 3][i] for i in p) for p in parts]
    assert sorted(loads) == [8, 10] or sorted(loads) == [9, 9]
    with pytest.raises(ValueError):
        shard.partition([1], 0)
