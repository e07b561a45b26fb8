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


def _bench_worker(rank, world, port, q):
    # the benchmark's own multi-GPU partition (bench.build_views with world > 1): the
    # one batched_64 batch cut into tiles and balanced over the ranks
    import numpy as np

    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    names = bench.build_manifest_names()
    full = bench.build_views("batched_64", names.index)
    mine = bench.build_views("batched_64", names.index, world, rank, names)
    index = {v.seed: i for i, v in enumerate(full)}
    offs = np.cumsum([0] + [abi.rays_of(v) for v in full])
    cover = torch.zeros(int(offs[-1]), dtype=torch.int32)
    cv = cover.numpy()
    for t in mine:
        i = index[t.seed]
        v = full[i]
        block = cv[offs[i]:offs[i + 1]].reshape(v.spp, v.tile_h, v.tile_w)
        block[:, t.tile_y - v.tile_y:t.tile_y - v.tile_y + t.tile_h, t.tile_x - v.tile_x:t.tile_x - v.tile_x + t.tile_w] += 1
    load = torch.tensor([sum(shard.estimate_cost(t, names[t.formula]) for t in mine)], dtype=torch.float64)
    loads = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(loads, load)
    dist.all_reduce(cover)
    if rank == 0:
        q.put((int(cover.min()), int(cover.max()), [float(x.item()) for x in loads], len(mine)))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_partition_covers_the_batch_once():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_bench_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(300)
        assert p.exitcode == 0
    lo, hi, loads, ntiles = q.get(timeout=10)
    assert lo == 1 and hi == 1, "a ray of the batch is marched twice or never"
    assert max(loads) <= 1.1 * sum(loads) / world, loads


def test_tiles_draw_the_rays_of_the_whole_view():
    # jittered samples are keyed by their place in the frame: a view cut into tiles
    # marches exactly the rays of the uncut view (checked with the FP64 oracle)
    import numpy as np

    from oracle import pyoracle

    v = abi.make_view(0, 24, 16, (2.0, 1.0, -2.5), params=[8.0, 8.0], spp=4, seed=99)
    whole = pyoracle.render(v, "mandelbrot", precision=64)
    d = whole["depth64"].reshape(4, 16, 24)
    st = whole["steps"].reshape(4, 16, 24)
    for t in shard.split_tiles(v, 2, 2):
        part = pyoracle.render(t, "mandelbrot", precision=64)
        ys, xs = slice(t.tile_y, t.tile_y + t.tile_h), slice(t.tile_x, t.tile_x + t.tile_w)
        np.testing.assert_array_equal(part["depth64"].reshape(4, t.tile_h, t.tile_w), d[:, ys, xs])
        np.testing.assert_array_equal(part["steps"].reshape(4, t.tile_h, t.tile_w), st[:, ys, xs])
