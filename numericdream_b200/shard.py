"""Splitting a batch of views over GPUs (one process per GPU).

Rays are independent: a view or a tile of a view reads only scene constants, so
the pass shards without any data-path collective.  Each rank marches its share
and writes its own G-buffer; the host (or a caller's own gather) assembles the
frame.  Big views are first cut into tiles with the reference's tile convention
(the tile rectangle of tileTransform, src/gpu/fractal_renderer.zig:852-863), then
views and tiles are assigned to ranks by longest-processing-time-first on an
estimated cost so the slowest rank finishes as early as possible.
"""

from __future__ import annotations

from . import abi

# relative DE cost of one ray per formula (DE evaluations x FLOPs per evaluation,
# measured with the op-counting build on the benchmark views); others default to 1
FORMULA_COST = {"mandelbrot": 0.5, "amazingbox_box": 1.9, "menger3_ifs": 1.2, "pseudokleinian_kleinian": 3.6}


def split_tiles(view: abi.nd_view_desc, tiles_x: int, tiles_y: int) -> list:
    """Cut a view's rectangle into tiles_x x tiles_y tiles (same frame, same camera)."""
    out = []
    x0, y0, w, h = view.tile_x, view.tile_y, view.tile_w, view.tile_h
    for ty in range(tiles_y):
        for tx in range(tiles_x):
            a = x0 + (w * tx) // tiles_x
            b = x0 + (w * (tx + 1)) // tiles_x
            c = y0 + (h * ty) // tiles_y
            d = y0 + (h * (ty + 1)) // tiles_y
            if b <= a or d <= c:
                continue
            t = type(view).from_buffer_copy(view)
            t.tile_x, t.tile_y, t.tile_w, t.tile_h = a, c, b - a, d - c
            out.append(t)
    return out


def estimate_cost(view: abi.nd_view_desc, formula_name: str | None = None) -> float:
    return abi.rays_of(view) * FORMULA_COST.get(formula_name or "", 1.0)


def partition(costs, world: int) -> list:
    """Longest-processing-time-first: returns, per rank, the list of item indices."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += costs[i]
    for p in parts:
        p.sort()
    return parts


def shard_views(views, world: int, rank: int, names=None, max_rays_per_item: int = 1 << 20) -> list:
    """The views (or tiles) rank `rank` of `world` marches."""
    items = []
    for i, v in enumerate(views):
        n = abi.rays_of(v)
        if n > max_rays_per_item and world > 1:
            k = 1
            while n // (k * k) > max_rays_per_item:
                k += 1
            items.extend((t, i) for t in split_tiles(v, k, k))
        else:
            items.append((v, i))
    costs = [estimate_cost(t, names[i] if names else None) for t, i in items]
    parts = partition(costs, world)
    return [items[j][0] for j in parts[rank]]


def rank_views(views, world: int, rank: int, names=None) -> list:
    """One rank's share of a batch for a multi-GPU step: the batch's views cut into
    tiles of at most total_rays / (4 x world) rays each (at least 2^16), assigned by
    longest-processing-time-first.  Every ray of the batch lands on exactly one rank,
    and a tile draws the same rays as the same pixels of the uncut view (the tile
    rectangle is in frame pixels and the sample jitter is keyed by frame position).
    names maps a view's formula id to its name (for the cost estimate)."""
    if world <= 1:
        return list(views)
    total = sum(abi.rays_of(v) for v in views)
    per = max(1 << 16, total // (4 * world))
    nm = [names[v.formula] for v in views] if names is not None else None
    return shard_views(views, world, rank, names=nm, max_rays_per_item=per)
