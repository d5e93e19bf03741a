"""Cost-balanced block schedule of the full-z fused step (path 3).

The full-z kernel gives each block one tile of `tile_y` rows and a run of x
planes.  Planes cost more where the block also filters CPML state along x or
y: the x- and y-slab psi are read and written directly, and on a B200 such a
plane took about 1.5x an interior plane.  A uniform grid of equal chunks
therefore ends with the CPML blocks running alone.  This module instead cuts
each tile's x extent into runs of equal estimated cost and hands the runs out
so that every resident block slot of the GPU gets one run: one wave, no tail.

`balanced_schedule` returns the (blocks, 4) int32 table of
`fdtd_step_args.schedule`: (y tile index, first plane, end plane, 0).

`segment_schedule` balances the time-blocked kernel (fdtd_step_block), which
runs one block per SM: with so few blocks per tile, whole runs per tile
quantise badly, so a block's planes may continue into the next tile (a second
segment) and every block gets the same estimated cost.
"""

import numpy as np

# Longest plane run of a block in a batch (the run length sizes the block's
# shared-memory x-coefficient table).
MAX_RUN = 96

# Extra cost of a plane whose tile holds y-slab rows / whose x position is an
# x-slab plane, relative to an interior plane (B200, 20 nm bend: the best of
# sweeps over 0.6..1.5 / 0.5..1.3 at tile_y 5 and 6).
Y_WEIGHT = 0.9
X_WEIGHT = 0.7

# The same for the time-blocked kernel (fdtd_step_block): the extra cost of
# a y-slab tile plane / an x-slab plane and the cost of a block's extra
# segment, in planes of the general build, and the cost of a plane run by the
# interior build (no x/y CPML code).  Least-squares fits of per-block
# durations (globaltimer at block start and end) on the 20 nm bend at depth
# 2, tile 7, then the best of a sweep around them (B200).
BLOCK_Y_WEIGHT = 0.75
BLOCK_X_WEIGHT = 0.75
BLOCK_SEGMENT_COST = 3.4
BLOCK_INTERIOR_COST = 0.78


def plane_costs(shape, tile_y, coeff_e, coeff_h, wy=Y_WEIGHT, wx=X_WEIGHT):
    """(tiles, nx) estimated cost of each tile plane; coeff_* are the (3, L, 4)
    CPML tables (a, b, 1/kappa, rank) of E and H."""
    nx, ny, _ = shape
    tiles = (ny + tile_y - 1) // tile_y
    yrow = (coeff_e[1, :ny, 0] != 0) | (coeff_h[1, :ny, 0] != 0)
    xact = ((coeff_e[0, :nx, 0] != 0) | (coeff_h[0, :nx, 0] != 0)).astype(np.float64)
    ytile = np.array([yrow[t * tile_y:(t + 1) * tile_y].any() for t in range(tiles)], np.float64)
    return 1.0 + wy * ytile[:, None] + wx * xact[None, :]


def balanced_schedule(shape, tile_y, coeff_e, coeff_h, blocks, wy=Y_WEIGHT, wx=X_WEIGHT):
    """Split every tile's planes into runs of equal estimated cost, about
    `blocks` runs in all (at least one per tile)."""
    cost = plane_costs(shape, tile_y, coeff_e, coeff_h, wy, wx)
    nx = shape[0]
    tiles = cost.shape[0]
    per_tile = cost.sum(axis=1)
    share = per_tile / per_tile.sum() * max(int(blocks), tiles)
    runs = np.maximum(1, np.floor(share).astype(np.int64))
    while runs.sum() < max(int(blocks), tiles):
        runs[np.argmax(share - runs)] += 1
    runs = np.minimum(runs, nx)
    entries = []
    for t in range(tiles):
        cum = np.concatenate([[0.0], np.cumsum(cost[t])])
        cuts = [0]
        for j in range(1, int(runs[t])):
            cuts.append(int(np.searchsorted(cum, cum[-1] * j / runs[t])))
        cuts.append(nx)
        for a, b in zip(cuts[:-1], cuts[1:]):
            if b > a:
                entries.append((t, a, b, 0))
    return np.asarray(entries, np.int32).reshape(-1, 4)


def batch_schedule(grids, tile_y, blocks, wy=Y_WEIGHT, wx=X_WEIGHT, max_run=MAX_RUN):
    """Many grids in one launch: `grids` is a list of (shape, coeff_e,
    coeff_h); every (grid, tile) gets runs of equal estimated cost, at least
    `blocks` runs in all (one wave) and runs of about `max_run` planes at
    most (more waves when the tiles outnumber the slots).  Returns the (n, 4) int32
    table (grid, y tile, first plane, end plane) of fdtd_step_batch."""
    costs = [plane_costs(shape, tile_y, ce, ch, wy, wx) for shape, ce, ch in grids]
    per_tile = np.concatenate([c.sum(axis=1) for c in costs])
    nx_tile = np.concatenate([np.full(c.shape[0], shape[0]) for c, (shape, _, _) in zip(costs, grids)])
    least = -(-nx_tile // max_run)  # runs of at most max_run planes
    total = max(int(blocks), int(least.sum()))
    share = per_tile / per_tile.sum() * total
    runs = np.maximum(least, np.floor(share).astype(np.int64))
    while runs.sum() < total:
        runs[np.argmax(share - runs)] += 1
    entries, j = [], 0
    for g, (c, (shape, _, _)) in enumerate(zip(costs, grids)):
        nx = shape[0]
        for t in range(c.shape[0]):
            n = int(min(runs[j], nx))
            j += 1
            cum = np.concatenate([[0.0], np.cumsum(c[t])])
            cuts = [0] + [int(np.searchsorted(cum, cum[-1] * k / n)) for k in range(1, n)] + [nx]
            entries += [(g, t, a, b) for a, b in zip(cuts[:-1], cuts[1:]) if b > a]
    return np.asarray(entries, np.int32).reshape(-1, 4)


def _active(coeff, axis, n):
    """Planes / rows of `axis` with CPML state or 1/kappa != 1."""
    return (coeff[axis, :n, 0] != 0) | (coeff[axis, :n, 2] != 1)


def interior_region(shape, tile_y, depth, coeff_e, coeff_h):
    """The part of the grid the time-blocked kernel's interior build may run:
    (tile mask, x0, x1).  A tile qualifies when none of its computed rows
    (y0 - depth + 1 .. y0 + tile_y + depth - 2) carries y CPML; planes
    [x0, x1) qualify when every plane a segment of them touches (x0 - depth -
    1 .. x1 + depth) is free of x CPML.  x0 >= x1 when there is none."""
    nx, ny, _ = shape
    tiles = (ny + tile_y - 1) // tile_y
    ya = _active(coeff_e, 1, ny) | _active(coeff_h, 1, ny)
    rows = tile_y + 2 * depth - 1
    ok = np.zeros(tiles, bool)
    for t in range(tiles):
        yf = t * tile_y - (depth - 1)
        ok[t] = not ya[max(0, yf):min(ny, yf + rows)].any()
    free = ~(_active(coeff_e, 0, nx) | _active(coeff_h, 0, nx))
    best, start = (0, 0), None
    for x in range(nx + 1):
        if x < nx and free[x]:
            start = x if start is None else start
        elif start is not None:
            if x - start > best[1] - best[0]:
                best = (start, x)
            start = None
    f0, f1 = best
    x0 = f0 if f0 == 0 else f0 + depth + 1
    x1 = f1 if f1 == nx else f1 - depth - 1
    return ok, x0, x1


def _cut(intervals, costs, pieces, segment_cost):
    """Cut the intervals' planes, taken in order, into `pieces` consecutive
    runs of equal estimated cost (each interval start charged segment_cost
    of its average plane); returns a list per piece of (tile, first, end, 0)
    segments."""
    flat = np.concatenate([c.copy() for c in costs])
    starts = np.cumsum([0] + [len(c) for c in costs])
    for j, c in enumerate(costs):
        flat[starts[j]] += segment_cost * c.mean()
    total = len(flat)
    pieces = max(1, min(int(pieces), total))
    cum = np.concatenate([[0.0], np.cumsum(flat)])
    cuts = np.searchsorted(cum, cum[-1] * np.arange(pieces + 1) / pieces)
    cuts[0], cuts[-1] = 0, total
    cuts = np.maximum.accumulate(cuts)
    lists = []
    for a, b in zip(cuts[:-1], cuts[1:]):
        segs = []
        while a < b:
            j = int(np.searchsorted(starts, a, side="right")) - 1
            t, xa, _ = intervals[j]
            n = min(int(b), int(starts[j + 1])) - int(a)
            first = xa + int(a - starts[j])
            segs.append((t, first, first + n, 0))
            a += n
        if segs:
            lists.append(segs)
    return lists


def _pack(lists):
    M = max(len(s) for s in lists)
    out = np.full((len(lists), M, 4), -1, np.int32)
    out[..., 3] = 0
    for i, segs in enumerate(lists):
        out[i, :len(segs)] = segs
    return out.reshape(-1, 4), M


def split_segment_schedule(shape, tile_y, depth, coeff_e, coeff_h, blocks, wy=BLOCK_Y_WEIGHT,
                           wx=BLOCK_X_WEIGHT, segment_cost=BLOCK_SEGMENT_COST,
                           interior_cost=BLOCK_INTERIOR_COST):
    """segment_schedule with the interior split off: the CPML-free tiles'
    planes [x0, x1) (interior_region) go to the first blocks, which run the
    kernel's interior build at `interior_cost` per plane; the rest of the
    grid (CPML slabs and their halo margins) to the others.  Blocks are
    shared out in proportion to the two parts' estimated costs.  Returns
    ((blocks * M, 4) entries, M, interior blocks)."""
    ok, x0, x1 = interior_region(shape, tile_y, depth, coeff_e, coeff_h)
    cost = plane_costs(shape, tile_y, coeff_e, coeff_h, wy, wx)
    nx = shape[0]
    inner, inner_c, outer, outer_c = [], [], [], []
    for t in range(cost.shape[0]):
        if ok[t] and x1 > x0:
            inner.append((t, x0, x1))
            inner_c.append(np.full(x1 - x0, interior_cost))
            for a, b in ((0, x0), (x1, nx)):
                if b > a:
                    outer.append((t, a, b))
                    outer_c.append(cost[t, a:b])
        else:
            outer.append((t, 0, nx))
            outer_c.append(cost[t])
    if not inner:
        runs, M = segment_schedule(shape, tile_y, coeff_e, coeff_h, blocks, wy, wx, segment_cost)
        return runs, M, 0
    w_in = sum(c.sum() + segment_cost * c.mean() for c in inner_c)
    w_out = sum(c.sum() + segment_cost * c.mean() for c in outer_c)
    blocks = max(2 if outer else 1, int(blocks))
    n_in = int(round(blocks * w_in / (w_in + w_out))) if outer else blocks
    n_in = min(max(n_in, 1), blocks - (1 if outer else 0))
    lists = _cut(inner, inner_c, n_in, segment_cost)
    n_in = len(lists)
    if outer:
        lists += _cut(outer, outer_c, blocks - n_in, segment_cost)
    runs, M = _pack(lists)
    return runs, M, n_in


def segment_schedule(shape, tile_y, coeff_e, coeff_h, blocks, wy=Y_WEIGHT, wx=X_WEIGHT,
                     segment_cost=2.0):
    """Cut the tiles' planes, taken tile after tile, into `blocks` consecutive
    pieces of equal estimated cost; a piece crossing a tile boundary becomes
    several segments of its block, each charged `segment_cost` planes for its
    pipeline start and halo planes.  Returns ((blocks * M, 4) int32 entries
    (tile, first plane, end plane, 0), with tile -1 padding a block's list, and
    M, the most segments of a block)."""
    cost = plane_costs(shape, tile_y, coeff_e, coeff_h, wy, wx)
    tiles, nx = cost.shape
    blocks = max(1, min(int(blocks), tiles * nx))
    # a tile change costs segment_cost planes of the tile's average plane
    flat = cost.copy()
    flat[:, 0] += segment_cost * cost.mean(axis=1)
    cum = np.concatenate([[0.0], np.cumsum(flat.ravel())])
    cuts = np.searchsorted(cum, cum[-1] * np.arange(blocks + 1) / blocks)
    cuts[0], cuts[-1] = 0, tiles * nx
    cuts = np.maximum.accumulate(cuts)
    lists = []
    for a, b in zip(cuts[:-1], cuts[1:]):
        segs = []
        while a < b:
            t, xa = divmod(int(a), nx)
            xb = min(nx, xa + int(b - a))
            segs.append((t, xa, xb, 0))
            a += xb - xa
        lists.append(segs)
    lists = [s for s in lists if s]
    M = max(len(s) for s in lists)
    out = np.full((len(lists), M, 4), -1, np.int32)
    out[..., 3] = 0
    for i, segs in enumerate(lists):
        out[i, :len(segs)] = segs
    return out.reshape(-1, 4), M
