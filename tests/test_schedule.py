"""Cost-balanced block schedule of the full-z step (host logic, CPU)."""

import numpy as np

from warp_fdtd_b200.schedule import balanced_schedule, plane_costs


def _tables(shape, slab=11):
    tabs = []
    for _ in range(2):
        c = np.zeros((3, max(shape), 4), np.float32)
        c[:, :, 1:3] = 1
        for axis, n in enumerate(shape):
            c[axis, :slab, 0] = 0.1
            c[axis, n - slab:n, 0] = 0.1
        tabs.append(c)
    return tabs


def test_runs_cover_every_tile_plane_once():
    shape = (324, 324, 144)
    ce, ch = _tables(shape)
    runs = balanced_schedule(shape, 5, ce, ch, 296)
    assert runs.dtype == np.int32 and runs.shape[1] == 4
    tiles = (shape[1] + 4) // 5
    assert abs(len(runs) - 296) <= 2
    for t in range(tiles):
        mine = runs[runs[:, 0] == t]
        assert mine[0, 1] == 0 and mine[-1, 2] == shape[0]
        assert np.all(mine[1:, 1] == mine[:-1, 2])
        assert np.all(mine[:, 2] > mine[:, 1])


def test_runs_have_equal_estimated_cost():
    shape = (324, 324, 144)
    ce, ch = _tables(shape)
    cost = plane_costs(shape, 5, ce, ch)
    runs = balanced_schedule(shape, 5, ce, ch, 296)
    per_run = np.array([cost[t, a:b].sum() for t, a, b, _ in runs])
    # integer run counts per tile leave at most one run's rounding per tile
    assert per_run.max() / per_run.mean() < 1.25
    # tiles with y-slab rows get more, shorter runs than interior tiles
    counts = np.bincount(runs[:, 0])
    assert counts[0] > counts[30]


def test_small_grid_caps_runs_at_one_plane():
    shape = (13, 11, 36)
    ce, ch = _tables(shape, slab=2)
    runs = balanced_schedule(shape, 5, ce, ch, 296)
    assert np.all(runs[:, 2] - runs[:, 1] >= 1)
    assert len(runs) <= 3 * 13
    for t in range(3):
        mine = runs[runs[:, 0] == t]
        assert mine[0, 1] == 0 and mine[-1, 2] == 13 and np.all(mine[1:, 1] == mine[:-1, 2])


def test_split_schedule_keeps_interior_blocks_off_cpml():
    """The time-blocked kernel's schedule: every (tile, plane) once; the first
    `interior` blocks only get planes whose whole reach (x0 - depth - 1 ..
    x1 + depth) and rows carry no x/y CPML, as their build has no CPML code."""
    from warp_fdtd_b200.schedule import interior_region, split_segment_schedule

    shape, ty, depth = (324, 324, 144), 7, 2
    ce, ch = _tables(shape, slab=12)
    runs, M, nin = split_segment_schedule(shape, ty, depth, ce, ch, 148)
    assert runs.shape == (148 * M, 4) and 0 < nin < 148
    tiles = (shape[1] + ty - 1) // ty
    cover = np.zeros((tiles, shape[0]), int)
    for t, a, b, _ in runs:
        if t >= 0:
            cover[t, a:b] += 1
    assert (cover == 1).all()
    ok, x0, x1 = interior_region(shape, ty, depth, ce, ch)
    assert (x0, x1) == (12 + depth + 1, 324 - 12 - depth - 1)
    rows = ty + 2 * depth - 1
    xact = (ce[0, :324, 0] != 0) | (ch[0, :324, 0] != 0)
    yact = (ce[1, :324, 0] != 0) | (ch[1, :324, 0] != 0)
    for b in range(nin):
        for t, a, e, _ in runs[b * M:(b + 1) * M]:
            if t < 0:
                continue
            assert not xact[max(0, a - depth - 1):e + depth + 1].any()
            yf = t * ty - (depth - 1)
            assert not yact[max(0, yf):yf + rows].any()
    # without CPML on x and y every block is an interior block
    for c in (ce, ch):
        c[:2, :, 0] = 0
    runs, M, nin = split_segment_schedule(shape, ty, depth, ce, ch, 148)
    assert nin == 148
