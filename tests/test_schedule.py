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
