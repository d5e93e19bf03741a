"""The seeded uneven bend instances of `python -m warp_fdtd_b200.batch`
(config-4 style): sizes in the stated ranges, design boxes inside the grid
and clear of the source, detector planes and CPML."""

import json

import numpy as np

from warp_fdtd_b200.batch import _uneven_bends


def test_uneven_bend_instances(tmp_path):
    specs = _uneven_bends(tmp_path, 3, 1, 50)
    assert len(specs) == 3
    for case, box in specs:
        meta = json.loads((case / "manifest.json").read_text())
        inv = np.load(case / "inputs.npz")["inv_permittivity"]
        nx, ny, nz = inv.shape[1:]
        assert 160 + 20 <= nx <= 320 + 20 and 160 + 20 <= ny <= 320 + 20 and nz == 96 + 20
        x0, y0, z0, sx, sy, sz = box
        assert 60 <= sx == sy <= 120 and sz == 9  # 1.5-3 um square, 220 nm core
        assert 10 <= x0 and x0 + sx <= nx - 10 and 10 <= y0 and y0 + sy <= ny - 10
        assert 10 <= z0 and z0 + sz <= nz - 10
        src = next(o for o in meta["objects"] if o["class"] == "ModePlaneSource")
        assert src["grid_slice"][0][1] <= x0  # source plane before the box
        for o in meta["objects"]:
            if o["class"] == "ModeOverlapDetector":
                axis = o["propagation_axis"]
                lo, hi = o["grid_slice"][axis]
                start, size = (x0, sx) if axis == 0 else (y0, sy)
                assert hi <= start or lo >= start + size  # plane outside the box
