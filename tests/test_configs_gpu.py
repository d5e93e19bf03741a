"""Parity at the benchmark configurations' full sizes (CUDA vs CPU oracle).

* Straight Si guide, 50 nm cells, 100 x 80 x 60 (4 x 3 x 2 um + 10-cell
  CPML), Gaussian pulse at 1.55 um, 1000 steps, modal detectors at 1.50 /
  1.55 / 1.60 um: the whole trajectory, fields and float64 phasors bitwise.
* The 20 nm bend grid, 324 x 324 x 144 (the benchmark), 150 steps on the
  full grid: fields bitwise (the CPU oracle needs ~15 s for this)."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_straight_guide_config_full_trajectory(tmp_path):
    from oracle.model import OracleSolver
    from warp_fdtd_b200 import scene
    from warp_fdtd_b200.detectors import attach, measurements
    from warp_fdtd_b200.solver import Solver

    case = scene.straight_case(tmp_path / "straight")
    s = Solver(case)
    attach(s)
    s.compile()
    s.reset()
    s.run()
    o = OracleSolver(case).attach()
    o.run()
    f, of = s.fields(), o.fields()
    np.testing.assert_array_equal(f["E"], of["E"])
    np.testing.assert_array_equal(f["H"], of["H"])
    for m, om in zip(s.monitors, o.monitors):
        np.testing.assert_array_equal(m.phasor.cpu().numpy(), om.phasor)
    meas = measurements(s)
    assert len(meas["modal_transmission_spectrum"]) == 3
    assert all(np.isfinite(meas["modal_transmission_spectrum"]))


def test_bend_benchmark_grid_bitwise(tmp_path):
    from oracle.model import OracleSolver
    from warp_fdtd_b200 import scene
    from warp_fdtd_b200.solver import Solver

    steps = 150
    case = scene.bend_case(tmp_path / "bend", steps=steps)
    s = Solver(case)
    assert s.material_kind == 1 and s.shape == (324, 324, 144)
    s.reset()
    s.run()
    o = OracleSolver(case)
    o.run()
    f, of = s.fields(), o.fields()
    assert float(np.abs(of["H"]).max()) > 0
    np.testing.assert_array_equal(f["E"], of["E"])
    np.testing.assert_array_equal(f["H"], of["H"])
