"""Every fused-step path of the Solver against the CPU oracle, bitwise.

Seeded bundles with CPML slabs of different widths (>= 2 cells: the
reference finds a slab's axis from its longest array dimension,
solver.py:114-115) on all six faces (E and H tables differ, an inactive plane inside some slabs, optional 1/kappa != 1), a
plane source, a colocated flux detector and a three-frequency mode detector.
Fields and CPML state must equal the oracle's exactly; float64 phasors
exactly; float64 flux sums to 1e-12 (plane sums run in a different order).
These cases pin the single-step kernels (time_block=0); the time-blocked
kernel has its own cases in test_block_gpu.py."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from bundles import make_bundle  # noqa: E402

CASES = [
    # shape, steps, seed, slabs, path, material, kappa  (path 30: path 3 with 2 z cells per thread)
    ((13, 11, 36), 14, 1, ((2, 3), (3, 2), (2, 2)), 1, "f32", False),
    ((13, 11, 36), 14, 1, ((2, 3), (3, 2), (2, 2)), 2, "u8", False),
    ((13, 11, 36), 14, 1, ((2, 3), (3, 2), (2, 2)), 3, "u8", False),
    ((13, 11, 36), 14, 1, ((2, 3), (3, 2), (2, 2)), 3, "f32", True),
    ((11, 7, 30), 12, 2, ((3, 3), (2, 2), (4, 3)), 3, "f32", False),
    ((9, 20, 33), 12, 3, ((2, 2), (3, 3), (3, 2)), 3, "u8", False),
    ((17, 19, 64), 10, 4, ((3, 3), (3, 3), (5, 5)), 3, "u8", True),
    ((21, 26, 48), 10, 5, ((4, 4), (4, 4), (4, 4)), 2, "u8", False),
    ((8, 7, 6), 10, 6, ((2, 2), (2, 2), (2, 2)), 3, "f32", False),
    ((24, 12, 148), 8, 7, ((3, 3), (2, 2), (6, 6)), 3, "u8", False),
    ((13, 11, 36), 14, 1, ((2, 3), (3, 2), (2, 2)), 30, "u8", True),
    ((24, 12, 148), 8, 7, ((3, 3), (2, 2), (6, 6)), 30, "f32", False),
    # path 31: path 3 over the uniform chunk grid instead of the balanced schedule
    ((13, 11, 36), 14, 1, ((2, 3), (3, 2), (2, 2)), 31, "u8", False),
    ((24, 12, 148), 8, 7, ((3, 3), (2, 2), (6, 6)), 31, "f32", True),
]


@pytest.mark.parametrize("shape,steps,seed,slabs,path,material,kappa", CASES)
def test_solver_path_matches_oracle(tmp_path, shape, steps, seed, slabs, path, material, kappa):
    from oracle.model import OracleSolver
    from warp_fdtd_b200.solver import Solver
    from warp_fdtd_b200.detectors import attach

    case = make_bundle(tmp_path / "b", shape, steps, seed=seed, slabs=slabs, kappa=kappa)
    o = OracleSolver(case).attach()
    o.run()
    s = Solver(case, path=3 if path in (30, 31) else path, material=material,
               schedule="uniform" if path == 31 else "balanced", time_block=0)
    if path == 30:
        s._args.vector = 2
    attach(s)
    s.reset()
    s.run()
    assert int(s.kernel_status.item()) == 0
    f = s.fields()
    of = o.fields()
    np.testing.assert_array_equal(f["E"], of["E"])
    np.testing.assert_array_equal(f["H"], of["H"])
    np.testing.assert_array_equal(s.psi_e.cpu().numpy(), o.psi_e)
    np.testing.assert_array_equal(s.psi_h.cpu().numpy(), o.psi_h)
    mons = {m.name: m for m in s.monitors}
    for om in o.monitors:
        m = mons[om.name]
        if om.is_phasor:
            np.testing.assert_array_equal(m.phasor.cpu().numpy(), om.phasor)
        else:
            np.testing.assert_allclose(m.flux.cpu().numpy(), om.flux, rtol=1e-12, atol=1e-300)


def test_graph_replay_and_tiles_identical(tmp_path):
    from warp_fdtd_b200.solver import Solver
    from warp_fdtd_b200.detectors import attach

    case = make_bundle(tmp_path / "b", (19, 23, 44), 40, seed=9)
    ref = None
    for tile, graph_steps in [((0, 0, 0), 16), ((3, 0, 5), 7), ((7, 0, 19), 40), ((1, 0, 3), 3)]:
        s = Solver(case, tile=tile, graph_steps=graph_steps, path=3)
        attach(s)
        s.compile()
        s.reset()
        s.run()
        f = s.fields()
        ph = s.monitors[1].phasor.cpu().numpy()
        if ref is None:
            ref = (f, ph)
        else:
            np.testing.assert_array_equal(f["E"], ref[0]["E"])
            np.testing.assert_array_equal(f["H"], ref[0]["H"])
            np.testing.assert_array_equal(ph, ref[1])


def test_batched_dft_mid_trajectory_reads(tmp_path):
    """Phasors read between batch boundaries include the pending steps (folded
    into a copy) and later folds do not count them twice."""
    from oracle.model import OracleSolver
    from warp_fdtd_b200.solver import Solver
    from warp_fdtd_b200.detectors import attach

    case = make_bundle(tmp_path / "b", (12, 14, 40), 75, seed=12)
    o = OracleSolver(case).attach()
    s = Solver(case, graph_steps=64)
    attach(s)
    s.reset()
    mode = {m.name: m for m in s.monitors}["mode_in"]
    omode = {m.name: m for m in o.monitors}["mode_in"]
    for n in (20, 45):  # 20 < batch 32, 45 straddles the fold at 32
        while s._issued < n:
            s.launch_step()
        o.run(n - int(o.step[0]))
        got = mode.phasors()
        want = (omode.phasor[0][..., 0] + 1j * omode.phasor[0][..., 1]).reshape(6, *omode.shape)
        np.testing.assert_array_equal(got, want)
    while s._issued < s.steps:
        s.launch_step()
    o.run(s.steps - int(o.step[0]))
    np.testing.assert_array_equal(mode.phasor.cpu().numpy(), omode.phasor)
