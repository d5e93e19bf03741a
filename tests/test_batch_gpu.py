"""Batched uneven-size instances (BatchSolver) and the launch-shape
autotuner reproduce single-solver runs bit for bit."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _detectors(s):
    return {m.name: (m.phasor.cpu().numpy(), m.flux.cpu().numpy()) for m in s.monitors}


def _run_alone(case):
    from warp_fdtd_b200.detectors import attach
    from warp_fdtd_b200.solver import Solver

    s = Solver(case, graph_steps=8)
    attach(s)
    s.compile()
    s.run()
    return s.fields(), _detectors(s)


def test_batch_of_uneven_instances_matches_single_runs(tmp_path):
    from tests.bundles import make_bundle
    from warp_fdtd_b200.batch import BatchSolver
    from warp_fdtd_b200.detectors import attach
    from warp_fdtd_b200.solver import Solver

    cases = [make_bundle(tmp_path / f"b{i}", shape, steps, seed=i)
             for i, (shape, steps) in enumerate([((14, 12, 20), 30), ((20, 9, 36), 27),
                                                 ((11, 16, 28), 33)])]
    alone = [_run_alone(c) for c in cases]
    solvers = []
    for c in cases:
        s = Solver(c, graph_steps=8)
        attach(s)
        solvers.append(s)
    batch = BatchSolver(solvers, fused=False)  # uneven z: per-instance streams
    assert not batch.fused
    batch.compile()
    batch.run()
    for s, (fields, meas) in zip(solvers, alone):
        got = s.fields()
        for name in ("E", "H"):
            np.testing.assert_array_equal(got[name], fields[name])
        m = _detectors(s)
        assert m.keys() == meas.keys()
        for key in meas:
            for got_a, want_a in zip(m[key], meas[key]):
                np.testing.assert_array_equal(got_a, want_a)
    # a second trajectory after reset gives the same again
    batch.reset()
    batch.run()
    np.testing.assert_array_equal(solvers[0].fields()["E"], alone[0][0]["E"])


def test_autotune_keeps_the_fastest_shape_and_parity(tmp_path):
    from oracle.model import OracleSolver
    from tests.bundles import make_bundle
    from warp_fdtd_b200.solver import Solver

    case = make_bundle(tmp_path / "b", (16, 13, 36), 12, seed=4)
    s = Solver(case)
    timings = s.autotune(repeats=3)
    # the time-blocked kernel: (depth, tile rows, stages), per-step times
    best = min(timings, key=timings.get)
    assert best == (s.time_block, *s.block_shape[s.time_block])
    s0 = Solver(case, time_block=0)
    t0 = s0.autotune(repeats=3)
    assert t0 and min(t0, key=t0.get) == (s0.tile[0], s0.stages, s0.schedule_weights)
    s.reset()
    s.run()
    o = OracleSolver(case)
    o.run()
    f, of = s.fields(), o.fields()
    np.testing.assert_array_equal(f["E"], of["E"])
    np.testing.assert_array_equal(f["H"], of["H"])


def test_fused_batch_of_uneven_instances_matches_single_runs(tmp_path):
    """One batched launch per step over grids of different x/y extents (same z
    pitch and slab width) equals each grid run alone, bit for bit."""
    from tests.bundles import make_bundle
    from warp_fdtd_b200.batch import BatchSolver
    from warp_fdtd_b200.detectors import attach
    from warp_fdtd_b200.solver import Solver

    cases = [make_bundle(tmp_path / f"f{i}", shape, 26, seed=10 + i)
             for i, shape in enumerate([(14, 12, 28), (23, 9, 28), (11, 17, 28), (30, 21, 28)])]
    alone = [_run_alone(c) for c in cases]
    solvers = []
    for c in cases:
        s = Solver(c, graph_steps=8)
        attach(s)
        solvers.append(s)
    batch = BatchSolver(solvers, fused=True)
    assert batch.fused
    batch.compile()
    batch.run()
    for s, (fields, meas) in zip(solvers, alone):
        got = s.fields()
        for name in ("E", "H"):
            np.testing.assert_array_equal(got[name], fields[name])
        m = _detectors(s)
        for key in meas:
            for got_a, want_a in zip(m[key], meas[key]):
                np.testing.assert_array_equal(got_a, want_a)
    batch.reset()
    batch.run()
    np.testing.assert_array_equal(solvers[3].fields()["H"], alone[3][0]["H"])


def test_batch_adjoint_matches_single_instances(tmp_path):
    """Gradients of two uneven 40 nm bends batched on concurrent streams equal
    the instances run alone: losses bitwise (the forwards are deterministic),
    gradients up to the float32 atomics of the adjoint source injection."""
    from warp_fdtd_b200 import scene
    from warp_fdtd_b200.adjoint_driver import Adjoint
    from warp_fdtd_b200.batch import BatchAdjoint
    from warp_fdtd_b200.detectors import attach

    specs = [((2.8, 2.8, 1.2), 0.8, (27, 43, 20, 16, 16, 6)),
             ((3.2, 3.6, 1.2), 1.0, (35, 45, 20, 16, 16, 6))]
    rng = np.random.default_rng(12)

    def build():
        out = []
        for i, (interior, radius, box) in enumerate(specs):
            case = scene.bend_case(tmp_path / f"b{i}", spacing_nm=40.0, interior_um=interior,
                                   pml=8, steps=700, radius_um=radius, nwav=1,
                                   pulse_width_fs=50.0) if not (tmp_path / f"b{i}").exists() \
                else tmp_path / f"b{i}"
            adj = Adjoint(case, box=box, checkpoint_every=256)
            attach(adj)
            out.append(adj)
        return out

    params = [rng.uniform(0, 1, (16, 16)).astype(np.float32) for _ in specs]
    single = [adj.differentiate(p) for adj, p in zip(build(), params)]
    batched = BatchAdjoint(build()).differentiate(params)
    for (l0, g0), (l1, g1) in zip(single, batched):
        assert l0 == l1
        assert np.linalg.norm(g1 - g0) / np.linalg.norm(g0) < 1e-5


def test_batch_release_with_launches_queued_and_device_check(tmp_path):
    """A fused batch closed while its steps are still queued (no synchronise)
    keeps its results: close() waits before the parameter slots go back, and
    a second batch prepared at once on the same slots does not disturb the
    first.  A plan is refused on a device other than its own."""
    import copy
    import ctypes

    from tests.bundles import make_bundle
    from warp_fdtd_b200 import _lib
    from warp_fdtd_b200.batch import BatchSolver
    from warp_fdtd_b200.solver import Solver

    shapes = [(14, 12, 28), (23, 9, 28)]
    cases = [make_bundle(tmp_path / f"r{i}", sh, 20, seed=40 + i) for i, sh in enumerate(shapes)]
    steps = 9
    alone = []
    for c in cases:
        s = Solver(c)
        s.reset()
        for _ in range(steps):
            s.launch_step()
        alone.append(s.fields())
    first = [Solver(c) for c in cases]
    batch = BatchSolver(first, fused=True)
    assert batch.fused
    batch.reset()
    for _ in range(steps):
        batch.launch_step()  # queued, not synchronised
    batch.close()
    second = BatchSolver([Solver(c) for c in reversed(cases)], fused=True)
    second.reset()
    for _ in range(3):
        second.launch_step()
    torch.cuda.synchronize()
    for s, want in zip(first, alone):
        np.testing.assert_array_equal(s.fields()["E"], want["E"])
        np.testing.assert_array_equal(s.fields()["H"], want["H"])
    plan = copy.copy(second._plan)
    plan.device = plan.device + 1
    with pytest.raises(ValueError, match="device"):
        _lib.call("fdtd_step_batch", ctypes.byref(plan), second._ws, second._schedule.data_ptr(),
                  second._blocks, _lib.stream_handle())
    second.close()
