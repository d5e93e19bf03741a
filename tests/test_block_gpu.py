"""The time-blocked step (fdtd_step_block) against the CPU oracle, bitwise.

Depth 1 advances one step per launch, depth 2 two steps per launch with the
detectors fed from the snapshot of the intermediate step.  The same seeded
bundles as the path tests (CPML on all six faces with different E and H
tables, inactive planes inside slabs, optional 1/kappa != 1, padded and
unpadded z rows, uint8 and float32 materials, a plane source, a colocated
flux detector and a three-frequency mode detector): fields, CPML state,
H(n-1/2) and float64 phasors must equal the oracle's exactly; float64 flux
sums to 1e-12 (plane sums run in a different order)."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from bundles import make_bundle  # noqa: E402

CASES = [
    # shape, steps, seed, slabs, material, kappa, time_block, graph_steps (0: eager), tile
    ((13, 11, 36), 14, 1, ((2, 3), (3, 2), (2, 2)), "u8", False, 2, 0, 0),
    ((13, 11, 36), 14, 1, ((2, 3), (3, 2), (2, 2)), "f32", True, 2, 8, 0),
    ((13, 11, 36), 15, 1, ((2, 3), (3, 2), (2, 2)), "u8", True, 1, 0, 0),
    ((11, 7, 30), 12, 2, ((3, 3), (2, 2), (4, 3)), "f32", False, 2, 0, 2),
    ((9, 20, 33), 13, 3, ((2, 2), (3, 3), (3, 2)), "u8", False, 2, 5, 3),
    ((17, 19, 64), 10, 4, ((3, 3), (3, 3), (5, 5)), "u8", True, 2, 4, 0),
    ((17, 19, 64), 10, 4, ((3, 3), (3, 3), (5, 5)), "u8", True, 1, 4, 5),
    ((21, 26, 48), 11, 5, ((4, 4), (4, 4), (4, 4)), "u8", False, 2, 64, 1),
    ((8, 7, 6), 10, 6, ((2, 2), (2, 2), (2, 2)), "f32", False, 2, 0, 0),
    ((24, 12, 148), 9, 7, ((3, 3), (2, 2), (6, 6)), "u8", False, 2, 0, 0),
    ((24, 12, 148), 8, 7, ((3, 3), (2, 2), (6, 6)), "f32", True, 2, 3, 4),
    ((30, 33, 40), 17, 8, ((0, 5), (6, 0), (0, 0)), "u8", False, 2, 6, 0),
]


@pytest.mark.parametrize("shape,steps,seed,slabs,material,kappa,tb,gs,tile", CASES)
def test_block_matches_oracle(tmp_path, shape, steps, seed, slabs, material, kappa, tb, gs, tile):
    from oracle.model import OracleSolver
    from warp_fdtd_b200.solver import Solver
    from warp_fdtd_b200.detectors import attach

    case = make_bundle(tmp_path / "b", shape, steps, seed=seed, slabs=slabs, kappa=kappa)
    o = OracleSolver(case).attach()
    o.run()
    s = Solver(case, material=material, time_block=tb, graph_steps=gs or 64,
               tile=(tile, 0, 0) if tile else None)
    assert s.time_block == tb
    attach(s)
    if gs:
        s.compile()
    s.reset()
    s.run()
    assert int(s.kernel_status.item()) == 0
    f, of = s.fields(), o.fields()
    np.testing.assert_array_equal(f["E"], of["E"])
    np.testing.assert_array_equal(f["H"], of["H"])
    np.testing.assert_array_equal(s.hprev.cpu().numpy(), o.hprev)
    np.testing.assert_array_equal(s.psi_e.cpu().numpy(), o.psi_e)
    np.testing.assert_array_equal(s.psi_h.cpu().numpy(), o.psi_h)
    mons = {m.name: m for m in s.monitors}
    for om in o.monitors:
        m = mons[om.name]
        if om.is_phasor:
            np.testing.assert_array_equal(m.phasor.cpu().numpy(), om.phasor)
        else:
            np.testing.assert_allclose(m.flux.cpu().numpy(), om.flux, rtol=1e-12, atol=1e-300)


def test_block_depth2_single_launch_equals_two_steps(tmp_path):
    """One depth-2 launch from a mid-trajectory state (random fields) equals
    two depth-1 launches, fields and CPML state, bit for bit."""
    from warp_fdtd_b200 import _lib
    from warp_fdtd_b200.solver import Solver
    import ctypes

    case = make_bundle(tmp_path / "b", (19, 23, 44), 10, seed=11, kappa=True)
    a = Solver(case, time_block=2)
    b = Solver(case, time_block=2)
    rng = np.random.default_rng(3)
    E = rng.normal(size=(3, a.n)).astype(np.float32)
    H = rng.normal(size=(3, a.n)).astype(np.float32)
    for s in (a, b):
        s.reset()
        s.step.fill_(3)
        s._issued = 3  # parity 1: the launches read buffers 1
        s.set_fields(E, H)
    for x, y in ((a._psi_e[1], b._psi_e[1]), (a._psi_h[1], b._psi_h[1])):
        x.copy_(torch.from_numpy(rng.normal(size=x.shape).astype(np.float32)))
        y.copy_(x)
    stream = _lib.stream_handle(a.device)
    info = a._block[2]
    extra = a._pair_extra()
    _lib.call("fdtd_step_block", ctypes.byref(info["args"][0]), ctypes.byref(info["plan"]),
              ctypes.byref(extra), stream)
    one = b._block[1]
    for _ in range(2):
        _lib.call("fdtd_step_block", ctypes.byref(one["args"][0]), ctypes.byref(one["plan"]),
                  ctypes.byref(one["extra"]), stream)
        _lib.call("fdtd_advance", _lib.ptr(b.step), 1, stream)
    torch.cuda.synchronize()
    assert int(a.kernel_status.item()) == 0 and int(b.kernel_status.item()) == 0
    # depth 2 read buffers 1 and wrote buffers 0 (relation flipped); the two
    # single steps end in buffers 1
    a._issued = b._issued = 5
    a._rel = 1
    np.testing.assert_array_equal(a.E.cpu().numpy(), b.E.cpu().numpy())
    np.testing.assert_array_equal(a.H.cpu().numpy(), b.H.cpu().numpy())
    np.testing.assert_array_equal(a.psi_e.cpu().numpy(), b.psi_e.cpu().numpy())
    np.testing.assert_array_equal(a.psi_h.cpu().numpy(), b.psi_h.cpu().numpy())
    assert float(np.abs(a.E.cpu().numpy()).max()) > 0
