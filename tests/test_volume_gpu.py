"""Volume phasor observer on the GPU (fdtd_record_volume, VolumeMonitor)
against the oracle, an affine field and the plane detector's colocation, in
the manner of the reference's tests/test_volume.py."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _record(e, h, prev, points, weights, t, first, shape):
    """One call of the C ABI with E = e, H = h, H(n-1/2) = prev at step t."""
    from warp_fdtd_b200 import _lib

    n = int(np.prod(shape))
    dev = "cuda"
    E = [torch.zeros((3, n), device=dev), torch.from_numpy(np.ascontiguousarray(e, np.float32)).to(dev)]
    H = [torch.from_numpy(np.ascontiguousarray(prev, np.float32)).to(dev),
         torch.from_numpy(np.ascontiguousarray(h, np.float32)).to(dev)]
    if t & 1:  # odd steps read the new fields from buffer 0
        E.reverse()
        H.reverse()
    step = torch.tensor([t], dtype=torch.int32, device=dev)
    pos = torch.from_numpy(np.ascontiguousarray(points, np.float32)).to(dev)
    w = torch.from_numpy(np.ascontiguousarray(weights, np.float32)).to(dev)
    out = torch.zeros((6, len(points), 2), dtype=torch.float64, device=dev)
    _lib.call("fdtd_record_volume", E[0].data_ptr(), E[1].data_ptr(), H[0].data_ptr(),
              H[1].data_ptr(), step.data_ptr(), pos.data_ptr(), len(points), w.data_ptr(),
              len(weights), first, out.data_ptr(), *shape, shape[2], None)
    torch.cuda.synchronize()
    raw = out.cpu().numpy()
    return raw[..., 0] + 1j * raw[..., 1]


def test_affine_physical_sampling_and_time_centering():
    from tests.test_volume import affine_fields

    shape = (7, 8, 9)
    e, h, prev = affine_fields(shape)
    points = np.array([[2.1, 3.4, 4.2], [1.3, 2.5, 3.7], [4.8, 5.1, 6.3]], "f")
    weights = np.array([[0, 0], [0.2, 0.3]], "f")
    assert not _record(e, h, prev, points, weights, 0, 1, shape).any()
    got = _record(e, h, prev, points, weights, 1, 1, shape)
    for c in range(6):
        v = points[:, 0].astype(float) + 2 * points[:, 1] - 3 * points[:, 2] + c
        np.testing.assert_allclose(got[c], v * (1 if c < 3 else 3) * (0.2 + 0.3j), rtol=2e-6, atol=3e-6)


def test_matches_oracle_bitwise_with_zero_halos():
    from oracle.volume import record_volume

    shape = (6, 7, 9)
    n = int(np.prod(shape))
    rng = np.random.default_rng(5)
    e, h, prev = (rng.normal(size=(3, n)).astype("f") for _ in range(3))
    # points inside, on the faces and within half a cell outside the Yee taps
    points = np.concatenate([rng.uniform(0, 1, (40, 3)) * np.array(shape, "f"),
                             np.array([[0, 0, 0], [6, 7, 9], [0.2, 6.9, 8.8]], "f")]).astype("f")
    weights = np.array([[0.7, -0.4], [0.3, 0.25], [-0.2, 0.9]], "f")
    for t in (1, 2):
        got = _record(e, h, prev, points, weights, t, 1, shape)
        want = np.zeros((6, len(points)), complex)
        record_volume(e, h, prev, points, weights, t, want, shape, 1)
        np.testing.assert_array_equal(got, want)


def test_matches_plane_colocation_including_zero_halos():
    """Volume points at the Ez locations reproduce the exact plane colocation
    of the phasor recorder over the whole grid (reference tolerance)."""
    from warp_fdtd_b200 import _lib

    shape = (7, 8, 9)
    n = int(np.prod(shape))
    rng = np.random.default_rng(18)
    e, h, prev = (rng.normal(size=(3, n)).astype("f") for _ in range(3))
    pts = np.indices(shape).astype("f")
    pts[2] += 0.5
    points = pts.reshape(3, -1).T.copy()
    weights = np.array([[0.3, -0.2]], "f")
    vol = _record(e, h, prev, points, weights, 0, 0, shape)
    dev = "cuda"
    E1 = torch.from_numpy(e).to(dev)
    H1 = torch.from_numpy(h).to(dev)
    H0 = torch.from_numpy(prev).to(dev)
    E0 = torch.zeros_like(E1)
    step = torch.zeros(1, dtype=torch.int32, device=dev)
    idx = torch.zeros(1, dtype=torch.int32, device=dev)
    w = torch.from_numpy(weights).to(dev)
    ph = torch.zeros((1, 6, n, 2), dtype=torch.float64, device=dev)
    _lib.call("fdtd_record_phasor64", E0.data_ptr(), E1.data_ptr(), H0.data_ptr(), H1.data_ptr(),
              step.data_ptr(), idx.data_ptr(), 1, w.data_ptr(), 1, ph.data_ptr(), *shape,
              shape[2], 0, 0, 0, *shape, 1, None)
    torch.cuda.synchronize()
    raw = ph[0].cpu().numpy()
    plane = raw[..., 0] + 1j * raw[..., 1]
    np.testing.assert_allclose(vol, plane, rtol=2e-6, atol=2e-7)


def test_volume_monitor_is_passive_and_matches_the_mode_plane(tmp_path):
    from tests.bundles import make_bundle
    from warp_fdtd_b200.detectors import attach
    from warp_fdtd_b200.solver import Solver
    from warp_fdtd_b200.volume import VolumeMonitor

    case = make_bundle(tmp_path / "b", (12, 10, 20), 40, seed=3)
    base = Solver(case)
    attach(base)
    base.reset()
    base.run()
    s = Solver(case)
    attach(s)
    mode = next(m for m in s.monitors if m.name == "mode_in")
    nx, ny, nz = s.shape
    dx = s.meta["settings"]["spacing_nm"] * 1e-9
    y = mode.lo[1]
    axes = [s.data["x_edges_m"][0] + np.arange(nx) * dx,
            s.data["y_edges_m"][0] + np.array([y]) * dx,
            s.data["z_edges_m"][0] + (np.arange(nz) + 0.5) * dx]
    vol = VolumeMonitor(s, axes, mode)
    s.reset()
    s.run()
    # passive: every detector of the run agrees bit for bit
    for ma, mb in zip(base.monitors, s.monitors):
        assert ma.name == mb.name
        assert np.array_equal(ma.phasor.cpu().numpy(), mb.phasor.cpu().numpy())
        assert np.array_equal(ma.flux.cpu().numpy(), mb.flux.cpu().numpy())
    # the volume at the mode plane's Ez points reproduces its colocated phasors
    np.testing.assert_allclose(vol.phasors(), mode.phasors(0), rtol=2e-6,
                               atol=2e-7 * np.abs(mode.phasors(0)).max())
