"""The checkpointed exact adjoint against the reference's own gradient."""

import json

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from conftest import GOLDEN  # noqa: E402


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def grad20():
    from warp_fdtd_b200.adjoint import Adjoint
    from warp_fdtd_b200.detectors import attach

    d = np.load(GOLDEN / "gradient20" / "inputs.npz")
    p0 = d["parameters/p0"][..., 0]
    adj = Adjoint(GOLDEN / "gradient20", checkpoint_every=256)
    attach(adj)
    loss, grad = adj.differentiate(p0)
    return adj, p0, loss, grad


def test_gradient20_matches_warp(grad20):
    """results/warp/gradient20/gradient.npz: the reference's exact Warp adjoint
    (rel-L2 1.85e-6 against FDTDX's exact gradient)."""
    adj, p0, loss, grad = grad20
    warp = np.load(GOLDEN / "gradient20" / "warp_gradient.npz")
    ref = json.loads((GOLDEN / "gradient20" / "warp_result.json").read_text())
    print("T", -loss, "voxel rel", rel(adj.voxel_gradient(), warp["voxel_gradient"]),
          "grad rel", rel(grad, warp["gradient"]))
    assert abs(-loss - ref["measurements"]["modal_transmission"]) < 1e-5
    assert rel(adj.voxel_gradient(), warp["voxel_gradient"]) < 1e-4
    assert rel(grad, warp["gradient"]) < 1e-4
    fdtdx = np.load(GOLDEN / "gradient20" / "fdtdx_gradient.npz")["g0"][..., 0]
    assert rel(grad, fdtdx) < 1e-4


def test_checkpoint_interval_does_not_change_the_gradient(grad20):
    """Segments recomputed from checkpoints reproduce the forward bitwise (the
    loss is identical), so one full history (the reference's storage) gives the
    same gradient up to the reverse sweep's summation order: inject scatters
    with float32 atomics, as the reference does."""
    from warp_fdtd_b200.adjoint import Adjoint
    from warp_fdtd_b200.detectors import attach

    adj, p0, loss, grad = grad20
    full = Adjoint(GOLDEN / "gradient20", checkpoint_every=10 ** 9)
    attach(full)
    loss2, grad2 = full.differentiate(p0)
    assert loss2 == loss
    assert rel(full.grad.cpu().numpy(), adj.grad.cpu().numpy()) < 1e-5
    assert rel(grad2, grad) < 1e-5


def test_gradient_matches_central_differences(grad20):
    """The whole chain (parameters -> material map -> FDTD -> modal T) against
    central finite differences, h = 1e-3, on 16 seeded pixels drawn from the
    upper quartile of |gradient| (smaller entries move T by less than the
    float32 trajectory resolves; even in the quartile a few pixels change T by
    only ~1e-6, so the bar is on the aggregate and the median)."""
    from warp_fdtd_b200.detectors import measurements

    adj, p0, loss, grad = grad20
    g = np.asarray(grad, np.float64).ravel()
    rng = np.random.default_rng(16)
    top = np.flatnonzero(np.abs(g) >= np.quantile(np.abs(g), 0.75))
    pixels = rng.choice(top, 16, replace=False)
    h = 1e-3

    def transmission(p):
        adj.set_design(p.reshape(p0.shape))
        adj.reset()
        adj.run()
        return measurements(adj)["modal_transmission"]

    fd = []
    for j in pixels:
        pp, pm = p0.ravel().copy(), p0.ravel().copy()
        pp[j] += h
        pm[j] -= h
        fd.append(-(transmission(pp) - transmission(pm)) / (2 * h))
    fd = np.array(fd)
    err = np.abs(fd - g[pixels]) / np.abs(g[pixels])
    print("FD vs adjoint per-pixel relative errors:", np.round(err, 4), "rel-L2", rel(fd, g[pixels]))
    # measured on a B200: rel-L2 1.05e-2, median per-pixel error 6e-3, the two
    # smallest pixels at 0.12 and 0.18 (T moves by ~1e-6 there)
    assert rel(fd, g[pixels]) < 0.02
    assert np.median(err) < 0.01


def test_transmission_loss_autograd_function(grad20):
    """TransmissionLoss.apply(params, adjoint) is -T as a torch scalar, and
    backward() leaves upstream x the adjoint gradient in params.grad (here
    upstream 2.5 from loss * 2.5).  The forward is deterministic, so the loss
    equals differentiate()'s bit for bit; the reverse sweep's float32 atomics
    leave the gradient equal to ~1e-6."""
    from warp_fdtd_b200.adjoint_driver import TransmissionLoss

    adj, p0, loss, grad = grad20
    params = torch.tensor(p0, dtype=torch.float32, requires_grad=True)
    out = TransmissionLoss.apply(params, adj)
    assert out.shape == () and out.dtype == torch.float32 and out.requires_grad
    assert out.item() == np.float32(loss)
    (out * 2.5).backward()
    assert params.grad is not None and params.grad.shape == params.shape
    got = params.grad.numpy() / 2.5
    assert rel(got, grad) < 1e-5
    assert float(np.abs(got).max()) > 0
