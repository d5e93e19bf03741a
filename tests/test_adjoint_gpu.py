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
