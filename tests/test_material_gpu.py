"""Design-to-material map and its pullback (material.py) on the GPU."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from conftest import GOLDEN  # noqa: E402


def test_pullback_finite_difference():
    """Port of the reference's tests/test_material.py:7-22 (seed 51, 16x16, beta 50)."""
    from warp_fdtd_b200.material import Material

    rng = np.random.default_rng(51)
    p = rng.uniform(0.2, 0.8, (16, 16)).astype(np.float32)
    weights = rng.normal(size=p.shape).astype(np.float32)
    direction = rng.normal(size=p.shape).astype(np.float32)
    direction /= np.linalg.norm(direction)
    material = Material(p, 50)
    gradient = material.pullback(weights)
    analytic = float(np.sum(gradient.astype(float) * direction))
    errors = []
    for h in (0.01, 0.003, 0.001):
        plus = Material(p + h * direction, 50).inv_eps.cpu().numpy()
        minus = Material(p - h * direction, 50).inv_eps.cpu().numpy()
        finite = float(np.sum((plus.astype(float) - minus) * weights) / (2 * h))
        errors.append(abs(finite - analytic) / max(abs(analytic), 1e-12))
    assert min(errors) < 0.01


@pytest.mark.parametrize("shape,beta,eps_lo,contrast", [((16, 16), 50.0, 1.0, 11.25),
                                                        ((125, 125), 8.0, 2.085, 10.025)])
def test_forward_matches_oracle(shape, beta, eps_lo, contrast):
    from oracle.material import material
    from warp_fdtd_b200.material import Material

    rng = np.random.default_rng(0)
    p = rng.uniform(0, 1, shape).astype(np.float32)
    got = Material(p, beta, eps_lo=eps_lo, contrast=contrast).inv_eps.cpu().numpy()
    want = material(p, beta, eps_lo, contrast)
    # float32 map vs float64 oracle: the tanh projection's slope (up to beta/2)
    # amplifies float32 rounding of the filtered density
    assert np.abs(got - want).max() < 2e-5 * np.abs(want).max()


def test_pullback_matches_oracle_directional_derivative():
    """Analytic pullback vs a float64 central difference of the oracle map."""
    from oracle.material import material
    from warp_fdtd_b200.material import Material

    rng = np.random.default_rng(3)
    p = rng.uniform(0, 1, (40, 40)).astype(np.float64)
    g = rng.normal(size=p.shape)
    direction = rng.normal(size=p.shape)
    direction /= np.linalg.norm(direction)
    grad = Material(p.astype(np.float32), 8.0, eps_lo=2.085, contrast=10.025).pullback(g)
    analytic = float(np.sum(grad.astype(float) * direction))
    h = 1e-5
    fd = float(np.sum((material(p + h * direction, 8.0, 2.085, 10.025)
                       - material(p - h * direction, 8.0, 2.085, 10.025)) * g) / (2 * h))
    assert abs(analytic - fd) / abs(fd) < 2e-3


def test_material_reproduces_gradient20_design_box():
    """The map applied to the bundle's parameters reproduces the inverse
    permittivity FDTDX exported in the 20 nm bend's design box (100..180,
    20..100, 30..50); the reference reports 1.6e-6 for its own Warp map."""
    from warp_fdtd_b200.material import Material

    d = np.load(GOLDEN / "gradient20" / "inputs.npz")
    p0 = d["parameters/p0"][..., 0]
    box = d["inv_permittivity"][0, 100:180, 20:100, 30]
    got = Material(p0, 50.0).inv_eps.cpu().numpy()
    assert np.abs(got - box).max() < 5e-6
