"""CPU checks of the surrogate's oracle (oracle/surrogate.py): its bf16 rounding
against torch's, the adjoint identities of its layout operators, and its
hand-written backward against central finite differences of the exact
(float64, unrounded) network."""

import numpy as np
import pytest

from oracle import surrogate as osg


def test_round_bf16_matches_torch():
    torch = pytest.importorskip("torch")
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(100000).astype(np.float32) * 10 ** rng.uniform(
        -20, 20, 100000).astype(np.float32), np.array([0.0, -0.0, 1.0, 1.00390625, 1.01171875],
                                                      np.float32)])
    want = torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy()
    np.testing.assert_array_equal(osg.round_bf16(x).view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("C", [1, 3, 8])
def test_layout_adjoints(C):
    rng = np.random.default_rng(C)
    B, H, W = 2, 6, 8
    x = rng.standard_normal((B * H * W, C))
    y = rng.standard_normal((B * H * W, 9 * C))
    assert np.isclose(np.sum(osg.im2col(x, H, W) * y), np.sum(x * osg.col2im(y, H, W, C)))
    yp = rng.standard_normal((B * H * W // 4, C))
    assert np.isclose(np.sum(osg.pool(x, H, W) * yp), np.sum(x * osg.pool_backward(yp, H, W)))
    xs = rng.standard_normal((B * H * W // 4, C))
    assert np.isclose(np.sum(osg.upsample(xs, H // 2, W // 2) * x),
                      np.sum(xs * osg.upsample_backward(x, H // 2, W // 2)))


def test_im2col_taps():
    """Column tap*C + c holds x at (y + dy, x + dx), tap = (dy+1)*3 + (dx+1)."""
    H, W = 4, 5
    x = np.arange(H * W, dtype=np.float64).reshape(-1, 1) + 1
    col = osg.im2col(x, H, W).reshape(H, W, 9)
    assert col[1, 1, 0] == x[0 * W + 0, 0]  # dy=-1, dx=-1
    assert col[1, 1, 5] == x[1 * W + 2, 0]  # dy=0, dx=+1
    assert col[0, 0, 0] == 0 and col[H - 1, W - 1, 8] == 0


def test_oracle_backward_matches_finite_differences():
    """Directional derivative of L = sum(a*T) + sum(c*g) along a random
    parameter direction: backward() against central differences, float64."""
    base, nwav, size, B = 4, 3, (16, 16), 2
    p = osg.init_params(seed=1, base=base, nwav=nwav)
    rng = np.random.default_rng(2)
    # non-zero biases so that the ReLUs are not all at the same kink pattern
    for k in p:
        if k.endswith(".b"):
            p[k] = rng.uniform(0.0, 0.1, p[k].shape)
    x = rng.uniform(0, 1, (B,) + size)
    a = rng.standard_normal((B, nwav))
    c = rng.standard_normal((B,) + size)
    net = osg.OracleSurrogate(p, size, nwav, base, bf16=False, dtype=np.float64)
    T, g = net.forward(x)
    grads = net.backward(a, c)
    v = {k: rng.standard_normal(np.shape(val)) for k, val in p.items()}
    analytic = sum(np.sum(grads[k] * v[k]) for k in p)

    def L(h):
        q = {k: np.asarray(p[k], np.float64) + h * v[k] for k in p}
        n = osg.OracleSurrogate(q, size, nwav, base, bf16=False, dtype=np.float64)
        t, gg = n.forward(x)
        return np.sum(a * t) + np.sum(c * gg)

    h = 1e-6
    fd = (L(h) - L(-h)) / (2 * h)
    assert abs(fd - analytic) <= 1e-6 * abs(analytic), (fd, analytic)


def test_parameter_count_of_default_network():
    p = osg.init_params(base=32, nwav=8)
    n = sum(v.size for v in p.values())
    assert 1.0e6 < n < 1.3e6, n


def test_conv_as_gemm_equals_direct_correlation():
    """im2col(x) . W^T with W[cout, tap*C + c] is the 3 x 3 'same' correlation
    out[p, o] = sum over (dy, dx, c) of x[y+dy, x+dx, c] * W[o, ((dy+1)*3 + dx+1)*C + c]."""
    rng = np.random.default_rng(3)
    B, H, W, C, O = 2, 5, 7, 3, 4
    x = rng.standard_normal((B * H * W, C))
    w = rng.standard_normal((O, 9 * C))
    got = osg.im2col(x, H, W) @ w.T
    xi = x.reshape(B, H, W, C)
    want = np.zeros((B, H, W, O))
    for b in range(B):
        for yy in range(H):
            for xx in range(W):
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        sy, sx = yy + dy, xx + dx
                        if 0 <= sy < H and 0 <= sx < W:
                            tap = (dy + 1) * 3 + (dx + 1)
                            want[b, yy, xx] += w[:, tap * C:(tap + 1) * C] @ xi[b, sy, sx]
    np.testing.assert_allclose(got.reshape(B, H, W, O), want, rtol=1e-12, atol=1e-12)


def test_bf16_network_tracks_the_exact_network():
    """The bf16-rounded forward stays within bf16 accuracy of the float64 one."""
    p = osg.init_params(seed=5, base=8, nwav=4)
    rng = np.random.default_rng(6)
    for k in p:
        if k.endswith(".b"):
            p[k] = rng.uniform(0.0, 0.05, p[k].shape).astype(np.float32)
    x = rng.uniform(0, 1, (2, 16, 16))
    T16, g16 = osg.OracleSurrogate(p, (16, 16), 4, 8, bf16=True).forward(x.astype(np.float32))
    T64, g64 = osg.OracleSurrogate(p, (16, 16), 4, 8, bf16=False, dtype=np.float64).forward(x)
    assert np.linalg.norm(T16 - T64) / np.linalg.norm(T64) < 3e-2
    assert np.linalg.norm(g16 - g64) / np.linalg.norm(g64) < 3e-2
