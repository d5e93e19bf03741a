"""The surrogate's tcgen05 GEMM and network against float64 products and the
CPU oracle (oracle/surrogate.py)."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import surrogate as osg  # noqa: E402


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def _bf16(rng, shape, scale=1.0):
    return torch.from_numpy((rng.standard_normal(shape) * scale).astype(np.float32)).to(
        torch.bfloat16)


@pytest.mark.parametrize("layout", [0, 1])
@pytest.mark.parametrize("M,N,K", [(128, 32, 64), (200, 40, 72), (1000, 96, 288),
                                   (300, 130, 9), (64, 256, 1152), (517, 64, 1000)])
def test_gemm_matches_float64_product(M, N, K, layout):
    from warp_fdtd_b200 import surrogate as sg

    rng = np.random.default_rng(M + N + K)
    lda = (K + 7) // 8 * 8 + 8  # padded rows: the kernel reads K columns only
    A = _bf16(rng, (M, lda))
    B = _bf16(rng, (N, (K + 7) // 8 * 8))
    C = torch.full((M, N), float("nan"), dtype=torch.float32, device="cuda")
    sg.gemm(A.cuda(), B.cuda(), C, M, N, K, lda, B.shape[1], N, layout=layout)
    torch.cuda.synchronize()
    want = A[:, :K].double().numpy() @ B[:, :K].double().numpy().T
    got = C.cpu().numpy()
    assert np.isfinite(got).all()
    assert rel(got, want) < 2e-6, rel(got, want)
    assert sg.status() == 0


def test_gemm_epilogue_bias_relu_bf16_and_strided_output():
    from warp_fdtd_b200 import surrogate as sg

    rng = np.random.default_rng(5)
    M, N, K = 333, 48, 200
    A = _bf16(rng, (M, 200)).cuda()
    B = _bf16(rng, (N, 200)).cuda()
    bias = torch.from_numpy(rng.standard_normal(N).astype(np.float32)).cuda()
    out = torch.zeros((M, 80), dtype=torch.bfloat16, device="cuda")
    sg.gemm(A, B, out[:, 16:64], M, N, K, 200, 200, 80, bias=bias, relu=True)
    acc = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    sg.gemm(A, B, acc, M, N, K, 200, 200, N)
    torch.cuda.synchronize()
    want = osg.round_bf16(np.maximum(acc.cpu().numpy() + bias.cpu().numpy(), 0))
    got = out[:, 16:64].float().cpu().numpy()
    np.testing.assert_array_equal(got, want)
    assert (out[:, :16].float() == 0).all() and (out[:, 64:].float() == 0).all()
    # accumulate
    sg.gemm(A, B, acc, M, N, K, 200, 200, N, accumulate=True)
    torch.cuda.synchronize()
    want2 = A.double().cpu().numpy() @ B.double().cpu().numpy().T
    assert rel(acc.cpu().numpy(), 2 * want2) < 2e-6


@pytest.mark.parametrize("layout", [0, 1])
def test_gemm_split_k_and_reduce(layout):
    from warp_fdtd_b200 import _lib
    from warp_fdtd_b200 import surrogate as sg

    rng = np.random.default_rng(9)
    M, N, K = 288, 32, 51200
    A = _bf16(rng, (M, K)).cuda()
    B = _bf16(rng, (N, K)).cuda()
    part = torch.zeros(64 * M * N, dtype=torch.float32, device="cuda")
    used = sg.gemm(A, B, part, M, N, K, K, K, N, splits=37, split_stride=M * N, layout=layout)
    assert 1 < used <= 37
    out = torch.zeros((N, M), dtype=torch.float32, device="cuda")
    _lib.call("fdtd_sg_splitk_reduce", sg.ptr(part), used, M * N, M, N, N, sg.ptr(out), M, 1,
              None)
    torch.cuda.synchronize()
    want = (A.double().cpu().numpy() @ B.double().cpu().numpy().T).T
    assert rel(out.cpu().numpy(), want) < 2e-6
    assert sg.status() == 0


@pytest.fixture(scope="module")
def pair():
    from warp_fdtd_b200.surrogate import Surrogate

    size, nwav, B = (32, 48), 8, 2
    p = osg.init_params(seed=3, base=32, nwav=nwav)
    rng = np.random.default_rng(4)
    for k in p:
        if k.endswith(".b"):
            p[k] = rng.uniform(0.0, 0.05, p[k].shape).astype(np.float32)
    gpu = Surrogate(size, nwav, params=p)
    cpu = osg.OracleSurrogate(p, size, nwav, 32, bf16=True)
    x = rng.uniform(0, 1, (B,) + size).astype(np.float32)
    return gpu, cpu, x, rng


def test_forward_matches_oracle(pair):
    gpu, cpu, x, _ = pair
    T, g = gpu.forward(torch.from_numpy(x).cuda())
    Tc, gc = cpu.forward(x)
    torch.cuda.synchronize()
    eT, eg = rel(T.cpu().numpy(), Tc), rel(g.cpu().numpy(), gc)
    print("forward rel-L2: T", eT, "g", eg)
    # identical rounding points; the float32 accumulation order differs, which
    # flips an occasional bf16 rounding
    assert eT < 1e-2 and eg < 1e-2


def _backward_case(pair):
    gpu, cpu, x, rng = pair
    B = x.shape[0]
    dT = rng.standard_normal((B, gpu.nwav)).astype(np.float32)
    dg = rng.standard_normal((B, gpu.H, gpu.W)).astype(np.float32) / np.sqrt(gpu.H * gpu.W)
    gpu.forward(torch.from_numpy(x).cuda())
    gpu.backward(torch.from_numpy(dT).cuda(), torch.from_numpy(dg).cuda())
    return gpu, cpu, x, dT, dg, gpu.grads_numpy()


def cosine(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-300))


def test_backward_matches_oracle_on_the_same_activations(pair):
    """The oracle's backward run on the GPU forward's own stored activations:
    the reverse kernels (ReLU masks, col2im, pooling and upsampling adjoints,
    split-K weight-gradient GEMMs, heads) against the oracle, up to float32
    summation order."""
    from warp_fdtd_b200 import surrogate as sg

    gpu, cpu, x, dT, dg, got = _backward_case(pair)
    cpu.set_tape(gpu.activations(), x.shape[0])
    want = cpu.backward(dT, dg)
    worst = 0.0
    for k in want:
        e = rel(got[k], want[k])
        worst = max(worst, e)
        assert e < 2e-3, (k, e)
    print("backward on shared activations, worst rel-L2:", worst)
    assert sg.status() == 0


def test_backward_end_to_end_against_oracle(pair):
    """Forward and backward both the oracle's own: bf16 rounding flips in the
    forward move a few ReLU masks, so the comparison is by direction."""
    gpu, cpu, x, dT, dg, got = _backward_case(pair)
    cpu.forward(x)
    want = cpu.backward(dT, dg)
    worst = min(cosine(got[k], want[k]) for k in want)
    print("end-to-end gradient cosine, worst parameter:", worst)
    assert worst > 0.995


def test_training_reduces_the_loss():
    """Adam on a fixed synthetic task (targets are smooth functions of the
    density): the GPU forward/backward kernels must drive the loss down."""
    from warp_fdtd_b200.surrogate import Surrogate

    rng = np.random.default_rng(11)
    n, size, nwav = 64, (32, 32), 8
    x = rng.uniform(0, 1, (n,) + size).astype(np.float32)
    T = np.stack([x[:, :16].mean(axis=(1, 2)) * (1 + 0.1 * k) for k in range(nwav)], 1)
    g = (x - x.mean(axis=(1, 2), keepdims=True)).astype(np.float32)
    net = Surrogate(size, nwav, seed=1)
    xd, Td, gd = (torch.from_numpy(a.astype(np.float32)).cuda() for a in (x, T, g))
    losses = net.fit(xd, Td, gd, steps=150, batch=16, lr=2e-3, log_every=149)
    print("loss", losses)
    assert losses[-1][1] < 0.2 * losses[0][1]
