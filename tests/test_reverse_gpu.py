"""The fused reverse halves (fdtd_reverse_half) against the reference's
prepare -> gather sequence (adjoint.py:388-414), bitwise, and the adjoint
driver's gradient with and without them."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nz", [16, 15])
def test_reverse_halves_match_prepare_gather_bitwise(nz):
    """Rows of whole 16-byte vectors and ragged rows."""
    from warp_fdtd_b200 import _lib
    from warp_fdtd_b200 import adjoint as k
    from warp_fdtd_b200._lib import ptr

    rng = np.random.default_rng(3)
    nx, ny = 21, 18
    n = nx * ny * nz
    box = (4, 3, 5, 9, 7, 6)
    dn = box[3] * box[4] * box[5]
    courant = np.float32(0.99 / np.sqrt(3))
    f32 = lambda *s: torch.from_numpy(rng.standard_normal(s).astype(np.float32)).cuda()  # noqa
    coeff = {}
    for f in "EH":
        c = np.zeros((3, max(nx, ny, nz), 3), np.float32)
        c[:, :, 1:] = 1
        for axis, L in enumerate((nx, ny, nz)):  # 4-cell CPML slabs at both ends
            for pos in list(range(4)) + list(range(L - 4, L)):
                c[axis, pos] = rng.uniform(0.05, 0.9, 3)
        coeff[f] = torch.from_numpy(c).cuda()
    eps = torch.from_numpy(rng.uniform(0.08, 0.5, n).astype(np.float32)).cuda()
    qe, qh = f32(3, n), f32(3, n)
    psie, psih = f32(6, n), f32(6, n)
    hist = f32(4, 3, dn)
    grad = torch.zeros(dn, dtype=torch.float64, device="cuda")
    # fused copies: psi ping-pong pairs start from the same state
    fqe, fqh, fgrad = qe.clone(), qh.clone(), grad.clone()
    pe = [psie.clone(), torch.zeros_like(psie)]
    ph = [psih.clone(), torch.zeros_like(psih)]
    d = torch.empty((6, n), dtype=torch.float32, device="cuda")
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    hstep = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    coeff4 = {f: torch.nn.functional.pad(c, (0, 1)).contiguous() for f, c in coeff.items()}
    for t in (4, 3, 2, 1):  # reverse steps: even, odd, even, odd
        step.fill_(t)
        hstep.fill_(t % 4)
        k.prepare(qh, eps, psih, coeff["H"], d, nx, ny, nz, courant, 0)
        k.gather(qe, d, hist, grad, hstep, nx, ny, nz, *box, 1)
        k.prepare(qe, eps, psie, coeff["E"], d, nx, ny, nz, courant, 1)
        k.gather(qh, d, hist, grad, hstep, nx, ny, nz, *box, 0)
        # step parity 0 reads slot 0 of each pair
        _lib.call("fdtd_reverse_half", 1, ptr(fqe), ptr(fqh), ptr(eps), ptr(ph[0]), ptr(ph[1]),
                  ptr(coeff4["H"]), coeff["H"].shape[1], ptr(step), ptr(hist), ptr(fgrad),
                  ptr(hstep), nx, ny, nz, float(courant), *box, s)
        _lib.call("fdtd_reverse_half", 0, ptr(fqh), ptr(fqe), ptr(eps), ptr(pe[0]), ptr(pe[1]),
                  ptr(coeff4["E"]), coeff["E"].shape[1], ptr(step), None, None, None, nx, ny, nz,
                  float(courant), 0, 0, 0, 0, 0, 0, s)
        torch.cuda.synchronize()
        assert torch.equal(fqe, qe) and torch.equal(fqh, qh)
        assert torch.equal(fgrad, grad)
        out = 1 - (t & 1)  # the slot this step wrote
        x = torch.arange(n, device="cuda") // (ny * nz)
        y = (torch.arange(n, device="cuda") // nz) % ny
        z = torch.arange(n, device="cuda") % nz
        for axis, pos, L in ((0, x, nx), (1, y, ny), (2, z, nz)):
            sl = (pos < 4) | (pos >= L - 4)
            for slot in (2 * axis, 2 * axis + 1):
                assert torch.equal(pe[out][slot][sl], psie[slot][sl])
                assert torch.equal(ph[out][slot][sl], psih[slot][sl])
    assert float(grad.abs().max()) > 0


def test_adjoint_gradient_fused_and_unfused_reverse_agree():
    """The 20 nm bend's gradient with the fused halves and with the
    reference-signature kernels: equal up to the float32 atomics of inject
    (the two sweeps see the same values in a different atomic order)."""
    from conftest import GOLDEN
    from warp_fdtd_b200.adjoint import Adjoint
    from warp_fdtd_b200.detectors import attach

    d = np.load(GOLDEN / "gradient20" / "inputs.npz")
    p0 = d["parameters/p0"][..., 0]
    out = {}
    for fused in (True, False):
        adj = Adjoint(GOLDEN / "gradient20", checkpoint_every=256, fused_reverse=fused)
        attach(adj)
        loss, grad = adj.differentiate(p0)
        out[fused] = (loss, np.asarray(grad, np.float64), adj.grad.cpu().numpy())
        del adj
        torch.cuda.empty_cache()
    assert out[True][0] == out[False][0]
    for j in (1, 2):
        a, b = out[True][j], out[False][j]
        assert np.linalg.norm(a - b) / np.linalg.norm(b) < 1e-5
