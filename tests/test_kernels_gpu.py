"""Kernel-level parity: every CUDA kernel against the CPU oracle, and ports of
the reference's own kernel tests (tests/test_adjoint.py, tests/test_packed.py).

Bitwise equality is required wherever the arithmetic is deterministic: both
sides evaluate the same float32 expressions in the same order without FMA
contraction.  Atomically scattered sums (inject, flux) use tolerances."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

from oracle import cpu as ocpu  # noqa: E402


def T(a, dtype=None):
    a = np.ascontiguousarray(a)
    t = torch.from_numpy(a).cuda()
    return t if dtype is None else t.to(dtype)


def N(t):
    return t.detach().cpu().numpy()


def cpml_table(shape, rng, slabs=2, packed=False, vals=(-0.1, 0.8, 1.2)):
    c = np.zeros((3, max(shape), 3), np.float32)
    c[:, :, 1:] = 1
    for axis, length in enumerate(shape):
        for k in range(slabs):
            c[axis, [k, length - 1 - k]] = [vals[0] * (1 + 0.1 * k), vals[1], vals[2]]
    return c


def pack(c, shape):
    from warp_fdtd_b200.solver import pack_coefficients

    return pack_coefficients(c, shape)


@pytest.mark.parametrize("electric", [True, False])
@pytest.mark.parametrize("packed", [False, True])
@pytest.mark.parametrize("periodic", [0, 1])
def test_update_matches_oracle_bitwise(electric, packed, periodic):
    from warp_fdtd_b200 import kernels as k

    rng = np.random.default_rng(5)
    shape = (6, 7, 9)
    n = int(np.prod(shape))
    f = rng.normal(size=(3, n)).astype(np.float32)
    g = rng.normal(size=(3, n)).astype(np.float32)
    eps = rng.uniform(0.1, 1, n).astype(np.float32)
    c = cpml_table(shape, rng)
    if packed:
        c, size = pack(c, shape)
    else:
        size = n
    psi = (rng.normal(size=(6, size)) * 0.1).astype(np.float32)
    src = rng.normal(size=(3, shape[1] * shape[2])).astype(np.float32)
    waves = rng.normal(size=(3, 4)).astype(np.float32)
    step = np.array([2], np.int32)
    hprev = np.zeros((3, n), np.float32)
    args = dict(save_h_from=1, shape=shape, source_x=3, courant=0.4, periodic=periodic)
    # oracle
    fo, po, ho = f.copy(), psi.copy(), hprev.copy()
    ocpu.update(electric, fo, g, eps, po, c, src, waves, step, ho, args["save_h_from"],
                shape, 3, 0.4, periodic)
    # CUDA
    tf, tpsi, th = T(f), T(psi), T(hprev)
    kern = {(True, False): k.update_e, (False, False): k.update_h,
            (True, True): k.update_e_packed, (False, True): k.update_h_packed}[(electric, packed)]
    k.launch(kern, n, inputs=[tf, T(g), T(eps), tpsi, T(c), T(src), T(waves), T(step), th, 1,
                              *shape, 3, 0.4, periodic])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(N(tf), fo)
    np.testing.assert_array_equal(N(tpsi), po)
    np.testing.assert_array_equal(N(th), ho)


def fused_args(shape, E, H, pe, ph, coeff4, eps, src, waves, step, source_x, courant,
               packed, psi_cols, material=None, table=None, tile=(0, 0, 0)):
    from warp_fdtd_b200 import _lib

    a = _lib.StepArgs()
    for j in range(2):
        a.E[j], a.H[j] = E[j].data_ptr(), H[j].data_ptr()
        a.psi_e[j], a.psi_h[j] = pe[j].data_ptr(), ph[j].data_ptr()
    a.psi_cols = psi_cols
    a.coeff_e, a.coeff_h = coeff4[0].data_ptr(), coeff4[1].data_ptr()
    a.clen = int(coeff4[0].shape[1])
    a.packed = int(packed)
    a.inv_eps = eps.data_ptr()
    if material is not None:
        a.material_kind = 1
        a.material = material.data_ptr()
        a.material_table = table.data_ptr()
        a.material_count = int(table.numel())
    a.src_e, a.src_h = src[0].data_ptr(), src[1].data_ptr()
    a.waves_e, a.waves_h = waves[0].data_ptr(), waves[1].data_ptr()
    a.waves_cols = int(waves[0].shape[1])
    a.source_x = source_x
    a.courant = courant
    a.step = step.data_ptr()
    a.nx, a.ny, a.nz = shape
    a.tile_y, a.tile_z, a.chunk_x = tile
    return a


@pytest.mark.parametrize(
    "shape,tile,packed,u8,path",
    [
        ((13, 11, 37), (4, 8, 5), False, False, 1),
        ((13, 11, 37), (8, 32, 0), True, False, 1),
        ((9, 20, 33), (3, 16, 2), False, True, 1),
        ((5, 6, 7), (16, 64, 64), False, False, 1),
        ((13, 11, 36), (4, 8, 5), False, False, 2),
        ((13, 11, 36), (8, 32, 0), True, False, 2),
        ((9, 20, 32), (3, 16, 2), False, True, 2),
        ((17, 19, 64), (0, 0, 0), True, True, 0),
        ((5, 6, 8), (16, 64, 64), False, False, 2),
        ((21, 26, 48), (12, 48, 7), False, True, 2),
    ],
)
def test_fused_step_matches_oracle_sequence(shape, tile, packed, u8, path):
    """The fused E+H kernel == oracle update_e then update_h, bitwise, over
    several steps, including CPML slabs on all faces, the source plane, ragged
    tiles/chunks and both material and psi storages."""
    from warp_fdtd_b200 import _lib

    rng = np.random.default_rng(11)
    n = int(np.prod(shape))
    steps = 6
    ce = cpml_table(shape, rng, slabs=3)
    chh = cpml_table(shape, rng, slabs=2, vals=(-0.13, 0.75, 1.1))
    ce4, size_e = pack(ce, shape)
    ch4, size_h = pack(chh, shape)
    psi_cols = max(size_e, size_h) if packed else n
    table = rng.uniform(0.08, 1.0, 5).astype(np.float32)
    idx = rng.integers(0, len(table), n).astype(np.uint8)
    eps = table[idx] if u8 else rng.uniform(0.08, 1.0, n).astype(np.float32)
    src = [rng.normal(size=(3, shape[1] * shape[2])).astype(np.float32) for _ in range(2)]
    waves = [rng.normal(size=(3, steps)).astype(np.float32) for _ in range(2)]
    E0 = (rng.normal(size=(3, n)) * 0.3).astype(np.float32)
    H0 = (rng.normal(size=(3, n)) * 0.3).astype(np.float32)
    source_x = shape[0] // 2
    courant = 0.99 / np.sqrt(3)
    # oracle: kernel-level sequence, full psi storage
    oE, oH = E0.copy(), H0.copy()
    ope = np.zeros((6, n), np.float32)
    oph = np.zeros((6, n), np.float32)
    dummy = np.zeros((3, 1), np.float32)
    for t in range(steps):
        st = np.array([t], np.int32)
        ocpu.update(True, oE, oH, eps, ope, ce, src[1], waves[1], st, dummy, 1 << 30, shape,
                    source_x, courant)
        ocpu.update(False, oH, oE, eps, oph, chh, src[0], waves[0], st, dummy, 1 << 30, shape,
                    source_x, courant)
    # CUDA fused with ping-pong buffers
    E = [T(E0), torch.zeros_like(T(E0))]
    H = [T(H0), torch.zeros_like(T(H0))]
    pe = [torch.zeros((6, psi_cols), device="cuda") for _ in range(2)]
    ph = [torch.zeros((6, psi_cols), device="cuda") for _ in range(2)]
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    tsrc = [T(s) for s in src]
    twav = [T(w) for w in waves]
    # every tensor whose pointer goes into the argument block stays referenced
    keep = dict(ce=T(ce4), ch=T(ch4), eps=T(eps), idx=T(idx), table=T(table))
    a = fused_args(shape, E, H, pe, ph, (keep["ce"], keep["ch"]), keep["eps"], tsrc, twav, step,
                   source_x, float(courant), packed, psi_cols,
                   material=keep["idx"] if u8 else None, table=keep["table"] if u8 else None,
                   tile=tile)
    a.path = path
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    a.error = err.data_ptr()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(steps):
        _lib.call("fdtd_step_fused", a, stream)
        _lib.call("fdtd_advance", step.data_ptr(), 1, stream)
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    cur = steps & 1
    np.testing.assert_array_equal(N(E[cur]), oE)
    np.testing.assert_array_equal(N(H[cur]), oH)
    # psi state: compare active cells (full storage only is addressed by cell)
    if not packed:
        for field, (got, want, c) in enumerate(((pe[cur], ope, ce), (ph[cur], oph, chh))):
            x, y, z = np.indices(shape)
            coords = [x, y, z]
            g = N(got).reshape(6, *shape)
            w = want.reshape(6, *shape)
            for axis in range(3):
                active = c[axis, coords[axis], 0] != 0
                for slot in (2 * axis, 2 * axis + 1):
                    np.testing.assert_array_equal(g[slot][active], w[slot][active])


def test_cpml_full_state_transpose():
    """Port of the reference's tests/test_adjoint.py:11-57 (seed 71, 6x7x8)."""
    from warp_fdtd_b200 import kernels as k
    from warp_fdtd_b200 import adjoint as adj

    rng = np.random.default_rng(71)
    shape = (6, 7, 8)
    n = int(np.prod(shape))
    initial = [rng.normal(size=(c, n)).astype(np.float32) * 0.1 for c in (3, 3, 6, 6)]
    cot = [rng.normal(size=a.shape).astype(np.float32) * 0.1 for a in initial]
    e, h, pe, ph = [T(a) for a in initial]
    qe, qh, qpe, qph = [T(a) for a in cot]
    eps = T(rng.uniform(0.2, 1, n).astype(np.float32))
    ce = np.zeros((3, max(shape), 3), np.float32)
    ce[:, :, 1:] = 1
    ch = ce.copy()
    for axis, length in enumerate(shape):
        ce[axis, [0, length - 1]] = [-0.1, 0.8, 1.2]
        ch[axis, [0, length - 1]] = [-0.13, 0.75, 1.1]
    ce, ch = T(ce), T(ch)
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    dummy = torch.zeros((3, n), device="cuda")
    shared = [dummy, dummy, step, dummy, 1, *shape, -1, 0.4, 0]
    k.launch(k.update_e, n, inputs=[e, h, eps, pe, ce, *shared])
    k.launch(k.update_h, n, inputs=[h, e, eps, ph, ch, *shared])
    outputs = [N(a) for a in (e, h, pe, ph)]
    d = torch.empty_like(pe)
    hist = torch.zeros((1, 3, 1), device="cuda")
    grad = torch.zeros(1, device="cuda")
    k.launch(adj.prepare, n, inputs=[qh, eps, qph, ch, d, *shape, 0.4, 0])
    args = [d, hist, grad, step, *shape, 0, 0, 0, 0, 0, 0]
    k.launch(adj.gather, n, inputs=[qe, *args, 1])
    k.launch(adj.prepare, n, inputs=[qe, eps, qpe, ce, d, *shape, 0.4, 1])
    k.launch(adj.gather, n, inputs=[qh, *args, 0])
    transposed = [N(a) for a in (qe, qh, qpe, qph)]
    lhs = sum(np.sum(a.astype(float) * b) for a, b in zip(outputs, cot))
    rhs = sum(np.sum(a.astype(float) * b) for a, b in zip(initial, transposed))
    assert abs(lhs - rhs) / max(abs(lhs), abs(rhs)) < 2e-6


def test_space_time_colocation_transpose():
    """Port of the reference's tests/test_adjoint.py:60-127 (seed 17)."""
    from warp_fdtd_b200 import kernels as k
    from warp_fdtd_b200 import adjoint as adj
    from warp_fdtd_b200.detectors import record

    rng = np.random.default_rng(17)
    shape = (6, 7, 8)
    n = int(np.prod(shape))
    e, h, hp = [T(rng.normal(size=(3, n)).astype(np.float32)) for _ in range(3)]
    sx, sy, sz = 1, 7, 8
    count = sx * sy * sz
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    indices = torch.zeros(1, dtype=torch.int32, device="cuda")
    weights = T(np.array([[0.3, 0.7]], np.float32))
    ph = torch.zeros((6, count, 2), device="cuda")
    flux = torch.zeros(1, device="cuda")
    area = torch.ones(count, device="cuda")
    k.launch(record, count, inputs=[e, h, hp, step, weights, indices, ph, flux, area, *shape,
                                    2, 0, 0, sy, sz, 0, 1, 1])
    source_np = rng.normal(size=(6, count, 2)).astype(np.float32)
    source = T(source_np)
    qe = torch.zeros_like(e)
    qh = torch.zeros_like(h)
    args = [qe, qh, source, weights, step, *shape, 2, 0, 0, sy, sz]
    k.launch(adj.inject, count, inputs=[*args, 0])
    rhs = np.sum(N(qe).astype(float) * N(e)) + np.sum(N(qh).astype(float) * N(h))
    qh.zero_()
    k.launch(adj.inject, count, inputs=[*args, 1])
    rhs += np.sum(N(qh).astype(float) * N(hp))
    v = N(ph)
    lhs = np.sum(source_np[..., 0].astype(float) * v[..., 0]
                 - source_np[..., 1].astype(float) * v[..., 1])
    assert abs(lhs - rhs) / max(abs(lhs), abs(rhs)) < 2e-6


def test_packed_asymmetric_full_state():
    """Port of the reference's tests/test_packed.py:12-91 (seed 8, 7x8x9):
    packed CPML storage is bitwise a storage change, every active psi too."""
    from warp_fdtd_b200 import kernels as k

    shape = (7, 8, 9)
    n = int(np.prod(shape))
    rng = np.random.default_rng(8)
    fields = rng.normal(size=(2, 3, n)).astype("f")
    eps = T(rng.uniform(0.1, 1, n).astype("f"))
    states = []
    for packed in (False, True):
        e, h = [T(v) for v in fields]
        histories, coeffs = [], []
        for field in range(2):
            c = np.zeros((3, max(shape), 3), "f")
            c[..., 1:] = 1
            for axis, length in enumerate(shape):
                active = [0, length - 1] if field == 0 else [1, 2, length - 2]
                if axis == 1:
                    active = active[:1]
                c[axis, active] = [-0.12, 0.8, 0.9]
            pc, size = pack(c, shape)
            coeffs.append(T(pc if packed else c))
            histories.append(torch.zeros((6, size if packed else n), device="cuda"))
        states.append((e, h, histories, coeffs))
    dummy = torch.zeros((3, 1), device="cuda")
    step = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(20):
        for packed, (e, h, histories, coeffs) in enumerate(states):
            kernels = (k.update_e_packed, k.update_h_packed) if packed else (k.update_e, k.update_h)
            for field, kernel in enumerate(kernels):
                k.launch(kernel, n, inputs=[e if field == 0 else h, h if field == 0 else e, eps,
                                            histories[field], coeffs[field], dummy, dummy, step,
                                            dummy, 1000, *shape, -1, 0.2, 0])
    for component in range(2):
        np.testing.assert_array_equal(N(states[0][component]), N(states[1][component]))
    x, y, z = np.indices(shape)
    for field in range(2):
        packed = N(states[1][3][field])
        full_history = N(states[0][2][field]).reshape(6, *shape)
        compact_history = N(states[1][2][field])
        for axis, length in enumerate(shape):
            rank = packed[axis, :length, 3].astype(int)
            coords = [x, y, z]
            index = (
                (rank[x] * shape[1] + y) * shape[2] + z
                if axis == 0
                else ((rank[y] * shape[0] + x) * shape[2] + z if axis == 1
                      else (rank[z] * shape[0] + x) * shape[1] + y)
            )
            active = packed[axis, coords[axis], 0] != 0
            for slot in (2 * axis, 2 * axis + 1):
                np.testing.assert_array_equal(full_history[slot][active],
                                              compact_history[slot, index[active]])


@pytest.mark.parametrize("exact", [0, 1])
def test_record_phasor64_and_flux64_match_oracle(exact):
    from warp_fdtd_b200 import _lib

    rng = np.random.default_rng(3)
    shape = (9, 10, 11)
    n = int(np.prod(shape))
    e_new, h_new, h_old = [rng.normal(size=(3, n)).astype(np.float32) for _ in range(3)]
    t = 3  # odd step: new fields live in buffer 0, H(n-1/2) in buffer 1
    E = [T(e_new), T(np.zeros_like(e_new))]
    H = [T(h_new), T(h_old)]
    step = T(np.array([t], np.int32))
    steps, K = 5, 3
    weights = rng.normal(size=(K, steps, 2)).astype(np.float32)
    lo, sh = (4, 1, 2), (1, 8, 9)
    count = int(np.prod(sh))
    indices = np.array([-1, 0, -1, 2, 1], np.int32)
    ph = torch.zeros((K, 6, count, 2), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # keep every device tensor referenced until the kernels have run
    t_idx, t_w = T(indices), T(weights)
    _lib.call("fdtd_record_phasor64", E[0].data_ptr(), E[1].data_ptr(), H[0].data_ptr(),
              H[1].data_ptr(), step.data_ptr(), t_idx.data_ptr(), steps, t_w.data_ptr(), K,
              ph.data_ptr(), *shape, shape[2], *lo, *sh, exact, stream)
    want = np.zeros((K, 6, count, 2))
    ocpu.lib().oracle_record_phasor(e_new, h_new, h_old, n, t, weights, K, steps, want, *shape,
                                    *lo, *sh, exact)
    np.testing.assert_array_equal(N(ph), want)
    area = rng.uniform(0.5, 1.5, count).astype(np.float32)
    t_area = T(area)
    flux = torch.zeros(3, dtype=torch.float64, device="cuda")
    for axis in range(3):
        _lib.call("fdtd_record_flux64", E[0].data_ptr(), E[1].data_ptr(), H[0].data_ptr(),
                  H[1].data_ptr(), step.data_ptr(), t_idx.data_ptr(), steps, t_area.data_ptr(),
                  flux.data_ptr(), 3, *shape, shape[2], *lo, *sh, axis, exact, stream)
        total = ocpu.lib().oracle_flux_sum(e_new, h_new, h_old, n, area, *shape, *lo, *sh,
                                           axis, exact)
        got = N(flux)[indices[t]]
        assert abs(got - total) <= 1e-12 * max(1.0, abs(total)), (axis, got, total)
        flux.zero_()


def test_prepare_gather_match_oracle_bitwise():
    from warp_fdtd_b200 import kernels as k
    from warp_fdtd_b200 import adjoint as adj

    rng = np.random.default_rng(21)
    shape = (6, 7, 8)
    n = int(np.prod(shape))
    q = rng.normal(size=(3, n)).astype(np.float32)
    eps = rng.uniform(0.2, 1, n).astype(np.float32)
    psi = rng.normal(size=(6, n)).astype(np.float32)
    c = cpml_table(shape, rng)
    box = (1, 2, 1, 3, 4, 5)
    hist = rng.normal(size=(2, 3, 60)).astype(np.float32)
    for electric in (0, 1):
        d_o = np.zeros((6, n), np.float32)
        psi_o = psi.copy()
        ocpu.prepare(q, eps, psi_o, c, d_o, shape, 0.4, electric)
        td, tpsi = torch.zeros((6, n), device="cuda"), T(psi)
        k.launch(adj.prepare, n, inputs=[T(q), T(eps), tpsi, T(c), td, *shape, 0.4, electric])
        torch.cuda.synchronize()
        np.testing.assert_array_equal(N(td), d_o)
        np.testing.assert_array_equal(N(tpsi), psi_o)
        for from_h in (0, 1):
            q_o = q.copy()
            g_o = np.zeros(60, np.float32)
            ocpu.gather(q_o, d_o, hist, g_o, 1, shape, box, from_h)
            tq, tg = T(q), torch.zeros(60, device="cuda")
            step = T(np.array([1], np.int32))
            k.launch(adj.gather, n, inputs=[tq, td, T(hist), tg, step, *shape, *box, from_h])
            torch.cuda.synchronize()
            np.testing.assert_array_equal(N(tq), q_o)
            np.testing.assert_array_equal(N(tg), g_o)


def test_record_curl_and_write_design_match_oracle():
    from warp_fdtd_b200 import kernels as k
    from warp_fdtd_b200 import adjoint as adj

    rng = np.random.default_rng(4)
    shape = (6, 7, 8)
    n = int(np.prod(shape))
    h = rng.normal(size=(3, n)).astype(np.float32)
    box = (1, 2, 3, 4, 3, 2)
    dn = 4 * 3 * 2
    hist_o = np.zeros((3, 3, dn), np.float32)
    ocpu.record_curl(h, hist_o, 2, shape, box, 0.4)
    th = torch.zeros((3, 3, dn), device="cuda")
    k.launch(adj.record_curl, dn, inputs=[T(h), th, T(np.array([2], np.int32)), *shape, *box, 0.4])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(N(th), hist_o)
    plane = rng.normal(size=(4, 3)).astype(np.float32)
    eps = rng.normal(size=n).astype(np.float32)
    eps_o = eps.copy()
    ocpu.lib().oracle_write_design(plane, eps_o, *shape, *box)
    te = T(eps)
    k.launch(adj.write_design, dn, inputs=[T(plane), te, *shape, *box])
    torch.cuda.synchronize()
    np.testing.assert_array_equal(N(te), eps_o)


def test_inject_matches_oracle():
    from warp_fdtd_b200 import kernels as k
    from warp_fdtd_b200 import adjoint as adj

    rng = np.random.default_rng(9)
    shape = (6, 7, 8)
    n = int(np.prod(shape))
    lo, sh = (2, 0, 0), (1, 7, 8)
    count = 56
    source = rng.normal(size=(6, count, 2)).astype(np.float32)
    weights = rng.normal(size=(3, 2)).astype(np.float32)
    for old in (0, 1):
        qe_o = np.zeros((3, n), np.float32)
        qh_o = np.zeros((3, n), np.float32)
        ocpu.inject(qe_o, qh_o, source, weights, 1, shape, lo, sh, old)
        qe, qh = torch.zeros((3, n), device="cuda"), torch.zeros((3, n), device="cuda")
        k.launch(adj.inject, count, inputs=[qe, qh, T(source), T(weights),
                                            T(np.array([1], np.int32)), *shape, *lo, 7, 8, old])
        torch.cuda.synchronize()
        np.testing.assert_allclose(N(qe), qe_o, rtol=1e-6, atol=1e-6)
        np.testing.assert_allclose(N(qh), qh_o, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("nplanes", [2, 5, 8])
def test_inject_many_matches_per_plane_oracle(nplanes):
    """fdtd_inject_many over planes of uneven extents (some overlapping, some
    on the grid's edge) equals the oracle's inject applied plane by plane,
    within float32 atomic-order tolerance; a zero-weight step adds nothing."""
    import ctypes

    from warp_fdtd_b200 import _lib

    rng = np.random.default_rng(30 + nplanes)
    shape = (9, 11, 13)
    nx, ny, nz = shape
    n = int(np.prod(shape))
    steps = 4
    planes, keep = [], []
    for k in range(nplanes):
        sx, sy, sz = int(rng.integers(1, 4)), int(rng.integers(1, ny + 1)), int(rng.integers(1, nz + 1))
        if k == 1:  # overlaps plane 0 exactly
            (x0, y0, z0), (sx, sy, sz) = planes[0][0], planes[0][1]
        else:
            x0, y0, z0 = (int(rng.integers(0, d - s + 1)) for d, s in zip(shape, (sx, sy, sz)))
        count = sx * sy * sz
        src = rng.normal(size=(6, count, 2)).astype(np.float32)
        w = rng.normal(size=(steps, 2)).astype(np.float32)
        w[2] = 0.0  # a step without a source
        planes.append(((x0, y0, z0), (sx, sy, sz), src, w))
    for t in (1, 2):
        for old in (0, 1):
            qe_o = np.zeros((3, n), np.float32)
            qh_o = np.zeros((3, n), np.float32)
            for lo, sh, src, w in planes:
                ocpu.inject(qe_o, qh_o, src, w, t, shape, lo, sh, old)
            arr = (_lib.InjectPlane * nplanes)()
            for pl, (lo, sh, src, w) in zip(arr, planes):
                s_t, w_t = T(src), T(w)
                keep += [s_t, w_t]
                pl.source, pl.weights = s_t.data_ptr(), w_t.data_ptr()
                pl.x0, pl.y0, pl.z0 = lo
                pl.sx, pl.sy, pl.sz = sh
            qe, qh = torch.zeros((3, n), device="cuda"), torch.zeros((3, n), device="cuda")
            step = T(np.array([t], np.int32))
            _lib.call("fdtd_inject_many", qe.data_ptr(), qh.data_ptr(), arr, nplanes,
                      step.data_ptr(), nx, ny, nz, old, None)
            torch.cuda.synchronize()
            np.testing.assert_allclose(N(qe), qe_o, rtol=1e-5, atol=1e-5)
            np.testing.assert_allclose(N(qh), qh_o, rtol=1e-5, atol=1e-5)
            if t == 2:
                assert not N(qe).any() and not N(qh).any()
