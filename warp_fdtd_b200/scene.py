"""Scene generator: input bundles for the straight-guide and 90-degree-bend workloads.

The reference never builds geometry: FDTDX produced every array of its bundles
(baseline/export_case.py:52-167 writes them; the solver only reads them,
warp_fdtd/solver.py:60-66).  The silicon-photonics workloads this repository
benchmarks have no such bundle, so this module writes them in the same format
(inputs.npz + manifest.json, see bundle.py), with

* a cell-centre raster of the guide (uint8-friendly: two materials),
* CPML coefficients graded like the committed bundles: for a slab of L cells,
  sigma(u) = sigma_end * u**m, alpha(u) = alpha_start + (alpha_end -
  alpha_start) * u**m_alpha, kappa(u) likewise, with u the depth into the slab
  (0 at the inner face, 1 at the outer), E samples at u = (L - 1 - i) / L and
  H samples half a cell deeper-to-shallower (mirrored for the high-side
  slab), b = exp(-(sigma / kappa + alpha) dt / eps0) and
  a = sigma / (sigma kappa + kappa^2 alpha) (b - 1).  `cpml_arrays` reproduces
  the exported pml_a/pml_b/inv_kappa arrays of the reference bundles from
  their manifest parameters (tests/test_oracle.py);
* the TE0 eigenmode of the Yee grid itself on the guide's cross-section
  (full-vectorial, the leapfrog's discrete curls with its numerical
  dispersion) for the source, and the same mode passed through the
  recorder's colocation for the mode detectors: on the straight guide the
  source launches the grid's own mode, so modal T is 1 and the backward
  overlap R is ~1e-8 (FDTDX's continuum mode solver is not reproduced);
* pulsed sources (GaussianPulseProfile, HannPulseProfile) and K-frequency DFT
  detectors ("frequencies_hz").
"""

import math

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from .bundle import write_bundle

C0 = 299792458.0
EPS0 = 8.8541878128e-12
ETA0 = 376.730313668
EPS_SI = 12.11
EPS_SIO2 = 2.085


# ---------------------------------------------------------------- CPML

def cpml_sigma_max(thickness, dx, order=3.0, reflection=1e-6):
    """Polynomial-grading maximum conductivity for a target normal reflection."""
    return -(order + 1) * math.log(reflection) / (2 * ETA0 * thickness * dx)


def cpml_arrays(thickness, direction, field, dt, sigma_start=0.0, sigma_end=0.0,
                sigma_order=3.0, alpha_start=0.0, alpha_end=0.0, alpha_order=1.0,
                kappa_start=1.0, kappa_end=1.0, kappa_order=3.0):
    """(a, b, inv_kappa) float32 for one slab, innermost-to-outermost ordering
    as stored along the slab's axis (low side '-' starts at the outer face)."""
    i = np.arange(thickness, dtype=np.float64)
    if direction == "-":
        u = (thickness - 1 - i) / thickness
        if field == "H":
            u = u - 0.5 / thickness
    else:
        u = i / thickness
        if field == "E":
            u = u - 0.5 / thickness
    u = np.clip(u, 0.0, 1.0)
    sigma = sigma_start + (sigma_end - sigma_start) * u ** sigma_order
    alpha = alpha_start + (alpha_end - alpha_start) * u ** alpha_order
    kappa = kappa_start + (kappa_end - kappa_start) * u ** kappa_order
    b = np.exp(-(sigma / kappa + alpha) * dt / EPS0)
    den = sigma * kappa + kappa * kappa * alpha
    a = np.where(den > 0, sigma / np.where(den > 0, den, 1.0) * (b - 1.0), 0.0)
    return a.astype(np.float32), b.astype(np.float32), (1.0 / kappa).astype(np.float32)


def add_cpml(arrays, objects, shape, cells, dt, dx, frequency_hz):
    """Six CPML slabs of `cells` cells, grading parameters as the committed
    bundles use (R = 1e-6, cubic sigma, alpha_start = 2 pi f eps0 / 100)."""
    params = dict(sigma_start=0.0, sigma_end=cpml_sigma_max(cells, dx), sigma_order=3.0,
                  alpha_start=2 * math.pi * frequency_hz * EPS0 / 100, alpha_end=0.0,
                  alpha_order=1.0, kappa_start=1.0, kappa_end=1.0, kappa_order=3.0)
    k = 0
    for axis, length in enumerate(shape):
        for direction in ("-", "+"):
            name = f"Object_{k}"
            k += 1
            sl = [[0, shape[0]], [0, shape[1]], [0, shape[2]]]
            sl[axis] = [0, cells] if direction == "-" else [length - cells, length]
            dims = [1, 1, 1]
            dims[axis] = cells
            for field in "EH":
                a, b, ik = cpml_arrays(cells, direction, field, dt, **params)
                arrays[f"{name}/pml_a_{field}"] = a.reshape(dims)
                arrays[f"{name}/pml_b_{field}"] = b.reshape(dims)
                arrays[f"{name}/inv_kappa_{field}"] = ik.reshape(dims)
            objects.append(dict(name=name, **{"class": "PerfectlyMatchedLayer"},
                                grid_slice=sl, direction=direction, **params))


# ---------------------------------------------------------------- modes

def _forward_difference(nu, nv, d, along):
    """Forward difference (f[next] - f) / d on an nu x nv grid flattened row
    major, along u (0) or v (1), with zero beyond the last row / column."""
    n = nu * nv
    step = nv if along == 0 else 1
    upper = np.ones(n - step)
    if along == 1:
        upper[np.arange(1, n) % nv == 0] = 0.0  # no wrap into the next row
    return sp.diags([-np.ones(n), upper], [0, step], format="csr") / d


def yee_mode(eps, d, dt, wavelength, horizontal=0, n_guess=None):
    """Fundamental TE-like eigenmode of the Yee grid itself on a cross-section.

    `eps[i, j]` is the permittivity of the cells of the plane, indexed by the
    local transverse axes (u, v); the mode travels along w, with (u, v, w) a
    cyclic permutation of (x, y, z) so that the Yee lattice reads the same:
    Eu at (i+1/2, j), Ev at (i, j+1/2), Ew at (i, j) a half cell further in
    w, Hu at (i, j+1/2), Hv at (i+1/2, j), both a half cell further in w, and
    Hw at (i+1/2, j+1/2).  Every cell uses its one permittivity for all three
    E components, as the solver's update does.

    With fields ~ exp(i (w t - beta w)) the leapfrog's differences are exact
    for k~ = 2 sin(w dt / 2) / (c dt) and beta~ = 2 sin(beta d / 2) / d, and
    eliminating Ew, Hw (discrete div H = 0) leaves beta~^2 [Hu; Hv] =
    P [Hu; Hv] with, for D_u, D_v the forward and -D^T the backward
    differences,

        P = [[k~^2 e + e D_v e^-1 B_v + B_u D_u,   B_u D_v - e D_v e^-1 B_u],
             [B_v D_u - e D_u e^-1 B_v,   k~^2 e + B_v D_v + e D_u e^-1 B_u]].

    So the profile is the discrete mode of the update itself, not of
    Maxwell's equations: a source built from it launches (almost) nothing
    else, and a detector overlap with it rejects the backward mode.

    TE-like means the E component along the local axis `horizontal` (0: u,
    1: v) dominates, so the vertical H (the other local axis) dominates H.

    Returns (beta, E, H): the true propagation constant (rad/m) and the
    (3, nu, nv) complex phasors in local components (u, v, w), each at its
    own Yee position; the transverse parts are real, Ew and Hw imaginary."""
    nu, nv = eps.shape
    omega = 2 * math.pi * C0 / wavelength
    k = 2 * math.sin(omega * dt / 2) / (C0 * dt)
    e = sp.diags(eps.ravel().astype(np.float64))
    ie = sp.diags(1.0 / eps.ravel().astype(np.float64))
    Du, Dv = _forward_difference(nu, nv, d, 0), _forward_difference(nu, nv, d, 1)
    Bu, Bv = -Du.T.tocsr(), -Dv.T.tocsr()
    P = sp.bmat([[k * k * e + e @ Dv @ ie @ Bv + Bu @ Du, Bu @ Dv - e @ Dv @ ie @ Bu],
                 [Bv @ Du - e @ Du @ ie @ Bv, k * k * e + Bv @ Dv + e @ Du @ ie @ Bu]],
                format="csc")
    n_top = math.sqrt(float(eps.max())) if n_guess is None else n_guess
    vals, vecs = spla.eigs(P, k=4, sigma=(k * n_top) ** 2, which="LM")
    best = None
    n = nu * nv
    for val, vec in zip(vals, vecs.T):
        bt2 = float(np.real(val))
        if bt2 <= 0 or abs(np.imag(val)) > 1e-6 * abs(bt2):
            continue
        hu, hv = vec[:n], vec[n:]
        # TE-like: horizontal E (Eu ~ beta Hv, Ev ~ -beta Hu) dominates
        vertical, other = (hv, hu) if horizontal == 0 else (hu, hv)
        te = np.sum(np.abs(vertical) ** 2) > np.sum(np.abs(other) ** 2)
        if te and (best is None or bt2 > best[0]):
            best = (bt2, vec)
    if best is None:
        raise ValueError("No guided TE-like mode found")
    bt2, vec = best
    vec = vec / vec[np.argmax(np.abs(vec))]
    bt = math.sqrt(bt2)
    hu, hv = np.real(vec[:n]), np.real(vec[n:])
    hw = (Du @ hu + Dv @ hv) / (1j * bt)
    ew = (Bu @ hv - Bv @ hu) / (1j * k * eps.ravel())
    eu = (Bv @ hw + 1j * bt * hv) / (1j * k * eps.ravel())
    ev = (-1j * bt * hu - Bu @ hw) / (1j * k * eps.ravel())
    beta = 2 / d * math.asin(min(1.0, bt * d / 2))
    shape = (nu, nv)
    E = np.stack([eu.reshape(shape), ev.reshape(shape), ew.reshape(shape)])
    H = np.stack([hu.reshape(shape).astype(complex), hv.reshape(shape).astype(complex),
                  hw.reshape(shape)])
    return beta, E, H


def _to_global(local, axis):
    """(3, nu, nv) local-component plane arrays -> global components on the
    plane's (a, b) index order: axis 0: (u, v, w) = (y, z, x), plane (y, z);
    axis 1: (u, v, w) = (z, x, y), plane (x, z)."""
    if axis == 0:
        return np.stack([local[2], local[0], local[1]])
    return np.stack([local[1].T, local[2].T, local[0].T])


def _colocated(E, H, axis, beta, d, omega, dt):
    """The detectors' colocation (detectors.py:27-62) applied to the mode:
    E and H (3, a, b) global-component profiles of the plane, each the
    amplitude at its own Yee position w_c (the field there being profile *
    exp(-i beta w_c)), averaged onto the common point of each cell the way the
    recorder averages the grid, with H's two time levels averaged
    (cos(w dt / 2)).  Returns the (3, a, b) colocated E and H, phases
    relative to exp(-i beta w) at the plane itself."""
    # components half a cell further along the propagation axis: E_w, H_u, H_v
    half_e = [c == axis for c in range(3)]
    half_h = [c != axis for c in range(3)]

    def at(F, half, c, sx=0, sy=0, sz=0):
        """Component c of F at (x + sx, y + sy, z + sz), sx, sy in {-1, 0},
        sz in {0, 1}, zero outside the plane."""
        sw = sx if axis == 0 else sy  # cells back along the propagation axis
        G = F[c] * np.exp(-1j * beta * d * (sw + 0.5 * half[c]))
        if (sy if axis == 0 else sx):  # one cell back along the plane's first axis
            G = np.concatenate([np.zeros_like(G[:1]), G[:-1]], axis=0)
        if sz:
            G = np.concatenate([G[:, 1:], np.zeros_like(G[:, :1])], axis=1)
        return G

    def mean(F, half, c, shifts):
        return sum(at(F, half, c, *sh) for sh in shifts) / len(shifts)

    ec = np.stack([
        mean(E, half_e, 0, [(0, 0, 0), (-1, 0, 0), (0, 0, 1), (-1, 0, 1)]),
        mean(E, half_e, 1, [(0, 0, 0), (0, -1, 0), (0, 0, 1), (0, -1, 1)]),
        at(E, half_e, 2),
    ])
    hc = np.stack([
        mean(H, half_h, 0, [(0, 0, 0), (0, -1, 0)]),
        mean(H, half_h, 1, [(0, 0, 0), (-1, 0, 0)]),
        mean(H, half_h, 2, [(sx, sy, sz) for sx in (0, -1) for sy in (0, -1) for sz in (0, 1)]),
    ]) * math.cos(omega * dt / 2)
    return ec, hc


def mode_fields(eps_plane, d, dt, wavelength, axis):
    """The Yee-grid TE0 mode (yee_mode) on a plane normal to `axis` (0: x,
    plane eps[y, z]; 1: y, plane eps[x, z]) propagating in +axis.

    Returns (n_eff, source, detector): `source` = (E, H) float32 (3, a, b),
    the real transverse components at their Yee positions (longitudinal
    components zero: the plane source injects only the transverse ones);
    `detector` = (E, H) complex64, the mode as the recorder sees it after
    colocation.  Both normalised so that the colocated sum over cells of
    Re(E x H*)_axis = 2 (unit modal power in the detectors' overlap,
    detectors.py:203-211)."""
    local = eps_plane if axis == 0 else eps_plane.T
    beta, El, Hl = yee_mode(local, d, dt, wavelength, horizontal=0 if axis == 0 else 1)
    E, H = _to_global(El, axis), _to_global(Hl, axis)
    omega = 2 * math.pi * C0 / wavelength
    Ec, Hc = _colocated(E, H, axis, beta, d, omega, dt)
    power = float(np.sum(np.real(np.cross(Ec, Hc.conj(), axis=0)[axis])))
    if not power > 0:
        raise ValueError("Mode solve gave no forward power")
    scale = math.sqrt(2.0 / power)
    tr = [c for c in range(3) if c != axis]
    src_E = np.zeros(E.shape, np.float32)
    src_H = np.zeros(H.shape, np.float32)
    src_E[tr] = np.real(E[tr]) * scale
    src_H[tr] = np.real(H[tr]) * scale
    return beta * C0 / omega, (src_E, src_H), ((Ec * scale).astype(np.complex64),
                                               (Hc * scale).astype(np.complex64))


# ---------------------------------------------------------------- geometry

def bend_raster(shape, dx, pml, radius, width, height, x_turn, y_guide):
    """Boolean core mask: +x input guide at y = y_guide (centre), a quarter
    circle of `radius` from (x_turn, y_guide) to (x_turn + radius, y_guide +
    radius), and a +y output guide at x = x_turn + radius.  Lengths in metres,
    measured from the interior's lower corner (after `pml` cells)."""
    nx, ny, nz = shape
    x = (np.arange(nx) + 0.5 - pml) * dx
    y = (np.arange(ny) + 0.5 - pml) * dx
    z = (np.arange(nz) + 0.5) * dx
    X, Y = np.meshgrid(x, y, indexing="ij")
    half = width / 2
    straight_in = (X <= x_turn) & (np.abs(Y - y_guide) <= half)
    cx, cy = x_turn, y_guide + radius
    r = np.hypot(X - cx, Y - cy)
    arc = (X >= x_turn) & (Y <= cy) & (np.abs(r - radius) <= half)
    straight_out = (Y >= cy) & (np.abs(X - (x_turn + radius)) <= half)
    plane = straight_in | arc | straight_out
    zc = nz * dx / 2
    zmask = np.abs(z - zc) <= height / 2
    return plane[:, :, None] & zmask[None, None, :]


def straight_raster(shape, dx, pml, width, height):
    nx, ny, nz = shape
    y = (np.arange(ny) + 0.5) * dx
    z = (np.arange(nz) + 0.5) * dx
    ym = np.abs(y - ny * dx / 2) <= width / 2
    zm = np.abs(z - nz * dx / 2) <= height / 2
    return np.broadcast_to(ym[None, :, None] & zm[None, None, :], shape)


# ---------------------------------------------------------------- bundles

def _detector_schedule(steps):
    return np.arange(steps, dtype=np.int32), np.ones(steps, np.float32)


def write_scene(path, core, dx, pml, steps, source_x, frequency_hz, pulse, detectors,
                wavelengths, settings):
    """Assemble and write a bundle.  `detectors` lists (name, axis, position)
    mode planes, or (name, axis, position, "-") for the backward-travelling
    mode (its transverse H negated: the reflected power); `pulse` is the
    source object's temporal-profile fields."""
    shape = core.shape
    nx, ny, nz = shape
    dt = 0.99 / math.sqrt(3) * dx / C0
    eps = np.where(core, EPS_SI, EPS_SIO2)
    inv_eps = (1.0 / eps).astype(np.float32)
    arrays = {"inv_permittivity": inv_eps[None], "inv_permeability": np.array(1.0)}
    for a, L in zip("xyz", shape):
        arrays[f"{a}_edges_m"] = (np.arange(L + 1) * dx).astype(np.float32)
    objects = []
    add_cpml(arrays, objects, shape, pml, dt, dx, frequency_hz)
    lam0 = C0 / frequency_hz
    n_eff, (Em, Hm), _ = mode_fields(eps[source_x], dx, dt, lam0, 0)
    arrays["source/_E"] = Em[:, None]
    arrays["source/_H"] = Hm[:, None]
    arrays["source/_neff"] = np.array(n_eff, np.complex64)
    # the H profile sits half a cell ahead along x: delay it by n_eff dx / (2 c dt) steps
    delay = np.float32(-0.5 * n_eff * dx / (C0 * dt))
    off_e = np.zeros((3, 1, ny, nz), np.float32)
    off_h = np.zeros((3, 1, ny, nz), np.float32)
    off_e[0] = delay
    off_h[1:] = delay
    arrays["source/_time_offset_E"] = off_e
    arrays["source/_time_offset_H"] = off_h
    arrays["source/_time_step_to_on_idx"] = np.arange(steps, dtype=np.int32)
    objects.append(dict(name="source", **{"class": "ModePlaneSource"},
                        grid_slice=[[source_x, source_x + 1], [0, ny], [0, nz]],
                        direction="+", propagation_axis=0, horizontal_axis=1, vertical_axis=2,
                        mode_index=0, static_amplitude_factor=1.0, frequency_hz=frequency_hz,
                        phase_shift=0.0, profile_phase_shift=0.0, **pulse))
    freqs = [C0 / w for w in wavelengths]
    idx, window = _detector_schedule(steps)
    for name, axis, pos, *way in detectors:
        direction = way[0] if way else "+"
        sl = [[0, nx], [0, ny], [0, nz]]
        sl[axis] = [pos, pos + 1]
        plane_eps = eps[pos] if axis == 0 else eps[:, pos]
        me, mh = [], []
        for w in wavelengths:
            _, _, (E, H) = mode_fields(plane_eps, dx, dt, w, axis)
            if direction == "-":  # backward mode: transverse H and longitudinal E flip
                H = H.copy()
                E = E.copy()
                for c in range(3):
                    if c == axis:
                        E[c] = -E[c]
                    else:
                        H[c] = -H[c]
            me.append(np.expand_dims(E, axis + 1))
            mh.append(np.expand_dims(H, axis + 1))
        arrays[f"{name}/_mode_E"] = np.stack(me).astype(np.complex64)
        arrays[f"{name}/_mode_H"] = np.stack(mh).astype(np.complex64)
        arrays[f"{name}/_time_step_to_arr_idx"] = idx
        arrays[f"{name}/_window_at_time_step_arr"] = window
        objects.append(dict(name=name, **{"class": "ModeOverlapDetector"}, grid_slice=sl,
                            direction=direction, propagation_axis=axis, mode_index=0,
                            window_sum=float(window.sum()), frequencies_hz=freqs))
    meta = {"settings": dict(spacing_nm=dx * 1e9, precision="float32",
                             exact_interpolation=True, pml_cells=pml, **settings),
            "dt_s": dt, "time_steps": int(steps), "objects": objects,
            "convention": "Normalised fields (H' = eta0 H), Yee staggering, CPML; "
                          "written by warp_fdtd_b200.scene"}
    return write_bundle(path, arrays, meta)


def straight_case(path, spacing_nm=50.0, interior_um=(4.0, 3.0, 2.0), pml=10, steps=1000,
                  wavelengths_um=(1.50, 1.55, 1.60), width_nm=500.0, height_nm=220.0):
    """Straight Si wire (500 x 220 nm, eps 12.11) in SiO2 (2.085), Gaussian pulse
    at 1.55 um, K-wavelength modal detector at the output (and input)."""
    dx = spacing_nm * 1e-9
    inner = [int(round(v * 1e-6 / dx)) for v in interior_um]
    shape = tuple(n + 2 * pml for n in inner)
    core = straight_raster(shape, dx, pml, width_nm * 1e-9, height_nm * 1e-9)
    f0 = C0 / 1.55e-6
    sigma_t = 8e-15
    pulse = dict(temporal_profile="GaussianPulseProfile", pulse_sigma_s=sigma_t,
                 pulse_delay_s=4 * sigma_t)
    sx = pml + 3
    dets = [("mode_in", 0, sx + 2), ("mode_reflected", 0, sx + 2, "-"),
            ("mode_out", 0, shape[0] - pml - 3)]
    return write_scene(path, np.ascontiguousarray(core), dx, pml, steps, sx, f0, pulse, dets,
                       [w * 1e-6 for w in wavelengths_um],
                       dict(scene="straight", domain_um=list(interior_um)))


def bend_case(path, spacing_nm=20.0, interior_um=(6.0, 6.0, 2.4), pml=12, steps=4000,
              radius_um=2.0, nwav=5, width_nm=500.0, height_nm=220.0, pulse_width_fs=200.0):
    """90-degree Si bend (radius 2 um, 500 x 220 nm) in SiO2, Hann-windowed
    pulse (200 fs full width by default) at 1.55 um, modal input (forward and
    backward) and output detectors at `nwav` wavelengths in 1.50-1.60 um.
    At 20 nm, 4000 steps are 152 fs of light: the pulse is still being
    emitted when the run ends, so the transmission is not a converged
    device figure; the workload is the fixed step count."""
    dx = spacing_nm * 1e-9
    inner = [int(round(v * 1e-6 / dx)) for v in interior_um]
    shape = tuple(n + 2 * pml for n in inner)
    R = radius_um * 1e-6
    y_guide = 1.5e-6
    x_turn = interior_um[0] * 1e-6 - 1.5e-6 - R
    core = bend_raster(shape, dx, pml, R, width_nm * 1e-9, height_nm * 1e-9, x_turn, y_guide)
    f0 = C0 / 1.55e-6
    width = pulse_width_fs * 1e-15
    pulse = dict(temporal_profile="HannPulseProfile", pulse_width_s=width,
                 pulse_delay_s=width / 2)
    sx = pml + 3
    x_out_guide = pml + int(round((x_turn + R) / dx))
    dets = [("mode_in", 0, sx + 3), ("mode_reflected", 0, sx + 3, "-"),
            ("mode_out", 1, shape[1] - pml - 4)]
    del x_out_guide
    return write_scene(path, np.ascontiguousarray(core), dx, pml, steps, sx, f0, pulse, dets,
                       list(np.linspace(1.50e-6, 1.60e-6, nwav)),
                       dict(scene="bend", domain_um=list(interior_um), radius_um=radius_um))
