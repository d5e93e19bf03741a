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
  their manifest parameters (tests/test_scene.py);
* a semi-vectorial finite-difference eigenmode of the guide cross-section for
  the source and the mode detectors (the dominant transverse E component and
  its H partner n_eff * E; parity with FDTDX's full-vectorial mode solver is
  not claimed);
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

def solve_mode(eps, d, wavelength, n_guess):
    """Fundamental scalar mode of a 2-D permittivity map eps[u, v] (grid step
    d): (d2/du2 + d2/dv2 + k0^2 eps) f = beta^2 f with zero boundary values.
    Returns (n_eff, f) with f normalised to max |f| = 1 and positive."""
    nu, nv = eps.shape
    k0 = 2 * math.pi / wavelength
    main = np.full(nu * nv, -4.0 / d ** 2) + k0 ** 2 * eps.ravel()
    off_v = np.full(nu * nv - 1, 1.0 / d ** 2)
    off_v[np.arange(1, nu * nv) % nv == 0] = 0.0
    off_u = np.full(nu * nv - nv, 1.0 / d ** 2)
    A = sp.diags([main, off_v, off_v, off_u, off_u], [0, 1, -1, nv, -nv], format="csc")
    sigma = (k0 * n_guess) ** 2
    vals, vecs = spla.eigs(A, k=1, sigma=sigma, which="LM")
    beta2 = float(np.real(vals[0]))
    f = np.real(vecs[:, 0]).reshape(nu, nv)
    f /= f[np.unravel_index(np.argmax(np.abs(f)), f.shape)]
    return math.sqrt(max(beta2, 0.0)) / k0, f


def mode_fields(eps_plane, d, wavelength, axis, n_guess=2.6):
    """E and H (3, nu, nv) of the fundamental TE-like mode on a plane normal to
    `axis` (0: x, 1: y) propagating in +axis, with the dominant E along the
    plane's horizontal in-plane axis and H' = eta0 H = n_eff x E.  Normalised
    so that sum over cells of (E x H)_axis = 2 (unit modal power in the
    detectors' overlap, detectors.py:203-211)."""
    n_eff, f = solve_mode(eps_plane, d, wavelength, n_guess)
    E = np.zeros((3,) + f.shape)
    H = np.zeros((3,) + f.shape)
    if axis == 0:   # plane (y, z); E_y dominant, H_z = n_eff E_y  -> (E x H)_x = Ey Hz
        E[1] = f
        H[2] = n_eff * f
    else:           # plane (x, z); E_x dominant, H_z = -n_eff E_x -> (E x H)_y = -Ex Hz
        E[0] = f
        H[2] = -n_eff * f
    s = np.sum(np.cross(E, H, axis=0)[axis])
    scale = math.sqrt(2.0 / s)
    return n_eff, (E * scale).astype(np.float32), (H * scale).astype(np.float32)


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
    mode planes; `pulse` is the source object's temporal-profile fields."""
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
    n_eff, Em, Hm = mode_fields(eps[source_x], dx, lam0, 0)
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
    for name, axis, pos in detectors:
        sl = [[0, nx], [0, ny], [0, nz]]
        sl[axis] = [pos, pos + 1]
        plane_eps = eps[pos] if axis == 0 else eps[:, pos]
        me, mh = [], []
        for w in wavelengths:
            _, E, H = mode_fields(plane_eps, dx, w, axis)
            me.append(np.expand_dims(E, axis + 1))
            mh.append(np.expand_dims(H, axis + 1))
        arrays[f"{name}/_mode_E"] = np.stack(me).astype(np.complex64)
        arrays[f"{name}/_mode_H"] = np.stack(mh).astype(np.complex64)
        arrays[f"{name}/_time_step_to_arr_idx"] = idx
        arrays[f"{name}/_window_at_time_step_arr"] = window
        objects.append(dict(name=name, **{"class": "ModeOverlapDetector"}, grid_slice=sl,
                            direction="+", propagation_axis=axis, mode_index=0,
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
    dets = [("mode_in", 0, sx + 2), ("mode_out", 0, shape[0] - pml - 3)]
    return write_scene(path, np.ascontiguousarray(core), dx, pml, steps, sx, f0, pulse, dets,
                       [w * 1e-6 for w in wavelengths_um],
                       dict(scene="straight", domain_um=list(interior_um)))


def bend_case(path, spacing_nm=20.0, interior_um=(6.0, 6.0, 2.4), pml=12, steps=4000,
              radius_um=2.0, nwav=5, width_nm=500.0, height_nm=220.0, pulse_width_fs=100.0):
    """90-degree Si bend (radius 2 um, 500 x 220 nm) in SiO2, Hann-enveloped pulse
    at 1.55 um, modal input/output detectors at `nwav` wavelengths in 1.50-1.60 um."""
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
    dets = [("mode_in", 0, sx + 3), ("mode_out", 1, shape[1] - pml - 4)]
    del x_out_guide
    return write_scene(path, np.ascontiguousarray(core), dx, pml, steps, sx, f0, pulse, dets,
                       list(np.linspace(1.50e-6, 1.60e-6, nwav)),
                       dict(scene="bend", domain_um=list(interior_um), radius_um=radius_um))
