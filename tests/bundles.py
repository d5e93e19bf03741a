"""Small seeded input bundles for parity tests (test utility).

Builds bundles in the reference's format (inputs.npz + manifest.json) with
CPML slabs of different widths and strengths on every face (E and H tables
differ), a plane source, a colocated flux detector and a multi-frequency mode
detector, so the CUDA paths and the CPU oracle can be compared on identical
inputs of any shape."""

import numpy as np

from warp_fdtd_b200.bundle import write_bundle

C0 = 299792458.0


def make_bundle(path, shape, steps, seed=0, slabs=((2, 3), (3, 2), (2, 2)), materials=5,
                source_x=None, exact=True, nfreq=3, kappa=False):
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    dx = 50e-9
    dt = 0.99 / np.sqrt(3) * dx / C0
    table = rng.uniform(0.08, 1.0, materials).astype(np.float32)
    inv_eps = table[rng.integers(0, materials, shape)].astype(np.float32)
    arrays = {"inv_permittivity": inv_eps[None], "inv_permeability": np.array(1.0)}
    for a, L in zip("xyz", shape):
        arrays[f"{a}_edges_m"] = (np.arange(L + 1) * dx).astype(np.float32)
    objs = []
    k = 0
    for axis, (lo_w, hi_w) in enumerate(slabs):
        L = shape[axis]
        for side, w in ((0, lo_w), (1, hi_w)):
            if w == 0:
                continue
            name = f"Object_{k}"
            k += 1
            sl = [[0, nx], [0, ny], [0, nz]]
            sl[axis] = [0, w] if side == 0 else [L - w, L]
            dims = [1, 1, 1]
            dims[axis] = w
            for f, scale in (("E", 1.0), ("H", 1.3)):
                a = (-rng.uniform(0.02, 0.2, w) * scale).astype(np.float32)
                a[rng.integers(0, w)] = 0.0 if w > 2 else a[0]  # an inactive plane inside a slab
                b = rng.uniform(0.6, 0.95, w).astype(np.float32)
                ik = (rng.uniform(0.8, 1.0, w) if kappa else np.ones(w)).astype(np.float32)
                arrays[f"{name}/pml_a_{f}"] = a.reshape(dims)
                arrays[f"{name}/pml_b_{f}"] = b.reshape(dims)
                arrays[f"{name}/inv_kappa_{f}"] = ik.reshape(dims)
            objs.append({"name": name, "class": "PerfectlyMatchedLayer", "grid_slice": sl})
    sx = nx // 3 if source_x is None else source_x
    for f in "EH":
        arrays[f"source/_{f}"] = rng.normal(size=(3, 1, ny, nz)).astype(np.float32)
        off = np.zeros((3, 1, ny, nz), np.float32)
        off[1] = 0.25
        arrays[f"source/_time_offset_{f}"] = off
    arrays["source/_time_step_to_on_idx"] = np.arange(steps, dtype=np.int32)
    f0 = C0 / 1.55e-6
    objs.append({"name": "source", "class": "ModePlaneSource",
                 "grid_slice": [[sx, sx + 1], [0, ny], [0, nz]], "direction": "+",
                 "propagation_axis": 0, "temporal_profile": "SingleFrequencyProfile",
                 "frequency_hz": f0, "phase_shift": 0.0, "profile_phase_shift": np.pi,
                 "num_startup_periods": 1, "static_amplitude_factor": 1.0})
    # flux detector (x-normal plane) and a mode detector with nfreq frequencies
    fx = min(nx - 2, sx + 2)
    fl = [[fx, fx + 1], [1, ny - 1], [1, nz - 1]]
    idx = np.full(steps, -1, np.int32)
    idx[steps // 3:] = np.arange(steps - steps // 3)
    arrays["flux/_time_step_to_arr_idx"] = idx
    objs.append({"name": "flux", "class": "PoyntingFluxDetector", "grid_slice": fl,
                 "direction": "+", "propagation_axis": 0})
    ml = [[0, nx], [ny // 2, ny // 2 + 1], [0, nz]]
    arrays["mode_in/_time_step_to_arr_idx"] = np.where(np.arange(steps) >= steps // 4,
                                                      np.arange(steps), -1).astype(np.int32)
    win = np.hanning(steps).astype(np.float32)
    arrays["mode_in/_window_at_time_step_arr"] = win
    pl = (nx, 1, nz)
    arrays["mode_in/_mode_E"] = (rng.normal(size=(1, 3, *pl)) + 1j * rng.normal(size=(1, 3, *pl))).astype(np.complex64)
    arrays["mode_in/_mode_H"] = (rng.normal(size=(1, 3, *pl)) + 1j * rng.normal(size=(1, 3, *pl))).astype(np.complex64)
    freqs = [C0 / w for w in np.linspace(1.5e-6, 1.6e-6, nfreq)]
    objs.append({"name": "mode_in", "class": "ModeOverlapDetector", "grid_slice": ml,
                 "direction": "+", "propagation_axis": 1, "window_sum": float(win.sum()),
                 "frequencies_hz": freqs})
    meta = {"settings": {"spacing_nm": 50.0, "precision": "float32",
                         "exact_interpolation": bool(exact)},
            "dt_s": dt, "time_steps": int(steps), "objects": objs}
    return write_bundle(path, arrays, meta)
