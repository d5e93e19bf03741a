"""CPU oracle of a whole forward run on an exported input bundle.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker; the product never imports it.

This is an independent NumPy restatement of the reference's host setup and
detector post-processing, driving the C kernels in oracle/fdtd_oracle.c:

* bundle checks, Courant number and buffers: warp_fdtd/solver.py:54-104;
* CPML coefficient table: solver.py:105-131, packing solver.py:16-29;
* source waveforms in float32 arithmetic: solver.py:132-182;
* step order E, H, detectors, advance: solver.py:194-237;
* detector weights/areas: detectors.py:110-168; modal power
  detectors.py:203-211; measurements detectors.py:223-232; attach
  detectors.py:214-220.

Bundle extensions this repository writes for its own scenes (absent from the
reference's bundles, which therefore take the reference path unchanged):
pulsed source profiles ("GaussianPulseProfile", "HannPulseProfile") and a
detector key "frequencies_hz" listing K DFT frequencies (default: the source
frequency, as the reference does).
"""

import hashlib
import json
from pathlib import Path

import numpy as np

from . import cpu

C0 = 299792458.0


def load_bundle(case):
    path = Path(case)
    meta = json.loads((path / "manifest.json").read_text())
    raw = path / "inputs.npz"
    if hashlib.sha256(raw.read_bytes()).hexdigest() != meta["inputs_sha256"]:
        raise ValueError("Input bundle checksum mismatch")
    with np.load(raw) as data:
        arrays = {n: data[n] for n in data.files}
    return meta, arrays


def cpml_table(meta, data, shape, field):
    """solver.py:105-123: coeff[axis, pos] = (a, b, 1/kappa), default (0,1,1)."""
    coeff = np.zeros((3, max(shape), 3), np.float32)
    coeff[:, :, 1:] = 1
    covered = np.zeros((3, max(shape)), bool)
    for obj in meta["objects"]:
        if obj["class"] != "PerfectlyMatchedLayer":
            continue
        name = obj["name"]
        dims = data[f"{name}/pml_a_{field}"].shape
        axis = int(np.argmax(dims))
        lo, hi = obj["grid_slice"][axis]
        if covered[axis, lo:hi].any():
            raise ValueError("Overlapping CPML slabs unsupported")
        covered[axis, lo:hi] = True
        for j, key in enumerate((f"pml_a_{field}", f"pml_b_{field}", f"inv_kappa_{field}")):
            coeff[axis, lo:hi, j] = data[f"{name}/{key}"].ravel()
    return coeff


def pack_table(coeff, shape):
    """solver.py:16-29: append the per-axis rank of each active plane."""
    packed = np.zeros((*coeff.shape[:2], 4), np.float32)
    packed[..., :3] = coeff
    sizes = []
    for axis, length in enumerate(shape):
        active = coeff[axis, :length, 0] != 0
        packed[axis, :length, 3] = np.maximum(np.cumsum(active) - 1, 0)
        sizes.append(int(active.sum()) * (int(np.prod(shape)) // length))
    return packed, max(1, *sizes)


def envelope(src, t):
    """Temporal envelope, float32 arithmetic (t is float32 seconds)."""
    kind = src["temporal_profile"]
    if kind == "SingleFrequencyProfile":
        # solver.py:178-180
        return np.clip(t / np.float32(src["num_startup_periods"] / src["frequency_hz"]), 0, 1)
    if kind == "GaussianPulseProfile":
        s = np.float32(src["pulse_sigma_s"])
        u = (t - np.float32(src["pulse_delay_s"])) / s
        return np.exp(np.float32(-0.5) * u * u).astype(np.float32)
    if kind == "HannPulseProfile":
        width = np.float32(src["pulse_width_s"])
        u = (t - np.float32(src["pulse_delay_s"])) / width + np.float32(0.5)
        inside = (u >= 0) & (u <= 1)
        s = np.sin(np.float32(np.pi) * u)
        return np.where(inside, s * s, np.float32(0)).astype(np.float32)
    raise ValueError(f"Unsupported temporal profile {kind}")


def source_waves(meta, data, steps, field):
    """solver.py:162-181, float32 operation by operation."""
    src = next(o for o in meta["objects"] if o["class"] == "ModePlaneSource")
    name = src["name"]
    offsets = data[f"{name}/_time_offset_{field}"].reshape(3, -1)
    half_step = np.float32(0.5 if field == "E" else 0.0)
    t = (np.arange(steps, dtype=np.float32)[None, :] + half_step + offsets[:, :1]) * np.float32(
        meta["dt_s"]
    )
    period = np.float32(1 / src["frequency_hz"])
    phase = (
        np.float32(2 * np.pi) * t / period
        + np.float32(src["phase_shift"])
        + np.float32(src["profile_phase_shift"])
    )
    ramp = envelope(src, t)
    wave = ramp * np.cos(phase) * np.float32(src["static_amplitude_factor"])
    return np.ascontiguousarray(wave, np.float32)


class OracleMonitor:
    """detectors.py:109-211 with K DFT frequencies and float64 phasors."""

    def __init__(self, s, obj):
        self.obj = obj
        self.name = obj["name"]
        cls = obj["class"]
        if cls not in ("ModeOverlapDetector", "PhasorDetector", "PoyntingFluxDetector"):
            raise ValueError(f"Unsupported detector {cls}")
        self.is_phasor = cls in ("ModeOverlapDetector", "PhasorDetector")
        self.lo = [a for a, b in obj["grid_slice"]]
        self.shape = tuple(hi - lo for lo, hi in obj["grid_slice"])
        self.n = int(np.prod(self.shape))
        self.exact = bool(self.is_phasor or s.meta["settings"].get("exact_interpolation", False))
        self.indices = np.ascontiguousarray(s.data[self.name + "/_time_step_to_arr_idx"], np.int32)
        self.first = int(np.flatnonzero(self.indices >= 0)[0])
        src = next(o for o in s.meta["objects"] if o["class"] == "ModePlaneSource")
        self.freqs = [float(f) for f in obj.get("frequencies_hz", [src["frequency_hz"]])]
        K = len(self.freqs)
        weights = np.zeros((K, s.steps), np.complex64)
        if self.is_phasor:
            t = np.arange(s.steps, dtype=np.float32) * np.float32(s.meta["dt_s"])
            for k, f in enumerate(self.freqs):
                phase = np.float32(2 * np.pi * f) * t
                weights[k] = (
                    np.exp(1j * phase).astype(np.complex64)
                    * np.float32(2 / obj["window_sum"])
                    * s.data[self.name + "/_window_at_time_step_arr"]
                )
        self.weights = np.ascontiguousarray(
            np.stack((weights.real, weights.imag), axis=-1), np.float32
        )  # (K, steps, 2)
        self.phasor = np.zeros((K, 6, self.n, 2), np.float64)
        self.flux = np.zeros(int(self.indices.max()) + 1, np.float64)
        self.axis = obj.get("propagation_axis", 2)
        widths = []
        for a, axis in enumerate("xyz"):
            lo, hi = obj["grid_slice"][a]
            v = (
                np.diff(s.data[axis + "_edges_m"])[lo:hi]
                if a != self.axis
                else np.ones(hi - lo, np.float32)
            )
            sh = [1, 1, 1]
            sh[a] = len(v)
            widths.append(v.reshape(sh))
        self.area = np.broadcast_to(widths[0] * widths[1] * widths[2], self.shape).copy()
        if cls == "ModeOverlapDetector":
            self.area /= self.area.mean()
        self.area_flat = np.ascontiguousarray(self.area.ravel(), np.float32)

    def record(self, s, t, prev):
        index = self.indices[t]
        if index < 0:
            return
        nx, ny, nz = s.shape
        L = cpu.lib(s.dtype == np.float64)
        if self.is_phasor:
            L.oracle_record_phasor(
                s.E, s.H, prev, s.n, int(t), self.weights, self.weights.shape[0],
                self.weights.shape[1], self.phasor, nx, ny, nz, *self.lo, *self.shape,
                int(self.exact),
            )
        else:
            total = L.oracle_flux_sum(
                s.E, s.H, prev, s.n, self.area_flat, nx, ny, nz, *self.lo, *self.shape,
                int(self.axis), int(self.exact),
            )
            self.flux[index] += total

    def phasors(self, k=0):
        raw = self.phasor[k]
        return (raw[..., 0] + 1j * raw[..., 1]).reshape(6, *self.shape)

    def power(self, s, k=0):
        """detectors.py:203-211, in complex128."""
        ph = self.phasors(k)
        me = s.data[self.name + "/_mode_E"]
        mh = s.data[self.name + "/_mode_H"]
        em = me[k if me.shape[0] > 1 else 0]
        hm = mh[k if mh.shape[0] > 1 else 0]
        integrand = (
            np.cross(em, ph[3:].conj(), axis=0) + np.cross(ph[:3].conj(), hm, axis=0)
        )[self.axis]
        alpha = np.sum(integrand * self.area) / 4
        return float(abs(alpha) ** 2)


class OracleSolver:
    """Host-side restatement of solver.py's Solver for a CPU run."""

    def __init__(self, case, cpml_storage="full", dtype=np.float32):
        """dtype float64 runs the same restatement in double (liboracle64):
        the inputs are the float32 run's, widened."""
        self.meta, self.data = load_bundle(case)
        m, d = self.meta, self.data
        eps = d["inv_permittivity"]
        self.shape = tuple(int(v) for v in eps.shape[1:])
        self.n = int(np.prod(self.shape))
        self.steps = int(m["time_steps"])
        factor = m["settings"].get("courant_factor", 0.99)
        self.courant = factor / np.sqrt(3)
        self.eps = np.ascontiguousarray(eps.reshape(-1), np.float32)
        self.E = np.zeros((3, self.n), np.float32)
        self.H = np.zeros((3, self.n), np.float32)
        self.hprev = np.zeros((3, self.n), np.float32)
        self.step = np.zeros(1, np.int32)
        self.coeffs = {}
        self.cpml_storage = cpml_storage
        for field in "EH":
            c = cpml_table(m, d, self.shape, field)
            if cpml_storage == "packed":
                c, size = pack_table(c, self.shape)
            else:
                size = self.n
            self.coeffs[field] = np.ascontiguousarray(c)
            setattr(self, "psi_" + field.lower(), np.zeros((6, size), np.float32))
        src = next(o for o in m["objects"] if o["class"] == "ModePlaneSource")
        self.source_x = src["grid_slice"][0][0]
        self.sources = {
            f: np.ascontiguousarray(d[f"{src['name']}/_{f}"].reshape(3, -1), np.float32)
            for f in "EH"
        }
        self.waves = {f: source_waves(m, d, self.steps, f) for f in "EH"}
        self.monitors = []
        self.save_h_from = self.steps
        self.dtype = np.dtype(dtype)
        if self.dtype == np.float64:
            wide = lambda a: np.ascontiguousarray(a, np.float64)
            self.eps, self.E, self.H, self.hprev = map(wide, (self.eps, self.E, self.H, self.hprev))
            self.psi_e, self.psi_h = wide(self.psi_e), wide(self.psi_h)
            self.coeffs = {f: wide(c) for f, c in self.coeffs.items()}
            self.sources = {f: wide(a) for f, a in self.sources.items()}
            self.waves = {f: wide(a) for f, a in self.waves.items()}

    def attach(self):
        """detectors.py:214-220."""
        for obj in self.meta["objects"]:
            if obj["class"].endswith("Detector"):
                mon = OracleMonitor(self, obj)
                if self.dtype == np.float64:
                    mon.weights = np.ascontiguousarray(mon.weights, np.float64)
                    mon.area_flat = np.ascontiguousarray(mon.area_flat, np.float64)
                self.monitors.append(mon)
                if mon.exact:
                    self.save_h_from = min(self.save_h_from, mon.first)
        return self

    def reset(self):
        for a in (self.E, self.H, self.hprev, self.psi_e, self.psi_h, self.step):
            a[...] = 0
        for mon in self.monitors:
            mon.phasor[...] = 0
            mon.flux[...] = 0

    def launch_step(self):
        t = int(self.step[0])
        cpu.update(True, self.E, self.H, self.eps, self.psi_e, self.coeffs["E"],
                   self.sources["H"], self.waves["H"], self.step, self.hprev,
                   self.save_h_from, self.shape, self.source_x, self.courant)
        cpu.update(False, self.H, self.E, self.eps, self.psi_h, self.coeffs["H"],
                   self.sources["E"], self.waves["E"], self.step, self.hprev,
                   self.save_h_from, self.shape, self.source_x, self.courant)
        for mon in self.monitors:
            mon.record(self, t, self.hprev)
        self.step[0] += 1

    def run(self, steps=None):
        for _ in range(self.steps if steps is None else steps):
            self.launch_step()

    def fields(self):
        return {"E": self.E.reshape(3, *self.shape).copy(),
                "H": self.H.reshape(3, *self.shape).copy()}

    def measurements(self, k=0):
        """detectors.py:223-232."""
        powers = {
            m.name: m.power(self, k)
            for m in self.monitors
            if m.obj["class"] == "ModeOverlapDetector"
        }
        if powers:
            powers["modal_transmission"] = powers["mode_out"] / powers["mode_in"]
            if "mode_reflected" in powers:
                powers["modal_reflection"] = powers["mode_reflected"] / powers["mode_in"]
        return powers
