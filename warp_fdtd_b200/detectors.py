"""Drop-in for warp_fdtd/detectors.py: colocated phasor and flux detectors.

`Monitor`, `attach` and `measurements` keep the reference's names, arguments
and results (detectors.py:109-232).  Differences, all in accuracy's favour:

* phasors accumulate in float64 (K frequencies at once; the reference keeps
  one complex64 phasor at the source frequency);
* flux bins are float64 plane sums instead of float32 atomics;
* monitors that sample the same plane with the same weights (the reference
  bundles' mode_in and mode_reflected) share one accumulator.

The kernel-level `record` (detectors.py:65-106) with the reference's float32
semantics is exported as a launchable for code that drives kernels directly.
"""

import numpy as np
import torch

from . import _lib
from .kernels import Kernel
from ._lib import ptr


def _record(e, h, prev, step, weights, indices, phasor, flux, area, nx, ny, nz, x0, y0, z0,
            sy, sz, axis, exact, is_phasor, count=None, stream=None):
    """detectors.py:65-106; launch size count = sx*sy*sz (sx inferred from area)."""
    count = int(area.numel()) if count is None else int(count)
    sx = count // (int(sy) * int(sz))
    _lib.call(
        "fdtd_record", ptr(e), ptr(h), ptr(prev), int(e.shape[1]), ptr(step), ptr(weights),
        ptr(indices), ptr(phasor), ptr(flux), ptr(area), int(nx), int(ny), int(nz), int(x0),
        int(y0), int(z0), sx, int(sy), int(sz), int(axis), int(exact), int(is_phasor),
        stream if stream is not None else _lib.stream_handle(),
    )


record = Kernel("record", _record, lambda *a: int(a[8].numel()))


class Monitor:
    def __init__(self, solver, obj):
        self.obj = obj
        self.name = obj["name"]
        self.is_phasor = obj["class"] in ("ModeOverlapDetector", "PhasorDetector")
        if obj["class"] not in ("ModeOverlapDetector", "PhasorDetector", "PoyntingFluxDetector"):
            raise ValueError(f"Unsupported detector {obj['class']}")
        self.shape = tuple(hi - lo for lo, hi in obj["grid_slice"])
        self.n = int(np.prod(self.shape))
        self.lo = [a for a, b in obj["grid_slice"]]
        nx, ny, nz = solver.shape
        for a, (lo, hi) in enumerate(obj["grid_slice"]):
            if not 0 <= lo < hi <= solver.shape[a]:
                raise ValueError(f"Detector {self.name} lies outside the grid")
        self.exact = bool(
            self.is_phasor or solver.meta["settings"].get("exact_interpolation", False)
        )
        indices = np.ascontiguousarray(solver.data[self.name + "/_time_step_to_arr_idx"], np.int32)
        if indices.shape != (solver.steps,):
            raise ValueError(f"Detector {self.name} schedule must have one entry per step")
        dev = solver.device
        self.indices = torch.from_numpy(indices).to(dev)
        self.first = int(np.flatnonzero(indices >= 0)[0])
        src = next(o for o in solver.meta["objects"] if o["class"] == "ModePlaneSource")
        self.frequencies = [float(f) for f in obj.get("frequencies_hz", [src["frequency_hz"]])]
        K = len(self.frequencies)
        weights = np.zeros((K, solver.steps), np.complex64)
        if self.is_phasor:
            # detectors.py:133-141, per frequency
            t = np.arange(solver.steps, dtype=np.float32) * np.float32(solver.meta["dt_s"])
            window = solver.data[self.name + "/_window_at_time_step_arr"]
            for j, f in enumerate(self.frequencies):
                phase = np.float32(2 * np.pi * f) * t
                weights[j] = (
                    np.exp(1j * phase).astype(np.complex64)
                    * np.float32(2 / obj["window_sum"])
                    * window
                )
        self.weights_numpy = weights
        self.weights = torch.from_numpy(
            np.ascontiguousarray(np.stack((weights.real, weights.imag), axis=-1), np.float32)
        ).to(dev)
        self.phasor = torch.zeros((K, 6, self.n if self.is_phasor else 1, 2),
                                  dtype=torch.float64, device=dev)
        self.flux = torch.zeros(int(indices.max()) + 1, dtype=torch.float64, device=dev)
        self.axis = obj.get("propagation_axis", 2)
        widths = []
        for a, axis in enumerate("xyz"):
            lo, hi = obj["grid_slice"][a]
            v = (
                np.diff(solver.data[axis + "_edges_m"])[lo:hi]
                if a != self.axis
                else np.ones(hi - lo, np.float32)
            )
            sh = [1, 1, 1]
            sh[a] = len(v)
            widths.append(v.reshape(sh))
        self.area_numpy = np.broadcast_to(widths[0] * widths[1] * widths[2], self.shape).copy()
        if obj["class"] == "ModeOverlapDetector":
            self.area_numpy /= self.area_numpy.mean()
        self.area = torch.from_numpy(
            np.ascontiguousarray(self.area_numpy.ravel(), np.float32)).to(dev)
        self.shared = None  # monitor whose accumulator this one aliases
        self._solver = solver
        # Phasor DFTs are batched: each step stages the float32 samples, a fold
        # every `batch` steps adds them to the float64 phasors in time order.
        self.batch = int(np.gcd(int(solver.graph_steps), 32)) if self.is_phasor else 1
        self.stage = (torch.zeros((self.batch, 6, self.n), dtype=torch.float32, device=dev)
                      if self.is_phasor else None)
        self._folded = 0  # steps already folded (host mirror)

    def _key(self):
        return (tuple(map(tuple, self.obj["grid_slice"])), self.exact, self.is_phasor,
                self.weights_numpy.tobytes(), self.indices.cpu().numpy().tobytes())

    def reset(self):
        if self.shared is None:
            self.phasor.zero_()
            self.flux.zero_()
        self._folded = 0

    def fold(self, s, issued, into=None):
        """Add the steps staged since the last batch boundary to the phasors
        (the window comes from the device step counter).  Folds happen at
        every multiple of `batch` steps and after the last step; `into`
        receives a partial window instead (see phasors)."""
        if self.shared is not None or not self.is_phasor:
            return
        _lib.call("fdtd_dft_fold", ptr(s.step), ptr(self.indices), int(self.indices.numel()),
                  ptr(self.weights), int(self.weights.shape[0]), ptr(self.stage), self.batch,
                  ptr(self.phasor if into is None else into), self.n,
                  _lib.stream_handle(s.device))
        if into is None:
            self._folded = issued

    def launch(self, s, E=None, H=None):
        """Record the step just computed; E, H are the (entry 0, entry 1)
        pointer pairs the recorder picks from by the step parity (default:
        the solver's field buffers)."""
        if self.shared is not None:
            return
        nx, ny, nz = s.shape
        stream = _lib.stream_handle(s.device)
        E = E or s._ord(s._E)
        H = H or s._ord(s._H)
        common = (E[0], E[1], H[0], H[1], ptr(s.step))
        steps = int(self.indices.numel())
        if self.is_phasor:
            _lib.call(
                "fdtd_record_stage", *common, ptr(self.indices), steps, ptr(self.stage),
                self.batch, nx, ny, nz, s._pitch, *self.lo, *self.shape, int(self.exact),
                stream,
            )
        else:
            _lib.call(
                "fdtd_record_flux64", *common, ptr(self.indices), steps, ptr(self.area),
                ptr(self.flux), int(self.flux.numel()), nx, ny, nz, s._pitch, *self.lo,
                *self.shape, int(self.axis), int(self.exact), stream,
            )

    def _accumulator(self):
        owner = self.shared or self
        acc = owner.phasor
        if owner.is_phasor and owner._folded < self._solver._issued:
            # mid-batch read: add the pending steps to a copy
            acc = owner.phasor.clone()
            owner.fold(self._solver, self._solver._issued, into=acc)
        return acc

    def phasors(self, k=0):
        raw = self._accumulator()[k].cpu().numpy()
        return (raw[..., 0] + 1j * raw[..., 1]).reshape(6, *self.shape)

    def all_phasors(self):
        """Every frequency's phasors, (K, 6, *shape) complex128, in one copy
        (the float64 (re, im) pairs read as complex numbers in place)."""
        raw = np.ascontiguousarray(self._accumulator().cpu().numpy())
        return raw.view(np.complex128)[..., 0].reshape(raw.shape[0], 6, *self.shape)

    def powers(self, s, ph_all):
        """power() at every frequency of `ph_all` (all_phasors()).  Only the
        normal component of the two cross products is formed, with
        np.cross's own products and order, so each value equals power()'s."""
        me = s.data[self.name + "/_mode_E"]
        mh = s.data[self.name + "/_mode_H"]
        b, c = (self.axis + 1) % 3, (self.axis + 2) % 3
        out = []
        for k in range(ph_all.shape[0]):
            ph = ph_all[k]
            em = me[k if me.shape[0] > 1 else 0]
            hm = mh[k if mh.shape[0] > 1 else 0]
            hc = ph[3:].conj()
            ec = ph[:3].conj()
            integrand = (em[b] * hc[c] - em[c] * hc[b]) + (ec[b] * hm[c] - ec[c] * hm[b])
            alpha = np.sum(integrand * self.area_numpy) / 4
            out.append(float(abs(alpha) ** 2))
        return out

    def power(self, s, k=0, ph=None):
        """detectors.py:203-211 (complex128 overlap on the host); `ph` the
        frequency's phasors when the caller already holds them."""
        ph = self.phasors(k) if ph is None else ph
        me = s.data[self.name + "/_mode_E"]
        mh = s.data[self.name + "/_mode_H"]
        em = me[k if me.shape[0] > 1 else 0]
        hm = mh[k if mh.shape[0] > 1 else 0]
        integrand = (
            np.cross(em, ph[3:].conj(), axis=0) + np.cross(ph[:3].conj(), hm, axis=0)
        )[self.axis]
        alpha = np.sum(integrand * self.area_numpy) / 4
        return float(abs(alpha) ** 2)


def attach(solver):
    """detectors.py:214-220, plus accumulator sharing for identical planes."""
    for obj in solver.meta["objects"]:
        if obj["class"].endswith("Detector"):
            m = Monitor(solver, obj)
            key = m._key()
            for other in solver.monitors:
                if other.shared is None and other._key() == key:
                    m.shared = other
                    m.phasor = other.phasor
                    m.flux = other.flux
                    break
            solver.monitors.append(m)
            if m.exact:
                solver.save_h_from = min(solver.save_h_from, m.first)


def measurements(solver, k=0):
    """detectors.py:223-232 at frequency index k; with K > 1 frequencies the
    per-frequency values are added as `<name>_spectrum` lists."""
    modal = [m for m in solver.monitors if m.obj["class"] == "ModeOverlapDetector"]
    # one device-to-host copy per accumulator (monitors of one plane share it)
    # and every frequency's power from it
    held, spectra = {}, {}
    for m in modal:
        key = id(m.shared or m)
        if key not in held:
            held[key] = m.all_phasors()
        spectra[m.name] = m.powers(solver, held[key])
    powers = {m.name: spectra[m.name][k] for m in modal}
    if powers:
        powers["modal_transmission"] = powers["mode_out"] / powers["mode_in"]
        if "mode_reflected" in powers:
            powers["modal_reflection"] = powers["mode_reflected"] / powers["mode_in"]
        K = min(len(m.frequencies) for m in modal)
        if K > 1:
            for m in modal:
                powers[m.name + "_spectrum"] = spectra[m.name][:K]
            powers["modal_transmission_spectrum"] = [
                a / b for a, b in zip(powers["mode_out_spectrum"], powers["mode_in_spectrum"])
            ]
            powers["frequencies_hz"] = modal[0].frequencies[:K]
    return powers
