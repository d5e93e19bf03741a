"""Drop-in for warp_fdtd/volume.py's VolumeMonitor: passive full-volume
phasors at fixed physical points.

All six components are sampled at the same physical point (trilinear
interpolation of the Yee-staggered fields, zero outside the grid) and H is
centred in time as the mean of H(n+1/2) and H(n-1/2), then accumulated with a
window monitor's DFT weights (volume.py:92-151).  The recorder is the CUDA
kernel behind fdtd_record_volume; accumulators are float64 (the reference
keeps complex64).  Sampling costs a launch per step and is never part of the
solver's benchmark.
"""

import numpy as np
import torch

from . import _lib
from ._lib import ptr


class VolumeMonitor:
    def __init__(self, solver, axes_m, window_monitor, k=0):
        """volume.py:92-124: `axes_m` are three increasing physical axes (m);
        `window_monitor` (a phasor Monitor) supplies the first step and the
        DFT weights, at its frequency index `k`."""
        self.axes_m = tuple(np.asarray(a, dtype=np.float64) for a in axes_m)
        if len(self.axes_m) != 3 or any(
            a.ndim != 1 or not a.size or not np.isfinite(a).all() or np.any(np.diff(a) <= 0)
            for a in self.axes_m
        ):
            raise ValueError("Three finite increasing sampling axes required")
        self.shape = tuple(len(a) for a in self.axes_m)
        self.n = int(np.prod(self.shape))
        self.obj = {"class": "VolumeDiagnostic", "name": "volume"}
        self.name = "volume"
        self.first = window_monitor.first
        self.weights = window_monitor.weights[k].contiguous()
        self.exact = True
        self.is_phasor = False  # no staged batches: accumulates every step
        self.shared = None
        self.batch = 1
        self._folded = 0
        # nominal spacing avoids accumulated errors from float32 edge subtraction
        dx = solver.meta["settings"]["spacing_nm"] * 1e-9
        axes = [(a - float(solver.data[c + "_edges_m"][0])) / dx for a, c in zip(self.axes_m, "xyz")]
        if any(np.any(a < 0) or np.any(a > n) for a, n in zip(axes, solver.shape)):
            raise ValueError("Sampling points must lie within the physical grid")
        points = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)
        self.positions = torch.from_numpy(np.ascontiguousarray(points, np.float32)).to(solver.device)
        self.phasor = torch.zeros((6, self.n, 2), dtype=torch.float64, device=solver.device)
        solver.monitors.append(self)
        solver.save_h_from = min(solver.save_h_from, self.first)

    def launch(self, s, E=None, H=None):
        nx, ny, nz = s.shape
        E = E or s._ord(s._E)
        H = H or s._ord(s._H)
        _lib.call("fdtd_record_volume", E[0], E[1], H[0], H[1],
                  ptr(s.step), ptr(self.positions), self.n, ptr(self.weights),
                  int(self.weights.shape[0]), int(self.first), ptr(self.phasor), nx, ny, nz,
                  s._pitch, _lib.stream_handle(s.device))

    def fold(self, s, issued, into=None):
        return

    def reset(self):
        self.phasor.zero_()
        self._folded = 0

    def phasors(self):
        raw = self.phasor.cpu().numpy()
        return (raw[..., 0] + 1j * raw[..., 1]).reshape(6, *self.shape)
