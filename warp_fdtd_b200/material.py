"""Drop-in for warp_fdtd/material.py: the design-to-material map and its pullback.

`Material(params, beta)` applies, as the reference does (material.py:58-102),
a (2r+1)^2 Gaussian filter with clamped edges (r = 9, sigma = 3 cells), then the
subpixel-smoothed tanh projection, then inv_eps = 1 / (eps_lo + contrast * v)
(reference: eps_lo = 1, contrast = 11.25).  The reverse mode is written out by
hand in CUDA (fdtd_material_backward) instead of a Warp Tape.  Extra keyword
arguments select the filter radius / sigma and the permittivity range, e.g.
the benchmark's design map: eps 2.085 - 12.11 (eps_lo=2.085, contrast=10.025).
"""

import numpy as np
import torch

from . import _lib
from ._lib import ptr


def gaussian_weights(radius=9, sigma=3.0):
    """material.py:73-75, float32 arithmetic."""
    xy = np.arange(-radius, radius + 1, dtype=np.float32)
    w = np.exp(-(xy[:, None] ** 2 + xy[None, :] ** 2) / np.float32(2 * sigma * sigma))
    w = w.astype(np.float32)
    w /= w.sum()
    return w


class Material:
    def __init__(self, params, beta, eps_lo=1.0, contrast=11.25, radius=9, sigma=3.0,
                 device="cuda:0"):
        params = np.asarray(params)
        if (
            params.ndim != 2
            or min(params.shape) < 2
            or not np.isfinite(params).all()
            or not np.isfinite(beta)
            or beta <= 0
        ):
            raise ValueError("Require finite 2D parameters and positive finite beta")
        self.device = torch.device(device)
        self.shape = params.shape
        self.beta = float(beta)
        self.eps_lo = float(eps_lo)
        self.contrast = float(contrast)
        self.radius = int(radius)
        self.p = torch.from_numpy(np.ascontiguousarray(params, np.float32)).to(self.device)
        self.weights = torch.from_numpy(gaussian_weights(radius, sigma)).to(self.device)
        self.filtered = torch.empty_like(self.p)
        self.inv_eps = torch.empty_like(self.p)
        px, py = self.shape
        _lib.call("fdtd_material_forward", ptr(self.p), ptr(self.weights), self.radius,
                  ptr(self.filtered), ptr(self.inv_eps), px, py, self.beta, self.eps_lo,
                  self.contrast, _lib.stream_handle(self.device))

    def pullback(self, gradient):
        """d(sum(gradient * inv_eps)) / d params, as a float32 NumPy array."""
        g = torch.as_tensor(np.ascontiguousarray(gradient, np.float32)).to(self.device)
        if tuple(g.shape) != tuple(self.shape):
            raise ValueError("gradient must have the parameters' shape")
        px, py = self.shape
        scratch = torch.empty(2 * px * py, dtype=torch.float32, device=self.device)
        grad = torch.empty_like(self.p)
        _lib.call("fdtd_material_backward", ptr(self.p), ptr(self.weights), self.radius, ptr(g),
                  ptr(scratch), ptr(grad), px, py, self.beta, self.eps_lo, self.contrast,
                  _lib.stream_handle(self.device))
        return grad.cpu().numpy()
