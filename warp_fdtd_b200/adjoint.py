"""Drop-in for warp_fdtd/adjoint.py: the exact discrete adjoint.

Kernel-level launchables with the reference's argument lists
(record_curl, prepare, gather, inject, retreat, write_design; adjoint.py:17-228,
472-490) run through the C ABI.  The `Adjoint` driver is defined in
adjoint_driver.py and re-exported here.
"""

import torch

from . import _lib
from .kernels import Kernel, retreat  # noqa: F401  (retreat: adjoint.py:226-228)
from ._lib import ptr


def _s(stream):
    return stream if stream is not None else _lib.stream_handle()


def _record_curl(h, hist, step, nx, ny, nz, x0, y0, z0, sx, sy, sz, courant, stream=None):
    if hist.dim() != 3 or hist.shape[1] != 3 or hist.shape[2] != int(sx) * int(sy) * int(sz):
        raise ValueError("hist must be (steps, 3, sx*sy*sz)")
    _lib.call("fdtd_record_curl", ptr(h), int(h.shape[1]), ptr(hist), ptr(step), int(nx),
              int(ny), int(nz), int(x0), int(y0), int(z0), int(sx), int(sy), int(sz),
              float(courant), _s(stream))


def _prepare(q, eps, psi, coeff, d, nx, ny, nz, courant, electric, stream=None):
    if coeff.dim() != 3 or coeff.shape[2] != 3:
        raise ValueError("prepare takes the full (3, L, 3) CPML table")
    _lib.call("fdtd_prepare", ptr(q), ptr(eps), ptr(psi), ptr(coeff), int(coeff.shape[1]),
              ptr(d), int(nx), int(ny), int(nz), float(courant), int(electric), _s(stream))


def _gather(q, d, hist, grad, step, nx, ny, nz, x0, y0, z0, sx, sy, sz, from_h, stream=None):
    if grad.dtype not in (torch.float32, torch.float64):
        raise ValueError("grad must be float32 or float64")
    _lib.call("fdtd_gather", ptr(q), ptr(d), ptr(hist), ptr(grad),
              int(grad.dtype == torch.float64), ptr(step), int(nx), int(ny), int(nz), int(x0),
              int(y0), int(z0), int(sx), int(sy), int(sz), int(from_h), _s(stream))


def _inject(qe, qh, source, weights, step, nx, ny, nz, x0, y0, z0, sy, sz, old_h_only,
            stream=None):
    count = int(source.shape[1])
    sx = count // (int(sy) * int(sz))
    _lib.call("fdtd_inject", ptr(qe), ptr(qh), ptr(source), ptr(weights), ptr(step), int(nx),
              int(ny), int(nz), int(x0), int(y0), int(z0), sx, int(sy), int(sz),
              int(old_h_only), _s(stream))


def _write_design(plane, eps, nx, ny, nz, x0, y0, z0, sx, sy, sz, stream=None):
    if tuple(plane.shape) != (int(sx), int(sy)):
        raise ValueError("plane must be (sx, sy)")
    _lib.call("fdtd_write_design", ptr(plane), ptr(eps), int(nx), int(ny), int(nz), int(x0),
              int(y0), int(z0), int(sx), int(sy), int(sz), _s(stream))


def _n(*a):
    return int(a[0]) * int(a[1]) * int(a[2])


record_curl = Kernel("record_curl", _record_curl, lambda *a: int(a[9]) * int(a[10]) * int(a[11]))
prepare = Kernel("prepare", _prepare, lambda *a: int(a[5]) * int(a[6]) * int(a[7]))
gather = Kernel("gather", _gather, lambda *a: int(a[5]) * int(a[6]) * int(a[7]))
inject = Kernel("inject", _inject, lambda *a: int(a[2].shape[1]))
write_design = Kernel("write_design", _write_design,
                      lambda *a: int(a[8]) * int(a[9]) * int(a[10]))


def __getattr__(name):
    if name == "Adjoint":
        from .adjoint_driver import Adjoint

        return Adjoint
    raise AttributeError(name)
