"""Kernel-level drop-ins for warp_fdtd/kernels.py (and the detector/adjoint kernels).

The reference launches Warp kernels directly, e.g. (tests/test_adjoint.py:37-41)

    wp.launch(k.update_e, n, inputs=[e, h, eps, pe, ce, src, waves, step, hprev,
                                      save_h_from, nx, ny, nz, source_x, courant,
                                      periodic], device=device)

Here the same kernels are objects taking the same inputs in the same order, as
torch CUDA tensors, and `launch(kernel, dim, inputs=[...])` mirrors wp.launch.
Each call goes through the C ABI (include/warp_fdtd_b200.h) on the current
torch stream.  Array conventions: a Warp array2d(float) of shape (r, c) is a
float32 tensor (r, c); array2d(vec3|vec4) of shape (3, L) is (3, L, 3|4);
array(vec2) of length m is (m, 2); int arrays are int32.
"""

import torch

from . import _lib
from ._lib import ptr


def _cols(t, rows):
    if t.dim() != 2 or t.shape[0] < rows:
        raise ValueError(f"expected a ({rows}, cols) array, got {tuple(t.shape)}")
    return int(t.shape[1])


def _check(t, dtype, name):
    if t.dtype != dtype:
        raise ValueError(f"{name} must be {dtype}, got {t.dtype}")
    return t


class Kernel:
    """A launchable with the reference kernel's input list."""

    def __init__(self, name, fn, dim_of):
        self.name = name
        self._fn = fn
        self._dim_of = dim_of

    def __call__(self, *inputs, stream=None):
        return self._fn(*inputs, stream=stream)

    def __repr__(self):
        return f"<warp_fdtd_b200 kernel {self.name}>"


def launch(kernel, dim, inputs, device=None, stream=None):
    """Counterpart of wp.launch for the kernels in this module.

    `dim` is checked against the launch size the kernel derives from its
    inputs (n cells, plane cells or design cells), as Warp would index them."""
    expected = kernel._dim_of(*inputs)
    if int(dim) != expected:
        raise ValueError(f"{kernel.name}: launch dim {dim} != {expected} implied by inputs")
    if device is not None:
        with torch.cuda.device(torch.device(device)):
            return kernel(*inputs, stream=stream)
    return kernel(*inputs, stream=stream)


def _stream(stream):
    return stream if stream is not None else _lib.stream_handle()


def _make_update(electric, packed):
    def fn(f, g, inv_eps, psi, coeff, source, waves, step, hprev, save_h_from, nx, ny, nz,
           source_x, courant, periodic, stream=None):
        for t, nm in ((f, "f"), (g, "g"), (psi, "psi"), (source, "source"), (waves, "waves"),
                      (hprev, "hprev"), (coeff, "coeff")):
            _check(t, torch.float32, nm)
        _check(step, torch.int32, "step")
        cw = 4 if packed else 3
        if coeff.dim() != 3 or coeff.shape[0] != 3 or coeff.shape[2] != cw:
            raise ValueError(f"coeff must be (3, L, {cw}) for this kernel")
        if electric:
            _check(inv_eps, torch.float32, "inv_eps")
        _lib.call(
            "fdtd_update", int(electric), int(packed), ptr(f), ptr(g), _cols(f, 3),
            ptr(inv_eps) if inv_eps is not None else None, ptr(psi), _cols(psi, 6),
            ptr(coeff), int(coeff.shape[1]), ptr(source), _cols(source, 1), ptr(waves),
            _cols(waves, 1), ptr(step), ptr(hprev), _cols(hprev, 1), int(save_h_from),
            int(nx), int(ny), int(nz), int(source_x), float(courant), int(periodic),
            _stream(stream),
        )

    def dim_of(*a):
        return int(a[10]) * int(a[11]) * int(a[12])

    tag = ("update_e" if electric else "update_h") + ("_packed" if packed else "")
    return Kernel(tag, fn, dim_of)


# kernels.py:145-148
update_e = _make_update(True, False)
update_h = _make_update(False, False)
update_e_packed = _make_update(True, True)
update_h_packed = _make_update(False, True)


def _advance(step, stream=None):
    _lib.call("fdtd_advance", ptr(_check(step, torch.int32, "step")), 1, _stream(stream))


def _retreat(step, stream=None):
    _lib.call("fdtd_advance", ptr(_check(step, torch.int32, "step")), -1, _stream(stream))


# kernels.py:151-153 and adjoint.py:226-228
advance = Kernel("advance", _advance, lambda *a: 1)
retreat = Kernel("retreat", _retreat, lambda *a: 1)


def pack_index(full, coeff4, shape):
    """Gather a (6, n) by-cell CPML state into the reference's packed layout
    (kernels.py:50-74 index formula) given the (3, L, 4) ranked table."""
    nx, ny, nz = shape
    c = coeff4.detach().cpu()
    sizes = []
    for axis, length in enumerate(shape):
        sizes.append(int((c[axis, :length, 0] != 0).sum()) * (nx * ny * nz // length))
    out = torch.zeros((6, max(1, *sizes)), dtype=full.dtype, device=full.device)
    f = full.view(6, nx, ny, nz)
    for axis, length in enumerate(shape):
        for pos in range(length):
            if float(c[axis, pos, 0]) == 0.0:
                continue
            r = int(c[axis, pos, 3])
            for slot in (2 * axis, 2 * axis + 1):
                if axis == 0:
                    out[slot, r * ny * nz:(r + 1) * ny * nz] = f[slot, pos].reshape(-1)
                elif axis == 1:
                    out[slot, r * nx * nz:(r + 1) * nx * nz] = f[slot, :, pos].reshape(-1)
                else:
                    out[slot, r * nx * ny:(r + 1) * nx * ny] = f[slot, :, :, pos].reshape(-1)
    return out
