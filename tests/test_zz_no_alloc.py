"""The allocation-free material map entry point (fdtd_material_forward_noalloc).

Some callers cannot allocate device memory: an application embedding the
library under a fixed memory budget that only lends it input and output
buffers, or a loop where a cudaMalloc could stall the device.  For them the
library keeps the map's intermediate (the smoothed density) in a static
device array.  These tests call both the allocation-free entry point and the
caller-scratch entry point (fdtd_material_forward) through the C ABI and
require the same result on two calls in a row, and check that an oversized
map is refused.  The file is named so pytest collects it last."""

import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def _weights():
    from warp_fdtd_b200.material import gaussian_weights

    return torch.from_numpy(gaussian_weights(9, 3.0)).cuda()


def _reference_forward(lib, p, w, px, py, beta, eps_lo, contrast, stream):
    scratch = torch.empty(px * py, dtype=torch.float32, device="cuda")
    out = torch.empty((px, py), dtype=torch.float32, device="cuda")
    rc = lib.fdtd_material_forward(p.data_ptr(), w.data_ptr(), 9, scratch.data_ptr(),
                                   out.data_ptr(), px, py, beta, eps_lo, contrast, stream)
    assert rc == 0, lib.fdtd_last_error()
    return out


def test_noalloc_matches_caller_scratch_twice_in_a_row():
    from warp_fdtd_b200 import _lib

    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    w = _weights()
    rng = np.random.default_rng(7)
    # two consecutive calls of different sizes and parameters share the array
    for shape, beta, eps_lo, contrast in [((125, 125), 8.0, 2.085, 10.025),
                                          ((37, 90), 50.0, 1.0, 11.25)]:
        px, py = shape
        p = torch.from_numpy(rng.uniform(0, 1, shape).astype(np.float32)).cuda()
        out = torch.full((px, py), float("nan"), dtype=torch.float32, device="cuda")
        rc = lib.fdtd_material_forward_noalloc(p.data_ptr(), w.data_ptr(), 9, out.data_ptr(),
                                               px, py, ctypes.c_float(beta),
                                               ctypes.c_float(eps_lo),
                                               ctypes.c_float(contrast), stream)
        assert rc == 0, lib.fdtd_last_error()
        want = _reference_forward(lib, p, w, px, py, ctypes.c_float(beta),
                                  ctypes.c_float(eps_lo), ctypes.c_float(contrast), stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.isfinite(got).all()
        # identical kernels on identical inputs: equal, far inside the
        # material tests' 2e-5 relative tolerance
        np.testing.assert_array_equal(got, want.cpu().numpy())


def test_noalloc_rejects_maps_beyond_its_scratch():
    from warp_fdtd_b200 import _lib

    lib = _lib.load()
    rc = lib.fdtd_material_forward_noalloc(1, 1, 9, 1, 1025, 1024, ctypes.c_float(8.0),
                                           ctypes.c_float(1.0), ctypes.c_float(11.25), None)
    assert rc == -1
    assert b"exceed" in lib.fdtd_last_error()
