"""The C-ABI library loads and exports every entry point include/*.h declares.

Runs on CPU: loading the shared library needs no GPU and no compute call is
made."""

import ctypes
import re

import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for header in (ROOT / "include").glob("*.h"):
        text = header.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"^\s*(?:const\s+)?(?:\w+\s+)*\w+\s*\*?\s*(fdtd_\w+)\s*\(", text,
                                flags=re.M))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from warp_fdtd_b200 import build as b

    b.build()
    return ctypes.CDLL(str(b.LIB))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "fdtd_step_fused" in names and "fdtd_update" in names
    assert len(names) >= 17


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_header():
    from warp_fdtd_b200 import _lib

    assert sorted(_lib.EXPORTS) == declared_symbols()


def test_version_and_error_string(lib):
    lib.fdtd_version.restype = ctypes.c_int
    assert lib.fdtd_version() >= 100
    lib.fdtd_last_error.restype = ctypes.c_char_p
    assert isinstance(lib.fdtd_last_error(), bytes)


def test_argument_errors_need_no_gpu(lib):
    """Invalid sizes are rejected on the host before any launch."""
    lib.fdtd_last_error.restype = ctypes.c_char_p
    rc = lib.fdtd_advance(None, 1, None)
    assert rc == -1
    assert b"null" in lib.fdtd_last_error()


def test_new_entry_points_reject_bad_arguments(lib):
    """Batches, grouped staging, the volume recorder and the launch-shape
    queries check their arguments on the host."""
    from warp_fdtd_b200 import _lib

    L = _lib.load()
    assert L.fdtd_batch_workspace_bytes(0) == 0
    assert L.fdtd_batch_workspace_bytes(3) > 0
    plan = _lib.BatchPlan()
    assert L.fdtd_batch_prepare(None, 0, None, 0, ctypes.byref(plan)) == -1
    assert L.fdtd_step_batch(ctypes.byref(plan), None, None, 0, None) == -1
    assert L.fdtd_batch_release(ctypes.byref(plan)) == -1
    assert L.fdtd_advance_many(None, 0, 1, None) == -1
    assert L.fdtd_record_stage_many(None, None, None, None, None, None, 0, 8, 8, 8, 8, None, 0,
                                    None) == -1
    assert L.fdtd_record_volume(None, None, None, None, None, None, 0, None, 1, 0, None, 4, 4, 4,
                                4, None) == -1
    a = _lib.StepArgs()
    assert L.fdtd_step_defaults(ctypes.byref(a)) == -1
    blocks, sms = ctypes.c_int(), ctypes.c_int()
    assert L.fdtd_step_occupancy(ctypes.byref(a), ctypes.byref(blocks), ctypes.byref(sms)) == -1
    assert b"full-z" in L.fdtd_last_error()


def test_surrogate_and_reverse_entry_points_reject_bad_arguments(lib):
    """The surrogate's GEMM and layer kernels and the fused reverse halves
    check their arguments on the host, before any launch."""
    from warp_fdtd_b200 import _lib

    L = _lib.load()
    g = _lib.SgGemmArgs()
    assert L.fdtd_sg_gemm(ctypes.byref(g), None) == -1  # null operands
    g.A, g.B, g.C = 16, 32, 48
    g.M, g.N, g.K, g.lda, g.ldb, g.ldc = 128, 32, 64, 64, 64, 32
    g.lda = 60  # not a multiple of 8
    assert L.fdtd_sg_gemm(ctypes.byref(g), None) == -1
    g.lda, g.A = 64, 17  # misaligned A
    assert L.fdtd_sg_gemm(ctypes.byref(g), None) == -1
    g.A, g.K, g.lda, g.ldb = 16, 1000, 1000, 1000
    g.splits, g.relu = 4, 1  # split K (16 chunks of 64) with an epilogue
    assert L.fdtd_sg_gemm(ctypes.byref(g), None) == -1
    g.relu, g.splits, g.layout = 0, 1, 2  # unknown operand layout
    assert L.fdtd_sg_gemm(ctypes.byref(g), None) == -1
    assert b"layout" in L.fdtd_last_error()
    g.splits = 37  # more than the 16 chunks of 64
    assert L.fdtd_sg_gemm_splits(ctypes.byref(g)) == 16
    g.splits = 5
    assert L.fdtd_sg_gemm_splits(ctypes.byref(g)) == 4  # 4 chunks each
    assert L.fdtd_sg_im2col(None, 1, 1, 4, 4, 1, None, 16, None) == -1
    assert L.fdtd_sg_im2col(16, 1, 1, 4, 4, 1, 32, 8, None) == -1  # ldcol < 9 C
    assert L.fdtd_sg_pool(16, 8, 1, 5, 4, 8, 32, 8, None) == -1  # odd H
    assert L.fdtd_sg_transpose(16, 4, 8, 8, 32, 4, None) == -1  # lds < cols
    assert L.fdtd_sg_splitk_reduce(16, 2, 10, 4, 4, 4, 32, 4, 0, None) == -1  # stride
    assert L.fdtd_sg_adam(16, 16, 16, 16, 10, 1e-3, 0.9, 0.999, 1e-8, 0, None) == -1
    # fused reverse halves
    assert L.fdtd_reverse_half(1, None, None, None, None, None, None, 8, None, None, None,
                               None, 4, 4, 4, 0.5, 0, 0, 0, 0, 0, 0, None) == -1
    assert L.fdtd_reverse_half(0, 16, 32, 48, 64, 64, 96, 8, 112, None, None, None, 4, 4, 4,
                               0.5, 0, 0, 0, 0, 0, 0, None) == -1  # psi0 == psi1
    assert L.fdtd_reverse_half(0, 16, 32, 48, 64, 80, 100, 8, 112, None, None, None, 4, 4, 4,
                               0.5, 0, 0, 0, 0, 0, 0, None) == -1  # misaligned table
    assert L.fdtd_reverse_half(0, 16, 32, 48, 64, 80, 96, 3, 112, None, None, None, 4, 4, 4,
                               0.5, 0, 0, 0, 0, 0, 0, None) == -1  # clen < max dim
    assert L.fdtd_reverse_half(0, 16, 32, None, 64, 80, 96, 8, 112, None, None, None, 4, 4, 4,
                               0.5, 0, 0, 0, 0, 0, 0, None) == -1  # electric half needs eps
    assert L.fdtd_reverse_half(1, 16, 32, 48, 64, 80, 96, 8, 112, 128, 144, 160, 4, 4, 4, 0.5,
                               2, 0, 0, 4, 4, 4, None) == -1  # design box outside the grid


def test_inject_many_and_block_step_reject_bad_arguments(lib):
    """fdtd_inject_many and the time-blocked step check their arguments on
    the host, before any launch."""
    from warp_fdtd_b200 import _lib

    L = _lib.load()
    planes = (_lib.InjectPlane * 9)()
    for pl in planes:
        pl.source, pl.weights, pl.sx, pl.sy, pl.sz = 16, 32, 1, 2, 2
    args = (16, 32)
    assert L.fdtd_inject_many(*args, planes, 9, 48, 4, 4, 4, 0, None) == -1  # > 8 planes
    assert L.fdtd_inject_many(*args, planes, 0, 48, 4, 4, 4, 0, None) == -1  # no plane
    planes[1].source = None
    assert L.fdtd_inject_many(*args, planes, 2, 48, 4, 4, 4, 0, None) == -1  # null source
    assert b"plane 1" in L.fdtd_last_error()
    planes[1].source, planes[1].sy = 16, 0
    assert L.fdtd_inject_many(*args, planes, 2, 48, 4, 4, 4, 0, None) == -1  # empty extent
    assert L.fdtd_inject_many(None, 32, planes, 1, 48, 4, 4, 4, 0, None) == -1  # null field
    a = _lib.StepArgs()
    plan = _lib.BlockPlan()
    assert L.fdtd_step_block_prepare(ctypes.byref(a), 3, ctypes.byref(plan)) == -1  # depth 3
    assert L.fdtd_step_block_prepare(None, 2, ctypes.byref(plan)) == -1
    assert L.fdtd_step_block_prepare(ctypes.byref(a), 2, ctypes.byref(plan)) == -1  # empty grid
    assert L.fdtd_step_block(ctypes.byref(a), None, None, None) == -1
    plan.depth = 2
    assert L.fdtd_step_block(ctypes.byref(a), ctypes.byref(plan), None, None) == -1


def test_pair_staging_rejects_bad_arguments(lib):
    """fdtd_record_stage_pair checks its fields, planes and counter on the
    host, before any launch (odd T would let a fold fall inside the pair)."""
    from warp_fdtd_b200 import _lib

    L = _lib.load()
    fields = (ctypes.c_void_p * 8)(*([16] * 8))
    planes = (_lib.StagePlane * 1)()
    pl = planes[0]
    pl.indices, pl.stage, pl.nsteps, pl.T = 16, 32, 10, 4
    pl.sx, pl.sy, pl.sz = 1, 4, 4
    step, counter = 64, 80
    call = lambda f, n, c: L.fdtd_record_stage_pair(f, step, planes, n, 4, 4, 4, 4, c, None)  # noqa
    assert call(fields, 0, counter) == -1  # no plane
    assert call(fields, 9, counter) == -1  # more than eight
    assert call(fields, 1, None) == -1  # no completion counter
    fields[5] = None
    assert call(fields, 1, counter) == -1 and b"null field pointer 5" in L.fdtd_last_error()
    fields[5] = 16
    pl.T = 1
    assert call(fields, 1, counter) == -1 and b"T >= 2" in L.fdtd_last_error()
