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
