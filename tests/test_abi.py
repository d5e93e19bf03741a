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
        names.update(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(fdtd_\w+)\s*\(", text, flags=re.M))
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
