"""ctypes binding of the CPU oracle library (oracle/fdtd_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg as the checker.  The product never imports it.
"""

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "build" / "liboracle.so"

_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64 = ctypes.c_longlong
_int = ctypes.c_int

LIB64_PATH = HERE / "build" / "liboracle64.so"

_libs = {}


def build():
    """Compile the oracle with its Makefile (gcc, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)


def lib(f64=False):
    """The float32 restatement, or with f64 the same compiled in double
    (every float argument then float64 / c_double)."""
    if f64 not in _libs:
        path = LIB64_PATH if f64 else LIB_PATH
        if not path.exists():
            build()
        _libs[f64] = _load(path, f64)
    return _libs[f64]


def _load(path, f64):
    _rp = np.ctypeslib.ndpointer(np.float64 if f64 else np.float32, flags="C_CONTIGUOUS")
    _rs = ctypes.c_double if f64 else ctypes.c_float
    L = ctypes.CDLL(str(path))
    L.oracle_update.argtypes = [
        _int, _int, _rp, _rp, _i64, _rp, _rp, _i64, _rp, _int,
        _rp, _i64, _rp, _i64, _i32p, _rp, _i64, _int, _int, _int, _int,
        _int, _rs, _int,
    ]
    L.oracle_record_phasor.argtypes = [
        _rp, _rp, _rp, _i64, _int, _rp, _int, _i64, _f64p,
        _int, _int, _int, _int, _int, _int, _int, _int, _int, _int,
    ]
    L.oracle_record_phasor_f32.argtypes = [
        _rp, _rp, _rp, _i64, _int, _rp, _rp,
        _int, _int, _int, _int, _int, _int, _int, _int, _int, _int,
    ]
    L.oracle_flux_sum.argtypes = [
        _rp, _rp, _rp, _i64, _rp, _int, _int, _int, _int, _int, _int,
        _int, _int, _int, _int, _int,
    ]
    L.oracle_flux_sum.restype = ctypes.c_double
    L.oracle_record_curl.argtypes = [
        _rp, _i64, _rp, _i64, _int, _int, _int, _int, _int, _int, _int,
        _int, _int, _int, _rs,
    ]
    L.oracle_prepare.argtypes = [
        _rp, _rp, _rp, _rp, _int, _rp, _int, _int, _int, _rs, _int,
    ]
    L.oracle_gather.argtypes = [
        _rp, _rp, _rp, _i64, ctypes.c_void_p, _int, _int, _int, _int, _int,
        _int, _int, _int, _int, _int, _int, _int,
    ]
    L.oracle_inject.argtypes = [
        _rp, _rp, _rp, _rp, _int, _int, _int, _int, _int, _int, _int,
        _int, _int, _int, _int,
    ]
    L.oracle_write_design.argtypes = [
        _rp, _rp, _int, _int, _int, _int, _int, _int, _int, _int, _int,
    ]
    L.oracle_run_steps.argtypes = [
        _rp, _rp, _rp, _rp, _rp, _rp, _rp, _int, _rp, _rp,
        _rp, _rp, _i64, _int, _int, _int, _int, _int, _int, _rs,
    ]
    L.oracle_num_threads.restype = _int
    return L


def f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def update(electric, f, g, inv_eps, psi, coeff, source, waves, step, hprev,
           save_h_from, shape, source_x, courant, periodic=0):
    """kernels.py:77-142 on host arrays; f, psi, hprev are updated in place.

    Arrays must already be C-contiguous float32 (int32 for step)."""
    nx, ny, nz = shape
    packed = int(coeff.shape[-1] == 4)
    lib(f.dtype == np.float64).oracle_update(
        int(electric), packed, f, g, f.shape[1], inv_eps, psi, psi.shape[1],
        coeff, coeff.shape[1], source, source.shape[1], waves, waves.shape[1],
        step, hprev, hprev.shape[1], int(save_h_from), nx, ny, nz, int(source_x),
        float(courant), int(periodic),
    )


def prepare(q, eps, psi, coeff, d, shape, courant, electric):
    nx, ny, nz = shape
    lib().oracle_prepare(q, eps, psi, coeff, coeff.shape[1], d, nx, ny, nz,
                         float(courant), int(electric))


def gather(q, d, hist, grad, t, shape, box, from_h):
    nx, ny, nz = shape
    design_n = hist.shape[2]
    is64 = int(grad.dtype == np.float64)
    lib().oracle_gather(q, d, hist, design_n, grad.ctypes.data, is64, int(t), nx, ny,
                        nz, *box, int(from_h))


def inject(qe, qh, source, weights, t, shape, lo, plane_shape, old_h_only):
    nx, ny, nz = shape
    lib().oracle_inject(qe, qh, source, weights, int(t), nx, ny, nz, *lo,
                        *plane_shape, int(old_h_only))


def record_curl(h, hist, t, shape, box, courant):
    nx, ny, nz = shape
    lib().oracle_record_curl(h, h.shape[1], hist, hist.shape[2], int(t), nx, ny, nz,
                             *box, float(courant))


def num_threads():
    return int(lib().oracle_num_threads())
