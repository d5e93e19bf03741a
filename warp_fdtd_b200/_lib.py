"""ctypes binding of libwarp_fdtd_b200.so (the C ABI in include/warp_fdtd_b200.h).

The library is the only compute path: if it is missing or fails to load, every
entry point raises; nothing falls back to the CPU.
"""

import ctypes
from pathlib import Path

import torch

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libwarp_fdtd_b200.so"

FDTD_OK = 0
FDTD_ERR_ARG = -1
FDTD_ERR_CUDA = -2

_p = ctypes.c_void_p
_i = ctypes.c_int
_ll = ctypes.c_longlong
_f = ctypes.c_float


class StepArgs(ctypes.Structure):
    """Mirror of `fdtd_step_args`."""

    _fields_ = [
        ("E", _p * 2),
        ("H", _p * 2),
        ("psi_e", _p * 2),
        ("psi_h", _p * 2),
        ("psi_cols", _ll),
        ("coeff_e", _p),
        ("coeff_h", _p),
        ("clen", _i),
        ("packed", _i),
        ("psi_rx", _i),
        ("psi_ry", _i),
        ("psi_rz", _i),
        ("material_kind", _i),
        ("inv_eps", _p),
        ("material", _p),
        ("material_table", _p),
        ("material_count", _i),
        ("src_e", _p),
        ("src_h", _p),
        ("waves_e", _p),
        ("waves_h", _p),
        ("waves_cols", _ll),
        ("source_x", _i),
        ("courant", _f),
        ("step", _p),
        ("nx", _i),
        ("ny", _i),
        ("nz", _i),
        ("pitch_z", _i),
        ("material_pitch", _i),
        ("tile_y", _i),
        ("tile_z", _i),
        ("chunk_x", _i),
        ("path", _i),
        ("vector", _i),
        ("stages", _i),
        ("error", _p),
        ("schedule", _p),
        ("schedule_blocks", _i),
    ]


class StagePlane(ctypes.Structure):
    """Mirror of `fdtd_stage_plane`."""

    _fields_ = [("indices", _p), ("stage", _p)] + [
        (name, _i) for name in ("nsteps", "T", "x0", "y0", "z0", "sx", "sy", "sz", "exact")]


class BatchPlan(ctypes.Structure):
    """Mirror of `fdtd_batch_plan`."""

    _fields_ = [(name, _i) for name in ("count", "smem_bytes", "threads", "material_kind",
                                        "stages", "vector", "full_rows", "base", "device")]


BLOCK_GROUPS_MAX = 64
SNAP_BOXES_MAX = 8


class BlockPlan(ctypes.Structure):
    """Mirror of `fdtd_block_plan`."""

    _fields_ = ([(name, _i) for name in ("depth", "tile_y", "stages", "rows", "threads",
                                         "groups_plain", "groups_slab")]
                + [("group", ctypes.c_ubyte * BLOCK_GROUPS_MAX), ("scratch_block_bytes", _ll)]
                + [(name, _i) for name in ("pair_blocks", "device", "blocks_per_sm", "sms")])


class BlockExtra(ctypes.Structure):
    """Mirror of `fdtd_block_extra`."""

    _fields_ = [("scratch", _p), ("scratch_bytes", _ll), ("snap_e", _p), ("snap_h", _p),
                ("segments", _i), ("nsnap", _i), ("snap_box", (_i * 6) * SNAP_BOXES_MAX),
                ("interior_blocks", _i)]


class InjectPlane(ctypes.Structure):
    """Mirror of `fdtd_inject_plane`."""

    _fields_ = [("source", _p), ("weights", _p)] + [
        (name, _i) for name in ("x0", "y0", "z0", "sx", "sy", "sz")]


class SgGemmArgs(ctypes.Structure):
    """Mirror of `fdtd_sg_gemm_args`."""

    _fields_ = [("A", _p), ("lda", _i), ("B", _p), ("ldb", _i), ("C", _p), ("ldc", _i),
                ("c_bf16", _i), ("bias", _p), ("M", _i), ("N", _i), ("K", _i), ("splits", _i),
                ("split_stride", _ll), ("accumulate", _i), ("relu", _i), ("layout", _i)]


# name -> argtypes (all return int status)
_SIGNATURES = {
    "fdtd_update": [_i, _i, _p, _p, _ll, _p, _p, _ll, _p, _i, _p, _ll, _p, _ll, _p, _p, _ll,
                    _i, _i, _i, _i, _i, _f, _i, _p],
    "fdtd_advance": [_p, _i, _p],
    "fdtd_step_occupancy": [ctypes.POINTER(StepArgs), _p, _p],
    "fdtd_step_defaults": [ctypes.POINTER(StepArgs)],
    "fdtd_batch_prepare": [ctypes.POINTER(StepArgs), _i, _p, _ll, ctypes.POINTER(BatchPlan)],
    "fdtd_step_batch": [ctypes.POINTER(BatchPlan), _p, _p, _i, _p],
    "fdtd_advance_many": [_p, _i, _i, _p],
    "fdtd_batch_release": [ctypes.POINTER(BatchPlan)],
    "fdtd_record_stage_many": [_p, _p, _p, _p, _p, ctypes.POINTER(StagePlane), _i, _i, _i, _i,
                               _i, _p, _i, _p],
    "fdtd_record_stage_pair": [_p, _p, ctypes.POINTER(StagePlane), _i, _i, _i, _i, _i, _p, _p],
    "fdtd_record_volume": [_p, _p, _p, _p, _p, _p, _ll, _p, _i, _i, _p, _i, _i, _i, _i, _p],
    "fdtd_record": [_p, _p, _p, _ll, _p, _p, _p, _p, _p, _p, _i, _i, _i, _i, _i, _i, _i, _i,
                    _i, _i, _i, _i, _p],
    "fdtd_record_curl": [_p, _ll, _p, _p, _i, _i, _i, _i, _i, _i, _i, _i, _i, _f, _p],
    "fdtd_record_curl_pp": [_p, _p, _i, _p, _p, _p, _i, _i, _i, _i, _i, _i, _i, _i, _i, _f, _p],
    "fdtd_prepare": [_p, _p, _p, _p, _i, _p, _i, _i, _i, _f, _i, _p],
    "fdtd_gather": [_p, _p, _p, _p, _i, _p, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _p],
    "fdtd_inject": [_p, _p, _p, _p, _p, _i, _i, _i, _i, _i, _i, _i, _i, _i, _i, _p],
    "fdtd_write_design": [_p, _p, _i, _i, _i, _i, _i, _i, _i, _i, _i, _p],
    "fdtd_material_smooth": [_p, _p, _i, _p, _i, _i, _p],
    "fdtd_material_smooth_adjoint": [_p, _p, _i, _p, _i, _i, _p],
    "fdtd_material_subpixel": [_p, _p, _i, _i, _f, _f, _f, _p],
    "fdtd_material_subpixel_adjoint": [_p, _p, _p, _i, _i, _f, _f, _f, _p],
    "fdtd_material_forward": [_p, _p, _i, _p, _p, _i, _i, _f, _f, _f, _p],
    "fdtd_material_forward_noalloc": [_p, _p, _i, _p, _i, _i, _f, _f, _f, _p],
    "fdtd_material_backward": [_p, _p, _i, _p, _p, _p, _i, _i, _f, _f, _f, _p],
    "fdtd_step_fused": [ctypes.POINTER(StepArgs), _p],
    "fdtd_step_block_prepare": [ctypes.POINTER(StepArgs), _i, ctypes.POINTER(BlockPlan)],
    "fdtd_step_block": [ctypes.POINTER(StepArgs), ctypes.POINTER(BlockPlan),
                        ctypes.POINTER(BlockExtra), _p],
    "fdtd_record_phasor64": [_p, _p, _p, _p, _p, _p, _i, _p, _i, _p, _i, _i, _i, _i, _i, _i,
                             _i, _i, _i, _i, _i, _p],
    "fdtd_record_stage": [_p, _p, _p, _p, _p, _p, _i, _p, _i, _i, _i, _i, _i, _i, _i, _i, _i,
                          _i, _i, _i, _p],
    "fdtd_dft_fold": [_p, _p, _i, _p, _i, _p, _i, _p, _ll, _p],
    "fdtd_inject_many": [_p, _p, ctypes.POINTER(InjectPlane), _i, _p, _i, _i, _i, _i, _p],
    "fdtd_reverse_half": [_i, _p, _p, _p, _p, _p, _p, _i, _p, _p, _p, _p, _i, _i, _i, _f, _i,
                          _i, _i, _i, _i, _i, _p],
    "fdtd_sg_gemm": [ctypes.POINTER(SgGemmArgs), _p],
    "fdtd_sg_gemm_splits": [ctypes.POINTER(SgGemmArgs)],
    "fdtd_sg_status": [ctypes.POINTER(_i), _i],
    "fdtd_sg_im2col": [_p, _i, _i, _i, _i, _i, _p, _i, _p],
    "fdtd_sg_transpose": [_p, _i, _ll, _i, _p, _ll, _p],
    "fdtd_sg_col2im": [_p, _i, _i, _i, _i, _i, _p, _i, _i, _p],
    "fdtd_sg_relu_backward": [_p, _i, _p, _i, _ll, _i, _p, _i, _p, _p, _p],
    "fdtd_sg_pool": [_p, _i, _i, _i, _i, _i, _p, _i, _p],
    "fdtd_sg_pool_backward": [_p, _i, _i, _i, _i, _i, _p, _i, _i, _p],
    "fdtd_sg_upsample": [_p, _i, _i, _i, _i, _i, _p, _i, _p],
    "fdtd_sg_upsample_backward": [_p, _i, _i, _i, _i, _i, _p, _i, _i, _p],
    "fdtd_sg_gap_linear": [_p, _i, _i, _i, _i, _p, _p, _i, _p, _p, _p],
    "fdtd_sg_gap_linear_backward": [_p, _p, _p, _i, _i, _i, _i, _p, _p, _p, _i, _i, _p],
    "fdtd_sg_head": [_p, _i, _ll, _i, _p, _p, _p, _p],
    "fdtd_sg_head_backward": [_p, _p, _i, _ll, _i, _p, _p, _i, _p, _p, _p, _p],
    "fdtd_sg_mse": [_p, _p, _ll, _f, _p, _p, _p],
    "fdtd_sg_adam": [_p, _p, _p, _p, _ll, _f, _f, _f, _f, _i, _p],
    "fdtd_sg_cast_weights": [_p, _i, _i, _p, _i, _p, _p],
    "fdtd_sg_splitk_reduce": [_p, _i, _ll, _i, _i, _i, _p, _i, _i, _p],
    "fdtd_sg_to_bf16": [_p, _p, _ll, _p],
    "fdtd_record_flux64": [_p, _p, _p, _p, _p, _p, _i, _p, _p, _i, _i, _i, _i, _i, _i, _i, _i,
                           _i, _i, _i, _i, _i, _p],
}

EXPORTS = sorted(_SIGNATURES) + ["fdtd_batch_workspace_bytes", "fdtd_last_error",
                                 "fdtd_version"]

_lib = None


class FdtdError(RuntimeError):
    pass


def load():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FdtdError(
                f"{LIB_PATH.name} is not built; run `python -m warp_fdtd_b200.build`"
            )
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, argtypes in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = argtypes
            fn.restype = _i
        lib.fdtd_last_error.restype = ctypes.c_char_p
        lib.fdtd_last_error.argtypes = []
        lib.fdtd_version.restype = _i
        lib.fdtd_batch_workspace_bytes.argtypes = [_i]
        lib.fdtd_batch_workspace_bytes.restype = _ll
        _lib = lib
    return _lib


def call(name, *args):
    """Call an entry point and raise on a non-zero status."""
    lib = load()
    status = getattr(lib, name)(*args)
    if status != FDTD_OK:
        msg = lib.fdtd_last_error().decode(errors="replace")
        if status == FDTD_ERR_ARG:
            raise ValueError(msg)
        raise FdtdError(msg)
    return status


def ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    if t is None:
        return None
    if not isinstance(t, torch.Tensor):
        raise TypeError(f"expected a torch.Tensor, got {type(t).__name__}")
    if t.device.type != "cuda":
        raise ValueError("warp_fdtd_b200 kernels take CUDA tensors only")
    if not t.is_contiguous():
        raise ValueError("warp_fdtd_b200 kernels take contiguous tensors only")
    return t.data_ptr()


def stream_handle(device=None):
    return torch.cuda.current_stream(device).cuda_stream
