"""warp_fdtd_b200: the uniform-grid 3-D FDTD path of warp-fdtd, B200-native.

Modules mirror the reference package warp_fdtd: solver (Solver,
pack_coefficients, owned_array_bytes), kernels (kernel-level launchables),
detectors (Monitor, attach, measurements, record), adjoint (Adjoint and the
adjoint kernels), material (Material).  All compute runs in the CUDA library
libwarp_fdtd_b200.so through the C ABI in include/warp_fdtd_b200.h.
"""

__version__ = "0.1.0"
