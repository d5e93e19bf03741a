"""NumPy restatement of the reference's volume phasor observer
(warp_fdtd/volume.py:24-89: trilinear, offset, record_volume).

TEST INFRASTRUCTURE ONLY (checker for warp_fdtd_b200.volume and
fdtd_record_volume).  The sampled value follows the reference's float32
operation order; the accumulation is float64, as in the CUDA recorder."""

import numpy as np

F = np.float32
# Yee offsets of Ex, Ey, Ez, Hx, Hy, Hz (volume.py:44-57)
OFFSETS = np.array([[0.5, 0, 0], [0, 0.5, 0], [0, 0, 0.5], [0, 0.5, 0.5], [0.5, 0, 0.5],
                    [0.5, 0.5, 0]], np.float32)


def trilinear(f, comp, p, shape):
    """volume.py:24-41 for one point p (float32 vec3); f is (3, n)."""
    nx, ny, nz = shape
    ix, iy, iz = (int(np.floor(v)) for v in p)
    tx, ty, tz = F(p[0] - F(ix)), F(p[1] - F(iy)), F(p[2] - F(iz))
    value = F(0)
    for a in range(2):
        for b in range(2):
            for c in range(2):
                x, y, z = ix + a, iy + b, iz + c
                if 0 <= x < nx and 0 <= y < ny and 0 <= z < nz:
                    w = F(F((tx if a else F(F(1) - tx)) * (ty if b else F(F(1) - ty)))
                          * (tz if c else F(F(1) - tz)))
                    value = F(value + F(w * f[comp, (x * ny + y) * nz + z]))
    return value


def record_volume(e, h, prev, positions, weights, t, phasor, shape, first):
    """volume.py:60-89: phasor (6, n) complex128 += weights[t] * sample."""
    if t < first:
        return
    w = weights[t]
    for i, pos in enumerate(np.asarray(positions, np.float32)):
        for c in range(6):
            p = (pos - OFFSETS[c]).astype(np.float32)
            if c < 3:
                value = trilinear(e, c, p, shape)
            else:
                value = F(F(0.5) * F(trilinear(h, c - 3, p, shape) + trilinear(prev, c - 3, p, shape)))
            phasor[c, i] += complex(float(w[0]) * float(value), float(w[1]) * float(value))
