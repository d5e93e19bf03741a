// Shared helpers for the B200 FDTD kernels.
//
// Layout (the reference's, warp_fdtd/kernels.py:25): a field is (3, n) float32
// with n = nx*ny*nz and flat index i = (x*ny + y)*nz + z, z fastest.  Every
// kernel is built with --fmad=false so each float expression rounds exactly as
// written; operand order follows the reference source, which makes results
// bitwise comparable with the CPU oracle built with -ffp-contract=off.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/warp_fdtd_b200.h"

typedef long long i64;

namespace wfb {

// Record a CUDA error from the last launch and map it to an ABI status code.
int launch_status(const char *where);
void set_error(const char *fmt, ...);

__device__ __forceinline__ bool inside(int x, int y, int z, int nx, int ny, int nz) {
    return x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz;
}

// Flat index of (x, y, z) with z rows of `pitch` elements (pitch = nz for the
// reference layout).
__device__ __forceinline__ i64 flat(int x, int y, int z, int ny, int pitch) {
    return ((i64)x * ny + y) * pitch + z;
}

// kernels.py:8-26 `sample` (zero padding, optional periodic wrap).
__device__ __forceinline__ void sample3(const float *__restrict__ f, i64 cols, int x, int y,
                                        int z, int nx, int ny, int nz, int periodic,
                                        float out[3], int pitch = -1) {
    if (periodic) {
        x = (x + nx) % nx;
        y = (y + ny) % ny;
        z = (z + nz) % nz;
    }
    if (!inside(x, y, z, nx, ny, nz)) {
        out[0] = out[1] = out[2] = 0.0f;
        return;
    }
    i64 i = flat(x, y, z, ny, pitch < 0 ? nz : pitch);
    out[0] = f[i];
    out[1] = f[cols + i];
    out[2] = f[2 * cols + i];
}

// detectors.py:26-62 `colocate`, shared by the reference-signature recorder and
// the float64 multi-frequency recorder.
__device__ __forceinline__ void colocate(const float *__restrict__ e,
                                         const float *__restrict__ h,
                                         const float *__restrict__ prev, i64 cols, int x,
                                         int y, int z, int nx, int ny, int nz, float ec[3],
                                         float hc[3], int pitch = -1) {
    float e0[3], ex[3], ey[3], ez[3], exz[3], eyz[3];
    sample3(e, cols, x, y, z, nx, ny, nz, 0, e0, pitch);
    sample3(e, cols, x - 1, y, z, nx, ny, nz, 0, ex, pitch);
    sample3(e, cols, x, y - 1, z, nx, ny, nz, 0, ey, pitch);
    sample3(e, cols, x, y, z + 1, nx, ny, nz, 0, ez, pitch);
    sample3(e, cols, x - 1, y, z + 1, nx, ny, nz, 0, exz, pitch);
    sample3(e, cols, x, y - 1, z + 1, nx, ny, nz, 0, eyz, pitch);
    ec[0] = 0.25f * (((e0[0] + ex[0]) + ez[0]) + exz[0]);
    ec[1] = 0.25f * (((e0[1] + ey[1]) + ez[1]) + eyz[1]);
    ec[2] = e0[2];
    const int ox[8] = {0, 1, 0, 1, 0, 1, 0, 1};
    const int oy[8] = {0, 0, 1, 1, 0, 0, 1, 1};
    const int oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    float hv[8][3];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float a[3], b[3];
        sample3(h, cols, x - ox[k], y - oy[k], z + oz[k], nx, ny, nz, 0, a, pitch);
        sample3(prev, cols, x - ox[k], y - oy[k], z + oz[k], nx, ny, nz, 0, b, pitch);
#pragma unroll
        for (int c = 0; c < 3; ++c) hv[k][c] = 0.5f * (a[c] + b[c]);
    }
    // hv order: h0, hx, hy, hxy, hz, hxz, hyz, hxyz
    hc[0] = 0.5f * (hv[0][0] + hv[2][0]);
    hc[1] = 0.5f * (hv[0][1] + hv[1][1]);
    hc[2] = 0.125f * (((((((hv[0][2] + hv[1][2]) + hv[2][2]) + hv[3][2]) + hv[4][2]) +
                        hv[5][2]) +
                       hv[6][2]) +
                      hv[7][2]);
}

__device__ __forceinline__ void plane_sample(const float *__restrict__ e,
                                             const float *__restrict__ h,
                                             const float *__restrict__ prev, i64 cols, int x,
                                             int y, int z, int nx, int ny, int nz, int exact,
                                             float ee[3], float hh[3], int pitch = -1) {
    if (exact) {
        colocate(e, h, prev, cols, x, y, z, nx, ny, nz, ee, hh, pitch);
    } else {
        sample3(e, cols, x, y, z, nx, ny, nz, 0, ee, pitch);
        sample3(h, cols, x, y, z, nx, ny, nz, 0, hh, pitch);
    }
}

__device__ __forceinline__ float cross_axis(const float a[3], const float b[3], int axis) {
    if (axis == 0) return a[1] * b[2] - a[2] * b[1];
    if (axis == 1) return a[2] * b[0] - a[0] * b[2];
    return a[0] * b[1] - a[1] * b[0];
}

}  // namespace wfb
