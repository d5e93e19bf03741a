// Kernel-level replacements of the reference's Warp kernels (group 1 of the
// C ABI).  One thread per cell (or per plane / design cell), the same
// arguments and in-place semantics as the Warp launches they replace, so the
// reference's own kernel-level tests (tests/test_adjoint.py, test_packed.py)
// can drive them directly.  The Solver's forward path uses step_fused.cu.
#include <stdarg.h>
#include <stdio.h>

#include "common.cuh"

namespace wfb {

static thread_local char g_error[512] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

int launch_status(const char *where) {
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        set_error("%s: %s", where, cudaGetErrorString(err));
        return FDTD_ERR_CUDA;
    }
    return FDTD_OK;
}

static inline unsigned blocks_for(i64 n, int threads) {
    return (unsigned)((n + threads - 1) / threads);
}

// kernels.py:29-74 `cpml` / `cpml_packed`.
template <bool PACKED>
__device__ __forceinline__ float cpml(float d, float *__restrict__ psi, i64 psi_cols,
                                      const float *__restrict__ coeff, int clen, int axis,
                                      int position, int slot, i64 i, int nx, int ny, int nz) {
    constexpr int CW = PACKED ? 4 : 3;
    const float *c = coeff + ((i64)axis * clen + position) * CW;
    float a = c[0];
    if (a != 0.0f) {
        i64 index = i;
        if (PACKED) {
            i64 plane = (i64)(int)c[3];
            i64 nyz = (i64)ny * nz;
            index = plane * nyz + i % nyz;
            if (axis == 1)
                index = plane * nx * nz + (i / nyz) * nz + i % nz;
            else if (axis == 2)
                index = plane * nx * ny + i / nz;
        }
        float *ps = psi + (i64)slot * psi_cols + index;
        float p = c[1] * (*ps) + a * d;
        *ps = p;
        return c[2] * d + p;
    }
    return c[2] * d;
}

// kernels.py:77-142 `make_update(electric, packed)`.
template <bool ELECTRIC, bool PACKED>
__global__ void update_kernel(float *__restrict__ f, const float *__restrict__ g, i64 fg_cols,
                              const float *__restrict__ inv_eps, float *__restrict__ psi,
                              i64 psi_cols, const float *__restrict__ coeff, int clen,
                              const float *__restrict__ source, i64 source_cols,
                              const float *__restrict__ waves, i64 waves_cols,
                              const int *__restrict__ step, float *__restrict__ hprev,
                              i64 hprev_cols, int save_h_from, int nx, int ny, int nz,
                              int source_x, float courant, int periodic) {
    const i64 n = (i64)nx * ny * nz;
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int z = (int)(i % nz);
    int y = (int)((i / nz) % ny);
    int x = (int)(i / ((i64)ny * nz));
    float v[3], a[3], b[3], c[3], dx[3], dy[3], dz[3];
    sample3(g, fg_cols, x, y, z, nx, ny, nz, periodic, v);
    if (ELECTRIC) {
        sample3(g, fg_cols, x - 1, y, z, nx, ny, nz, periodic, a);
        sample3(g, fg_cols, x, y - 1, z, nx, ny, nz, periodic, b);
        sample3(g, fg_cols, x, y, z - 1, nx, ny, nz, periodic, c);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            dx[k] = v[k] - a[k];
            dy[k] = v[k] - b[k];
            dz[k] = v[k] - c[k];
        }
    } else {
        sample3(g, fg_cols, x + 1, y, z, nx, ny, nz, periodic, a);
        sample3(g, fg_cols, x, y + 1, z, nx, ny, nz, periodic, b);
        sample3(g, fg_cols, x, y, z + 1, nx, ny, nz, periodic, c);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            dx[k] = a[k] - v[k];
            dy[k] = b[k] - v[k];
            dz[k] = c[k] - v[k];
        }
    }
    float dxz = cpml<PACKED>(dx[2], psi, psi_cols, coeff, clen, 0, x, 0, i, nx, ny, nz);
    float dxy = cpml<PACKED>(dx[1], psi, psi_cols, coeff, clen, 0, x, 1, i, nx, ny, nz);
    float dyx = cpml<PACKED>(dy[0], psi, psi_cols, coeff, clen, 1, y, 2, i, nx, ny, nz);
    float dyz = cpml<PACKED>(dy[2], psi, psi_cols, coeff, clen, 1, y, 3, i, nx, ny, nz);
    float dzy = cpml<PACKED>(dz[1], psi, psi_cols, coeff, clen, 2, z, 4, i, nx, ny, nz);
    float dzx = cpml<PACKED>(dz[0], psi, psi_cols, coeff, clen, 2, z, 5, i, nx, ny, nz);
    float curl[3] = {dyz - dzy, dzx - dxz, dxy - dyx};
    float old[3] = {f[i], f[fg_cols + i], f[2 * fg_cols + i]};
    float value[3];
    const int t = step[0];
    if (ELECTRIC) {
        const float ie = inv_eps[i];
#pragma unroll
        for (int k = 0; k < 3; ++k) value[k] = old[k] + (courant * curl[k]) * ie;
        if (x == source_x) {
            i64 s = (i64)y * nz + z;
            value[1] = value[1] + ((source[2 * source_cols + s] * waves[2 * waves_cols + t]) * courant) * ie;
            value[2] = value[2] - ((source[source_cols + s] * waves[waves_cols + t]) * courant) * ie;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) value[k] = old[k] - courant * curl[k];
        if (t >= save_h_from) {
            hprev[i] = old[0];
            hprev[hprev_cols + i] = old[1];
            hprev[2 * hprev_cols + i] = old[2];
        }
        if (x == source_x) {
            i64 s = (i64)y * nz + z;
            value[1] = value[1] - (source[2 * source_cols + s] * waves[2 * waves_cols + t]) * courant;
            value[2] = value[2] + (source[source_cols + s] * waves[waves_cols + t]) * courant;
        }
    }
    f[i] = value[0];
    f[fg_cols + i] = value[1];
    f[2 * fg_cols + i] = value[2];
}

__global__ void advance_kernel(int *step, int delta) { step[0] += delta; }

// The step counters of many grids, one thread each.
__global__ void advance_many_kernel(int *const *steps, int count, int delta) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) steps[i][0] += delta;
}

// detectors.py:65-106 `record` (float32 phasor, float32 atomic flux).
__global__ void record_kernel(const float *__restrict__ e, const float *__restrict__ h,
                              const float *__restrict__ prev, i64 cols,
                              const int *__restrict__ step, const float2 *__restrict__ weights,
                              const int *__restrict__ indices, float2 *__restrict__ phasor,
                              float *__restrict__ flux, const float *__restrict__ area,
                              int nx, int ny, int nz, int x0, int y0, int z0, int sx, int sy,
                              int sz, int axis, int exact, int is_phasor) {
    const i64 count = (i64)sx * sy * sz;
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int t = step[0];
    const int index = indices[t];
    if (index < 0) return;
    int x = x0 + (int)(i / ((i64)sy * sz));
    int y = y0 + (int)((i / sz) % sy);
    int z = z0 + (int)(i % sz);
    float ee[3], hh[3];
    plane_sample(e, h, prev, cols, x, y, z, nx, ny, nz, exact, ee, hh);
    if (is_phasor) {
        float2 w = weights[t];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            float2 p = phasor[(i64)c * count + i];
            p.x = p.x + w.x * ee[c];
            p.y = p.y + w.y * ee[c];
            phasor[(i64)c * count + i] = p;
            float2 q = phasor[(i64)(c + 3) * count + i];
            q.x = q.x + w.x * hh[c];
            q.y = q.y + w.y * hh[c];
            phasor[(i64)(c + 3) * count + i] = q;
        }
    } else {
        float power = cross_axis(ee, hh, axis) * area[i];
        atomicAdd(flux + index, power);
    }
}

// adjoint.py:17-43 `record_curl`.
__global__ void record_curl_kernel(const float *__restrict__ h, i64 cols,
                                   float *__restrict__ hist, const int *__restrict__ step,
                                   int nx, int ny, int nz, int x0, int y0, int z0, int sx,
                                   int sy, int sz, float courant) {
    const i64 dn = (i64)sx * sy * sz;
    i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= dn) return;
    int x = x0 + (int)(j / ((i64)sy * sz));
    int y = y0 + (int)((j / sz) % sy);
    int z = z0 + (int)(j % sz);
    float v[3], a[3], b[3], c[3];
    sample3(h, cols, x, y, z, nx, ny, nz, 0, v);
    sample3(h, cols, x - 1, y, z, nx, ny, nz, 0, a);
    sample3(h, cols, x, y - 1, z, nx, ny, nz, 0, b);
    sample3(h, cols, x, y, z - 1, nx, ny, nz, 0, c);
    float dx[3], dy[3], dz[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dx[k] = v[k] - a[k];
        dy[k] = v[k] - b[k];
        dz[k] = v[k] - c[k];
    }
    float curl[3] = {dy[2] - dz[1], dz[0] - dx[2], dx[1] - dy[0]};
    const i64 t = step[0];
#pragma unroll
    for (int k = 0; k < 3; ++k) hist[(t * 3 + k) * dn + j] = courant * curl[k];
}

// record_curl over ping-pong, pitched buffers.
__global__ void record_curl_pp_kernel(const float *__restrict__ H0, const float *__restrict__ H1,
                                      int pitch, const int *__restrict__ step,
                                      const int *__restrict__ hist_step,
                                      float *__restrict__ hist, int nx, int ny, int nz, int x0,
                                      int y0, int z0, int sx, int sy, int sz, float courant) {
    const i64 dn = (i64)sx * sy * sz;
    i64 j = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= dn) return;
    const float *h = (step[0] & 1) ? H1 : H0;
    const i64 cols = (i64)nx * ny * pitch;
    int x = x0 + (int)(j / ((i64)sy * sz));
    int y = y0 + (int)((j / sz) % sy);
    int z = z0 + (int)(j % sz);
    float v[3], a[3], b[3], c[3];
    sample3(h, cols, x, y, z, nx, ny, nz, 0, v, pitch);
    sample3(h, cols, x - 1, y, z, nx, ny, nz, 0, a, pitch);
    sample3(h, cols, x, y - 1, z, nx, ny, nz, 0, b, pitch);
    sample3(h, cols, x, y, z - 1, nx, ny, nz, 0, c, pitch);
    float dx[3], dy[3], dz[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        dx[k] = v[k] - a[k];
        dy[k] = v[k] - b[k];
        dz[k] = v[k] - c[k];
    }
    float curl[3] = {dy[2] - dz[1], dz[0] - dx[2], dx[1] - dy[0]};
    const i64 t = hist_step[0];
#pragma unroll
    for (int k = 0; k < 3; ++k) hist[(t * 3 + k) * dn + j] = courant * curl[k];
}

// adjoint.py:46-88 `prepare`.
__global__ void prepare_kernel(const float *__restrict__ q, const float *__restrict__ eps,
                               float *__restrict__ psi, const float *__restrict__ coeff,
                               int clen, float *__restrict__ d, int nx, int ny, int nz,
                               float courant, int electric) {
    const i64 n = (i64)nx * ny * nz;
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int x = (int)(i / ((i64)ny * nz));
    int y = (int)((i / nz) % ny);
    int z = (int)(i % nz);
    float factor = -courant;
    if (electric) factor = courant * eps[i];
    float v[3] = {factor * q[i], factor * q[n + i], factor * q[2 * n + i]};
#pragma unroll
    for (int axis = 0; axis < 3; ++axis) {
        int pos = axis == 0 ? x : (axis == 1 ? y : z);
        const float *co = coeff + ((i64)axis * clen + pos) * 3;
        int a = (axis + 1) % 3, b = (axis + 2) % 3;
        float q1 = -v[a];
        float q2 = v[b];
        float d1 = co[2] * q1;
        float d2 = co[2] * q2;
        if (co[0] != 0.0f) {
            float p1 = psi[(2 * axis) * n + i] + q1;
            float p2 = psi[(2 * axis + 1) * n + i] + q2;
            d1 = d1 + co[0] * p1;
            d2 = d2 + co[0] * p2;
            psi[(2 * axis) * n + i] = co[1] * p1;
            psi[(2 * axis + 1) * n + i] = co[1] * p2;
        }
        d[(2 * axis) * n + i] = d1;
        d[(2 * axis + 1) * n + i] = d2;
    }
}

// adjoint.py:91-104 `read`.
__device__ __forceinline__ float read_d(const float *__restrict__ d, i64 n, int slot, int x,
                                        int y, int z, int nx, int ny, int nz) {
    if (!inside(x, y, z, nx, ny, nz)) return 0.0f;
    return d[(i64)slot * n + flat(x, y, z, ny, nz)];
}

// adjoint.py:107-162 `gather`.
template <bool GRAD64>
__global__ void gather_kernel(float *__restrict__ q, const float *__restrict__ d,
                              const float *__restrict__ hist, void *__restrict__ grad,
                              const int *__restrict__ step, int nx, int ny, int nz, int x0,
                              int y0, int z0, int sx, int sy, int sz, int from_h) {
    const i64 n = (i64)nx * ny * nz;
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int x = (int)(i / ((i64)ny * nz));
    int y = (int)((i / nz) % ny);
    int z = (int)(i % nz);
    const int delta = from_h ? -1 : 1;
    float v[3];
    v[0] = (read_d(d, n, 2, x, y + delta, z, nx, ny, nz) - d[2 * n + i]) +
           (read_d(d, n, 5, x, y, z + delta, nx, ny, nz) - d[5 * n + i]);
    v[1] = (read_d(d, n, 1, x + delta, y, z, nx, ny, nz) - d[n + i]) +
           (read_d(d, n, 4, x, y, z + delta, nx, ny, nz) - d[4 * n + i]);
    v[2] = (read_d(d, n, 0, x + delta, y, z, nx, ny, nz) - d[i]) +
           (read_d(d, n, 3, x, y + delta, z, nx, ny, nz) - d[3 * n + i]);
    if (!from_h) {
        v[0] = -v[0];
        v[1] = -v[1];
        v[2] = -v[2];
    }
    float value[3] = {q[i] + v[0], q[n + i] + v[1], q[2 * n + i] + v[2]};
    q[i] = value[0];
    q[n + i] = value[1];
    q[2 * n + i] = value[2];
    if (from_h && x >= x0 && x < x0 + sx && y >= y0 && y < y0 + sy && z >= z0 && z < z0 + sz) {
        const i64 dn = (i64)sx * sy * sz;
        i64 j = ((i64)(x - x0) * sy + (y - y0)) * sz + (z - z0);
        const float *hh = hist + (i64)step[0] * 3 * dn;
        if (GRAD64) {
            double *g = (double *)grad;
            g[j] = g[j] + (((double)hh[j] * value[0] + (double)hh[dn + j] * value[1]) +
                           (double)hh[2 * dn + j] * value[2]);
        } else {
            float *g = (float *)grad;
            g[j] = g[j] + ((hh[j] * value[0] + hh[dn + j] * value[1]) + hh[2 * dn + j] * value[2]);
        }
    }
}

// adjoint.py:165-178 `add`.
__device__ __forceinline__ void add_q(float *q, i64 n, int c, int x, int y, int z, int nx,
                                      int ny, int nz, float value) {
    if (inside(x, y, z, nx, ny, nz)) atomicAdd(q + (i64)c * n + flat(x, y, z, ny, nz), value);
}

// adjoint.py:181-223 `inject` for plane cell i of one plane.
__device__ __forceinline__ void inject_cell(float *__restrict__ qe, float *__restrict__ qh,
                                            const float2 *__restrict__ source,
                                            const float2 *__restrict__ weights,
                                            const int *__restrict__ step, int nx, int ny,
                                            int nz, int x0, int y0, int z0, int sx, int sy,
                                            int sz, int old_h_only, i64 i) {
    const i64 n = (i64)nx * ny * nz;
    const i64 count = (i64)sx * sy * sz;
    float2 w = weights[step[0]];
    if (!(fabsf(w.x) + fabsf(w.y) > 0.0f)) return;
    int x = x0 + (int)(i / ((i64)sy * sz));
    int y = y0 + (int)((i / sz) % sy);
    int z = z0 + (int)(i % sz);
    float v[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        float2 a = source[(i64)c * count + i];
        v[c] = a.x * w.x - a.y * w.y;
    }
    if (!old_h_only) {
        for (int dz = 0; dz < 2; ++dz) {
            for (int dx = 0; dx < 2; ++dx) add_q(qe, n, 0, x - dx, y, z + dz, nx, ny, nz, 0.25f * v[0]);
            for (int dy = 0; dy < 2; ++dy) add_q(qe, n, 1, x, y - dy, z + dz, nx, ny, nz, 0.25f * v[1]);
        }
        add_q(qe, n, 2, x, y, z, nx, ny, nz, v[2]);
    }
    for (int dy = 0; dy < 2; ++dy) add_q(qh, n, 0, x, y - dy, z, nx, ny, nz, 0.25f * v[3]);
    for (int dx = 0; dx < 2; ++dx) add_q(qh, n, 1, x - dx, y, z, nx, ny, nz, 0.25f * v[4]);
    for (int dx = 0; dx < 2; ++dx)
        for (int dy = 0; dy < 2; ++dy)
            for (int dz = 0; dz < 2; ++dz)
                add_q(qh, n, 2, x - dx, y - dy, z + dz, nx, ny, nz, 0.0625f * v[5]);
}

__global__ void inject_kernel(float *__restrict__ qe, float *__restrict__ qh,
                              const float2 *__restrict__ source,
                              const float2 *__restrict__ weights,
                              const int *__restrict__ step, int nx, int ny, int nz, int x0,
                              int y0, int z0, int sx, int sy, int sz, int old_h_only) {
    const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (i64)sx * sy * sz) return;
    inject_cell(qe, qh, source, weights, step, nx, ny, nz, x0, y0, z0, sx, sy, sz, old_h_only,
                i);
}

// Several planes' injections in one launch: thread i belongs to the plane
// whose cell range [start[k], start[k+1]) holds it.
struct InjectPlanes {
    fdtd_inject_plane p[FDTD_INJECT_PLANES_MAX];
    i64 start[FDTD_INJECT_PLANES_MAX + 1];
    int count;
};

__global__ void inject_many_kernel(float *__restrict__ qe, float *__restrict__ qh,
                                   const __grid_constant__ InjectPlanes planes,
                                   const int *__restrict__ step, int nx, int ny, int nz,
                                   int old_h_only) {
    const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= planes.start[planes.count]) return;
    int k = 0;
    while (k + 1 < planes.count && i >= planes.start[k + 1]) ++k;
    const fdtd_inject_plane &pl = planes.p[k];
    inject_cell(qe, qh, (const float2 *)pl.source, (const float2 *)pl.weights, step, nx, ny, nz,
                pl.x0, pl.y0, pl.z0, pl.sx, pl.sy, pl.sz, old_h_only, i - planes.start[k]);
}

// adjoint.py:472-490 `write_design`.
__global__ void write_design_kernel(const float *__restrict__ plane, float *__restrict__ eps,
                                    int nx, int ny, int nz, int x0, int y0, int z0, int sx,
                                    int sy, int sz) {
    const i64 dn = (i64)sx * sy * sz;
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= dn) return;
    int x = (int)(i / ((i64)sy * sz));
    int y = (int)((i / sz) % sy);
    int z = (int)(i % sz);
    eps[flat(x0 + x, y0 + y, z0 + z, ny, nz)] = plane[(i64)x * sy + y];
}

}  // namespace wfb

using namespace wfb;

static cudaStream_t as_stream(void *s) { return (cudaStream_t)s; }

extern "C" {

const char *fdtd_last_error(void) { return wfb::g_error; }

int fdtd_version(void) { return 100; }

int fdtd_update(int electric, int packed, float *f, const float *g, long long fg_cols,
                const float *inv_eps, float *psi, long long psi_cols, const float *coeff,
                int clen, const float *source, long long source_cols, const float *waves,
                long long waves_cols, const int *step, float *hprev, long long hprev_cols,
                int save_h_from, int nx, int ny, int nz, int source_x, float courant,
                int periodic, void *stream) {
    if (nx <= 0 || ny <= 0 || nz <= 0 || !f || !g || !psi || !coeff || !step ||
        (electric && !inv_eps)) {
        set_error("fdtd_update: invalid sizes or null pointer");
        return FDTD_ERR_ARG;
    }
    const i64 n = (i64)nx * ny * nz;
    if (fg_cols < n || clen < (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz))) {
        set_error("fdtd_update: field columns %lld or coefficient length %d too small", fg_cols, clen);
        return FDTD_ERR_ARG;
    }
    if (!packed && psi_cols < n) {
        set_error("fdtd_update: full CPML storage needs psi_cols >= n");
        return FDTD_ERR_ARG;
    }
    const int T = 256;
    dim3 grid(blocks_for(n, T));
    cudaStream_t st = as_stream(stream);
#define LAUNCH(E, P)                                                                        \
    update_kernel<E, P><<<grid, T, 0, st>>>(f, g, fg_cols, inv_eps, psi, psi_cols, coeff,   \
                                            clen, source, source_cols, waves, waves_cols,   \
                                            step, hprev, hprev_cols, save_h_from, nx, ny,  \
                                            nz, source_x, courant, periodic)
    if (electric) {
        if (packed) LAUNCH(true, true); else LAUNCH(true, false);
    } else {
        if (packed) LAUNCH(false, true); else LAUNCH(false, false);
    }
#undef LAUNCH
    return launch_status("fdtd_update");
}

int fdtd_advance(int *step, int delta, void *stream) {
    if (!step) {
        set_error("fdtd_advance: null step");
        return FDTD_ERR_ARG;
    }
    advance_kernel<<<1, 1, 0, as_stream(stream)>>>(step, delta);
    return launch_status("fdtd_advance");
}

int fdtd_advance_many(int *const *steps, int count, int delta, void *stream) {
    if (!steps || count < 1) {
        set_error("fdtd_advance_many: null steps or count < 1");
        return FDTD_ERR_ARG;
    }
    advance_many_kernel<<<(count + 127) / 128, 128, 0, as_stream(stream)>>>(steps, count, delta);
    return launch_status("fdtd_advance_many");
}

int fdtd_record(const float *e, const float *h, const float *prev, long long cols,
                const int *step, const float *weights, const int *indices, float *phasor,
                float *flux, const float *area, int nx, int ny, int nz, int x0, int y0,
                int z0, int sx, int sy, int sz, int axis, int exact, int is_phasor,
                void *stream) {
    const i64 count = (i64)sx * sy * sz;
    if (count <= 0 || axis < 0 || axis > 2 || !e || !h || !step || !weights || !indices ||
        (is_phasor && !phasor) || (!is_phasor && (!flux || !area)) || (exact && !prev)) {
        set_error("fdtd_record: invalid arguments");
        return FDTD_ERR_ARG;
    }
    record_kernel<<<blocks_for(count, 256), 256, 0, as_stream(stream)>>>(
        e, h, prev, cols, step, (const float2 *)weights, indices, (float2 *)phasor, flux, area,
        nx, ny, nz, x0, y0, z0, sx, sy, sz, axis, exact, is_phasor);
    return launch_status("fdtd_record");
}

int fdtd_record_curl(const float *h, long long cols, float *hist, const int *step, int nx,
                     int ny, int nz, int x0, int y0, int z0, int sx, int sy, int sz,
                     float courant, void *stream) {
    const i64 dn = (i64)sx * sy * sz;
    if (dn <= 0 || !h || !hist || !step) {
        set_error("fdtd_record_curl: invalid arguments");
        return FDTD_ERR_ARG;
    }
    record_curl_kernel<<<blocks_for(dn, 256), 256, 0, as_stream(stream)>>>(
        h, cols, hist, step, nx, ny, nz, x0, y0, z0, sx, sy, sz, courant);
    return launch_status("fdtd_record_curl");
}

int fdtd_record_curl_pp(const float *H0, const float *H1, int pitch_z, const int *step,
                        const int *hist_step, float *hist, int nx, int ny, int nz, int x0,
                        int y0, int z0, int sx, int sy, int sz, float courant, void *stream) {
    const i64 dn = (i64)sx * sy * sz;
    if (pitch_z <= 0) pitch_z = nz;
    if (dn <= 0 || !H0 || !H1 || !step || !hist_step || !hist || pitch_z < nz || x0 < 0 ||
        y0 < 0 || z0 < 0 || x0 + sx > nx || y0 + sy > ny || z0 + sz > nz) {
        set_error("fdtd_record_curl_pp: invalid arguments");
        return FDTD_ERR_ARG;
    }
    record_curl_pp_kernel<<<blocks_for(dn, 256), 256, 0, as_stream(stream)>>>(
        H0, H1, pitch_z, step, hist_step, hist, nx, ny, nz, x0, y0, z0, sx, sy, sz, courant);
    return launch_status("fdtd_record_curl_pp");
}

int fdtd_prepare(const float *q, const float *eps, float *psi, const float *coeff, int clen,
                 float *d, int nx, int ny, int nz, float courant, int electric,
                 void *stream) {
    const i64 n = (i64)nx * ny * nz;
    if (n <= 0 || !q || !psi || !coeff || !d || (electric && !eps)) {
        set_error("fdtd_prepare: invalid arguments");
        return FDTD_ERR_ARG;
    }
    prepare_kernel<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(
        q, eps, psi, coeff, clen, d, nx, ny, nz, courant, electric);
    return launch_status("fdtd_prepare");
}

int fdtd_gather(float *q, const float *d, const float *hist, void *grad, int grad_f64,
                const int *step, int nx, int ny, int nz, int x0, int y0, int z0, int sx,
                int sy, int sz, int from_h, void *stream) {
    const i64 n = (i64)nx * ny * nz;
    if (n <= 0 || !q || !d || !step || (from_h && (sx * sy * sz) > 0 && (!hist || !grad))) {
        set_error("fdtd_gather: invalid arguments");
        return FDTD_ERR_ARG;
    }
    if (grad_f64)
        gather_kernel<true><<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(
            q, d, hist, grad, step, nx, ny, nz, x0, y0, z0, sx, sy, sz, from_h);
    else
        gather_kernel<false><<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(
            q, d, hist, grad, step, nx, ny, nz, x0, y0, z0, sx, sy, sz, from_h);
    return launch_status("fdtd_gather");
}

int fdtd_inject(float *qe, float *qh, const float *source, const float *weights,
                const int *step, int nx, int ny, int nz, int x0, int y0, int z0, int sx,
                int sy, int sz, int old_h_only, void *stream) {
    const i64 count = (i64)sx * sy * sz;
    if (count <= 0 || !qe || !qh || !source || !weights || !step) {
        set_error("fdtd_inject: invalid arguments");
        return FDTD_ERR_ARG;
    }
    inject_kernel<<<blocks_for(count, 256), 256, 0, as_stream(stream)>>>(
        qe, qh, (const float2 *)source, (const float2 *)weights, step, nx, ny, nz, x0, y0, z0,
        sx, sy, sz, old_h_only);
    return launch_status("fdtd_inject");
}

int fdtd_inject_many(float *qe, float *qh, const fdtd_inject_plane *planes, int nplanes,
                     const int *step, int nx, int ny, int nz, int old_h_only, void *stream) {
    if (!qe || !qh || !planes || !step || nplanes < 1 || nplanes > FDTD_INJECT_PLANES_MAX ||
        nx < 1 || ny < 1 || nz < 1) {
        set_error("fdtd_inject_many: invalid arguments (1 to %d planes)",
                  FDTD_INJECT_PLANES_MAX);
        return FDTD_ERR_ARG;
    }
    InjectPlanes pp;
    pp.count = nplanes;
    pp.start[0] = 0;
    for (int k = 0; k < nplanes; ++k) {
        const fdtd_inject_plane &pl = planes[k];
        if (!pl.source || !pl.weights || pl.sx < 1 || pl.sy < 1 || pl.sz < 1) {
            set_error("fdtd_inject_many: plane %d has no source, weights or cells", k);
            return FDTD_ERR_ARG;
        }
        pp.p[k] = pl;
        pp.start[k + 1] = pp.start[k] + (i64)pl.sx * pl.sy * pl.sz;
    }
    inject_many_kernel<<<blocks_for(pp.start[nplanes], 256), 256, 0, as_stream(stream)>>>(
        qe, qh, pp, step, nx, ny, nz, old_h_only);
    return launch_status("fdtd_inject_many");
}

int fdtd_write_design(const float *plane, float *eps, int nx, int ny, int nz, int x0,
                      int y0, int z0, int sx, int sy, int sz, void *stream) {
    const i64 dn = (i64)sx * sy * sz;
    if (dn <= 0 || !plane || !eps || x0 < 0 || y0 < 0 || z0 < 0 || x0 + sx > nx ||
        y0 + sy > ny || z0 + sz > nz) {
        set_error("fdtd_write_design: box outside the grid or null pointer");
        return FDTD_ERR_ARG;
    }
    write_design_kernel<<<blocks_for(dn, 256), 256, 0, as_stream(stream)>>>(
        plane, eps, nx, ny, nz, x0, y0, z0, sx, sy, sz);
    return launch_status("fdtd_write_design");
}

}  // extern "C"
