// Float64 detector recorders for the fused forward path (detectors.py:65-106
// generalised to K DFT frequencies).  They run after fdtd_step_fused on the
// same stream and pick the ping-pong buffers by the step parity, so a CUDA
// graph of steps replays them unchanged.
#include "common.cuh"

namespace wfb {

__global__ void record_phasor64_kernel(const float *__restrict__ E0, const float *__restrict__ E1,
                                       const float *__restrict__ H0, const float *__restrict__ H1,
                                       const int *__restrict__ step,
                                       const int *__restrict__ indices, int nsteps,
                                       const float2 *__restrict__ weights, int nfreq,
                                       double2 *__restrict__ phasor, int nx, int ny, int nz,
                                       int pitch, int x0, int y0, int z0, int sx, int sy, int sz,
                                       int exact) {
    const i64 count = (i64)sx * sy * sz;
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int t = step[0];
    if (t < 0 || t >= nsteps || indices[t] < 0) return;
    const i64 wsteps = nsteps;
    const int s = t & 1;
    const float *e = s ? E0 : E1;
    const float *h = s ? H0 : H1;
    const float *prev = s ? H1 : H0;
    const i64 n = (i64)nx * ny * pitch;
    int x = x0 + (int)(i / ((i64)sy * sz));
    int y = y0 + (int)((i / sz) % sy);
    int z = z0 + (int)(i % sz);
    float ee[3], hh[3];
    plane_sample(e, h, prev, n, x, y, z, nx, ny, nz, exact, ee, hh, pitch);
    for (int k = 0; k < nfreq; ++k) {
        float2 w = weights[(i64)k * wsteps + t];
        double wr = w.x, wi = w.y;
        if (wr == 0.0 && wi == 0.0) continue;
#pragma unroll
        for (int c = 0; c < 6; ++c) {
            double v = c < 3 ? (double)ee[c] : (double)hh[c - 3];
            double2 *p = phasor + ((i64)k * 6 + c) * count + i;
            double2 acc = *p;
            acc.x = acc.x + wr * v;
            acc.y = acc.y + wi * v;
            *p = acc;
        }
    }
}

__global__ void record_flux64_kernel(const float *__restrict__ E0, const float *__restrict__ E1,
                                     const float *__restrict__ H0, const float *__restrict__ H1,
                                     const int *__restrict__ step,
                                     const int *__restrict__ indices, int nsteps,
                                     const float *__restrict__ area, double *__restrict__ flux,
                                     int nbins, int nx, int ny, int nz, int pitch, int x0,
                                     int y0, int z0, int sx, int sy, int sz, int axis,
                                     int exact) {
    __shared__ double partial[32];
    const i64 count = (i64)sx * sy * sz;
    const int t = step[0];
    if (t < 0 || t >= nsteps) return;
    const int index = indices[t];
    if (index < 0 || index >= nbins) return;
    const int s = t & 1;
    const float *e = s ? E0 : E1;
    const float *h = s ? H0 : H1;
    const float *prev = s ? H1 : H0;
    const i64 n = (i64)nx * ny * pitch;
    double acc = 0.0;
    for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += (i64)gridDim.x * blockDim.x) {
        int x = x0 + (int)(i / ((i64)sy * sz));
        int y = y0 + (int)((i / sz) % sy);
        int z = z0 + (int)(i % sz);
        float ee[3], hh[3];
        plane_sample(e, h, prev, n, x, y, z, nx, ny, nz, exact, ee, hh, pitch);
        float power = cross_axis(ee, hh, axis) * area[i];
        acc += (double)power;
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) partial[warp] = acc;
    __syncthreads();
    if (warp == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        acc = lane < nw ? partial[lane] : 0.0;
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if (lane == 0) atomicAdd(flux + index, acc);
    }
}

__global__ void record_stage_kernel(const float *__restrict__ E0, const float *__restrict__ E1,
                                    const float *__restrict__ H0, const float *__restrict__ H1,
                                    const int *__restrict__ step,
                                    const int *__restrict__ indices, int nsteps,
                                    float *__restrict__ stage, int T, int nx, int ny, int nz,
                                    int pitch, int x0, int y0, int z0, int sx, int sy, int sz,
                                    int exact) {
    const i64 count = (i64)sx * sy * sz;
    i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int t = step[0];
    if (t < 0 || t >= nsteps || indices[t] < 0) return;
    const int s = t & 1;
    const float *e = s ? E0 : E1;
    const float *h = s ? H0 : H1;
    const float *prev = s ? H1 : H0;
    const i64 n = (i64)nx * ny * pitch;
    int x = x0 + (int)(i / ((i64)sy * sz));
    int y = y0 + (int)((i / sz) % sy);
    int z = z0 + (int)(i % sz);
    float ee[3], hh[3];
    plane_sample(e, h, prev, n, x, y, z, nx, ny, nz, exact, ee, hh, pitch);
    float *dst = stage + (i64)(t % T) * 6 * count + i;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        dst[(i64)c * count] = ee[c];
        dst[(i64)(c + 3) * count] = hh[c];
    }
}

// volume.py:24-41: component `comp` of f trilinearly interpolated at grid
// position (px, py, pz); taps outside the grid count as zero.  Same float32
// operation order as the reference.
__device__ __forceinline__ float trilinear(const float *__restrict__ f, i64 n, int comp, float px,
                                           float py, float pz, int nx, int ny, int nz,
                                           int pitch) {
    const int ix = (int)floorf(px), iy = (int)floorf(py), iz = (int)floorf(pz);
    const float tx = px - (float)ix, ty = py - (float)iy, tz = pz - (float)iz;
    float value = 0.0f;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
            for (int c = 0; c < 2; ++c) {
                const int x = ix + a, y = iy + b, z = iz + c;
                if (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz) {
                    const float w = ((a ? tx : 1.0f - tx) * (b ? ty : 1.0f - ty)) * (c ? tz : 1.0f - tz);
                    value = value + w * f[comp * n + ((i64)x * ny + y) * pitch + z];
                }
            }
    return value;
}

// volume.py:60-89 with float64 accumulators: one thread per sampling point;
// component c is sampled at the point minus its Yee offset, H as the mean of
// H(n+1/2) and H(n-1/2).
__global__ void record_volume_kernel(const float *__restrict__ E0, const float *__restrict__ E1,
                                     const float *__restrict__ H0, const float *__restrict__ H1,
                                     const int *__restrict__ step,
                                     const float *__restrict__ positions, i64 count,
                                     const float2 *__restrict__ weights, int nsteps, int first,
                                     double2 *__restrict__ phasor, int nx, int ny, int nz,
                                     int pitch) {
    const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const int t = step[0];
    if (t < first || t < 0 || t >= nsteps) return;
    const float2 w = weights[t];
    const int s = t & 1;
    const float *e = s ? E0 : E1;
    const float *h = s ? H0 : H1;
    const float *prev = s ? H1 : H0;
    const i64 n = (i64)nx * ny * pitch;
    const float px = positions[3 * i], py = positions[3 * i + 1], pz = positions[3 * i + 2];
    // Yee offsets of Ex, Ey, Ez, Hx, Hy, Hz (volume.py:44-57)
    const float ox[6] = {0.5f, 0.0f, 0.0f, 0.0f, 0.5f, 0.5f};
    const float oy[6] = {0.0f, 0.5f, 0.0f, 0.5f, 0.0f, 0.5f};
    const float oz[6] = {0.0f, 0.0f, 0.5f, 0.5f, 0.5f, 0.0f};
#pragma unroll
    for (int c = 0; c < 6; ++c) {
        const float qx = px - ox[c], qy = py - oy[c], qz = pz - oz[c];
        float value;
        if (c < 3)
            value = trilinear(e, n, c, qx, qy, qz, nx, ny, nz, pitch);
        else
            value = 0.5f * (trilinear(h, n, c - 3, qx, qy, qz, nx, ny, nz, pitch) +
                            trilinear(prev, n, c - 3, qx, qy, qz, nx, ny, nz, pitch));
        double2 *p = phasor + (i64)c * count + i;
        double2 acc = *p;
        acc.x = acc.x + (double)w.x * (double)value;
        acc.y = acc.y + (double)w.y * (double)value;
        *p = acc;
    }
}

// fdtd_record_stage over several planes in one launch (blockIdx.y = plane).
struct StagePlanes {
    fdtd_stage_plane p[FDTD_STAGE_PLANES_MAX];
};

// With `done` set, the block that finishes last also advances step[0] by
// `delta` (every block has read it by then) and rearms the counter.
__device__ __forceinline__ void stage_block_done(int *step, unsigned *done, int delta) {
    if (!done) return;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned blocks = gridDim.x * gridDim.y * gridDim.z;
        if (atomicAdd(done, 1u) == blocks - 1) {
            step[0] += delta;
            *done = 0;
            __threadfence();
        }
    }
}

// Field pointers of the steps one launch stages: blockIdx.z selects the step
// (t + blockIdx.z) and its pointer set.
struct StageFields {
    const float *E0[2], *E1[2], *H0[2], *H1[2];
};

__global__ void record_stage_many_kernel(const StageFields f, int *step, const StagePlanes planes,
                                         int nx, int ny, int nz, int pitch, unsigned *done,
                                         int delta) {
    const fdtd_stage_plane &pl = planes.p[blockIdx.y];
    const i64 count = (i64)pl.sx * pl.sy * pl.sz;
    const i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    const int z = blockIdx.z;
    const float *__restrict__ E0 = f.E0[z], *__restrict__ E1 = f.E1[z];
    const float *__restrict__ H0 = f.H0[z], *__restrict__ H1 = f.H1[z];
    const int t = *(volatile int *)step + z;
    if (i < count && t >= 0 && t < pl.nsteps && pl.indices[t] >= 0) {
        const int s = t & 1;
        const float *e = s ? E0 : E1;
        const float *h = s ? H0 : H1;
        const float *prev = s ? H1 : H0;
        const i64 n = (i64)nx * ny * pitch;
        const int x = pl.x0 + (int)(i / ((i64)pl.sy * pl.sz));
        const int y = pl.y0 + (int)((i / pl.sz) % pl.sy);
        const int z = pl.z0 + (int)(i % pl.sz);
        float ee[3], hh[3];
        plane_sample(e, h, prev, n, x, y, z, nx, ny, nz, pl.exact, ee, hh, pitch);
        float *dst = pl.stage + (i64)(t % pl.T) * 6 * count + i;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            dst[(i64)c * count] = ee[c];
            dst[(i64)(c + 3) * count] = hh[c];
        }
    }
    stage_block_done(step, done, delta);  // every thread of the block reaches it
}

// One thread per (component, cell) and group of up to FOLD_K frequencies: the
// thread reads its cell's staged samples once and feeds every frequency of
// its group; each phasor still sums its steps in time order.  The window's
// weights are staged in shared memory ([k][t] float2).
constexpr int FOLD_K = 8;

__global__ void dft_fold_kernel(const int *__restrict__ step, const int *__restrict__ indices,
                                int nsteps, const float2 *__restrict__ weights, int nfreq,
                                const float *__restrict__ stage, int T,
                                double2 *__restrict__ phasor, i64 count) {
    extern __shared__ float2 wsm[];  // [nfreq][T]
    __shared__ int valid[256];
    const int s = step[0];
    if (s <= 0) return;
    const int t0 = ((s - 1) / T) * T;
    const int n = s - t0;
    for (int j = threadIdx.x; j < nfreq * T; j += blockDim.x) {
        const int k = j / T, dt = j - k * T;
        const int t = t0 + dt;
        wsm[j] = (dt < n && t < nsteps) ? weights[(i64)k * nsteps + t] : make_float2(0.f, 0.f);
    }
    for (int j = threadIdx.x; j < T; j += blockDim.x) {
        const int t = t0 + j;
        valid[j] = (j < n && t < nsteps && indices[t] >= 0) ? 1 : 0;
    }
    __syncthreads();
    const int groups = (nfreq + FOLD_K - 1) / FOLD_K;
    const i64 gid = (i64)blockIdx.x * blockDim.x + threadIdx.x;
    if (gid >= (i64)groups * 6 * count) return;
    const int kg = (int)(gid / (6 * count));
    const i64 rem = gid - (i64)kg * 6 * count;
    const int c = (int)(rem / count);
    const i64 i = rem - (i64)c * count;
    const int k0 = kg * FOLD_K, kn = min(FOLD_K, nfreq - k0);
    double2 acc[FOLD_K];
#pragma unroll
    for (int q = 0; q < FOLD_K; ++q)
        if (q < kn) acc[q] = phasor[((i64)(k0 + q) * 6 + c) * count + i];
    constexpr int CH = 8;  // samples in flight per thread
    for (int d0 = 0; d0 < n; d0 += CH) {
        float v[CH];
#pragma unroll
        for (int j = 0; j < CH; ++j) {
            const int dt = d0 + j;
            v[j] = dt < n && valid[dt] ? stage[((i64)((t0 + dt) % T) * 6 + c) * count + i] : 0.0f;
        }
#pragma unroll
        for (int j = 0; j < CH; ++j) {
            const int dt = d0 + j;
            if (dt >= n || !valid[dt]) continue;
            const double vv = (double)v[j];
#pragma unroll
            for (int q = 0; q < FOLD_K; ++q) {
                if (q >= kn) break;
                const float2 w = wsm[(k0 + q) * T + dt];
                const double wr = w.x, wi = w.y;
                if (wr == 0.0 && wi == 0.0) continue;
                acc[q].x = acc[q].x + wr * vv;
                acc[q].y = acc[q].y + wi * vv;
            }
        }
    }
#pragma unroll
    for (int q = 0; q < FOLD_K; ++q)
        if (q < kn) phasor[((i64)(k0 + q) * 6 + c) * count + i] = acc[q];
}

}  // namespace wfb

using namespace wfb;

extern "C" {

int fdtd_record_phasor64(const float *E0, const float *E1, const float *H0, const float *H1,
                         const int *step, const int *indices, int nsteps,
                         const float *weights, int nfreq, double *phasor, int nx, int ny,
                         int nz, int pitch_z, int x0, int y0, int z0, int sx, int sy, int sz,
                         int exact, void *stream) {
    const i64 count = (i64)sx * sy * sz;
    if (pitch_z <= 0) pitch_z = nz;
    if (count <= 0 || nfreq < 1 || nsteps < 1 || pitch_z < nz || !E0 || !E1 || !H0 || !H1 ||
        !step || !indices || !weights || !phasor || x0 < 0 || y0 < 0 || z0 < 0 ||
        x0 + sx > nx || y0 + sy > ny || z0 + sz > nz) {
        set_error("fdtd_record_phasor64: invalid arguments");
        return FDTD_ERR_ARG;
    }
    record_phasor64_kernel<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        E0, E1, H0, H1, step, indices, nsteps, (const float2 *)weights, nfreq,
        (double2 *)phasor, nx, ny, nz, pitch_z, x0, y0, z0, sx, sy, sz, exact);
    return launch_status("fdtd_record_phasor64");
}

int fdtd_record_flux64(const float *E0, const float *E1, const float *H0, const float *H1,
                       const int *step, const int *indices, int nsteps, const float *area,
                       double *flux, int nbins, int nx, int ny, int nz, int pitch_z, int x0,
                       int y0, int z0, int sx, int sy, int sz, int axis, int exact,
                       void *stream) {
    const i64 count = (i64)sx * sy * sz;
    if (pitch_z <= 0) pitch_z = nz;
    if (count <= 0 || axis < 0 || axis > 2 || nsteps < 1 || nbins < 1 || pitch_z < nz ||
        !E0 || !E1 || !H0 || !H1 || !step || !indices || !area || !flux || x0 < 0 || y0 < 0 ||
        z0 < 0 || x0 + sx > nx || y0 + sy > ny || z0 + sz > nz) {
        set_error("fdtd_record_flux64: invalid arguments");
        return FDTD_ERR_ARG;
    }
    i64 blocks = (count + 255) / 256;
    if (blocks > 148) blocks = 148;
    record_flux64_kernel<<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(
        E0, E1, H0, H1, step, indices, nsteps, area, flux, nbins, nx, ny, nz, pitch_z, x0, y0,
        z0, sx, sy, sz, axis, exact);
    return launch_status("fdtd_record_flux64");
}

int fdtd_record_stage(const float *E0, const float *E1, const float *H0, const float *H1,
                      const int *step, const int *indices, int nsteps, float *stage, int T,
                      int nx, int ny, int nz, int pitch_z, int x0, int y0, int z0, int sx,
                      int sy, int sz, int exact, void *stream) {
    const i64 count = (i64)sx * sy * sz;
    if (pitch_z <= 0) pitch_z = nz;
    if (count <= 0 || T < 1 || T > 256 || nsteps < 1 || pitch_z < nz || !E0 || !E1 || !H0 ||
        !H1 || !step || !indices || !stage || x0 < 0 || y0 < 0 || z0 < 0 || x0 + sx > nx ||
        y0 + sy > ny || z0 + sz > nz) {
        set_error("fdtd_record_stage: invalid arguments");
        return FDTD_ERR_ARG;
    }
    record_stage_kernel<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        E0, E1, H0, H1, step, indices, nsteps, stage, T, nx, ny, nz, pitch_z, x0, y0, z0, sx, sy,
        sz, exact);
    return launch_status("fdtd_record_stage");
}

int fdtd_dft_fold(const int *step, const int *indices, int nsteps, const float *weights,
                  int nfreq, const float *stage, int T, double *phasor, long long count,
                  void *stream) {
    if (!step || !indices || !weights || !stage || !phasor || nfreq < 1 || nfreq > 64 ||
        T < 1 || T > 256 || nfreq * T > 6144 || count < 1 || nsteps < 1) {
        set_error("fdtd_dft_fold: invalid arguments");
        return FDTD_ERR_ARG;
    }
    const i64 work = (i64)((nfreq + FOLD_K - 1) / FOLD_K) * 6 * count;
    const size_t smem = (size_t)nfreq * T * sizeof(float2);
    dft_fold_kernel<<<(unsigned)((work + 255) / 256), 256, smem, (cudaStream_t)stream>>>(
        step, indices, nsteps, (const float2 *)weights, nfreq, stage, T, (double2 *)phasor,
        count);
    return launch_status("fdtd_dft_fold");
}

int fdtd_record_volume(const float *E0, const float *E1, const float *H0, const float *H1,
                       const int *step, const float *positions, long long count,
                       const float *weights, int nsteps, int first, double *phasor, int nx,
                       int ny, int nz, int pitch_z, void *stream) {
    if (pitch_z <= 0) pitch_z = nz;
    if (count <= 0 || nsteps < 1 || nx < 1 || ny < 1 || nz < 1 || pitch_z < nz || !E0 || !E1 ||
        !H0 || !H1 || !step || !positions || !weights || !phasor) {
        set_error("fdtd_record_volume: invalid arguments");
        return FDTD_ERR_ARG;
    }
    record_volume_kernel<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        E0, E1, H0, H1, step, positions, (i64)count, (const float2 *)weights, nsteps, first,
        (double2 *)phasor, nx, ny, nz, pitch_z);
    return launch_status("fdtd_record_volume");
}

int fdtd_record_stage_many(const float *E0, const float *E1, const float *H0, const float *H1,
                           int *step, const fdtd_stage_plane *planes, int nplanes, int nx,
                           int ny, int nz, int pitch_z, unsigned *advance_counter, int delta,
                           void *stream) {
    if (pitch_z <= 0) pitch_z = nz;
    if (!planes || nplanes < 1 || nplanes > FDTD_STAGE_PLANES_MAX || !E0 || !E1 || !H0 || !H1 ||
        !step || pitch_z < nz) {
        set_error("fdtd_record_stage_many: invalid arguments");
        return FDTD_ERR_ARG;
    }
    StagePlanes sp;
    i64 most = 0;
    for (int j = 0; j < nplanes; ++j) {
        const fdtd_stage_plane &pl = planes[j];
        const i64 count = (i64)pl.sx * pl.sy * pl.sz;
        if (count <= 0 || pl.T < 1 || pl.T > 256 || pl.nsteps < 1 || !pl.indices || !pl.stage ||
            pl.x0 < 0 || pl.y0 < 0 || pl.z0 < 0 || pl.x0 + pl.sx > nx || pl.y0 + pl.sy > ny ||
            pl.z0 + pl.sz > nz) {
            set_error("fdtd_record_stage_many: invalid plane %d", j);
            return FDTD_ERR_ARG;
        }
        sp.p[j] = pl;
        most = count > most ? count : most;
    }
    StageFields f;
    f.E0[0] = f.E0[1] = E0;
    f.E1[0] = f.E1[1] = E1;
    f.H0[0] = f.H0[1] = H0;
    f.H1[0] = f.H1[1] = H1;
    record_stage_many_kernel<<<dim3((unsigned)((most + 255) / 256), (unsigned)nplanes), 256, 0,
                               (cudaStream_t)stream>>>(f, step, sp, nx, ny, nz, pitch_z,
                                                       advance_counter, delta);
    return launch_status("fdtd_record_stage_many");
}

int fdtd_record_stage_pair(const float *const *fields, int *step, const fdtd_stage_plane *planes,
                           int nplanes, int nx, int ny, int nz, int pitch_z,
                           unsigned *advance_counter, void *stream) {
    if (pitch_z <= 0) pitch_z = nz;
    if (!fields || !planes || nplanes < 1 || nplanes > FDTD_STAGE_PLANES_MAX || !step ||
        !advance_counter || pitch_z < nz) {
        set_error("fdtd_record_stage_pair: invalid arguments");
        return FDTD_ERR_ARG;
    }
    for (int j = 0; j < 8; ++j)
        if (!fields[j]) {
            set_error("fdtd_record_stage_pair: null field pointer %d", j);
            return FDTD_ERR_ARG;
        }
    StagePlanes sp;
    i64 most = 0;
    for (int j = 0; j < nplanes; ++j) {
        const fdtd_stage_plane &pl = planes[j];
        const i64 count = (i64)pl.sx * pl.sy * pl.sz;
        if (count <= 0 || pl.T < 2 || pl.T > 256 || pl.nsteps < 1 || !pl.indices || !pl.stage ||
            pl.x0 < 0 || pl.y0 < 0 || pl.z0 < 0 || pl.x0 + pl.sx > nx || pl.y0 + pl.sy > ny ||
            pl.z0 + pl.sz > nz) {
            set_error("fdtd_record_stage_pair: invalid plane %d (T >= 2 needed)", j);
            return FDTD_ERR_ARG;
        }
        sp.p[j] = pl;
        most = count > most ? count : most;
    }
    StageFields f;
    for (int k = 0; k < 2; ++k) {
        f.E0[k] = fields[4 * k];
        f.E1[k] = fields[4 * k + 1];
        f.H0[k] = fields[4 * k + 2];
        f.H1[k] = fields[4 * k + 3];
    }
    record_stage_many_kernel<<<dim3((unsigned)((most + 255) / 256), (unsigned)nplanes, 2), 256, 0,
                               (cudaStream_t)stream>>>(f, step, sp, nx, ny, nz, pitch_z,
                                                       advance_counter, 2);
    return launch_status("fdtd_record_stage_pair");
}

}  // extern "C"
