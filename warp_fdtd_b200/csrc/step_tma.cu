// Fused Yee leapfrog step with a TMA + mbarrier pipeline (sm_100a).
//
// Same decomposition and arithmetic as the shared-memory path in
// step_fused.cu (a block owns a tile_y x tile_z column of the y-z plane and a
// chunk of x planes, marching along x, E computed one plane ahead of H), but
// the planes are staged by the Tensor Memory Accelerator:
//
//   * a ring of S stages, each holding one x plane of
//       H(p) on the tile plus a -y/-z halo (box z: tile_z + 8 from z0 - 4),
//       E(p) on the tile plus a +y/+z halo (box z: tile_z + 4 from z0),
//       the material (uint8 box z: tile_z + 16, or float32 like E);
//   * one elected thread issues cp.async.bulk.tensor loads for plane p+S-1
//     while the block computes plane p; completion is tracked by one
//     mbarrier per stage (expect_tx / complete_tx);
//   * coordinates outside the grid are zero-filled by the TMA unit, which is
//     exactly the reference's zero padding (kernels.py:23-24), so the stencil
//     needs no bounds branches for loads.
// Every TMA box starts at a z coordinate that is a multiple of 4 floats (16 B)
// or 16 bytes for uint8, as the hardware requires; the halo offsets are
// absorbed by widening the box and indexing from the remainder in shared
// memory.  No multicast is used.
//
// Every wait is bounded: if a stage does not complete within the limit the
// block records the failure in `error`, waits (bounded) for its own copies in
// flight and exits, so a fault can never hang the GPU.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "common.cuh"
#include "step_internal.h"
#include "tma_util.cuh"

namespace wfb {

struct TmaMaps {
    CUtensorMap E[2];  // fields, 4-D (z, y, x, component)
    CUtensorMap H[2];
    CUtensorMap M;     // material: 3-D uint8 or float32 (z, y, x)
};

struct TmaParams {
    fdtd_step_args a;
    TmaLayout L;
};

// kernels.py:29-74: CPML-filtered difference; psi read from the old buffer,
// the new value written (for owned cells) to the new buffer.
__device__ __forceinline__ float cpml_pp2(float d, float4 c, const float *__restrict__ psi_o,
                                          float *__restrict__ psi_n, i64 psi_cols, int slot,
                                          i64 index, bool own) {
    if (c.x != 0.0f) {
        float p = c.y * psi_o[(i64)slot * psi_cols + index] + c.x * d;
        if (own) psi_n[(i64)slot * psi_cols + index] = p;
        return c.z * d + p;
    }
    return c.z * d;
}

template <bool PACKED>
__device__ __forceinline__ i64 psi_idx(int axis, float rank, i64 i, int x, int y, int z, int nx,
                                       int ny, int nz) {
    if (!PACKED) return i;
    i64 plane = (i64)(int)rank;
    if (axis == 0) return plane * ny * nz + (i64)y * nz + z;
    if (axis == 1) return plane * nx * nz + (i64)x * nz + z;
    return plane * nx * ny + (i64)x * ny + y;
}

// A coefficient (a, b, 1/kappa) changes the difference unless a == 0 and
// 1/kappa == 1, where the reference returns 1 * d == d exactly.
__device__ __forceinline__ bool cpml_active(float4 c) { return c.x != 0.0f || c.z != 1.0f; }

template <int V>
__device__ __forceinline__ void ldv(const float *p, float (&o)[V]) {
    if constexpr (V == 4) {
        const float4 v = *(const float4 *)p;
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    } else if constexpr (V == 2) {
        const float2 v = *(const float2 *)p;
        o[0] = v.x; o[1] = v.y;
    } else {
        o[0] = p[0];
    }
}

template <int V>
__device__ __forceinline__ void stv(float *p, const float (&o)[V]) {
    if constexpr (V == 4) {
        *(float4 *)p = make_float4(o[0], o[1], o[2], o[3]);
    } else if constexpr (V == 2) {
        *(float2 *)p = make_float2(o[0], o[1]);
    } else {
        p[0] = o[0];
    }
}

// Store V consecutive cells of a row to global memory: one vector store when
// all lie inside the grid (gz0 + V <= nz), else one store per inside cell.
template <int V>
__device__ __forceinline__ void stg_row(float *p, const float (&o)[V], int gz0, int nz) {
    if (gz0 + V <= nz) {
        stv<V>(p, o);
    } else {
#pragma unroll
        for (int j = 0; j < V; ++j)
            if (gz0 + j < nz) p[j] = o[j];
    }
}

// E update of V consecutive cells (ez0 .. ez0+V-1) of row ey of plane p, with
// the arithmetic of kernels.py:101-127 cell by cell.  The tile part is stored;
// the +y halo row and the +z halo column (V == 1 call) are only kept in the
// shared-memory ring for the H update.
template <int MAT, bool PACKED, bool CPML, int V>
__device__ __forceinline__ void e_vec(const fdtd_step_args &a, const TmaLayout &L, int ey,
                                      int ez0, int p, int y0, int z0, i64 pbase, int t,
                                      bool store_plane, bool wave_ok, float4 cx,
                                      const float4 *cy_t, const float4 *cz_t,
                                      const unsigned char *stc, const unsigned char *stp,
                                      const float *mtab, float *Ecur, int RE, int REz,
                                      float *__restrict__ En, const float *__restrict__ pe_o,
                                      float *__restrict__ pe_n, i64 cols) {
    const int ny = a.ny, nz = a.nz, pitch = a.pitch_z, TY = L.ty, TZ = L.tz, HZ = L.hz;
    const int gy = y0 + ey, gz0 = z0 + ez0;
    const int c = ey * REz + ez0;
    float r0[V], r1[V], r2[V];
    if (p >= a.nx || gy >= ny || gz0 >= nz) {
#pragma unroll
        for (int j = 0; j < V; ++j) r0[j] = r1[j] = r2[j] = 0.0f;
        stv<V>(Ecur + c, r0);
        stv<V>(Ecur + RE + c, r1);
        stv<V>(Ecur + 2 * RE + c, r2);
        return;
    }
    const float *Hc = (const float *)stc;
    const float *Hp = (const float *)stp;
    const float *Eo = (const float *)(stc + L.off_e);
    const int HS = (TY + 2) * HZ, ES = (TY + 1) * L.ez;
    const int h = (ey + 1) * HZ + ez0 + 4;
    float dx[3][V], dy[3][V], dz[3][V];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
        float hc[V], hp[V], hym[V];
        ldv<V>(Hc + q * HS + h, hc);
        ldv<V>(Hp + q * HS + h, hp);
        ldv<V>(Hc + q * HS + h - HZ, hym);
        float zm = Hc[q * HS + h - 1];
#pragma unroll
        for (int j = 0; j < V; ++j) {
            dx[q][j] = hc[j] - hp[j];
            dy[q][j] = hc[j] - hym[j];
            dz[q][j] = hc[j] - zm;
            zm = hc[j];
        }
    }
    float eo0[V], eo1[V], eo2[V];
    const int e = ey * L.ez + ez0;
    ldv<V>(Eo + e, eo0);
    ldv<V>(Eo + ES + e, eo1);
    ldv<V>(Eo + 2 * ES + e, eo2);
    float ie[V];
    if (MAT == 1) {
        const unsigned char *m = stc + L.off_m + ey * L.mz + ez0;
#pragma unroll
        for (int j = 0; j < V; ++j) ie[j] = mtab[m[j]];
    } else {
        ldv<V>((const float *)(stc + L.off_m) + ey * L.mz + ez0, ie);
    }
    const float courant = a.courant;
    const i64 i0 = pbase + (gy * pitch + gz0);
    const bool own_row = store_plane && ey < TY && ez0 < TZ;
#pragma unroll
    for (int j = 0; j < V; ++j) {
        const int gz = gz0 + j;
        float c0, c1, c2;
        if (CPML) {
            const float4 cy = cy_t[ey], cz = cz_t[ez0 + j];
            const i64 i = i0 + j;
            const bool own = own_row && gz < nz;
            const i64 ix = psi_idx<PACKED>(0, cx.w, i, p, gy, gz, a.nx, ny, nz);
            const i64 iy = psi_idx<PACKED>(1, cy.w, i, p, gy, gz, a.nx, ny, nz);
            const i64 iz = psi_idx<PACKED>(2, cz.w, i, p, gy, gz, a.nx, ny, nz);
            const float dxz = cpml_pp2(dx[2][j], cx, pe_o, pe_n, a.psi_cols, 0, ix, own);
            const float dxy = cpml_pp2(dx[1][j], cx, pe_o, pe_n, a.psi_cols, 1, ix, own);
            const float dyx = cpml_pp2(dy[0][j], cy, pe_o, pe_n, a.psi_cols, 2, iy, own);
            const float dyz = cpml_pp2(dy[2][j], cy, pe_o, pe_n, a.psi_cols, 3, iy, own);
            const float dzy = cpml_pp2(dz[1][j], cz, pe_o, pe_n, a.psi_cols, 4, iz, own);
            const float dzx = cpml_pp2(dz[0][j], cz, pe_o, pe_n, a.psi_cols, 5, iz, own);
            c0 = dyz - dzy;
            c1 = dzx - dxz;
            c2 = dxy - dyx;
        } else {
            c0 = dy[2][j] - dz[1][j];
            c1 = dz[0][j] - dx[2][j];
            c2 = dx[1][j] - dy[0][j];
        }
        float v0 = eo0[j] + (courant * c0) * ie[j];
        float v1 = eo1[j] + (courant * c1) * ie[j];
        float v2 = eo2[j] + (courant * c2) * ie[j];
        if (p == a.source_x && wave_ok && gz < nz) {
            const i64 sidx = (i64)gy * nz + gz;
            const i64 syz = (i64)ny * nz;
            v1 = v1 + ((a.src_h[2 * syz + sidx] * a.waves_h[2 * a.waves_cols + t]) * courant) * ie[j];
            v2 = v2 - ((a.src_h[syz + sidx] * a.waves_h[a.waves_cols + t]) * courant) * ie[j];
        }
        const bool in = gz < nz;
        r0[j] = in ? v0 : 0.0f;
        r1[j] = in ? v1 : 0.0f;
        r2[j] = in ? v2 : 0.0f;
    }
    stv<V>(Ecur + c, r0);
    stv<V>(Ecur + RE + c, r1);
    stv<V>(Ecur + 2 * RE + c, r2);
    if (own_row) {
        stg_row<V>(En + i0, r0, gz0, nz);
        stg_row<V>(En + cols + i0, r1, gz0, nz);
        stg_row<V>(En + 2 * cols + i0, r2, gz0, nz);
    }
}

// H update of V consecutive owned cells of row hy of plane q (kernels.py:128-137).
template <bool PACKED, bool CPML, int V>
__device__ __forceinline__ void h_vec(const fdtd_step_args &a, const TmaLayout &L, int hy,
                                      int hz0, int q, int y0, int z0, i64 qbase, int t,
                                      bool wave_ok, float4 cx, const float4 *cy_t,
                                      const float4 *cz_t, const unsigned char *stq,
                                      const float *Eq, const float *Ep, int RE, int REz,
                                      float *__restrict__ Hn, const float *__restrict__ ph_o,
                                      float *__restrict__ ph_n, i64 cols) {
    const int ny = a.ny, nz = a.nz, pitch = a.pitch_z, TY = L.ty, HZ = L.hz;
    const int gy = y0 + hy, gz0 = z0 + hz0;
    if (gy >= ny || gz0 >= nz) return;
    const int e = hy * REz + hz0;
    float dx[3][V], dy[3][V], dz[3][V];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
        float eq[V], ep[V], eyp[V];
        ldv<V>(Eq + r * RE + e, eq);
        ldv<V>(Ep + r * RE + e, ep);
        ldv<V>(Eq + r * RE + e + REz, eyp);
        const float zlast = Eq[r * RE + e + V];
#pragma unroll
        for (int j = 0; j < V; ++j) {
            const float zp = j + 1 < V ? eq[j + 1 < V ? j + 1 : 0] : zlast;
            dx[r][j] = ep[j] - eq[j];
            dy[r][j] = eyp[j] - eq[j];
            dz[r][j] = zp - eq[j];
        }
    }
    const float *Hq = (const float *)stq;
    const int HS = (TY + 2) * HZ;
    const int h = (hy + 1) * HZ + hz0 + 4;
    float hq0[V], hq1[V], hq2[V];
    ldv<V>(Hq + h, hq0);
    ldv<V>(Hq + HS + h, hq1);
    ldv<V>(Hq + 2 * HS + h, hq2);
    const float courant = a.courant;
    const i64 i0 = qbase + (gy * pitch + gz0);
    float r0[V], r1[V], r2[V];
#pragma unroll
    for (int j = 0; j < V; ++j) {
        const int gz = gz0 + j;
        float c0, c1, c2;
        if (CPML) {
            const float4 cy = cy_t[hy], cz = cz_t[hz0 + j];
            const i64 i = i0 + j;
            const bool own = gz < nz;
            const i64 ix = psi_idx<PACKED>(0, cx.w, i, q, gy, gz, a.nx, ny, nz);
            const i64 iy = psi_idx<PACKED>(1, cy.w, i, q, gy, gz, a.nx, ny, nz);
            const i64 iz = psi_idx<PACKED>(2, cz.w, i, q, gy, gz, a.nx, ny, nz);
            const float dxz = cpml_pp2(dx[2][j], cx, ph_o, ph_n, a.psi_cols, 0, ix, own);
            const float dxy = cpml_pp2(dx[1][j], cx, ph_o, ph_n, a.psi_cols, 1, ix, own);
            const float dyx = cpml_pp2(dy[0][j], cy, ph_o, ph_n, a.psi_cols, 2, iy, own);
            const float dyz = cpml_pp2(dy[2][j], cy, ph_o, ph_n, a.psi_cols, 3, iy, own);
            const float dzy = cpml_pp2(dz[1][j], cz, ph_o, ph_n, a.psi_cols, 4, iz, own);
            const float dzx = cpml_pp2(dz[0][j], cz, ph_o, ph_n, a.psi_cols, 5, iz, own);
            c0 = dyz - dzy;
            c1 = dzx - dxz;
            c2 = dxy - dyx;
        } else {
            c0 = dy[2][j] - dz[1][j];
            c1 = dz[0][j] - dx[2][j];
            c2 = dx[1][j] - dy[0][j];
        }
        float v0 = hq0[j] - courant * c0;
        float v1 = hq1[j] - courant * c1;
        float v2 = hq2[j] - courant * c2;
        if (q == a.source_x && wave_ok && gz < nz) {
            const i64 sidx = (i64)gy * nz + gz;
            const i64 syz = (i64)ny * nz;
            v1 = v1 - (a.src_e[2 * syz + sidx] * a.waves_e[2 * a.waves_cols + t]) * courant;
            v2 = v2 + (a.src_e[syz + sidx] * a.waves_e[a.waves_cols + t]) * courant;
        }
        r0[j] = v0;
        r1[j] = v1;
        r2[j] = v2;
    }
    stg_row<V>(Hn + i0, r0, gz0, nz);
    stg_row<V>(Hn + cols + i0, r1, gz0, nz);
    stg_row<V>(Hn + 2 * cols + i0, r2, gz0, nz);
}

// Threads are laid out (z, y): threadIdx.x is the z offset in the tile
// (blockDim.x == tile_z), threadIdx.y strides over rows, so no index needs a
// division.  The +z halo column of E is computed by threadIdx.x == 0.
template <int MAT, bool PACKED, int V>
__global__ void __launch_bounds__(256, 3)
    tma_step_kernel(const __grid_constant__ TmaMaps maps, const __grid_constant__ TmaParams prm) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const fdtd_step_args &a = prm.a;
    const TmaLayout &L = prm.L;
    const int nx = a.nx, ny = a.ny, nz = a.nz, pitch = a.pitch_z;
    const i64 cols = (i64)nx * ny * pitch;
    const i64 plane_cells = (i64)ny * pitch;
    const int TY = L.ty, TZ = L.tz, S = L.stages;
    const int REz = TZ + 4, RE = (TY + 1) * REz;  // E ring rows padded to 16 B

    uint64_t *bars = (uint64_t *)smem;
    unsigned char *stage0 = smem + L.off_stages;
    float *Es = (float *)(smem + L.off_enew);  // [2][3][RE]
    float *mtab = (float *)(smem + L.off_mtab);
    float4 *coef = (float4 *)(smem + L.off_coef);  // ce_y[TY+1] ce_z[TZ+1] ch_y[TY+1] ch_z[TZ+1]
    float4 *cey = coef, *cez = coef + (TY + 1), *chy = cez + (TZ + 1), *chz = chy + (TY + 1);

    const int tiles_z = (nz + TZ - 1) / TZ;
    const int tiles_y = (ny + TY - 1) / TY;
    int b = blockIdx.x;
    const int tzi = b % tiles_z;
    b /= tiles_z;
    const int tyi = b % tiles_y;
    const int chunk = b / tiles_y;
    const int y0 = tyi * TY, z0 = tzi * TZ;
    const int xa = chunk * a.chunk_x;
    if (xa >= nx) return;
    const int xb = min(xa + a.chunk_x, nx);
    const int last = xb - xa + 1;  // planes k = 0..last are xa-1 .. xb

    const int t = a.step[0];
    const int s = t & 1;
    const CUtensorMap *mapE = &maps.E[s];
    const CUtensorMap *mapH = &maps.H[s];
    float *__restrict__ En = a.E[s ^ 1];
    float *__restrict__ Hn = a.H[s ^ 1];
    const float *__restrict__ pe_o = a.psi_e[s];
    float *__restrict__ pe_n = a.psi_e[s ^ 1];
    const float *__restrict__ ph_o = a.psi_h[s];
    float *__restrict__ ph_n = a.psi_h[s ^ 1];
    const float4 *__restrict__ ce = (const float4 *)a.coeff_e;
    const float4 *__restrict__ ch = (const float4 *)a.coeff_h;
    const int clen = a.clen;
    const int tx = threadIdx.x, tyv = threadIdx.y, BY = blockDim.y;
    const int tid = tyv * blockDim.x + tx, nth = blockDim.x * blockDim.y;
    const bool wave_ok = t >= 0 && t < a.waves_cols;

    auto stage_ptr = [&](int k) { return stage0 + (size_t)(k % S) * L.stage_bytes; };
    auto issue = [&](int k) {
        unsigned char *st = stage_ptr(k);
        uint64_t *bar = bars + (k % S);
        const int p = xa - 1 + k;
        mbar_expect_tx(bar, L.tx_bytes);
        tma_load_4d(st, mapH, z0 - 4, y0 - 1, p, 0, bar);
        tma_load_4d(st + L.off_e, mapE, z0, y0, p, 0, bar);
        tma_load_3d(st + L.off_m, &maps.M, z0, y0, p, bar);
    };

    if (tid == 0) {
        for (int j = 0; j < S; ++j) mbar_init(bars + j, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (MAT == 1) {
        for (int j = tid; j < 256; j += nth)
            mtab[j] = j < a.material_count ? a.material_table[j] : 0.0f;
    }
    // tile coefficient tables (positions past the grid read as identity)
    bool act = false;
    const float4 ident = make_float4(0.f, 1.f, 1.f, 0.f);
    for (int j = tid; j <= TY; j += nth) {
        const int gy = y0 + j;
        const float4 e = gy < ny ? __ldg(ce + clen + gy) : ident;
        const float4 h = gy < ny ? __ldg(ch + clen + gy) : ident;
        cey[j] = e;
        chy[j] = h;
        act |= (cpml_active(e) && j <= TY) || (cpml_active(h) && j < TY);
    }
    const bool ycp = __syncthreads_or(act);
    act = false;
    for (int j = tid; j <= TZ; j += nth) {
        const int gz = z0 + j;
        const float4 e = gz < nz ? __ldg(ce + 2 * clen + gz) : ident;
        const float4 h = gz < nz ? __ldg(ch + 2 * clen + gz) : ident;
        cez[j] = e;
        chz[j] = h;
        act |= (cpml_active(e) && j <= TZ) || (cpml_active(h) && j < TZ);
    }
    const bool yzcp = __syncthreads_or(act) || ycp;

    int issued;  // highest plane index whose load was issued
    if (tid == 0) {
        for (int k = 0; k <= last && k < S; ++k) issue(k);
    }
    issued = min(last, S - 1);

    const long limit = 1L << 24;
    bool timed_out = false;
    int done = -1;  // highest plane index this thread has seen complete
    if (mbar_wait_bounded(bars, 0, limit))
        done = 0;
    else
        timed_out = true;

    int k = 1;
    for (; k <= last; ++k) {
        const int p = xa - 1 + k;
        if (!timed_out) {
            if (mbar_wait_bounded(bars + (k % S), (k / S) & 1, limit))
                done = k;
            else
                timed_out = true;
        }
        const unsigned char *stc = stage_ptr(k);
        const unsigned char *stp = stage_ptr(k - 1);
        float *Ecur = Es + (k & 1) * 3 * RE;
        // ---- E update on the tile and its +y/+z halo ----
        if (!timed_out) {
            const bool store_plane = p < xb;
            const float4 cx = p < nx ? __ldg(ce + p) : ident;
            const bool cp = yzcp || cpml_active(cx);
            const i64 pbase = (i64)p * plane_cells;
            const int ez0 = tx * V;
            for (int ey = tyv; ey <= TY; ey += BY) {
#define ECELL(CP, W, EZ)                                                                        \
    e_vec<MAT, PACKED, CP, W>(a, L, ey, EZ, p, y0, z0, pbase, t, store_plane, wave_ok, cx, cey, \
                              cez, stc, stp, mtab, Ecur, RE, REz, En, pe_o, pe_n, cols)
                if (cp) {
                    ECELL(true, V, ez0);
                    if (tx == 0) ECELL(true, 1, TZ);
                } else {
                    ECELL(false, V, ez0);
                    if (tx == 0) ECELL(false, 1, TZ);
                }
#undef ECELL
            }
        }
        if (__syncthreads_or(timed_out)) {
            timed_out = true;
            break;
        }
        // ---- H update at plane q = p - 1 (needs E(q) and E(p)) ----
        const int q = p - 1;
        if (q >= xa) {
            const float *Eq = Es + ((k - 1) & 1) * 3 * RE;
            const float4 cx = __ldg(ch + q);
            const bool cp = yzcp || cpml_active(cx);
            const i64 qbase = (i64)q * plane_cells;
            for (int hy = tyv; hy < TY; hy += BY) {
                if (cp)
                    h_vec<PACKED, true, V>(a, L, hy, tx * V, q, y0, z0, qbase, t, wave_ok, cx, chy,
                                           chz, stp, Eq, Ecur, RE, REz, Hn, ph_o, ph_n, cols);
                else
                    h_vec<PACKED, false, V>(a, L, hy, tx * V, q, y0, z0, qbase, t, wave_ok, cx,
                                            chy, chz, stp, Eq, Ecur, RE, REz, Hn, ph_o, ph_n,
                                            cols);
            }
        }
        __syncthreads();
        // stage of plane k-1 is free: refill it with plane k-1+S
        if (k - 1 + S <= last) {
            if (tid == 0) issue(k - 1 + S);
            issued = k - 1 + S;
        }
    }
    if (timed_out) {
        if (tid == 0) {
            if (a.error) atomicExch(a.error, 1);
            // drain this block's copies still in flight before shared memory is released
            for (int j = done + 1; j <= issued; ++j)
                mbar_wait_bounded(bars + (j % S), (j / S) & 1, limit);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// host side

static inline size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

TmaLayout tma_layout(int ty, int tz, int stages, int mat) {
    TmaLayout L;
    L.ty = ty;
    L.tz = tz;
    L.stages = stages;
    L.hz = tz + 8;
    L.ez = tz + 4;
    L.mz = mat == 1 ? tz + 16 : tz + 4;
    size_t hb = (size_t)3 * (ty + 2) * L.hz * 4;
    size_t eb = (size_t)3 * (ty + 1) * L.ez * 4;
    size_t mb = (size_t)(ty + 1) * L.mz * (mat == 1 ? 1 : 4);
    L.off_e = (int)align_up(hb, 128);
    L.off_m = (int)(L.off_e + align_up(eb, 128));
    L.stage_bytes = (int)(L.off_m + align_up(mb, 128));
    L.tx_bytes = (unsigned)(hb + eb + mb);
    L.off_stages = 128;
    L.off_enew = (int)(L.off_stages + (size_t)stages * L.stage_bytes);
    size_t enew = (size_t)2 * 3 * (ty + 1) * (tz + 4) * 4;
    L.off_coef = (int)align_up(L.off_enew + enew, 16);
    size_t coef = (size_t)(2 * (ty + 1) + 2 * (tz + 1)) * 16;
    L.off_mtab = (int)align_up(L.off_coef + coef, 16);
    L.smem_bytes = (int)(L.off_mtab + (mat == 1 ? 256 * 4 : 0));
    return L;
}

bool tma_eligible(const fdtd_step_args &a) {
    auto al16 = [](const void *p) { return ((uintptr_t)p & 15) == 0; };
    if (a.pitch_z % 4 != 0) return false;
    if (a.material_kind == 1 && a.material_pitch % 16 != 0) return false;
    for (int j = 0; j < 2; ++j)
        if (!al16(a.E[j]) || !al16(a.H[j])) return false;
    if (a.material_kind == 1 ? !al16(a.material) : !al16(a.inv_eps)) return false;
    return true;
}

int launch_tma(const fdtd_step_args &a, cudaStream_t stream) {
    int rc = get_encoder();
    if (rc) return rc;
    const int ty = a.tile_y, tz = a.tile_z;
    // Every box must start on a 16-byte boundary in z: z0 = k * tile_z floats
    // (and z0 - 4 for the H halo box) needs tile_z % 4 == 0; the uint8
    // material box starting at z0 bytes needs tile_z % 16 == 0.
    if (tz % 4 != 0 || (a.material_kind == 1 && tz % 16 != 0) || tz > 64 || ty + 2 > 256) {
        set_error("fdtd_step_fused: TMA path needs tile_z %% 4 == 0 (%% 16 with uint8 "
                  "material), tile_z <= 64 and boxes <= 256");
        return FDTD_ERR_ARG;
    }
    int stages = a.stages > 0 ? a.stages : 4;
    if (stages < 2 || stages > 8) {
        set_error("fdtd_step_fused: stages must be 2..8");
        return FDTD_ERR_ARG;
    }
    TmaLayout L = tma_layout(ty, tz, stages, a.material_kind);
    while (L.smem_bytes > 200 * 1024 && stages > 2) L = tma_layout(ty, tz, --stages, a.material_kind);
    if (L.smem_bytes > 200 * 1024) {
        set_error("fdtd_step_fused: tile %dx%d needs %d bytes of shared memory", ty, tz, L.smem_bytes);
        return FDTD_ERR_ARG;
    }
    TmaMaps maps;
    const cuuint64_t nz = a.nz, ny = a.ny, nx = a.nx, pz = a.pitch_z;
    cuuint64_t fdims[4] = {nz, ny, nx, 3};
    cuuint64_t fstr[3] = {pz * 4, pz * ny * 4, pz * ny * nx * 4};
    cuuint32_t hbox[4] = {(cuuint32_t)L.hz, (cuuint32_t)(ty + 2), 1, 3};
    cuuint32_t ebox[4] = {(cuuint32_t)L.ez, (cuuint32_t)(ty + 1), 1, 3};
    for (int j = 0; j < 2; ++j) {
        if ((rc = encode(&maps.H[j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.H[j], fdims, fstr, hbox)))
            return rc;
        if ((rc = encode(&maps.E[j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.E[j], fdims, fstr, ebox)))
            return rc;
    }
    if (a.material_kind == 1) {
        const cuuint64_t mp = a.material_pitch;
        cuuint64_t mdims[3] = {nz, ny, nx};
        cuuint64_t mstr[2] = {mp, mp * ny};
        cuuint32_t mbox[3] = {(cuuint32_t)L.mz, (cuuint32_t)(ty + 1), 1};
        if ((rc = encode(&maps.M, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, a.material, mdims, mstr, mbox)))
            return rc;
    } else {
        cuuint64_t mdims[3] = {nz, ny, nx};
        cuuint64_t mstr[2] = {pz * 4, pz * ny * 4};
        cuuint32_t mbox[3] = {(cuuint32_t)L.mz, (cuuint32_t)(ty + 1), 1};
        if ((rc = encode(&maps.M, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, a.inv_eps, mdims, mstr, mbox)))
            return rc;
    }
    TmaParams prm;
    prm.a = a;
    prm.L = L;
    const int tiles = ((a.ny + ty - 1) / ty) * ((a.nz + tz - 1) / tz);
    const int chunks = (a.nx + a.chunk_x - 1) / a.chunk_x;
    dim3 grid((unsigned)(tiles * chunks));
    int V = a.vector > 0 ? a.vector : (tz % 4 == 0 && tz / 4 >= 8 ? 4 : (tz % 2 == 0 ? 2 : 1));
    if (tz % V != 0 || (V != 1 && V != 2 && V != 4)) {
        set_error("fdtd_step_fused: vector width %d must be 1, 2 or 4 and divide tile_z", V);
        return FDTD_ERR_ARG;
    }
    const int lanes = tz / V;
    int by = 256 / lanes;
    if (by > ty + 1) by = ty + 1;
    if (by < 1) by = 1;
    dim3 threads((unsigned)lanes, (unsigned)by);
#define LAUNCH(M, P, W)                                                                      \
    do {                                                                                     \
        cudaFuncSetAttribute(tma_step_kernel<M, P, W>,                                       \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L.smem_bytes);      \
        tma_step_kernel<M, P, W><<<grid, threads, L.smem_bytes, stream>>>(maps, prm);        \
    } while (0)
#define LAUNCH_V(M, P)                                                                       \
    do {                                                                                     \
        if (V == 4) LAUNCH(M, P, 4);                                                         \
        else if (V == 2) LAUNCH(M, P, 2);                                                    \
        else LAUNCH(M, P, 1);                                                                \
    } while (0)
    if (a.material_kind == 1) {
        if (a.packed) LAUNCH_V(1, true); else LAUNCH_V(1, false);
    } else {
        if (a.packed) LAUNCH_V(0, true); else LAUNCH_V(0, false);
    }
#undef LAUNCH_V
#undef LAUNCH
    return launch_status("fdtd_step_fused (TMA)");
}

}  // namespace wfb
