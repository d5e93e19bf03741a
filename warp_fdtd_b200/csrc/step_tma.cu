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

namespace wfb {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: false if the phase did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity, long limit) {
    for (long it = 0; it < limit; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if (it > 64) __nanosleep(32);
    }
    return false;
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, int c3, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1,
                                            int c2, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes "
        "[%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}

struct TmaMaps {
    CUtensorMap E[2];  // fields, 4-D (z, y, x, component)
    CUtensorMap H[2];
    CUtensorMap M;     // material: 3-D uint8 or float32 (z, y, x)
};

struct TmaParams {
    fdtd_step_args a;
    TmaLayout L;
};

template <int MAT, bool PACKED>
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

template <int MAT, bool PACKED>
__global__ void __launch_bounds__(256, 2)
    tma_step_kernel(const __grid_constant__ TmaMaps maps, const __grid_constant__ TmaParams prm) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const fdtd_step_args &a = prm.a;
    const TmaLayout &L = prm.L;
    const int nx = a.nx, ny = a.ny, nz = a.nz, pitch = a.pitch_z;
    const i64 cols = (i64)nx * ny * pitch;
    const int TY = L.ty, TZ = L.tz, S = L.stages;
    const int HZ = L.hz, EZ = L.ez, MZ = L.mz;        // smem row lengths of the boxes
    const int HS = (TY + 2) * HZ, ES = (TY + 1) * EZ;  // component strides in a stage
    const int REz = TZ + 1, RE = (TY + 1) * REz;       // E-new ring geometry

    uint64_t *bars = (uint64_t *)smem;
    unsigned char *stage0 = smem + L.off_stages;
    float *Es = (float *)(smem + L.off_enew);  // [2][3][RE]
    float *mtab = (float *)(smem + L.off_mtab);

    const int tiles_z = (nz + TZ - 1) / TZ;
    const int tiles_y = (ny + TY - 1) / TY;
    int b = blockIdx.x;
    const int tz = b % tiles_z;
    b /= tiles_z;
    const int ty = b % tiles_y;
    const int chunk = b / tiles_y;
    const int y0 = ty * TY, z0 = tz * TZ;
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
    const float courant = a.courant;
    const int tid = threadIdx.x, nth = blockDim.x;
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
    __syncthreads();
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
        const float *Hc = (const float *)stc;
        const float *Hp = (const float *)stp;
        const float *Eo = (const float *)(stc + L.off_e);
        float *Ecur = Es + (k & 1) * 3 * RE;
        // ---- E update on the tile and its +y/+z halo ----
        if (!timed_out) {
            const bool store_plane = p < xb;
            const float4 cx = p < nx ? __ldg(ce + p) : make_float4(0.f, 1.f, 1.f, 0.f);
            for (int c = tid; c < RE; c += nth) {
                const int ey = c / REz, ez = c - ey * REz;
                const int gy = y0 + ey, gz = z0 + ez;
                if (p >= nx || gy >= ny || gz >= nz) {
                    Ecur[c] = 0.0f;
                    Ecur[RE + c] = 0.0f;
                    Ecur[2 * RE + c] = 0.0f;
                    continue;
                }
                const bool own = store_plane && ey < TY && ez < TZ;
                const int h = (ey + 1) * HZ + ez + 4;
                float dx[3], dy[3], dz[3];
#pragma unroll
                for (int q = 0; q < 3; ++q) {
                    const float v = Hc[q * HS + h];
                    dx[q] = v - Hp[q * HS + h];
                    dy[q] = v - Hc[q * HS + h - HZ];
                    dz[q] = v - Hc[q * HS + h - 1];
                }
                const i64 i = flat(p, gy, gz, ny, pitch);
                const float4 cy = __ldg(ce + clen + gy);
                const float4 cz = __ldg(ce + 2 * clen + gz);
                const i64 ix = psi_idx<PACKED>(0, cx.w, i, p, gy, gz, nx, ny, nz);
                const i64 iy = psi_idx<PACKED>(1, cy.w, i, p, gy, gz, nx, ny, nz);
                const i64 iz = psi_idx<PACKED>(2, cz.w, i, p, gy, gz, nx, ny, nz);
                const float dxz = cpml_pp2<MAT, PACKED>(dx[2], cx, pe_o, pe_n, a.psi_cols, 0, ix, own);
                const float dxy = cpml_pp2<MAT, PACKED>(dx[1], cx, pe_o, pe_n, a.psi_cols, 1, ix, own);
                const float dyx = cpml_pp2<MAT, PACKED>(dy[0], cy, pe_o, pe_n, a.psi_cols, 2, iy, own);
                const float dyz = cpml_pp2<MAT, PACKED>(dy[2], cy, pe_o, pe_n, a.psi_cols, 3, iy, own);
                const float dzy = cpml_pp2<MAT, PACKED>(dz[1], cz, pe_o, pe_n, a.psi_cols, 4, iz, own);
                const float dzx = cpml_pp2<MAT, PACKED>(dz[0], cz, pe_o, pe_n, a.psi_cols, 5, iz, own);
                float ie;
                if (MAT == 1)
                    ie = mtab[stc[L.off_m + ey * MZ + ez]];
                else
                    ie = ((const float *)(stc + L.off_m))[ey * MZ + ez];
                const int e = ey * EZ + ez;
                float v0 = Eo[e] + (courant * (dyz - dzy)) * ie;
                float v1 = Eo[ES + e] + (courant * (dzx - dxz)) * ie;
                float v2 = Eo[2 * ES + e] + (courant * (dxy - dyx)) * ie;
                if (p == a.source_x && wave_ok) {
                    const i64 sidx = (i64)gy * nz + gz;
                    const i64 syz = (i64)ny * nz;
                    v1 = v1 + ((a.src_h[2 * syz + sidx] * a.waves_h[2 * a.waves_cols + t]) * courant) * ie;
                    v2 = v2 - ((a.src_h[syz + sidx] * a.waves_h[a.waves_cols + t]) * courant) * ie;
                }
                Ecur[c] = v0;
                Ecur[RE + c] = v1;
                Ecur[2 * RE + c] = v2;
                if (own) {
                    En[i] = v0;
                    En[cols + i] = v1;
                    En[2 * cols + i] = v2;
                }
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
            const float *Ep = Ecur;
            const float *Hq = Hp;
            const float4 cx = __ldg(ch + q);
            const int TT = TY * TZ;
            for (int c = tid; c < TT; c += nth) {
                const int hy = c / TZ, hz = c - hy * TZ;
                const int gy = y0 + hy, gz = z0 + hz;
                if (gy >= ny || gz >= nz) continue;
                const int e = hy * REz + hz;
                float dx[3], dy[3], dz[3];
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    const float v = Eq[r * RE + e];
                    dx[r] = Ep[r * RE + e] - v;
                    dy[r] = Eq[r * RE + e + REz] - v;
                    dz[r] = Eq[r * RE + e + 1] - v;
                }
                const i64 i = flat(q, gy, gz, ny, pitch);
                const float4 cy = __ldg(ch + clen + gy);
                const float4 cz = __ldg(ch + 2 * clen + gz);
                const i64 ix = psi_idx<PACKED>(0, cx.w, i, q, gy, gz, nx, ny, nz);
                const i64 iy = psi_idx<PACKED>(1, cy.w, i, q, gy, gz, nx, ny, nz);
                const i64 iz = psi_idx<PACKED>(2, cz.w, i, q, gy, gz, nx, ny, nz);
                const float dxz = cpml_pp2<MAT, PACKED>(dx[2], cx, ph_o, ph_n, a.psi_cols, 0, ix, true);
                const float dxy = cpml_pp2<MAT, PACKED>(dx[1], cx, ph_o, ph_n, a.psi_cols, 1, ix, true);
                const float dyx = cpml_pp2<MAT, PACKED>(dy[0], cy, ph_o, ph_n, a.psi_cols, 2, iy, true);
                const float dyz = cpml_pp2<MAT, PACKED>(dy[2], cy, ph_o, ph_n, a.psi_cols, 3, iy, true);
                const float dzy = cpml_pp2<MAT, PACKED>(dz[1], cz, ph_o, ph_n, a.psi_cols, 4, iz, true);
                const float dzx = cpml_pp2<MAT, PACKED>(dz[0], cz, ph_o, ph_n, a.psi_cols, 5, iz, true);
                const int h = (hy + 1) * HZ + hz + 4;
                float v0 = Hq[h] - courant * (dyz - dzy);
                float v1 = Hq[HS + h] - courant * (dzx - dxz);
                float v2 = Hq[2 * HS + h] - courant * (dxy - dyx);
                if (q == a.source_x && wave_ok) {
                    const i64 sidx = (i64)gy * nz + gz;
                    const i64 syz = (i64)ny * nz;
                    v1 = v1 - (a.src_e[2 * syz + sidx] * a.waves_e[2 * a.waves_cols + t]) * courant;
                    v2 = v2 + (a.src_e[syz + sidx] * a.waves_e[a.waves_cols + t]) * courant;
                }
                Hn[i] = v0;
                Hn[cols + i] = v1;
                Hn[2 * cols + i] = v2;
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

static PFN_cuTensorMapEncodeTiled_v12000 g_encode = nullptr;

static int get_encoder() {
    if (g_encode) return 0;
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    cudaError_t err = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (err != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
        set_error("fdtd_step_fused: cuTensorMapEncodeTiled unavailable");
        return FDTD_ERR_CUDA;
    }
    g_encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    return 0;
}

static int encode(CUtensorMap *map, CUtensorMapDataType dt, int rank, const void *base,
                  const cuuint64_t *dims, const cuuint64_t *strides, const cuuint32_t *box) {
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = g_encode(map, dt, rank, const_cast<void *>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("fdtd_step_fused: cuTensorMapEncodeTiled failed (%d)", (int)r);
        return FDTD_ERR_CUDA;
    }
    return 0;
}

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
    size_t enew = (size_t)2 * 3 * (ty + 1) * (tz + 1) * 4;
    L.off_mtab = (int)align_up(L.off_enew + enew, 16);
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
    if (tz % 4 != 0 || (a.material_kind == 1 && tz % 16 != 0) || tz + 16 > 256 || ty + 2 > 256) {
        set_error("fdtd_step_fused: TMA path needs tile_z %% 4 == 0 (%% 16 with uint8 "
                  "material) and boxes <= 256");
        return FDTD_ERR_ARG;
    }
    int stages = 4;
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
    const int threads = 256;
#define LAUNCH(M, P)                                                                         \
    do {                                                                                     \
        cudaFuncSetAttribute(tma_step_kernel<M, P>,                                          \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, L.smem_bytes);      \
        tma_step_kernel<M, P><<<grid, threads, L.smem_bytes, stream>>>(maps, prm);           \
    } while (0)
    if (a.material_kind == 1) {
        if (a.packed) LAUNCH(1, true); else LAUNCH(1, false);
    } else {
        if (a.packed) LAUNCH(0, true); else LAUNCH(0, false);
    }
#undef LAUNCH
    return launch_status("fdtd_step_fused (TMA)");
}

}  // namespace wfb
