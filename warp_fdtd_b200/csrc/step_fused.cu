// One fused Yee leapfrog step (E then H) over ping-pong buffers.
//
// This replaces the reference's two full-grid sweeps per step (update_e then
// update_h, warp_fdtd/kernels.py:77-148, launched by solver.py:194-237) with
// one sweep that reads E(n), H(n-1/2) once and writes E(n+1), H(n+1/2) once:
// 48 B of field traffic plus the material byte(s) per cell-step.
//
// Decomposition: a block owns a (tile_y x tile_z) column of the y-z plane and
// a chunk of x planes [xa, xb), and marches along x.  At plane p it
//   1. stages H(p) on the tile plus a one-cell -y/-z halo and E(p) on the
//      tile plus a +y/+z halo in shared memory,
//   2. computes E(p+1/2 step) on the tile and its +y/+z halo (the halo values
//      are recomputed redundantly; only tile cells are stored),
//   3. computes H at plane p-1 from E(p-1), E(p) held in shared memory.
// The x neighbour of E needs H(p-1) (kept from the previous iteration); the
// x neighbour of H needs E(p), computed one plane ahead.  At the chunk's end
// plane xb the block recomputes E(xb) without storing it.  Because halo cells
// are recomputed from the *old* fields and CPML state, every input is read
// from the buffers of parity s = step & 1 and every output goes to parity
// s ^ 1, so blocks never race on in-place data.
//
// Arithmetic follows kernels.py:101-140 operation by operation (built with
// --fmad=false), so a step is bitwise identical to the kernel-level
// update_e + update_h pair.
#include "common.cuh"
#include "step_internal.h"

namespace wfb {

struct StepCtx {
    int TY, TZ, RHz, RH, REz, RE;
    int y0, z0;
};

// kernels.py:29-74: CPML-filtered difference.  psi is read from the old
// buffer and, for cells this block owns, the new value is written to the new
// buffer (the reference updates it in place).
template <bool PACKED>
__device__ __forceinline__ float cpml_pp(float d, float4 c, const float *__restrict__ psi_o,
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
__device__ __forceinline__ i64 psi_index(int axis, float rank, i64 i, int x, int y, int z,
                                         int nx, int ny, int nz) {
    if (!PACKED) return i;
    i64 plane = (i64)(int)rank;
    if (axis == 0) return plane * ny * nz + (i64)y * nz + z;
    if (axis == 1) return plane * nx * nz + (i64)x * nz + z;
    return plane * nx * ny + (i64)x * ny + y;
}

template <int MAT, bool PACKED>
__global__ void __launch_bounds__(512) fused_step_kernel(const fdtd_step_args a) {
    extern __shared__ float smem[];
    const int nx = a.nx, ny = a.ny, nz = a.nz, pitch = a.pitch_z;
    const i64 n = (i64)nx * ny * pitch;
    const int TY = a.tile_y, TZ = a.tile_z;
    const int RHz = TZ + 2, RH = (TY + 2) * RHz;
    const int REz = TZ + 1, RE = (TY + 1) * REz;
    float *Hs = smem;             // [2][3][RH]
    float *Es = Hs + 6 * RH;      // [2][3][RE]
    float *mtab = Es + 6 * RE;    // [256] when MAT == 1

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

    const int t = a.step[0];
    const int s = t & 1;
    const float *__restrict__ Eo = a.E[s];
    float *__restrict__ En = a.E[s ^ 1];
    const float *__restrict__ Ho = a.H[s];
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

    if (MAT == 1) {
        for (int k = tid; k < 256; k += nth)
            mtab[k] = k < a.material_count ? a.material_table[k] : 0.0f;
    }

    // Stage H(p) over the tile with a -y/-z halo; zero outside the grid.
    auto load_h = [&](int p, int buf) {
        float *dst = Hs + buf * 3 * RH;
        for (int k = tid; k < RH; k += nth) {
            int ly = k / RHz, lz = k - ly * RHz;
            int gy = y0 - 1 + ly, gz = z0 - 1 + lz;
            float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
            if (p >= 0 && p < nx && gy >= 0 && gy < ny && gz >= 0 && gz < nz) {
                i64 i = flat(p, gy, gz, ny, pitch);
                v0 = Ho[i];
                v1 = Ho[n + i];
                v2 = Ho[2 * n + i];
            }
            dst[k] = v0;
            dst[RH + k] = v1;
            dst[2 * RH + k] = v2;
        }
    };

    load_h(xa - 1, (xa - 1) & 1);

    for (int p = xa; p <= xb; ++p) {
        const int cur = p & 1, prv = cur ^ 1;
        __syncthreads();
        // 1. stage H(p) and E(p)
        if (p < nx) {
            load_h(p, cur);
            float *dst = Es + cur * 3 * RE;
            for (int k = tid; k < RE; k += nth) {
                int ey = k / REz, ez = k - ey * REz;
                int gy = y0 + ey, gz = z0 + ez;
                float v0 = 0.0f, v1 = 0.0f, v2 = 0.0f;
                if (gy < ny && gz < nz) {
                    i64 i = flat(p, gy, gz, ny, pitch);
                    v0 = Eo[i];
                    v1 = Eo[n + i];
                    v2 = Eo[2 * n + i];
                }
                dst[k] = v0;
                dst[RE + k] = v1;
                dst[2 * RE + k] = v2;
            }
        }
        __syncthreads();
        // 2. E update on the tile and its +y/+z halo
        {
            float *E = Es + cur * 3 * RE;
            const float *Hc = Hs + cur * 3 * RH;
            const float *Hp = Hs + prv * 3 * RH;
            const bool store_plane = p < xb;
            const float4 cx = p < nx ? __ldg(ce + p) : make_float4(0.f, 1.f, 1.f, 0.f);
            for (int k = tid; k < RE; k += nth) {
                int ey = k / REz, ez = k - ey * REz;
                int gy = y0 + ey, gz = z0 + ez;
                if (p >= nx || gy >= ny || gz >= nz) {
                    E[k] = 0.0f;
                    E[RE + k] = 0.0f;
                    E[2 * RE + k] = 0.0f;
                    continue;
                }
                const bool own = store_plane && ey < TY && ez < TZ;
                const int hc = (ey + 1) * RHz + ez + 1;
                float dx[3], dy[3], dz[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    float v = Hc[c * RH + hc];
                    dx[c] = v - Hp[c * RH + hc];
                    dy[c] = v - Hc[c * RH + hc - RHz];
                    dz[c] = v - Hc[c * RH + hc - 1];
                }
                const i64 i = flat(p, gy, gz, ny, pitch);
                const float4 cy = __ldg(ce + clen + gy);
                const float4 cz = __ldg(ce + 2 * clen + gz);
                const i64 ix = psi_index<PACKED>(0, cx.w, i, p, gy, gz, nx, ny, nz);
                const i64 iy = psi_index<PACKED>(1, cy.w, i, p, gy, gz, nx, ny, nz);
                const i64 iz = psi_index<PACKED>(2, cz.w, i, p, gy, gz, nx, ny, nz);
                float dxz = cpml_pp<PACKED>(dx[2], cx, pe_o, pe_n, a.psi_cols, 0, ix, own);
                float dxy = cpml_pp<PACKED>(dx[1], cx, pe_o, pe_n, a.psi_cols, 1, ix, own);
                float dyx = cpml_pp<PACKED>(dy[0], cy, pe_o, pe_n, a.psi_cols, 2, iy, own);
                float dyz = cpml_pp<PACKED>(dy[2], cy, pe_o, pe_n, a.psi_cols, 3, iy, own);
                float dzy = cpml_pp<PACKED>(dz[1], cz, pe_o, pe_n, a.psi_cols, 4, iz, own);
                float dzx = cpml_pp<PACKED>(dz[0], cz, pe_o, pe_n, a.psi_cols, 5, iz, own);
                float curl0 = dyz - dzy, curl1 = dzx - dxz, curl2 = dxy - dyx;
                float ie;
                if (MAT == 1)
                    ie = mtab[a.material[flat(p, gy, gz, ny, a.material_pitch)]];
                else
                    ie = __ldg(a.inv_eps + i);
                float v0 = E[k] + (courant * curl0) * ie;
                float v1 = E[RE + k] + (courant * curl1) * ie;
                float v2 = E[2 * RE + k] + (courant * curl2) * ie;
                if (p == a.source_x && t < a.waves_cols) {
                    const i64 sidx = (i64)gy * nz + gz;
                    const i64 syz = (i64)ny * nz;
                    v1 = v1 + ((a.src_h[2 * syz + sidx] * a.waves_h[2 * a.waves_cols + t]) * courant) * ie;
                    v2 = v2 - ((a.src_h[syz + sidx] * a.waves_h[a.waves_cols + t]) * courant) * ie;
                }
                E[k] = v0;
                E[RE + k] = v1;
                E[2 * RE + k] = v2;
                if (own) {
                    En[i] = v0;
                    En[n + i] = v1;
                    En[2 * n + i] = v2;
                }
            }
        }
        __syncthreads();
        // 3. H update at plane q = p - 1
        const int q = p - 1;
        if (q >= xa) {
            const float *Eq = Es + prv * 3 * RE;
            const float *Ep = Es + cur * 3 * RE;
            const float *Hq = Hs + prv * 3 * RH;
            const float4 cx = __ldg(ch + q);
            const int TT = TY * TZ;
            for (int k = tid; k < TT; k += nth) {
                int hy = k / TZ, hz = k - hy * TZ;
                int gy = y0 + hy, gz = z0 + hz;
                if (gy >= ny || gz >= nz) continue;
                const int e = hy * REz + hz;
                float dx[3], dy[3], dz[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    float v = Eq[c * RE + e];
                    dx[c] = Ep[c * RE + e] - v;
                    dy[c] = Eq[c * RE + e + REz] - v;
                    dz[c] = Eq[c * RE + e + 1] - v;
                }
                const i64 i = flat(q, gy, gz, ny, pitch);
                const float4 cy = __ldg(ch + clen + gy);
                const float4 cz = __ldg(ch + 2 * clen + gz);
                const i64 ix = psi_index<PACKED>(0, cx.w, i, q, gy, gz, nx, ny, nz);
                const i64 iy = psi_index<PACKED>(1, cy.w, i, q, gy, gz, nx, ny, nz);
                const i64 iz = psi_index<PACKED>(2, cz.w, i, q, gy, gz, nx, ny, nz);
                float dxz = cpml_pp<PACKED>(dx[2], cx, ph_o, ph_n, a.psi_cols, 0, ix, true);
                float dxy = cpml_pp<PACKED>(dx[1], cx, ph_o, ph_n, a.psi_cols, 1, ix, true);
                float dyx = cpml_pp<PACKED>(dy[0], cy, ph_o, ph_n, a.psi_cols, 2, iy, true);
                float dyz = cpml_pp<PACKED>(dy[2], cy, ph_o, ph_n, a.psi_cols, 3, iy, true);
                float dzy = cpml_pp<PACKED>(dz[1], cz, ph_o, ph_n, a.psi_cols, 4, iz, true);
                float dzx = cpml_pp<PACKED>(dz[0], cz, ph_o, ph_n, a.psi_cols, 5, iz, true);
                const int hcell = (hy + 1) * RHz + hz + 1;
                float v0 = Hq[hcell] - courant * (dyz - dzy);
                float v1 = Hq[RH + hcell] - courant * (dzx - dxz);
                float v2 = Hq[2 * RH + hcell] - courant * (dxy - dyx);
                if (q == a.source_x && t < a.waves_cols) {
                    const i64 sidx = (i64)gy * nz + gz;
                    const i64 syz = (i64)ny * nz;
                    v1 = v1 - (a.src_e[2 * syz + sidx] * a.waves_e[2 * a.waves_cols + t]) * courant;
                    v2 = v2 + (a.src_e[syz + sidx] * a.waves_e[a.waves_cols + t]) * courant;
                }
                Hn[i] = v0;
                Hn[n + i] = v1;
                Hn[2 * n + i] = v2;
            }
        }
    }
}

static size_t smem_bytes(int TY, int TZ, int mat) {
    size_t RH = (size_t)(TY + 2) * (TZ + 2), RE = (size_t)(TY + 1) * (TZ + 1);
    return (6 * RH + 6 * RE + (mat == 1 ? 256 : 0)) * sizeof(float);
}

}  // namespace wfb

using namespace wfb;

// Default TMA tile: z extent a multiple of 4 that wastes the fewest cells of
// nz (ties to the size nearest 48), y extent likewise around 8-12 rows.
static int pick_tile(int n, const int *cands, int count) {
    int best = cands[0], waste_best = 1 << 30;
    for (int j = 0; j < count; ++j) {
        int c = cands[j];
        int waste = (n + c - 1) / c * c - n;
        if (waste < waste_best) {
            best = c;
            waste_best = waste;
        }
    }
    return best;
}

extern "C" int fdtd_step_fused(const fdtd_step_args *args, void *stream) {
    if (!args) {
        set_error("fdtd_step_fused: null args");
        return FDTD_ERR_ARG;
    }
    fdtd_step_args a = *args;
    if (a.nx <= 0 || a.ny <= 0 || a.nz <= 0 || !a.step || !a.coeff_e || !a.coeff_h) {
        set_error("fdtd_step_fused: invalid grid or null pointer");
        return FDTD_ERR_ARG;
    }
    if (a.pitch_z <= 0) a.pitch_z = a.nz;
    if (a.material_pitch <= 0) a.material_pitch = a.nz;
    if (a.pitch_z < a.nz || a.material_pitch < a.nz) {
        set_error("fdtd_step_fused: row pitch smaller than nz");
        return FDTD_ERR_ARG;
    }
    for (int k = 0; k < 2; ++k) {
        if (!a.E[k] || !a.H[k] || !a.psi_e[k] || !a.psi_h[k]) {
            set_error("fdtd_step_fused: null field or CPML buffer");
            return FDTD_ERR_ARG;
        }
    }
    if (a.packed < 0 || a.packed > 2) {
        set_error("fdtd_step_fused: unknown psi layout %d", a.packed);
        return FDTD_ERR_ARG;
    }
    if (a.packed == FDTD_PSI_FULL && a.psi_cols < (long long)a.nx * a.ny * a.pitch_z) {
        set_error("fdtd_step_fused: full CPML storage needs psi_cols >= nx*ny*pitch_z");
        return FDTD_ERR_ARG;
    }
    const int maxdim = a.nx > a.ny ? (a.nx > a.nz ? a.nx : a.nz) : (a.ny > a.nz ? a.ny : a.nz);
    if (a.clen < maxdim) {
        set_error("fdtd_step_fused: coefficient length %d < largest dimension %d", a.clen, maxdim);
        return FDTD_ERR_ARG;
    }
    if (a.material_kind == 1) {
        if (!a.material || !a.material_table || a.material_count < 1 || a.material_count > 256) {
            set_error("fdtd_step_fused: uint8 material needs a table of 1..256 entries");
            return FDTD_ERR_ARG;
        }
    } else if (a.material_kind != 0 || !a.inv_eps) {
        set_error("fdtd_step_fused: material_kind must be 0 (inv_eps) or 1 (uint8 index)");
        return FDTD_ERR_ARG;
    }
    if (a.source_x >= 0 && (!a.src_e || !a.src_h || !a.waves_e || !a.waves_h)) {
        set_error("fdtd_step_fused: source plane without profiles or waves");
        return FDTD_ERR_ARG;
    }
    int path = a.path;
    if (a.packed == FDTD_PSI_SLAB) {
        // the slab layout is only read by the full-z pipeline
        if (path != 0 && path != 3) {
            set_error("fdtd_step_fused: the slab psi layout needs path 3");
            return FDTD_ERR_ARG;
        }
        if (!fz_eligible(a)) {
            set_error("fdtd_step_fused: full-z path needs pitch_z %% 4 == 0, pitch_z <= 248, "
                      "psi_rz %% 4 == 0 and 16-byte aligned buffers");
            return FDTD_ERR_ARG;
        }
        path = 3;
    } else if (path == 3) {
        set_error("fdtd_step_fused: path 3 needs the slab psi layout");
        return FDTD_ERR_ARG;
    }
    if (path == 0) path = tma_eligible(a) ? 2 : 1;
    if (path == 2 && !tma_eligible(a)) {
        set_error("fdtd_step_fused: TMA path needs pitch_z %% 4 == 0, material_pitch %% 16 == 0 "
                  "and 16-byte aligned buffers");
        return FDTD_ERR_ARG;
    }
    if (path != 1 && path != 2 && path != 3) {
        set_error("fdtd_step_fused: path must be 0, 1, 2 or 3");
        return FDTD_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (path == 3) {
        if (a.schedule && (a.schedule_blocks < 1 || a.chunk_x < 1)) {
            set_error("fdtd_step_fused: a schedule needs schedule_blocks >= 1 and chunk_x >= "
                      "its longest entry");
            return FDTD_ERR_ARG;
        }
        fz_defaults(a);
        if (a.tile_y < 1 || a.chunk_x < 1) {
            set_error("fdtd_step_fused: invalid tile");
            return FDTD_ERR_ARG;
        }
        return launch_fz(a, st);
    }
    if (path == 2) {
        if (a.tile_z <= 0) {
            // uint8 material boxes must start on 16-byte boundaries: tile_z % 16 == 0
            const int cz[] = {48, 32, 64, 40, 56, 36, 44};
            const int cz8[] = {48, 32, 64, 16};
            a.tile_z = a.material_kind == 1 ? pick_tile(a.nz, cz8, 4) : pick_tile(a.nz, cz, 7);
        }
        if (a.tile_y <= 0) {
            const int cy[] = {8, 12, 10, 16, 6};
            a.tile_y = pick_tile(a.ny, cy, 5);
        }
        const int tiles = ((a.ny + a.tile_y - 1) / a.tile_y) * ((a.nz + a.tile_z - 1) / a.tile_z);
        if (a.chunk_x <= 0) {
            int want = 148 * 2;
            int chunks = (want + tiles - 1) / tiles;
            a.chunk_x = (a.nx + chunks - 1) / chunks;
        }
        if (a.tile_y < 1 || a.tile_z < 4 || a.chunk_x < 1) {
            set_error("fdtd_step_fused: invalid tile");
            return FDTD_ERR_ARG;
        }
        return launch_tma(a, st);
    }
    if (a.tile_y <= 0) a.tile_y = 8;
    if (a.tile_z <= 0) a.tile_z = 32;
    const int tiles = ((a.ny + a.tile_y - 1) / a.tile_y) * ((a.nz + a.tile_z - 1) / a.tile_z);
    if (a.chunk_x <= 0) {
        // about 8 resident blocks per SM on 148 SMs, one wave
        int want = 148 * 8;
        int chunks = (want + tiles - 1) / tiles;
        if (chunks < 1) chunks = 1;
        a.chunk_x = (a.nx + chunks - 1) / chunks;
        if (a.chunk_x < 4) a.chunk_x = 4 < a.nx ? 4 : a.nx;
    }
    if (a.tile_y * a.tile_z > 4096 || a.tile_y > 256 || a.tile_z > 256) {
        set_error("fdtd_step_fused: tile %dx%d too large", a.tile_y, a.tile_z);
        return FDTD_ERR_ARG;
    }
    const int chunks = (a.nx + a.chunk_x - 1) / a.chunk_x;
    const size_t smem = smem_bytes(a.tile_y, a.tile_z, a.material_kind);
    if (smem > 200 * 1024) {
        set_error("fdtd_step_fused: tile needs %zu bytes of shared memory", smem);
        return FDTD_ERR_ARG;
    }
    int threads = a.tile_y * a.tile_z;
    if (threads > 512) threads = 512;
    if (threads < 64) threads = 64;
    threads = (threads + 31) / 32 * 32;
    dim3 grid((unsigned)(tiles * chunks));
#define LAUNCH(M, P)                                                                          \
    do {                                                                                      \
        if (smem > 48 * 1024)                                                                 \
            cudaFuncSetAttribute(fused_step_kernel<M, P>,                                     \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);     \
        fused_step_kernel<M, P><<<grid, threads, smem, st>>>(a);                              \
    } while (0)
    if (a.material_kind == 1) {
        if (a.packed) LAUNCH(1, true); else LAUNCH(1, false);
    } else {
        if (a.packed) LAUNCH(0, true); else LAUNCH(0, false);
    }
#undef LAUNCH
    return launch_status("fdtd_step_fused");
}

extern "C" int fdtd_step_defaults(fdtd_step_args *args) {
    if (!args) {
        set_error("fdtd_step_defaults: null argument");
        return FDTD_ERR_ARG;
    }
    fdtd_step_args a = *args;
    if (a.pitch_z <= 0) a.pitch_z = a.nz;
    if (a.material_pitch <= 0) a.material_pitch = a.nz;
    if (a.nx <= 0 || a.ny <= 0 || a.nz <= 0 || a.packed != FDTD_PSI_SLAB || !fz_eligible(a)) {
        set_error("fdtd_step_defaults: arguments do not select the full-z path");
        return FDTD_ERR_ARG;
    }
    fz_defaults(a);
    args->tile_y = a.tile_y;
    if (!args->schedule) args->chunk_x = a.chunk_x;
    return 0;
}

extern "C" int fdtd_step_occupancy(const fdtd_step_args *args, int *blocks_per_sm, int *sms) {
    if (!args || !blocks_per_sm || !sms) {
        set_error("fdtd_step_occupancy: null argument");
        return FDTD_ERR_ARG;
    }
    fdtd_step_args a = *args;
    if (a.pitch_z <= 0) a.pitch_z = a.nz;
    if (a.material_pitch <= 0) a.material_pitch = a.nz;
    if (a.nx <= 0 || a.ny <= 0 || a.nz <= 0 || a.packed != FDTD_PSI_SLAB || !fz_eligible(a)) {
        set_error("fdtd_step_occupancy: arguments do not select the full-z path");
        return FDTD_ERR_ARG;
    }
    fz_defaults(a);
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(sms, cudaDevAttrMultiProcessorCount, dev);
    if (err != cudaSuccess) {
        set_error("fdtd_step_occupancy: %s", cudaGetErrorString(err));
        return FDTD_ERR_CUDA;
    }
    return fz_occupancy(a, blocks_per_sm);
}
