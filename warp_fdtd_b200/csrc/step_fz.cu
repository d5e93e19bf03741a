// Fused Yee leapfrog step over full-z tiles (path 3, the Solver's default).
//
// A block owns rows [y0, y0 + tile_y) of the y-z plane across the whole z
// extent and a chunk of x planes, marching along x with the E update one
// plane ahead of the H update (same scheme and arithmetic as step_fused.cu /
// step_tma.cu).  Because a tile spans all of z there is no z halo: the -z
// neighbour of z = 0 and the +z neighbour of z = nz - 1 are the grid's zero
// padding.  Each plane is staged by TMA in one ring stage:
//
//   H(p)   rows y0-1 .. y0+ty, z from -4 (box width pitch + 4; the -4 keeps
//          the box start 16-byte aligned and supplies z = -1 as zero fill)
//   E(p)   rows y0 .. y0+ty, z 0 .. pitch
//   material, and the z-slab CPML state of E (rows y0..y0+ty) and H (rows
//   y0..y0+ty-1), which the slab layout keeps contiguous in z-rank.
//
// A thread handles four consecutive z cells of one row (128-bit shared-memory
// loads and global stores) for both updates, so index arithmetic is hoisted
// out of the plane loop.  x- and y-slab CPML state is read directly (float4,
// coalesced) only in the planes / rows where it is active; whether a cell
// group takes the CPML branch is decided per thread from tile coefficient
// tables in shared memory.  Outside the slabs the reference's 1 * d == d, so
// the plain difference is used, bit for bit identical.
#include <mutex>
#include <new>

#include "common.cuh"
#include "step_internal.h"
#include "tma_util.cuh"

namespace wfb {

struct FzLayout {
    int ty, P, HB, MB, RZ, S;
    int off_h, off_e, off_m, off_pze, off_pzh;  // byte offsets inside a stage
    int stage_bytes;
    unsigned tx_bytes;
    int off_stages, off_ring, RW, off_coef, XK, off_mtab, smem_bytes;
};

struct FzMaps {
    CUtensorMap E[2], H[2], M, PZE[2], PZH[2];
};

struct FzParams {
    fdtd_step_args a;
    FzLayout L;
    long long xoff, yoff, zoff;  // slab-block offsets (elements) inside a psi buffer
};

__device__ __forceinline__ bool active(float4 c) { return c.x != 0.0f || c.z != 1.0f; }

// V consecutive floats held in registers (V = 2 or 4 z cells per thread).
template <int V>
struct VF {
    float v[V];
};

template <int V>
__device__ __forceinline__ VF<V> ldsv(const float *p) {
    VF<V> r;
    if constexpr (V == 4) {
        const float4 t = *(const float4 *)p;
        r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
    } else {
        const float2 t = *(const float2 *)p;
        r.v[0] = t.x; r.v[1] = t.y;
    }
    return r;
}

template <int V>
__device__ __forceinline__ VF<V> ldgv(const float *p) {
    VF<V> r;
    if constexpr (V == 4) {
        const float4 t = __ldg((const float4 *)p);
        r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
    } else {
        const float2 t = __ldg((const float2 *)p);
        r.v[0] = t.x; r.v[1] = t.y;
    }
    return r;
}

template <int V>
__device__ __forceinline__ void stv(float *p, const VF<V> &r) {
    if constexpr (V == 4)
        *(float4 *)p = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
    else
        *(float2 *)p = make_float2(r.v[0], r.v[1]);
}

template <int V>
__device__ __forceinline__ VF<V> zero_v() {
    VF<V> r;
#pragma unroll
    for (int j = 0; j < V; ++j) r.v[j] = 0.0f;
    return r;
}

// kernels.py:29-47 applied to one difference with its old psi value.
__device__ __forceinline__ float cpml1(float d, float4 c, float psi_old, float &psi_new) {
    if (c.x != 0.0f) {
        const float p = c.y * psi_old + c.x * d;
        psi_new = p;
        return c.z * d + p;
    }
    return c.z * d;
}

// CPML filter of the two differences an axis owns, for a cell group whose
// coefficient c is uniform (x: the plane, y: the row); psi in a slab block
// at `ib` (slot stride `slot`), read from `po`, written to `pn` if `own`.
template <int V>
__device__ __forceinline__ void cpml_axis(VF<V> &d0, VF<V> &d1, float4 c, const float *po,
                                          float *pn, i64 ib, i64 slot, bool own) {
    VF<V> p0 = zero_v<V>(), p1 = zero_v<V>(), n0 = zero_v<V>(), n1 = zero_v<V>();
    if (c.x != 0.0f) {
        p0 = ldgv<V>(po + ib);
        p1 = ldgv<V>(po + ib + slot);
    }
#pragma unroll
    for (int j = 0; j < V; ++j) {
        d0.v[j] = cpml1(d0.v[j], c, p0.v[j], n0.v[j]);
        d1.v[j] = cpml1(d1.v[j], c, p1.v[j], n1.v[j]);
    }
    if (own && c.x != 0.0f) {
        stv<V>(pn + ib, n0);
        stv<V>(pn + ib + slot, n1);
    }
}

// The same with the old psi values already in registers (p0 / p1 are read
// only where c.x != 0, which is where they were loaded).
template <int V>
__device__ __forceinline__ void cpml_axis_r(VF<V> &d0, VF<V> &d1, float4 c, const VF<V> &p0,
                                            const VF<V> &p1, float *pn, i64 ib, i64 slot,
                                            bool own) {
    VF<V> n0 = zero_v<V>(), n1 = zero_v<V>();
#pragma unroll
    for (int j = 0; j < V; ++j) {
        d0.v[j] = cpml1(d0.v[j], c, p0.v[j], n0.v[j]);
        d1.v[j] = cpml1(d1.v[j], c, p1.v[j], n1.v[j]);
    }
    if (own && c.x != 0.0f) {
        stv<V>(pn + ib, n0);
        stv<V>(pn + ib + slot, n1);
    }
}

// CPML filter of a cell group along z: per-cell coefficients from `cz`, the
// group's old psi pair staged at `po0` / `po1` (slab ranks rb .. rb+V-1), new
// values to `pn + ib` and `pn + ib + slot` if `store`.  Inactive cells of a
// slab window keep psi at zero.
template <int V>
__device__ __forceinline__ void cpml_z(VF<V> &d0, VF<V> &d1, const float4 *cz, bool has_psi,
                                       const float *po0, const float *po1, float *pn, i64 ib,
                                       i64 slot, bool store) {
    VF<V> z0, z1, u0 = zero_v<V>(), u1 = zero_v<V>();
    if (has_psi) {
        z0 = ldsv<V>(po0);
        z1 = ldsv<V>(po1);
    }
#pragma unroll
    for (int j = 0; j < V; ++j) {
        const float4 c = cz[j];
        d0.v[j] = cpml1(d0.v[j], c, z0.v[j], u0.v[j]);
        d1.v[j] = cpml1(d1.v[j], c, z1.v[j], u1.v[j]);
    }
    if (store && has_psi) {
        stv<V>(pn + ib, u0);
        stv<V>(pn + ib + slot, u1);
    }
}

// A cell group with z-slab psi must hold the aligned consecutive slab ranks
// rb .. rb+V-1 (one vector of the staged z-slab rows) inside the slab width.
template <int V>
__device__ __forceinline__ bool group_ranks_ok(const float4 *tab, int RZ) {
    const int rb = (int)tab[0].w;
    bool psi = false, ok = true;
#pragma unroll
    for (int j = 0; j < V; ++j)
        if (tab[j].x != 0.0f) {
            psi = true;
            ok &= (int)tab[j].w == rb + j;
        }
    return !psi || (ok && rb % V == 0 && rb + V <= RZ);
}

// FULLZ: rows hold no padding (nz == pitch_z), so no cell group needs the
// z < nz masks; dropping them frees registers the update's schedule uses.
// Body of one block: tile `tyi` over planes [xa, xb) of one grid.  `maps` and
// `prm` are the kernel parameters of a single-grid launch, or one entry of a
// batch's instance table in global memory.
template <int MAT, int S, int V, bool FULLZ>
__device__ __forceinline__ void fz_run(const FzMaps &maps, const FzParams &prm, int tyi, int xa,
                                       int xb) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const fdtd_step_args &a = prm.a;
    const FzLayout &L = prm.L;
    const int nx = a.nx, ny = a.ny, nz = a.nz, P = L.P, TY = L.ty;
    const i64 cols = (i64)nx * ny * P;
    const i64 plane = (i64)ny * P;
    const int HB = L.HB, RW = L.RW, RZ = L.RZ;
    const int HS = (TY + 2) * HB;   // H component stride in a stage
    const int ES = (TY + 1) * P;    // E component stride in a stage
    const int RS = (TY + 1) * RW;   // ring component stride
    const int lanes = P / V;

    uint64_t *bars = (uint64_t *)smem;
    int *meta = (int *)(smem + 64);  // [0] slab rank check failed
    unsigned char *stage0 = smem + L.off_stages;
    float *ring = (float *)(smem + L.off_ring);  // [3][TY+1][RW]: E of the last plane
    float4 *cey = (float4 *)(smem + L.off_coef);
    float4 *chy = cey + (TY + 1);
    float4 *cez = chy + (TY + 1);
    float4 *chz = cez + P;
    float4 *cex = chz + P;   // by stage index k: E coefficient of plane xa-1+k
    float4 *chx = cex + L.XK;  // ... H coefficient of plane xa-2+k
    float *mtab = (float *)(smem + L.off_mtab);

    if (xa >= xb) return;
    const int y0 = tyi * TY;
    const int last = xb - xa + 1;  // planes k = 0..last are xa-1 .. xb

    const int t = a.step[0];
    const int s = t & 1;
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
    const i64 xslot = (i64)a.psi_rx * plane;      // slot stride of the X block
    const i64 yslot = (i64)a.psi_ry * nx * P;     // ... of the Y block
    const i64 zslot = (i64)nx * ny * RZ;          // ... of the Z block

    auto stage_ptr = [&](int k) { return stage0 + (size_t)(k % S) * L.stage_bytes; };
    auto issue = [&](int k) {
        unsigned char *st = stage_ptr(k);
        uint64_t *bar = bars + (k % S);
        const int p = xa - 1 + k;
        mbar_expect_tx(bar, L.tx_bytes);
        tma_load_4d(st + L.off_h, &maps.H[s], -4, y0 - 1, p, 0, bar);
        tma_load_4d(st + L.off_e, &maps.E[s], 0, y0, p, 0, bar);
        tma_load_3d(st + L.off_m, &maps.M, 0, y0, p, bar);
        if (RZ > 0) {
            tma_load_4d(st + L.off_pze, &maps.PZE[s], 0, y0, p, 0, bar);
            tma_load_4d(st + L.off_pzh, &maps.PZH[s], 0, y0, p - 1, 0, bar);
        }
    };

    if (tid == 0) {
        for (int j = 0; j < S; ++j) mbar_init(bars + j, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (MAT == 1)
        for (int j = tid; j < 256; j += nth) mtab[j] = j < a.material_count ? a.material_table[j] : 0.0f;
    const float4 ident = make_float4(0.f, 1.f, 1.f, 0.f);
    for (int j = tid; j <= TY; j += nth) {
        const int y = y0 + j;
        cey[j] = y < ny ? __ldg(ce + clen + y) : ident;
        chy[j] = y < ny ? __ldg(ch + clen + y) : ident;
    }
    for (int j = tid; j < P; j += nth) {
        cez[j] = j < nz ? __ldg(ce + 2 * clen + j) : ident;
        chz[j] = j < nz ? __ldg(ch + 2 * clen + j) : ident;
    }
    for (int j = tid; j <= last; j += nth) {
        const int p = xa - 1 + j;
        cex[j] = p >= 0 && p < nx ? __ldg(ce + p) : ident;
        chx[j] = p >= 1 && p - 1 < nx ? __ldg(ch + p - 1) : ident;
    }
    // the ring's +z pad columns (z = P .. P+3) are the zero padding beyond the grid
    for (int j = tid; j < 3 * (TY + 1) * 4; j += nth) {
        const int r = j >> 2, c = j & 3;
        ring[r * RW + P + c] = 0.0f;
    }
    __syncthreads();
    if (tid == 0) {
        int bad = 0;
        for (int l = 0; l < lanes; ++l)
            if (!(group_ranks_ok<V>(cez + l * V, RZ) && group_ranks_ok<V>(chz + l * V, RZ))) bad = 1;
        meta[0] = bad;
    }
    __syncthreads();
    if (meta[0]) {
        if (tid == 0 && a.error) atomicExch(a.error, 2);
        return;  // nothing issued yet
    }
    const int ly = tid / lanes;           // this thread's row (E: ly <= TY, H: ly < TY)
    const int zv = (tid - ly * lanes) * V;  // first of this thread's V z cells
    const int gy = y0 + ly;
    // per-thread CPML activity of its row and its z cells
    const float4 my_cey = cey[ly], my_chy = chy[min(ly, TY - 1)];
    const bool yE = active(my_cey), yH = ly < TY && active(my_chy);
    bool zE = false, zH = false, zEp = false, zHp = false;
#pragma unroll
    for (int j = 0; j < V; ++j) {
        zE |= active(cez[zv + j]);
        zH |= active(chz[zv + j]);
        zEp |= cez[zv + j].x != 0.0f;
        zHp |= chz[zv + j].x != 0.0f;
    }
    const int rbe = (int)cez[zv].w, rbh = (int)chz[zv].w;

    int issued;
    if (tid == 0)
        for (int k = 0; k <= last && k < S; ++k) issue(k);
    issued = min(last, S - 1);
    const long limit = 1L << 24;
    bool timed_out = false;
    int done = -1;
    if (mbar_wait_bounded(bars, 0, limit))
        done = 0;
    else
        timed_out = true;

    const int h_off = (ly + 1) * HB + zv + 4;  // this cell group in an H box
    const int e_off = ly * P + zv;             // ... in an E box
    const int r_off = ly * RW + zv;            // ... in the E ring
    const int g_off = gy * P + zv;             // ... in a field plane (elements)
    const bool row_in = gy < ny;
    // H of the previous plane at this thread's cells: the E update's x
    // difference and the H update's old value, so a stage is free as soon as
    // the plane after it starts
    VF<V> hprev[3];
    {
        const float *H0 = (const float *)(stage0 + L.off_h);
#pragma unroll
        for (int c = 0; c < 3; ++c) hprev[c] = ldsv<V>(H0 + c * HS + h_off);
    }
    const int issuer = nth - 1;  // a thread of row TY, which has no H update

    int k = 1;
    for (; k <= last; ++k) {
        const int p = xa - 1 + k;
        const int q = p - 1;
        const float4 cxh = chx[k];
        const bool h_on = q >= xa && ly < TY && row_in;
        // x- and y-slab psi of the H plane q: in flight during the E update
        VF<V> xh0, xh1, yh0, yh1;
        if (h_on) {
            if (cxh.x != 0.0f) {
                const i64 ib = prm.xoff + ((i64)(int)cxh.w * ny + gy) * P + zv;
                xh0 = ldgv<V>(ph_o + ib);
                xh1 = ldgv<V>(ph_o + ib + xslot);
            }
            if (my_chy.x != 0.0f) {
                const i64 ib = prm.yoff + ((i64)(int)my_chy.w * nx + q) * P + zv;
                yh0 = ldgv<V>(ph_o + ib);
                yh1 = ldgv<V>(ph_o + ib + yslot);
            }
        }
        if (!timed_out) {
            if (mbar_wait_bounded(bars + (k % S), (k / S) & 1, limit))
                done = k;
            else
                timed_out = true;
        }
        const unsigned char *stc = stage_ptr(k);
        // ---------------- E update, rows y0 .. y0+TY ----------------
        // (kept in registers until the H update below has read plane q's E)
        VF<V> o[3] = {zero_v<V>(), zero_v<V>(), zero_v<V>()};
        if (!timed_out) {
            if (p < nx && row_in) {
                const float *Hc = (const float *)(stc + L.off_h);
                const float *Eo = (const float *)(stc + L.off_e);
                VF<V> dx[3], dy[3], dz[3];
#pragma unroll
                for (int q3 = 0; q3 < 3; ++q3) {
                    const VF<V> hc = ldsv<V>(Hc + q3 * HS + h_off);
                    const VF<V> &hp = hprev[q3];
                    const VF<V> hy = ldsv<V>(Hc + q3 * HS + h_off - HB);
                    float zm = Hc[q3 * HS + h_off - 1];
#pragma unroll
                    for (int j = 0; j < V; ++j) {
                        dx[q3].v[j] = hc.v[j] - hp.v[j];
                        dy[q3].v[j] = hc.v[j] - hy.v[j];
                        dz[q3].v[j] = hc.v[j] - zm;
                        zm = hc.v[j];
                    }
                }
                float ie[V];
                if (MAT == 1) {
                    const unsigned char *m = stc + L.off_m + ly * L.MB + zv;
                    if constexpr (V == 4) {
                        const uchar4 mm = *(const uchar4 *)m;
                        ie[0] = mtab[mm.x]; ie[1] = mtab[mm.y]; ie[2] = mtab[mm.z]; ie[3] = mtab[mm.w];
                    } else {
                        const uchar2 mm = *(const uchar2 *)m;
                        ie[0] = mtab[mm.x]; ie[1] = mtab[mm.y];
                    }
                } else {
                    const VF<V> t4 = ldsv<V>((const float *)(stc + L.off_m) + ly * L.MB + zv);
#pragma unroll
                    for (int j = 0; j < V; ++j) ie[j] = t4.v[j];
                }
                const float4 cx = cex[k];
                const bool own = p < xb && ly < TY;
                // CPML filter per axis (kernels.py:113-118): x is uniform over the
                // block's plane, y over the thread's row, z per cell of the group.
                // dx[2] = dxz, dx[1] = dxy, dy[0] = dyx, dy[2] = dyz, dz[1] = dzy, dz[0] = dzx
                if (active(cx))
                    cpml_axis<V>(dx[2], dx[1], cx, pe_o, pe_n,
                                 prm.xoff + ((i64)(int)cx.w * ny + gy) * P + zv, xslot, own);
                if (yE)
                    cpml_axis<V>(dy[0], dy[2], my_cey, pe_o, pe_n,
                                 prm.yoff + ((i64)(int)my_cey.w * nx + p) * P + zv, yslot, own);
                if (zE) {
                    const float *pz = (const float *)(stc + L.off_pze);  // [2][TY+1][RZ]
                    cpml_z<V>(dz[1], dz[0], cez + zv, zEp, pz + ly * RZ + rbe,
                              pz + (TY + 1) * RZ + ly * RZ + rbe, pe_n,
                              prm.zoff + ((i64)p * ny + gy) * RZ + rbe, zslot, own);
                }
                const VF<V> e0 = ldsv<V>(Eo + e_off), e1 = ldsv<V>(Eo + ES + e_off),
                            e2 = ldsv<V>(Eo + 2 * ES + e_off);
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    const float iej = ie[j];
                    float v0 = e0.v[j] + (courant * (dy[2].v[j] - dz[1].v[j])) * iej;
                    float v1 = e1.v[j] + (courant * (dz[0].v[j] - dx[2].v[j])) * iej;
                    float v2 = e2.v[j] + (courant * (dx[1].v[j] - dy[0].v[j])) * iej;
                    const int gz = zv + j;
                    if (p == a.source_x && wave_ok && (FULLZ || gz < nz)) {
                        const i64 sidx = (i64)gy * nz + gz;
                        const i64 syz = (i64)ny * nz;
                        v1 = v1 + ((a.src_h[2 * syz + sidx] * a.waves_h[2 * a.waves_cols + t]) * courant) * iej;
                        v2 = v2 - ((a.src_h[syz + sidx] * a.waves_h[a.waves_cols + t]) * courant) * iej;
                    }
                    const bool in = FULLZ || gz < nz;
                    o[0].v[j] = in ? v0 : 0.0f;
                    o[1].v[j] = in ? v1 : 0.0f;
                    o[2].v[j] = in ? v2 : 0.0f;
                }
                if (own) {
                    float *dst = En + (i64)p * plane + g_off;
                    stv<V>(dst, o[0]);
                    stv<V>(dst + cols, o[1]);
                    stv<V>(dst + 2 * cols, o[2]);
                }
            }
        }
        if (__syncthreads_or(timed_out)) {
            timed_out = true;
            break;
        }
        // plane k-1's stage is no longer read: refill it while the H update runs
        if (k - 1 + S <= last) {
            if (tid == issuer) issue(k - 1 + S);
            issued = k - 1 + S;
        }
        // ---------------- H update at plane q = p - 1, rows y0 .. y0+TY-1 ----------------
        if (h_on) {
            const float *Rq = ring;  // E of plane q
            VF<V> dx[3], dy[3], dz[3];
#pragma unroll
            for (int r = 0; r < 3; ++r) {
                const VF<V> eq = ldsv<V>(Rq + r * RS + r_off);
                const VF<V> &ep = o[r];
                const VF<V> eyp = ldsv<V>(Rq + r * RS + r_off + RW);
                const float zp = Rq[r * RS + r_off + V];
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    const float nxt = j + 1 < V ? eq.v[j + 1 < V ? j + 1 : 0] : zp;
                    dx[r].v[j] = ep.v[j] - eq.v[j];
                    dy[r].v[j] = eyp.v[j] - eq.v[j];
                    dz[r].v[j] = nxt - eq.v[j];
                }
            }
            if (active(cxh))
                cpml_axis_r<V>(dx[2], dx[1], cxh, xh0, xh1, ph_n,
                               prm.xoff + ((i64)(int)cxh.w * ny + gy) * P + zv, xslot, true);
            if (yH)
                cpml_axis_r<V>(dy[0], dy[2], my_chy, yh0, yh1, ph_n,
                               prm.yoff + ((i64)(int)my_chy.w * nx + q) * P + zv, yslot, true);
            if (zH) {
                const float *pz = (const float *)(stc + L.off_pzh);  // [2][TY][RZ], plane q
                cpml_z<V>(dz[1], dz[0], chz + zv, zHp, pz + ly * RZ + rbh,
                          pz + TY * RZ + ly * RZ + rbh, ph_n,
                          prm.zoff + ((i64)q * ny + gy) * RZ + rbh, zslot, true);
            }
            const VF<V> &h0 = hprev[0], &h1 = hprev[1], &h2 = hprev[2];
            VF<V> o[3];
#pragma unroll
            for (int j = 0; j < V; ++j) {
                float v0 = h0.v[j] - courant * (dy[2].v[j] - dz[1].v[j]);
                float v1 = h1.v[j] - courant * (dz[0].v[j] - dx[2].v[j]);
                float v2 = h2.v[j] - courant * (dx[1].v[j] - dy[0].v[j]);
                const int gz = zv + j;
                if (q == a.source_x && wave_ok && (FULLZ || gz < nz)) {
                    const i64 sidx = (i64)gy * nz + gz;
                    const i64 syz = (i64)ny * nz;
                    v1 = v1 - (a.src_e[2 * syz + sidx] * a.waves_e[2 * a.waves_cols + t]) * courant;
                    v2 = v2 + (a.src_e[syz + sidx] * a.waves_e[a.waves_cols + t]) * courant;
                }
                o[0].v[j] = v0;
                o[1].v[j] = v1;
                o[2].v[j] = v2;
            }
            float *dst = Hn + (i64)q * plane + g_off;
            stv<V>(dst, o[0]);
            stv<V>(dst + cols, o[1]);
            stv<V>(dst + 2 * cols, o[2]);
        }
        {
            const float *Hc = (const float *)(stc + L.off_h);
#pragma unroll
            for (int c = 0; c < 3; ++c) hprev[c] = ldsv<V>(Hc + c * HS + h_off);
        }
        __syncthreads();
        // every H update has read plane q's E: the ring takes plane p's
        stv<V>(ring + r_off, o[0]);
        stv<V>(ring + RS + r_off, o[1]);
        stv<V>(ring + 2 * RS + r_off, o[2]);
    }
    if (timed_out) {
        if (tid == 0) {
            if (a.error) atomicExch(a.error, 1);
            for (int j = done + 1; j <= issued; ++j)
                mbar_wait_bounded(bars + (j % S), (j / S) & 1, limit);
        }
        __syncthreads();
    }
}

// A block's (tile, plane range) from a schedule entry (tile, first plane, end
// plane) or the uniform tile x chunk grid; false (and error 3) for an entry
// outside the grid or longer than the shared-memory layout's chunk.
__device__ __forceinline__ bool fz_block_range(const fdtd_step_args &a, int ty, const int *entry,
                                               int &tyi, int &xa, int &xb) {
    const int tiles_y = (a.ny + ty - 1) / ty;
    if (entry) {
        tyi = entry[0];
        xa = entry[1];
        xb = entry[2];
        if (tyi < 0 || tyi >= tiles_y || xa < 0 || xb > a.nx || xb - xa > a.chunk_x) {
            if (threadIdx.x == 0 && a.error) atomicExch(a.error, 3);
            return false;
        }
    } else {
        tyi = blockIdx.x % tiles_y;
        xa = (blockIdx.x / tiles_y) * a.chunk_x;
        xb = min(xa + a.chunk_x, a.nx);
    }
    return true;
}

template <int MAT, int S, int V, bool FULLZ>
__global__ void __launch_bounds__(512)
    fz_step_kernel(const __grid_constant__ FzMaps maps, const __grid_constant__ FzParams prm) {
    const fdtd_step_args &a = prm.a;
    int tyi, xa, xb;
    if (!fz_block_range(a, prm.L.ty, a.schedule ? a.schedule + 4 * blockIdx.x : nullptr, tyi, xa, xb))
        return;
    fz_run<MAT, S, V, FULLZ>(maps, prm, tyi, xa, xb);
}

// One grid of a batch: its tensor maps and parameters (64-byte aligned for the
// tensor maps, read by TMA from global memory).
struct alignas(64) FzInstance {
    FzMaps maps;
    FzParams prm;
};

// Parameter blocks of the grids of live batches, by slot: constant memory,
// so a block reads its grid's (uniform) parameters through the constant
// cache; the tensor maps stay in the global instance table, where TMA reads
// them.
constexpr int FZ_BATCH_SLOTS = 128;
__constant__ FzParams g_batch_prm[FZ_BATCH_SLOTS];

// Many grids advanced by one launch: block b runs schedule entry b =
// (instance, tile, first plane, end plane); instance i uses constant slot
// base + i and entry i of the instance table.
template <int MAT, int S, int V, bool FULLZ>
__global__ void __launch_bounds__(512)
    fz_batch_kernel(const FzInstance *__restrict__ inst, int base, int count,
                    const int *__restrict__ sched) {
    const int *entry = sched + 4 * blockIdx.x;
    const int i = entry[0];
    if (i < 0 || i >= count) return;
    const FzParams &prm = g_batch_prm[base + i];
    int tyi, xa, xb;
    if (!fz_block_range(prm.a, prm.L.ty, entry + 1, tyi, xa, xb)) return;
    fz_run<MAT, S, V, FULLZ>(inst[i].maps, prm, tyi, xa, xb);
}

static inline size_t up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static FzLayout fz_layout(int ty, int P, int RZ, int S, int mat, int chunk_x) {
    FzLayout L;
    L.ty = ty;
    L.P = P;
    L.HB = P + 4;
    L.MB = mat == 1 ? (int)up(P, 16) : P;
    L.RZ = RZ;
    L.S = S;
    size_t hb = (size_t)3 * (ty + 2) * L.HB * 4;
    size_t eb = (size_t)3 * (ty + 1) * P * 4;
    size_t mb = (size_t)(ty + 1) * L.MB * (mat == 1 ? 1 : 4);
    size_t zeb = (size_t)2 * (ty + 1) * RZ * 4;
    size_t zhb = (size_t)2 * ty * RZ * 4;
    L.off_h = 0;
    L.off_e = (int)up(hb, 128);
    L.off_m = (int)(L.off_e + up(eb, 128));
    L.off_pze = (int)(L.off_m + up(mb, 128));
    L.off_pzh = (int)(L.off_pze + up(zeb, 128));
    L.stage_bytes = (int)(L.off_pzh + up(zhb, 128));
    L.tx_bytes = (unsigned)(hb + eb + mb + (RZ > 0 ? zeb + zhb : 0));
    L.off_stages = 128;
    L.RW = P + 4;
    L.off_ring = (int)(L.off_stages + (size_t)S * L.stage_bytes);
    size_t ring = (size_t)3 * (ty + 1) * L.RW * 4;
    L.off_coef = (int)up(L.off_ring + ring, 16);
    L.XK = chunk_x + 2;  // x coefficients of planes xa-1 .. xb (E) and xa-2 .. xb-1 (H)
    size_t coef = (size_t)(2 * (ty + 1) + 2 * P + 2 * L.XK) * 16;
    L.off_mtab = (int)up(L.off_coef + coef, 16);
    L.smem_bytes = (int)(L.off_mtab + (mat == 1 ? 256 * 4 : 0));
    return L;
}

bool fz_eligible(const fdtd_step_args &a) {
    if (a.packed != FDTD_PSI_SLAB) return false;
    if (a.pitch_z % 4 != 0 || a.pitch_z > 248) return false;
    if (a.material_kind == 1 && a.material_pitch % 16 != 0) return false;
    if (a.psi_rz % 4 != 0) return false;
    auto al16 = [](const void *p) { return ((uintptr_t)p & 15) == 0; };
    for (int j = 0; j < 2; ++j)
        if (!al16(a.E[j]) || !al16(a.H[j]) || !al16(a.psi_e[j]) || !al16(a.psi_h[j])) return false;
    return a.material_kind == 1 ? al16(a.material) : al16(a.inv_eps);
}

void fz_defaults(fdtd_step_args &a) {
    if (a.tile_y <= 0) {
        // the tallest tile whose block keeps two per SM (<= 256 threads at 128
        // registers, <= 112 KB with a three-stage ring and 40-plane runs)
        const int V = a.vector == 2 ? 2 : 4, lanes = a.pitch_z / V;
        a.tile_y = 1;
        for (int ty = 256 / lanes - 1; ty >= 1; --ty)
            if (fz_layout(ty, a.pitch_z, a.psi_rz, a.stages > 0 ? a.stages : 3, a.material_kind, 40)
                    .smem_bytes <= 112 * 1024) {
                a.tile_y = ty;
                break;
            }
    }
    if (a.chunk_x <= 0 && !a.schedule) {
        // about three waves of two resident blocks per SM, chunks of >= 16 planes
        const int tiles = (a.ny + a.tile_y - 1) / a.tile_y;
        const int want = 148 * 2 * 3;
        const int chunks = (want + tiles - 1) / tiles;
        a.chunk_x = (a.nx + chunks - 1) / chunks;
        if (a.chunk_x < 16) a.chunk_x = 16 < a.nx ? 16 : a.nx;
    }
}

using FzKernel = void (*)(FzMaps, FzParams);

template <int M, int SS>
static FzKernel fz_pick_v(int V, bool full) {
    if (full) return V == 4 ? fz_step_kernel<M, SS, 4, true> : fz_step_kernel<M, SS, 2, true>;
    return V == 4 ? fz_step_kernel<M, SS, 4, false> : fz_step_kernel<M, SS, 2, false>;
}

static FzKernel fz_pick(const fdtd_step_args &a, int S, int V) {
    const bool full = a.nz == a.pitch_z;
    if (a.material_kind == 1)
        return S == 2 ? fz_pick_v<1, 2>(V, full) : S == 3 ? fz_pick_v<1, 3>(V, full) : fz_pick_v<1, 4>(V, full);
    return S == 2 ? fz_pick_v<0, 2>(V, full) : S == 3 ? fz_pick_v<0, 3>(V, full) : fz_pick_v<0, 4>(V, full);
}

// Layout, stage count, z cells per thread and threads per block of a launch.
static int fz_shape(const fdtd_step_args &a, FzLayout &L, int &S, int &V, int &threads) {
    const int P = a.pitch_z, ty = a.tile_y, RZ = a.psi_rz;
    S = a.stages > 0 ? a.stages : 3;
    if (S < 2 || S > 4) {
        set_error("fdtd_step_fused: full-z path takes 2..4 stages");
        return FDTD_ERR_ARG;
    }
    L = fz_layout(ty, P, RZ, S, a.material_kind, a.chunk_x);
    while (L.smem_bytes > 220 * 1024 && S > 2) L = fz_layout(ty, P, RZ, --S, a.material_kind, a.chunk_x);
    V = a.vector == 2 ? 2 : 4;
    threads = P / V * (ty + 1);
    if (L.smem_bytes > 220 * 1024 || threads > 512 || ty + 2 > 256) {
        set_error("fdtd_step_fused: full-z tile of %d rows does not fit (%d bytes, %d threads)", ty,
                  L.smem_bytes, threads);
        return FDTD_ERR_ARG;
    }
    return 0;
}

int fz_occupancy(const fdtd_step_args &a, int *blocks_per_sm) {
    FzLayout L;
    int S, V, threads;
    int rc = fz_shape(a, L, S, V, threads);
    if (rc) return rc;
    FzKernel k = fz_pick(a, S, V);
    cudaError_t err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, L.smem_bytes);
    if (err == cudaSuccess)
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, k, threads, L.smem_bytes);
    if (err != cudaSuccess) {
        set_error("fdtd_step_occupancy: %s", cudaGetErrorString(err));
        return FDTD_ERR_CUDA;
    }
    return 0;
}

// Tensor maps and parameters of one grid's launch.
static int fz_build(const fdtd_step_args &a, FzMaps &maps, FzParams &prm, int &S, int &V,
                    int &nthreads) {
    int rc = get_encoder();
    if (rc) return rc;
    const int P = a.pitch_z, ty = a.tile_y, RZ = a.psi_rz;
    FzLayout L;
    if ((rc = fz_shape(a, L, S, V, nthreads))) return rc;
    const cuuint64_t nz = a.nz, ny = a.ny, nx = a.nx, pz = P;
    cuuint64_t fdims[4] = {nz, ny, nx, 3};
    cuuint64_t fstr[3] = {pz * 4, pz * ny * 4, pz * ny * nx * 4};
    cuuint32_t hbox[4] = {(cuuint32_t)L.HB, (cuuint32_t)(ty + 2), 1, 3};
    cuuint32_t ebox[4] = {(cuuint32_t)P, (cuuint32_t)(ty + 1), 1, 3};
    for (int j = 0; j < 2; ++j) {
        if ((rc = encode(&maps.H[j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.H[j], fdims, fstr, hbox)))
            return rc;
        if ((rc = encode(&maps.E[j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.E[j], fdims, fstr, ebox)))
            return rc;
    }
    cuuint64_t mdims[3] = {nz, ny, nx};
    cuuint32_t mbox[3] = {(cuuint32_t)L.MB, (cuuint32_t)(ty + 1), 1};
    if (a.material_kind == 1) {
        const cuuint64_t mp = a.material_pitch;
        cuuint64_t mstr[2] = {mp, mp * ny};
        if ((rc = encode(&maps.M, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, a.material, mdims, mstr, mbox)))
            return rc;
    } else {
        cuuint64_t mstr[2] = {pz * 4, pz * ny * 4};
        if ((rc = encode(&maps.M, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, a.inv_eps, mdims, mstr, mbox)))
            return rc;
    }
    prm.a = a;
    prm.L = L;
    prm.xoff = 0;
    prm.yoff = (long long)2 * a.psi_rx * a.ny * P;
    prm.zoff = prm.yoff + (long long)2 * a.psi_ry * a.nx * P;
    if (RZ > 0) {
        const cuuint64_t rz = RZ;
        cuuint64_t zdims[4] = {rz, ny, nx, 2};
        cuuint64_t zstr[3] = {rz * 4, rz * ny * 4, rz * ny * nx * 4};
        cuuint32_t zebox[4] = {(cuuint32_t)RZ, (cuuint32_t)(ty + 1), 1, 2};
        cuuint32_t zhbox[4] = {(cuuint32_t)RZ, (cuuint32_t)ty, 1, 2};
        for (int j = 0; j < 2; ++j) {
            if ((rc = encode(&maps.PZE[j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.psi_e[j] + prm.zoff,
                             zdims, zstr, zebox)))
                return rc;
            if ((rc = encode(&maps.PZH[j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.psi_h[j] + prm.zoff,
                             zdims, zstr, zhbox)))
                return rc;
        }
    } else {
        maps.PZE[0] = maps.PZE[1] = maps.PZH[0] = maps.PZH[1] = maps.M;  // never loaded
    }
    return 0;
}

int launch_fz(const fdtd_step_args &a, cudaStream_t stream) {
    FzMaps maps;
    FzParams prm;
    int S, V, nthreads, rc;
    if ((rc = fz_build(a, maps, prm, S, V, nthreads))) return rc;
    const int tiles = (a.ny + a.tile_y - 1) / a.tile_y;
    const int chunks = (a.nx + a.chunk_x - 1) / a.chunk_x;
    dim3 grid((unsigned)(a.schedule ? a.schedule_blocks : tiles * chunks));
    FzKernel kern = fz_pick(a, S, V);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, prm.L.smem_bytes);
    kern<<<grid, dim3((unsigned)nthreads), prm.L.smem_bytes, stream>>>(maps, prm);
    return launch_status("fdtd_step_fused (full-z TMA)");
}

// ------------------------------ batches ------------------------------

using FzBatchKernel = void (*)(const FzInstance *, int, int, const int *);

template <int M, int SS>
static FzBatchKernel fz_pick_batch_v(int V, bool full) {
    if (full) return V == 4 ? fz_batch_kernel<M, SS, 4, true> : fz_batch_kernel<M, SS, 2, true>;
    return V == 4 ? fz_batch_kernel<M, SS, 4, false> : fz_batch_kernel<M, SS, 2, false>;
}

static FzBatchKernel fz_pick_batch(int mat, int S, int V, bool full) {
    if (mat == 1)
        return S == 2 ? fz_pick_batch_v<1, 2>(V, full)
             : S == 3 ? fz_pick_batch_v<1, 3>(V, full) : fz_pick_batch_v<1, 4>(V, full);
    return S == 2 ? fz_pick_batch_v<0, 2>(V, full)
         : S == 3 ? fz_pick_batch_v<0, 3>(V, full) : fz_pick_batch_v<0, 4>(V, full);
}

}  // namespace wfb

using namespace wfb;

// Constant-memory slots of live batches, per device.
static std::mutex g_slot_mu;
static bool g_slot_used[64][FZ_BATCH_SLOTS];

static int fz_slots_take(int dev, int count) {
    std::lock_guard<std::mutex> lock(g_slot_mu);
    for (int b = 0; b + count <= FZ_BATCH_SLOTS; ++b) {
        bool free = true;
        for (int j = b; j < b + count && free; ++j) free = !g_slot_used[dev][j];
        if (free) {
            for (int j = b; j < b + count; ++j) g_slot_used[dev][j] = true;
            return b;
        }
    }
    return -1;
}

static void fz_slots_give(int dev, int base, int count) {
    std::lock_guard<std::mutex> lock(g_slot_mu);
    for (int j = base; j >= 0 && j < base + count && j < FZ_BATCH_SLOTS; ++j) g_slot_used[dev][j] = false;
}

extern "C" long long fdtd_batch_workspace_bytes(int count) {
    return count > 0 ? (long long)count * (long long)sizeof(FzInstance) : 0;
}

extern "C" int fdtd_batch_prepare(const fdtd_step_args *args, int count, void *workspace,
                                  long long workspace_bytes, fdtd_batch_plan *plan) {
    if (!args || count < 1 || !workspace || !plan ||
        workspace_bytes < fdtd_batch_workspace_bytes(count) || ((uintptr_t)workspace & 63)) {
        set_error("fdtd_batch_prepare: invalid arguments (workspace of "
                  "fdtd_batch_workspace_bytes(count), 64-byte aligned)");
        return FDTD_ERR_ARG;
    }
    FzInstance *host = new (std::nothrow) FzInstance[count];
    if (!host) {
        set_error("fdtd_batch_prepare: host allocation failed");
        return FDTD_ERR_CUDA;
    }
    int rc = 0, S0 = 0, V0 = 0, threads0 = 0;
    bool full0 = true;
    for (int i = 0; i < count && !rc; ++i) {
        fdtd_step_args a = args[i];
        if (a.pitch_z <= 0) a.pitch_z = a.nz;
        if (a.material_pitch <= 0) a.material_pitch = a.nz;
        a.schedule = nullptr;  // the batch schedule takes its place
        a.schedule_blocks = 0;
        if (a.nx <= 0 || a.ny <= 0 || a.nz <= 0 || !a.step || a.packed != FDTD_PSI_SLAB ||
            !fz_eligible(a) || a.tile_y < 1 || a.chunk_x < 1) {
            set_error("fdtd_batch_prepare: instance %d does not select the full-z path with a set "
                      "tile_y and chunk_x", i);
            rc = FDTD_ERR_ARG;
            break;
        }
        int S, V, threads;
        if ((rc = fz_build(a, host[i].maps, host[i].prm, S, V, threads))) break;
        const bool full = a.nz == a.pitch_z;
        if (i == 0) {
            S0 = S, V0 = V, threads0 = threads, full0 = full;
        } else if (S != S0 || V != V0 || threads != threads0 || full != full0 ||
                   host[i].prm.L.smem_bytes != host[0].prm.L.smem_bytes ||
                   a.material_kind != args[0].material_kind) {
            set_error("fdtd_batch_prepare: instance %d differs from instance 0 in row pitch, "
                      "z slab width, material kind, tile or stages", i);
            rc = FDTD_ERR_ARG;
        }
    }
    int dev = 0, base = -1;
    if (!rc) {
        cudaError_t err = cudaGetDevice(&dev);
        if (err == cudaSuccess && (dev < 0 || dev >= 64)) err = cudaErrorInvalidDevice;
        if (err == cudaSuccess && (base = fz_slots_take(dev, count)) < 0) {
            set_error("fdtd_batch_prepare: %d grids exceed the %d free parameter slots of live "
                      "batches (fdtd_batch_release frees them)", count, FZ_BATCH_SLOTS);
            rc = FDTD_ERR_ARG;
        }
        for (int i = 0; !rc && err == cudaSuccess && i < count; ++i)
            err = cudaMemcpyToSymbol(g_batch_prm, &host[i].prm, sizeof(FzParams),
                                     (size_t)(base + i) * sizeof(FzParams));
        if (!rc && err == cudaSuccess)
            err = cudaMemcpy(workspace, host, sizeof(FzInstance) * (size_t)count,
                             cudaMemcpyHostToDevice);
        if (!rc && err != cudaSuccess) {
            set_error("fdtd_batch_prepare: %s", cudaGetErrorString(err));
            rc = FDTD_ERR_CUDA;
        }
        if (rc && base >= 0) fz_slots_give(dev, base, count);
    }
    if (!rc) {
        plan->count = count;
        plan->base = base;
        plan->device = dev;
        plan->smem_bytes = host[0].prm.L.smem_bytes;
        plan->threads = threads0;
        plan->material_kind = args[0].material_kind;
        plan->stages = S0;
        plan->vector = V0;
        plan->full_rows = full0 ? 1 : 0;
    }
    delete[] host;
    return rc;
}

extern "C" int fdtd_step_batch(const fdtd_batch_plan *plan, const void *workspace,
                               const int *schedule, int blocks, void *stream) {
    if (!plan || !workspace || !schedule || blocks < 1 || plan->count < 1 || plan->base < 0) {
        set_error("fdtd_step_batch: invalid arguments");
        return FDTD_ERR_ARG;
    }
    // the parameter slots and the workspace live on the plan's device
    int dev = -1;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) {
        set_error("fdtd_step_batch: %s", cudaGetErrorString(err));
        return FDTD_ERR_CUDA;
    }
    if (dev != plan->device) {
        set_error("fdtd_step_batch: the plan was prepared on device %d, device %d is current",
                  plan->device, dev);
        return FDTD_ERR_ARG;
    }
    FzBatchKernel kern = fz_pick_batch(plan->material_kind, plan->stages, plan->vector,
                                       plan->full_rows != 0);
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, plan->smem_bytes);
    kern<<<(unsigned)blocks, (unsigned)plan->threads, plan->smem_bytes, (cudaStream_t)stream>>>(
        (const FzInstance *)workspace, plan->base, plan->count, schedule);
    return launch_status("fdtd_step_batch");
}

extern "C" int fdtd_batch_release(fdtd_batch_plan *plan) {
    if (!plan || plan->count < 1 || plan->base < 0 || plan->device < 0 || plan->device >= 64) {
        set_error("fdtd_batch_release: not a prepared plan");
        return FDTD_ERR_ARG;
    }
    fz_slots_give(plan->device, plan->base, plan->count);
    plan->count = 0;
    plan->base = -1;
    return 0;
}
