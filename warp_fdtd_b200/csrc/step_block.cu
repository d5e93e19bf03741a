// Time-blocked fused Yee leapfrog over full-z tiles: one launch advances E and
// H by D = 1 or 2 time steps (the work of D x solver.py:194-237's update_e +
// update_h launches, kernels.py:77-148), reading each plane of E(n), H(n-1/2)
// once and writing E(n+D), H(n+D-1/2) once.
//
// A block owns rows [y0, y0 + TY) of the y-z plane over the whole z extent
// and a run of x planes [xa, xb).  It marches along x; per iteration it
// stages one plane p of E, H (with a -y halo), material and the z-slab CPML
// state by TMA and computes, from left to right along the wavefront,
//
//   (a) E1(p)     = E(n+1)   rows y0-(D-1) .. y0+TY+D-1     (R = TY + 2D - 1 rows)
//   (b) H1(p-1)   = H(n+1/2) rows y0-(D-1) .. y0+TY+D-2
//   (c) E2(p-1)   = E(n+2)   rows y0 .. y0+TY               (D = 2)
//   (d) H2(p-2)   = H(n+3/2) rows y0 .. y0+TY-1             (D = 2)
//
// The y halo is recomputed (E needs H at y-1, H needs E at y+1), so blocks
// never exchange data.  E1 and E2 of the previous plane and H1 of the current
// one live in shared-memory rings; the H of the previous plane at a thread's
// own cells stays in registers.  Two block barriers per iteration: one per
// time step at D = 2.
//
// Threads: one per group of four consecutive z cells of one row.  Groups whose
// cells carry z CPML ("slab" groups) are packed into their own warps before
// the plain groups, so the z filter is a warp-uniform branch: plain warps never
// execute it.  x CPML is uniform over a plane, y CPML over a row.
//
// CPML state ping-pongs like the fields (slab layout, FDTD_PSI_SLAB): step 1
// reads psi[s]; with D = 2 its result (the state after step n+1) is kept for
// step 2 in a shared-memory ring (z) and in a block-private global scratch
// ring (x, y; L2-resident), and step 2 writes psi[s^1].
//
// Arithmetic is the reference's, operand for operand (kernels.py:29-47,
// 113-142), so every path is bitwise equal to the single-step kernels and the
// CPU oracle.  Every TMA box starts on a 16-byte boundary and no multicast is
// used; every mbarrier wait is bounded (on expiry the block sets the error
// word, drains its own copies and exits).
#include <cstring>
#include <new>

#include "common.cuh"
#include "step_internal.h"
#include "tma_util.cuh"

namespace wfb {
namespace blk {

struct Layout {
    int D, TY, R, P, HB, RW, MB, RZ, S;
    int HS, ES;  // component strides (floats) of H boxes / rings and E boxes / rings
    int off_h, off_e, off_m, off_pze, off_pzh, stage_bytes;
    unsigned tx_bytes;
    int off_stages, off_e1, off_h1, off_e2, off_zr, off_coef, off_mtab, smem_bytes;
};

struct Maps {
    CUtensorMap E[2], H[2], M, PZE[2], PZH[2];
};

struct Params {
    fdtd_step_args a;
    Layout L;
    long long xoff, yoff, zoff;  // slab-block offsets (elements) inside a psi buffer
    int ni, ns, ts;              // plain / slab groups per row, threads of the slab lanes
    unsigned char group[FDTD_BLOCK_GROUPS_MAX];  // z groups: plain ones, then slab ones
    unsigned char warp_rows[16];  // plain warps: which run of 32 plain lanes each takes
    float *scratch;              // D = 2: per-block x/y CPML ring
    long long scratch_block;     // floats per block
    float *snap_e, *snap_h;      // D = 2: E(n+1), H(n+1/2) inside the boxes
    int segments;                // schedule entries per block
    int interior_blocks;         // blocks [0, interior_blocks) run the build without x/y CPML
    int nsnap;
    int snap[FDTD_SNAP_BOXES_MAX][6];
};

__host__ __device__ constexpr size_t up(size_t v, size_t al) { return (v + al - 1) / al * al; }

// Row stride (floats) of the staged boxes and rings: at least P + 4, and
// congruent to 4 * ni modulo 32 so that plain lanes (consecutive groups, ni
// per row) stay on consecutive 16-byte bank groups across a row change.
__host__ __device__ constexpr int row_stride(int P, int ni) {
    for (int w = P + 4; w <= 256; w += 4)
        if ((w - 4 * ni) % 32 == 0) return w;
    return P + 4;
}

__host__ __device__ constexpr Layout layout(int D, int ty, int P, int RZ, int S, int mat, int ni) {
    Layout L{};
    L.D = D;
    L.TY = ty;
    L.R = ty + 2 * D - 1;
    L.P = P;
    L.HB = row_stride(P, ni);
    L.RW = L.HB;
    L.MB = mat == 1 ? (int)up(P, 16) : P;
    L.RZ = RZ;
    L.S = S;
    const int R = L.R;
    L.HS = (R + 1) * L.HB;
    L.ES = R * L.RW;
    const size_t hb = (size_t)3 * L.HS * 4;
    const size_t eb = (size_t)3 * L.ES * 4;
    const size_t mb = (size_t)R * L.MB * (mat == 1 ? 1 : 4);
    const size_t zb = (size_t)2 * R * RZ * 4;
    L.off_h = 0;
    L.off_e = (int)up(hb, 128);
    L.off_m = (int)(L.off_e + up(eb, 128));
    L.off_pze = (int)(L.off_m + up(mb, 128));
    L.off_pzh = (int)(L.off_pze + up(zb, 128));
    L.stage_bytes = (int)(L.off_pzh + up(zb, 128));
    L.tx_bytes = (unsigned)(hb + eb + mb + (RZ > 0 ? 2 * zb : 0));
    L.off_stages = 128;
    // rings hold two planes (slot = iteration parity)
    L.off_e1 = (int)(L.off_stages + (size_t)S * L.stage_bytes);
    L.off_h1 = (int)(L.off_e1 + 2 * up(eb, 16));
    L.off_e2 = (int)(L.off_h1 + (D == 2 ? 2 * up(hb, 16) : 0));
    L.off_zr = (int)(L.off_e2 + (D == 2 ? 2 * up(eb, 16) : 0));
    L.off_coef = (int)(L.off_zr + (D == 2 ? up((size_t)8 * R * RZ * 4, 16) : 0));
    const size_t coef = (size_t)(2 * R + 2 * P) * 16;
    L.off_mtab = (int)up(L.off_coef + coef, 16);
    L.smem_bytes = (int)(L.off_mtab + (mat == 1 ? 256 * 4 : 0));
    return L;
}


// Geometry of a launch as compile-time constants (GeoFixed, for shapes the
// library is built for: shared-memory offsets then fold into the load and
// store instructions) or read from the parameters at run time (GeoRT).
struct GeoRT {
    static constexpr bool fixed = false;
    static constexpr Layout L{};
};

template <int D_, int TY_, int P_, int RZ_, int S_, int MAT_, int NI_>
struct GeoFixed {
    static constexpr bool fixed = true;
    static constexpr Layout L = layout(D_, TY_, P_, RZ_, S_, MAT_, NI_);
};

// V consecutive z cells of one row held by a thread (a group of four).
template <int V>
struct VF {
    float v[V];
};

template <int V>
__device__ __forceinline__ VF<V> ldv(const float *p) {
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
__device__ __forceinline__ VF<V> zerov() {
    VF<V> r;
#pragma unroll
    for (int j = 0; j < V; ++j) r.v[j] = 0.0f;
    return r;
}

template <int V>
__device__ __forceinline__ VF<V> subv(const VF<V> &a, const VF<V> &b) {
    VF<V> r;
#pragma unroll
    for (int j = 0; j < V; ++j) r.v[j] = a.v[j] - b.v[j];
    return r;
}

__device__ __forceinline__ bool active(float4 c) { return c.x != 0.0f || c.z != 1.0f; }

// kernels.py:29-47 for one difference with an active state (a != 0):
// psi' = b * psi + a * d, returns d / kappa + psi'.
__device__ __forceinline__ float cp1(float d, float4 c, float po, float &pn) {
    const float p = c.y * po + c.x * d;
    pn = p;
    return c.z * d + p;
}

// The pair of differences an axis filters, with a coefficient uniform over the
// thread's cells (x: the plane, y: the row) and a != 0.
template <int V>
__device__ __forceinline__ void filt_u(VF<V> &d0, VF<V> &d1, float4 c, const VF<V> &p0,
                                       const VF<V> &p1, VF<V> &n0, VF<V> &n1) {
#pragma unroll
    for (int j = 0; j < V; ++j) {
        d0.v[j] = cp1(d0.v[j], c, p0.v[j], n0.v[j]);
        d1.v[j] = cp1(d1.v[j], c, p1.v[j], n1.v[j]);
    }
}

// ... with a == 0 and 1/kappa != 1: the reference's d / kappa.
template <int V>
__device__ __forceinline__ void scale_u(VF<V> &d0, VF<V> &d1, float k) {
#pragma unroll
    for (int j = 0; j < V; ++j) {
        d0.v[j] = k * d0.v[j];
        d1.v[j] = k * d1.v[j];
    }
}

// z axis: a coefficient per cell; inactive cells (a == 0) keep zero state and
// give d / kappa.  Both results are computed and one is selected: lanes of a
// warp hold different groups, and a branch per cell would split the warp.
template <int V>
__device__ __forceinline__ void filt_z(VF<V> &d0, VF<V> &d1, const float4 *cz, const VF<V> &p0,
                                       const VF<V> &p1, VF<V> &n0, VF<V> &n1) {
#pragma unroll
    for (int j = 0; j < V; ++j) {
        const float4 c = cz[j];
        const bool on = c.x != 0.0f;
        const float k0 = c.z * d0.v[j], k1 = c.z * d1.v[j];
        const float q0 = c.y * p0.v[j] + c.x * d0.v[j];
        const float q1 = c.y * p1.v[j] + c.x * d1.v[j];
        d0.v[j] = on ? k0 + q0 : k0;
        d1.v[j] = on ? k1 + q1 : k1;
        n0.v[j] = on ? q0 : 0.0f;
        n1.v[j] = on ? q1 : 0.0f;
    }
}

// Differences of an update (kernels.py:87-96): d/dx of components 1, 2, d/dy
// of 0, 2, d/dz of 0, 1 at the thread's cells.
template <int V>
struct Diff {
    VF<V> x1, x2, y0, y2, z0, z1;
};

// E update (electric): H at the thread's cells `hc` (staged at hs, component
// stride HS), the row below at hs - HB, the cell before the first at the end
// of the previous vector (hs - V; for z = 0 the box's zero pad), and H of the
// previous plane `hp`.
template <int V>
__device__ __forceinline__ Diff<V> e_diffs(const float *hs, int HS, int HB, const VF<V> *hc,
                                           const VF<V> *hp) {
    Diff<V> d;
    const VF<V> b0 = ldv<V>(hs - HB), b2 = ldv<V>(hs + 2 * HS - HB);
    // whole-vector loads: lanes read consecutive words, free of bank conflicts
    const float m0 = ldv<V>(hs - V).v[V - 1], m1 = ldv<V>(hs + HS - V).v[V - 1];
    d.x1 = subv<V>(hc[1], hp[1]);
    d.x2 = subv<V>(hc[2], hp[2]);
    d.y0 = subv<V>(hc[0], b0);
    d.y2 = subv<V>(hc[2], b2);
    d.z0.v[0] = hc[0].v[0] - m0;
    d.z1.v[0] = hc[1].v[0] - m1;
#pragma unroll
    for (int j = 1; j < V; ++j) {
        d.z0.v[j] = hc[0].v[j] - hc[0].v[j - 1];
        d.z1.v[j] = hc[1].v[j] - hc[1].v[j - 1];
    }
    return d;
}

// H update (magnetic): E of this plane `eq` (ring at es, component stride
// ES, row stride RW; the cell after the last at es + V, for the last cells of
// a row the ring's zero pad) and E of the next plane `en`.
template <int V>
__device__ __forceinline__ Diff<V> h_diffs(const float *es, int ES, int RW, const VF<V> *eq,
                                           const VF<V> *en) {
    Diff<V> d;
    const VF<V> u0 = ldv<V>(es + RW), u2 = ldv<V>(es + 2 * ES + RW);
    const float p0 = ldv<V>(es + V).v[0], p1 = ldv<V>(es + ES + V).v[0];
    d.x1 = subv<V>(en[1], eq[1]);
    d.x2 = subv<V>(en[2], eq[2]);
    d.y0 = subv<V>(u0, eq[0]);
    d.y2 = subv<V>(u2, eq[2]);
#pragma unroll
    for (int j = 0; j + 1 < V; ++j) {
        d.z0.v[j] = eq[0].v[j + 1] - eq[0].v[j];
        d.z1.v[j] = eq[1].v[j + 1] - eq[1].v[j];
    }
    d.z0.v[V - 1] = p0 - eq[0].v[V - 1];
    d.z1.v[V - 1] = p1 - eq[1].v[V - 1];
    return d;
}

// kernels.py:121-127: E += (courant * curl) * inv_eps, curl = (dyz - dzy,
// dzx - dxz, dxy - dyx) of the filtered differences.
template <int V>
__device__ __forceinline__ VF<V> e_comb(const VF<V> &o, const VF<V> &u, const VF<V> &w, float c,
                                        const VF<V> &ie) {
    VF<V> r;
#pragma unroll
    for (int j = 0; j < V; ++j) r.v[j] = o.v[j] + (c * (u.v[j] - w.v[j])) * ie.v[j];
    return r;
}

// kernels.py:128-129: H -= courant * curl.
template <int V>
__device__ __forceinline__ VF<V> h_comb(const VF<V> &o, const VF<V> &u, const VF<V> &w, float c) {
    VF<V> r;
#pragma unroll
    for (int j = 0; j < V; ++j) r.v[j] = o.v[j] - c * (u.v[j] - w.v[j]);
    return r;
}

// Pieces of the march that run only in CPML slabs, on the source plane or
// inside snapshot boxes.
template <int V>
struct Pair {
    VF<V> a, b;
};

// One axis's pair of differences with a coefficient uniform over the group and
// a != 0 (kernels.py:29-47): old state at src / src + sslot, new state to
// dst / dst + dslot unless dst is null.
template <int V>
__device__ __forceinline__ Pair<V> axis_cpml(Pair<V> d, float4 c, const float *src, long long sslot,
                                          float *dst, long long dslot) {
    const VF<V> p0 = ldv<V>(src), p1 = ldv<V>(src + sslot);
    VF<V> n0, n1;
    filt_u<V>(d.a, d.b, c, p0, p1, n0, n1);
    if (dst) {
        stv<V>(dst, n0);
        stv<V>(dst + dslot, n1);
    }
    return d;
}

// The z pair with per-cell coefficients cz (shared memory); state at src /
// src + sslot, new state to dst / dst + dslot unless dst is null, when `has`.
template <int V>
__device__ __forceinline__ Pair<V> z_cpml(Pair<V> d, const float4 *cz, bool has, const float *src,
                                          long long sslot, float *dst, long long dslot) {
    const VF<V> p0 = has ? ldv<V>(src) : zerov<V>(), p1 = has ? ldv<V>(src + sslot) : zerov<V>();
    VF<V> n0, n1;
    filt_z<V>(d.a, d.b, cz, p0, p1, n0, n1);
    if (has && dst) {
        stv<V>(dst, n0);
        stv<V>(dst + dslot, n1);
    }
    return d;
}

// kernels.py:130-137 (electric, with inverse permittivity) and 138-141
// (magnetic) plane source at time tw for the group's cells below nz:
// components 1 and 2 in `v`.
template <int V>
__device__ __noinline__ Pair<V> plane_source(Pair<V> v, VF<V> ie, bool electric, const float *src,
                                             const float *waves, long long wc, long long syz,
                                             int nz, int y, int zv, int tw, float C) {
    if (tw < 0 || tw >= wc) return v;
    const float w2 = waves[2 * wc + tw], w1 = waves[wc + tw];
#pragma unroll
    for (int j = 0; j < V; ++j) {
        const int gz = zv + j;
        if (gz < nz) {
            const long long si = (long long)y * nz + gz;
            if (electric) {
                v.a.v[j] = v.a.v[j] + ((src[2 * syz + si] * w2) * C) * ie.v[j];
                v.b.v[j] = v.b.v[j] - ((src[syz + si] * w1) * C) * ie.v[j];
            } else {
                v.a.v[j] = v.a.v[j] - (src[2 * syz + si] * w2) * C;
                v.b.v[j] = v.b.v[j] + (src[syz + si] * w1) * C;
            }
        }
    }
    return v;
}

// Snapshot of the group's three components (inline: the blocks owning a
// detector row store one every iteration, and one wave waits for its slowest
// block).
template <int V>
__device__ __forceinline__ void snap_store(float *base, long long off, long long cols, VF<V> v0,
                                           VF<V> v1, VF<V> v2) {
    float *dst = base + off;
    stv<V>(dst, v0);
    stv<V>(dst + cols, v1);
    stv<V>(dst + 2 * cols, v2);
}

// A slab group must hold the aligned consecutive ranks rb .. rb+3 of its
// window when any of its cells has CPML state.
__device__ __forceinline__ bool ranks_ok(const float4 *tab, int RZ) {
    const int rb = (int)tab[0].w;
    bool psi = false, ok = true;
#pragma unroll
    for (int j = 0; j < 4; ++j)
        if (tab[j].x != 0.0f) {
            psi = true;
            ok &= (int)tab[j].w == rb + j;
        }
    return !psi || (ok && rb % 4 == 0 && rb + 4 <= RZ);
}

// Segment `seg` of this block: a schedule entry (tile, first plane, end
// plane, 0) of block b at b * segments + seg (tile < 0: none), or the uniform
// tile x chunk grid.  false for no segment; an entry outside the grid or longer
// than chunk_x sets error 3.
__device__ __forceinline__ bool block_segment(const fdtd_step_args &a, int ty, int segments,
                                              int seg, int &tyi, int &xa, int &xb) {
    const int tiles_y = (a.ny + ty - 1) / ty;
    if (a.schedule) {
        const int *e = a.schedule + 4 * ((i64)blockIdx.x * segments + seg);
        tyi = e[0];
        xa = e[1];
        xb = e[2];
        if (tyi < 0) return false;
        if (tyi >= tiles_y || xa < 0 || xb > a.nx || xb - xa > a.chunk_x || xa >= xb) {
            if (threadIdx.x == 0 && a.error) atomicExch(a.error, 3);
            return false;
        }
        return true;
    }
    if (seg > 0) return false;
    tyi = blockIdx.x % tiles_y;
    xa = (blockIdx.x / tiles_y) * a.chunk_x;
    xb = min(xa + a.chunk_x, a.nx);
    return xa < xb;
}

// Shared-memory regions of a block.
struct Smem {
    uint64_t *bars;
    unsigned char *stage0;
    float *e1r0, *h1r0, *e2r0, *zr;  // rings of two planes (slot = iteration parity)
    int e_slot, h_slot;               // floats per ring slot
    float4 *cey, *chy, *cez, *chz;    // CPML coefficients by row of the tile and by z
    float *mtab;
};

// The march of one thread over the block's segments: V cells per thread,
// SLAB for the groups with z CPML.  Every thread of the block runs the same
// sequence of barriers whatever its V.
template <int MAT, int D, int V, class G, bool XY>
__device__ __forceinline__ void march(const Maps &maps, const Params &prm, const Smem &sm, int r,
                                      int zv, bool live, bool slab, int rbe, int rbh, bool zEp,
                                      bool zHp, const float4 *zce, const float4 *zch) {
    const fdtd_step_args &a = prm.a;
    const Layout &L = prm.L;
    const int nx = a.nx, ny = a.ny, nz = a.nz;
    const int P = G::fixed ? G::L.P : L.P, TY = G::fixed ? G::L.TY : L.TY;
    const int R = G::fixed ? G::L.R : L.R, S = G::fixed ? G::L.S : L.S;
    const int HB = G::fixed ? G::L.HB : L.HB, RW = G::fixed ? G::L.RW : L.RW;
    const int HS = G::fixed ? G::L.HS : L.HS, ES = G::fixed ? G::L.ES : L.ES;
    const int RZ = G::fixed ? G::L.RZ : L.RZ, MB = G::fixed ? G::L.MB : L.MB;
    const int off_h = G::fixed ? G::L.off_h : L.off_h, off_e = G::fixed ? G::L.off_e : L.off_e;
    const int off_m = G::fixed ? G::L.off_m : L.off_m;
    const int off_pze = G::fixed ? G::L.off_pze : L.off_pze;
    const int off_pzh = G::fixed ? G::L.off_pzh : L.off_pzh;
    const int stage_bytes = G::fixed ? G::L.stage_bytes : L.stage_bytes;
    const unsigned tx_bytes = G::fixed ? G::L.tx_bytes : L.tx_bytes;
    const i64 plane = (i64)ny * P;
    const i64 cols = (i64)nx * plane;
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
    const float C = a.courant;
    const int tid = threadIdx.x, nth = blockDim.x;
    const i64 xslot = (i64)a.psi_rx * plane;
    const i64 yslot = (i64)a.psi_ry * nx * P;
    const i64 zslot = (i64)nx * ny * RZ;
    const float4 ident = make_float4(0.f, 1.f, 1.f, 0.f);

    const int ho = (r + 1) * HB + 4 + zv;  // own cells in an H box / H ring
    const int eo = r * RW + zv;            // ... in an E box / E ring
    const int mo = r * MB + zv;
    const bool zpart = zv + V > nz;        // the vector holds padding cells
    float *scr = D == 2 ? prm.scratch + (i64)blockIdx.x * prm.scratch_block + (i64)r * P + zv
                        : nullptr;
    const i64 sc_comp = (i64)R * P;  // scratch: [slot][field][comp 4][R][P]
    const int zr_comp = R * RZ;      // z ring:  [slot][field][comp 2][R][RZ]
    const i64 syz = (i64)ny * nz;
    const i64 wc = a.waves_cols;
    const long limit = 1L << 24;
    const int issuer = nth - 1;

    int tyi, xa, xb, y0 = 0, yf = 0, K = 0, g0 = 0;
    int y = 0;
    bool row_in = false, own_row = false, yE = false, yH = false;
    float4 cye = ident, cyh = ident;
    unsigned snapmask = 0;
    int snap_lo = 0, snap_hi = 0;
    bool snap_multi = false;
    i64 grow = 0;  // own cells in a field plane (elements)

    // stages are numbered across the block's segments: stage g uses ring slot
    // g % S and mbarrier phase (g / S) & 1 (tracked incrementally below)
    auto issue = [&](int k, int slot) {
        unsigned char *st = sm.stage0 + (size_t)slot * stage_bytes;
        uint64_t *bar = sm.bars + slot;
        const int p = xa - D + k;
        mbar_expect_tx(bar, tx_bytes);
        tma_load_4d(st + off_h, &maps.H[s], -4, yf - 1, p, 0, bar);
        tma_load_4d(st + off_e, &maps.E[s], 0, yf, p, 0, bar);
        tma_load_3d(st + off_m, &maps.M, 0, yf, p, bar);
        if (RZ > 0) {
            tma_load_4d(st + off_pze, &maps.PZE[s], 0, yf, p, 0, bar);
            tma_load_4d(st + off_pzh, &maps.PZH[s], 0, yf, p - 1, 0, bar);
        }
    };
    // does a snapshot box holding this thread's row and cells cover owned plane pl?
    auto snap_hit = [&](int pl) {
        if (pl < snap_lo || pl >= snap_hi) return false;
        if (!snap_multi) return true;
        for (int b = 0; b < prm.nsnap; ++b)
            if (((snapmask >> b) & 1u) && pl >= prm.snap[b][0] && pl < prm.snap[b][1]) return true;
        return false;
    };
    auto zmask = [&](VF<V> *v) {
        if (zpart)
#pragma unroll
            for (int j = 0; j < V; ++j)
                if (zv + j >= nz)
#pragma unroll
                    for (int c = 0; c < 3; ++c) v[c].v[j] = 0.0f;
    };
    auto store3 = [&](float *base, i64 pl, const VF<V> *v) {
        float *dst = base + pl * plane + grow;
        stv<V>(dst, v[0]);
        stv<V>(dst + cols, v[1]);
        stv<V>(dst + 2 * cols, v[2]);
    };
    auto ld3 = [&](const float *base, int stride, VF<V> *v) {
        v[0] = ldv<V>(base);
        v[1] = ldv<V>(base + stride);
        v[2] = ldv<V>(base + 2 * stride);
    };
    auto st3 = [&](float *base, int stride, const VF<V> *v) {
        stv<V>(base, v[0]);
        stv<V>(base + stride, v[1]);
        stv<V>(base + 2 * stride, v[2]);
    };
    bool timed_out = false;
    int issued = -1, done = -1;  // stage indices of the current segment
    for (int seg = 0; seg < prm.segments && !timed_out; ++seg) {
        if (!block_segment(a, TY, prm.segments, seg, tyi, xa, xb)) break;
        if (seg > 0) g0 += K;
        y0 = tyi * TY;
        yf = y0 - (D - 1);
        K = xb - xa + 2 * D;
        __syncthreads();  // the previous segment's readers are done with tables and rings
        for (int j = tid; j < R; j += nth) {
            const int yy = yf + j;
            const bool in = yy >= 0 && yy < ny;
            sm.cey[j] = in ? __ldg(ce + clen + yy) : ident;
            sm.chy[j] = in ? __ldg(ch + clen + yy) : ident;
        }
        __syncthreads();
        if constexpr (!XY) {
            // this build has no x/y CPML code: the segment's rows and every
            // plane it touches (xa - D - 1 .. xb + D) must have none
            bool bad = false;
            for (int j = tid; j < R; j += nth) bad |= active(sm.cey[j]) || active(sm.chy[j]);
            for (int j = xa - D - 1 + tid; j <= xb + D; j += nth)
                if (j >= 0 && j < nx) bad |= active(__ldg(ce + j)) || active(__ldg(ch + j));
            if (__syncthreads_or(bad)) {
                if (tid == 0 && a.error) atomicExch(a.error, 4);
                break;
            }
        }
        y = yf + r;
        row_in = live && y >= 0 && y < ny;
        own_row = row_in && r >= D - 1 && r < D - 1 + TY;
        cye = sm.cey[r];
        cyh = sm.chy[r];
        yE = active(cye);
        yH = active(cyh);
        grow = (i64)y * P + zv;
        snapmask = 0;
        snap_lo = 0;
        snap_hi = 0;
        if (D == 2 && own_row)
            for (int b = 0; b < prm.nsnap; ++b)
                if (y >= prm.snap[b][2] && y < prm.snap[b][3] && zv + V > prm.snap[b][4] &&
                    zv < prm.snap[b][5]) {
                    snap_lo = snapmask ? min(snap_lo, prm.snap[b][0]) : prm.snap[b][0];
                    snap_hi = snapmask ? max(snap_hi, prm.snap[b][1]) : prm.snap[b][1];
                    snapmask |= 1u << b;
                }
        // planes of this segment the thread may snapshot: the boxes' union
        // within the owned planes; the exact per-box test runs only for
        // threads whose boxes' plane ranges leave gaps in that union
        snap_multi = false;
        if (__popc(snapmask) > 1) {
            int cur = snap_lo;
            for (int pass = 0; pass < FDTD_SNAP_BOXES_MAX; ++pass)
                for (int b = 0; b < prm.nsnap; ++b)
                    if (((snapmask >> b) & 1u) && prm.snap[b][0] <= cur && cur < prm.snap[b][1])
                        cur = prm.snap[b][1];
            snap_multi = cur < snap_hi;
        }
        snap_lo = max(snap_lo, xa);
        snap_hi = min(snap_hi, xb);

        const int slot0 = g0 % S;
        int phase = (g0 / S) & 1;
        issued = min(K - 1, S - 1);
        if (tid == issuer)
            for (int k = 0; k <= issued; ++k) issue(k, (slot0 + k) % S);
        timed_out = !mbar_wait_bounded(sm.bars + slot0, phase, limit);
        done = timed_out ? -1 : 0;
        // H of the previous plane at this thread's cells (step-1 input), H of
        // step 1 two planes back (step-2 input), the previous plane's inverse
        // permittivity
        VF<V> h0c[3], h1c[3], iep;
        ld3((const float *)(sm.stage0 + (size_t)slot0 * stage_bytes + off_h) + ho, HS, h0c);
        h1c[0] = h1c[1] = h1c[2] = zerov<V>();
        iep = zerov<V>();
        if (__syncthreads_or(timed_out)) timed_out = true;
        if (!timed_out && S < K) {
            if (tid == issuer) issue(S, slot0);
            issued = S;
        }
        int slot = slot0;

        for (int k = 1; k < K && !timed_out; ++k) {
            const int p = xa - D + k;
            const int q = p - 1, pe = p - 1, ph = p - 2;
            // plane-uniform x coefficients of the updates, in flight during the wait
            const float4 cxa = XY && p >= 0 && p < nx ? __ldg(ce + p) : ident;
            const float4 cxb = XY && q >= 0 && q < nx ? __ldg(ch + q) : ident;
            const float4 cxc = XY && D == 2 && pe >= 0 && pe < nx ? __ldg(ce + pe) : ident;
            const float4 cxd = XY && D == 2 && ph >= 0 && ph < nx ? __ldg(ch + ph) : ident;
            if (++slot == S) {
                slot = 0;
                phase ^= 1;
            }
            if (mbar_wait_bounded(sm.bars + slot, phase, limit))
                done = k;
            else
                timed_out = true;
            const unsigned char *st = sm.stage0 + (size_t)slot * stage_bytes;
            const float *Hb = (const float *)(st + off_h);
            const float *Eb = (const float *)(st + off_e);
            float *e1w = sm.e1r0 + (k & 1) * sm.e_slot;        // E1 of plane p (written now)
            const float *e1p = sm.e1r0 + (~k & 1) * sm.e_slot;  // E1 of plane p-1
            float *h1w = sm.h1r0 + (k & 1) * sm.h_slot;        // H1 of plane p-1 (written now)
            float *e2w = sm.e2r0 + (k & 1) * sm.e_slot;        // E2 of plane p-1 (written now)
            const float *e2p = sm.e2r0 + (~k & 1) * sm.e_slot;  // E2 of plane p-2

            // ---------------- (a) E1 at plane p, rows 0 .. R-1 ----------------
            VF<V> e1[3], ie;
            e1[0] = e1[1] = e1[2] = zerov<V>();
            if (MAT == 1) {
                if constexpr (V == 4) {
                    const uchar4 m = *(const uchar4 *)(st + off_m + mo);
                    ie.v[0] = sm.mtab[m.x];
                    ie.v[1] = sm.mtab[m.y];
                    ie.v[2] = sm.mtab[m.z];
                    ie.v[3] = sm.mtab[m.w];
                } else {
                    const uchar2 m = *(const uchar2 *)(st + off_m + mo);
                    ie.v[0] = sm.mtab[m.x];
                    ie.v[1] = sm.mtab[m.y];
                }
            } else {
                ie = ldv<V>((const float *)(st + off_m) + mo);
            }
            if (!timed_out && row_in && p >= 0 && p < nx) {
                VF<V> hcur[3];
                ld3(Hb + ho, HS, hcur);
                Diff<V> d = e_diffs<V>(Hb + ho, HS, HB, hcur, h0c);
                const float4 cx = cxa;
                const bool own = D == 1 && own_row && p >= xa && p < xb;
                if (XY && cx.x != 0.0f) {
                    const i64 ib = prm.xoff + ((i64)(int)cx.w * ny + y) * P + zv;
                    const Pair<V> f = axis_cpml<V>({d.x2, d.x1}, cx, pe_o + ib, xslot, D == 2 ? scr + (i64)((k & 1) * 2 + 0) * 4 * sc_comp : own ? pe_n + ib : nullptr, D == 2 ? sc_comp : xslot);
                    d.x2 = f.a;
                    d.x1 = f.b;
                } else if (XY && cx.z != 1.0f) {
                    scale_u<V>(d.x2, d.x1, cx.z);
                }
                if (XY && yE) {
                    if (cye.x != 0.0f) {
                        const i64 ib = prm.yoff + ((i64)(int)cye.w * nx + p) * P + zv;
                        const Pair<V> f = axis_cpml<V>({d.y0, d.y2}, cye, pe_o + ib, yslot, D == 2 ? scr + (i64)((k & 1) * 2 + 0) * 4 * sc_comp + 2 * sc_comp : own ? pe_n + ib : nullptr, D == 2 ? sc_comp : yslot);
                        d.y0 = f.a;
                        d.y2 = f.b;
                    } else {
                        scale_u<V>(d.y0, d.y2, cye.z);
                    }
                }
                if (slab) {
                    const i64 ib = prm.zoff + ((i64)p * ny + y) * RZ + rbe;
                    const Pair<V> f = z_cpml<V>({d.z1, d.z0}, zce, zEp, (const float *)(st + off_pze) + r * RZ + rbe, R * RZ, D == 2 ? sm.zr + ((k & 1) * 2 + 0) * 2 * zr_comp + r * RZ + rbe : own ? pe_n + ib : nullptr, D == 2 ? (i64)zr_comp : zslot);
                    d.z1 = f.a;
                    d.z0 = f.b;
                }
                VF<V> eo3[3];
                ld3(Eb + eo, ES, eo3);
                e1[0] = e_comb<V>(eo3[0], d.y2, d.z1, C, ie);
                e1[1] = e_comb<V>(eo3[1], d.z0, d.x2, C, ie);
                e1[2] = e_comb<V>(eo3[2], d.x1, d.y0, C, ie);
                if (p == a.source_x) {
                    const Pair<V> v = plane_source<V>({e1[1], e1[2]}, ie, true, a.src_h, a.waves_h, wc,
                                                syz, nz, y, zv, t, C);
                    e1[1] = v.a;
                    e1[2] = v.b;
                }
                zmask(e1);
                if (D == 1) {
                    if (own) store3(En, p, e1);
                } else if (snap_hit(p)) {
                    snap_store<V>(prm.snap_e, p * plane + grow, cols, e1[0], e1[1], e1[2]);
                }
            }
            if (live) st3(e1w + eo, ES, e1);

            // ---------------- (b) H1 at plane q = p-1, rows 0 .. R-2 ----------------
            VF<V> h1[3];
            h1[0] = h1[1] = h1[2] = zerov<V>();
            if (!timed_out && k >= 2 && r < R - 1 && row_in && q >= 0 && q < nx) {
                VF<V> eq[3];
                ld3(e1p + eo, ES, eq);
                Diff<V> d = h_diffs<V>(e1p + eo, ES, RW, eq, e1);
                const float4 cx = cxb;
                const bool own = D == 1 && own_row && q >= xa && q < xb;
                if (XY && cx.x != 0.0f) {
                    const i64 ib = prm.xoff + ((i64)(int)cx.w * ny + y) * P + zv;
                    const Pair<V> f = axis_cpml<V>({d.x2, d.x1}, cx, ph_o + ib, xslot, D == 2 ? scr + (i64)((k & 1) * 2 + 1) * 4 * sc_comp : own ? ph_n + ib : nullptr, D == 2 ? sc_comp : xslot);
                    d.x2 = f.a;
                    d.x1 = f.b;
                } else if (XY && cx.z != 1.0f) {
                    scale_u<V>(d.x2, d.x1, cx.z);
                }
                if (XY && yH) {
                    if (cyh.x != 0.0f) {
                        const i64 ib = prm.yoff + ((i64)(int)cyh.w * nx + q) * P + zv;
                        const Pair<V> f = axis_cpml<V>({d.y0, d.y2}, cyh, ph_o + ib, yslot, D == 2 ? scr + (i64)((k & 1) * 2 + 1) * 4 * sc_comp + 2 * sc_comp : own ? ph_n + ib : nullptr, D == 2 ? sc_comp : yslot);
                        d.y0 = f.a;
                        d.y2 = f.b;
                    } else {
                        scale_u<V>(d.y0, d.y2, cyh.z);
                    }
                }
                if (slab) {
                    const i64 ib = prm.zoff + ((i64)q * ny + y) * RZ + rbh;
                    const Pair<V> f = z_cpml<V>({d.z1, d.z0}, zch, zHp, (const float *)(st + off_pzh) + r * RZ + rbh, R * RZ, D == 2 ? sm.zr + ((k & 1) * 2 + 1) * 2 * zr_comp + r * RZ + rbh : own ? ph_n + ib : nullptr, D == 2 ? (i64)zr_comp : zslot);
                    d.z1 = f.a;
                    d.z0 = f.b;
                }
                h1[0] = h_comb<V>(h0c[0], d.y2, d.z1, C);
                h1[1] = h_comb<V>(h0c[1], d.z0, d.x2, C);
                h1[2] = h_comb<V>(h0c[2], d.x1, d.y0, C);
                if (q == a.source_x) {
                    const Pair<V> v = plane_source<V>({h1[1], h1[2]}, zerov<V>(), false, a.src_e,
                                                a.waves_e, wc, syz, nz, y, zv, t, C);
                    h1[1] = v.a;
                    h1[2] = v.b;
                }
                if (D == 1) {
                    if (own) store3(Hn, q, h1);
                } else if (snap_hit(q)) {
                    snap_store<V>(prm.snap_h, q * plane + grow, cols, h1[0], h1[1], h1[2]);
                }
            }
            if (D == 2 && r < R - 1) st3(h1w + ho, HS, h1);
            // H of plane p at this thread's cells, for the next plane's updates
            ld3(Hb + ho, HS, h0c);

            if (__syncthreads_or(timed_out)) {
                timed_out = true;
                break;
            }
            // stage k is no longer read: refill its slot with stage k + S
            if (k + S < K) {
                if (tid == issuer) issue(k + S, slot);
                issued = k + S;
            }
            if constexpr (D == 2) {
                // ---------------- (c) E2 at plane p-1, rows 1 .. R-2 ----------------
                VF<V> e2[3];
                e2[0] = e2[1] = e2[2] = zerov<V>();
                if (k >= 3 && r >= 1 && r < R - 1 && row_in && pe >= 0 && pe < nx) {
                    Diff<V> d = e_diffs<V>(h1w + ho, HS, HB, h1, h1c);
                    const int sl = (k - 1) & 1;
                    const float4 cx = cxc;
                    const bool own = own_row && pe >= xa && pe < xb;
                    if (XY && cx.x != 0.0f) {
                        const i64 ib = prm.xoff + ((i64)(int)cx.w * ny + y) * P + zv;
                        const Pair<V> f = axis_cpml<V>({d.x2, d.x1}, cx, scr + (i64)(sl * 2 + 0) * 4 * sc_comp, sc_comp, own ? pe_n + ib : nullptr, xslot);
                        d.x2 = f.a;
                        d.x1 = f.b;
                    } else if (XY && cx.z != 1.0f) {
                        scale_u<V>(d.x2, d.x1, cx.z);
                    }
                    if (XY && yE) {
                        if (cye.x != 0.0f) {
                            const i64 ib = prm.yoff + ((i64)(int)cye.w * nx + pe) * P + zv;
                            const Pair<V> f = axis_cpml<V>({d.y0, d.y2}, cye, scr + (i64)(sl * 2 + 0) * 4 * sc_comp + 2 * sc_comp, sc_comp, own ? pe_n + ib : nullptr, yslot);
                            d.y0 = f.a;
                            d.y2 = f.b;
                        } else {
                            scale_u<V>(d.y0, d.y2, cye.z);
                        }
                    }
                    if (slab) {
                        const i64 ib = prm.zoff + ((i64)pe * ny + y) * RZ + rbe;
                        const Pair<V> f = z_cpml<V>({d.z1, d.z0}, zce, zEp, sm.zr + (sl * 2 + 0) * 2 * zr_comp + r * RZ + rbe, zr_comp, own ? pe_n + ib : nullptr, zslot);
                        d.z1 = f.a;
                        d.z0 = f.b;
                    }
                    VF<V> eold[3];
                    ld3(e1p + eo, ES, eold);
                    e2[0] = e_comb<V>(eold[0], d.y2, d.z1, C, iep);
                    e2[1] = e_comb<V>(eold[1], d.z0, d.x2, C, iep);
                    e2[2] = e_comb<V>(eold[2], d.x1, d.y0, C, iep);
                    if (pe == a.source_x) {
                        const Pair<V> v = plane_source<V>({e2[1], e2[2]}, iep, true, a.src_h, a.waves_h,
                                                    wc, syz, nz, y, zv, t + 1, C);
                        e2[1] = v.a;
                        e2[2] = v.b;
                    }
                    zmask(e2);
                    if (own) store3(En, pe, e2);
                }
                if (live && r >= 1 && r < R - 1) st3(e2w + eo, ES, e2);

                // ---------------- (d) H2 at plane p-2, rows 1 .. R-3 ----------------
                if (k >= 4 && r >= 1 && r < R - 2 && row_in && ph >= xa && ph < xb) {
                    VF<V> eq[3];
                    ld3(e2p + eo, ES, eq);
                    Diff<V> d = h_diffs<V>(e2p + eo, ES, RW, eq, e2);
                    const int sl = (k - 1) & 1;
                    const float4 cx = cxd;
                    const bool own = own_row;
                    if (XY && cx.x != 0.0f) {
                        const i64 ib = prm.xoff + ((i64)(int)cx.w * ny + y) * P + zv;
                        const Pair<V> f = axis_cpml<V>({d.x2, d.x1}, cx, scr + (i64)(sl * 2 + 1) * 4 * sc_comp, sc_comp, own ? ph_n + ib : nullptr, xslot);
                        d.x2 = f.a;
                        d.x1 = f.b;
                    } else if (XY && cx.z != 1.0f) {
                        scale_u<V>(d.x2, d.x1, cx.z);
                    }
                    if (XY && yH) {
                        if (cyh.x != 0.0f) {
                            const i64 ib = prm.yoff + ((i64)(int)cyh.w * nx + ph) * P + zv;
                            const Pair<V> f = axis_cpml<V>({d.y0, d.y2}, cyh, scr + (i64)(sl * 2 + 1) * 4 * sc_comp + 2 * sc_comp, sc_comp, own ? ph_n + ib : nullptr, yslot);
                            d.y0 = f.a;
                            d.y2 = f.b;
                        } else {
                            scale_u<V>(d.y0, d.y2, cyh.z);
                        }
                    }
                    if (slab) {
                        const i64 ib = prm.zoff + ((i64)ph * ny + y) * RZ + rbh;
                        const Pair<V> f = z_cpml<V>({d.z1, d.z0}, zch, zHp, sm.zr + (sl * 2 + 1) * 2 * zr_comp + r * RZ + rbh, zr_comp, own ? ph_n + ib : nullptr, zslot);
                        d.z1 = f.a;
                        d.z0 = f.b;
                    }
                    VF<V> h2[3];
                    h2[0] = h_comb<V>(h1c[0], d.y2, d.z1, C);
                    h2[1] = h_comb<V>(h1c[1], d.z0, d.x2, C);
                    h2[2] = h_comb<V>(h1c[2], d.x1, d.y0, C);
                    if (ph == a.source_x) {
                        const Pair<V> v = plane_source<V>({h2[1], h2[2]}, zerov<V>(), false, a.src_e,
                                                    a.waves_e, wc, syz, nz, y, zv, t + 1, C);
                        h2[1] = v.a;
                        h2[2] = v.b;
                    }
                    if (own) store3(Hn, ph, h2);
                }
                h1c[0] = h1[0];
                h1c[1] = h1[1];
                h1c[2] = h1[2];
                iep = ie;
            }
        }
    }  // segments
    if (timed_out) {
        if (tid == 0) {
            if (a.error) atomicExch(a.error, 1);
            for (int j = done + 1; j <= issued; ++j)
                mbar_wait_bounded(sm.bars + ((g0 + j) % S), ((g0 + j) / S) & 1, limit);
        }
        __syncthreads();
    }
}

template <int MAT, int D, int NT, int MINB, class G>
__global__ void __launch_bounds__(NT, MINB)
    block_step_kernel(const __grid_constant__ Maps maps, const __grid_constant__ Params prm) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const fdtd_step_args &a = prm.a;
    const Layout &L = prm.L;
    {
        int tyi, xa, xb;
        if (!block_segment(a, L.TY, prm.segments, 0, tyi, xa, xb)) return;
    }
    const int nz = a.nz, P = L.P, R = L.R, S = L.S, RZ = L.RZ;
    const float4 *__restrict__ ce = (const float4 *)a.coeff_e;
    const float4 *__restrict__ ch = (const float4 *)a.coeff_h;
    const int clen = a.clen;
    const int tid = threadIdx.x, nth = blockDim.x;

    Smem sm;
    sm.bars = (uint64_t *)smem;
    int *meta = (int *)(smem + 64);
    sm.stage0 = smem + L.off_stages;
    sm.e1r0 = (float *)(smem + L.off_e1);
    sm.h1r0 = (float *)(smem + L.off_h1);
    sm.e2r0 = (float *)(smem + L.off_e2);
    sm.zr = (float *)(smem + L.off_zr);
    sm.e_slot = (L.off_h1 - L.off_e1) / 8;
    sm.h_slot = (L.off_e2 - L.off_h1) / 8;
    sm.cey = (float4 *)(smem + L.off_coef);
    sm.chy = sm.cey + R;
    sm.cez = sm.chy + R;
    sm.chz = sm.cez + P;
    sm.mtab = (float *)(smem + L.off_mtab);

    if (tid == 0) {
        for (int j = 0; j < S; ++j) mbar_init(sm.bars + j, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (MAT == 1)
        for (int j = tid; j < 256; j += nth) sm.mtab[j] = j < a.material_count ? a.material_table[j] : 0.0f;
    const float4 ident = make_float4(0.f, 1.f, 1.f, 0.f);
    for (int j = tid; j < P; j += nth) {
        sm.cez[j] = j < nz ? __ldg(ce + 2 * clen + j) : ident;
        sm.chz[j] = j < nz ? __ldg(ch + 2 * clen + j) : ident;
    }
    {
        // rings start at zero: their pad columns (z = -4..-1 of H, z >= P of
        // E) are the grid's zero padding and are never written
        const int n4 = (L.off_coef - L.off_e1) / 16;
        float4 *r4 = (float4 *)(smem + L.off_e1);
        for (int j = tid; j < n4; j += nth) r4[j] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    __syncthreads();
    if (tid == 0) {
        int bad = 0;
        for (int j = 0; j < prm.ni; ++j) {
            const int g = prm.group[j];
            for (int c = 0; c < 4; ++c)
                if (active(sm.cez[4 * g + c]) || active(sm.chz[4 * g + c])) bad = 1;
        }
        for (int j = 0; j < prm.ns; ++j) {
            const int g = prm.group[prm.ni + j];
            if (!(ranks_ok(sm.cez + 4 * g, RZ) && ranks_ok(sm.chz + 4 * g, RZ))) bad = 1;
        }
        meta[0] = bad;
    }
    __syncthreads();
    if (meta[0]) {
        if (tid == 0 && a.error) atomicExch(a.error, 2);
        return;  // nothing issued yet
    }

    // this thread's row r of the tile (y = yf + r) and group of four z cells;
    // the groups with z CPML run in warps of their own after the plain ones,
    // so the z filter is a warp-uniform branch.  One instruction stream for
    // all warps keeps the loop's code small.
    // (slab warps first: they carry the longest dependency chains)
    const bool slab = tid < prm.ts;
    int r, zv;
    if (slab) {
        r = tid / prm.ns;
        zv = 4 * prm.group[prm.ni + (tid - r * prm.ns)];
    } else {
        const int u = 32 * prm.warp_rows[(tid - prm.ts) >> 5] + (tid & 31);
        r = u / prm.ni;
        zv = 4 * prm.group[u - r * prm.ni];
    }
    const bool live = r < R;
    bool zEp = false, zHp = false;
    if (slab)
        for (int j = 0; j < 4; ++j) {
            zEp |= sm.cez[zv + j].x != 0.0f;
            zHp |= sm.chz[zv + j].x != 0.0f;
        }
    const int rbe = slab ? (int)sm.cez[zv].w : 0, rbh = slab ? (int)sm.chz[zv].w : 0;
    // the z coefficients stay in shared memory: registers held for them by
    // every thread would cost the plain threads more than the loads cost the
    // slab threads
    const float4 *zce = sm.cez + zv, *zch = sm.chz + zv;
    const int rr = live ? r : R - 1;
    // blocks scheduled on planes and rows free of x/y CPML run the build
    // without that code: its call sites and state would otherwise occupy
    // registers on every iteration
    if ((int)blockIdx.x < prm.interior_blocks)
        march<MAT, D, 4, G, false>(maps, prm, sm, rr, zv, live, slab, rbe, rbh, zEp, zHp, zce, zch);
    else
        march<MAT, D, 4, G, true>(maps, prm, sm, rr, zv, live, slab, rbe, rbh, zEp, zHp, zce, zch);
}

using Kernel = void (*)(Maps, Params);

// Register budgets: one block of up to 384 threads per SM (168 registers a
// thread), 448 (144) or 512 (128), or at depth 1 two blocks of up to 288 (96).
template <int NT, int MINB>
static Kernel pick_nt(int mat, int D) {
    if (mat == 1)
        return D == 2 ? block_step_kernel<1, 2, NT, MINB, GeoRT>
                      : block_step_kernel<1, 1, NT, MINB, GeoRT>;
    return D == 2 ? block_step_kernel<0, 2, NT, MINB, GeoRT> : block_step_kernel<0, 1, NT, MINB, GeoRT>;
}

// Shapes built with compile-time geometry: the 20 nm bend's rows (pitch 144,
// z CPML slabs 24 cells wide in rank, 30 plain groups a row, uint8
// material, two stages) at the tiles the autotuned defaults pick.
using GeoBend2 = GeoFixed<2, 7, 144, 24, 2, 1, 30>;
using GeoBend1 = GeoFixed<1, 8, 144, 24, 2, 1, 30>;

static bool same_layout(const Layout &a, const Layout &b) {
    return a.D == b.D && a.TY == b.TY && a.R == b.R && a.P == b.P && a.HB == b.HB &&
           a.RW == b.RW && a.MB == b.MB && a.RZ == b.RZ && a.S == b.S &&
           a.smem_bytes == b.smem_bytes && a.tx_bytes == b.tx_bytes;
}

static Kernel pick(int mat, int D, int threads, int pair, const Layout &L) {
    if (mat == 1 && D == 2 && threads <= 384 && same_layout(L, GeoBend2::L))
        return block_step_kernel<1, 2, 384, 1, GeoBend2>;
    if (mat == 1 && D == 1 && !pair && threads <= 384 && same_layout(L, GeoBend1::L))
        return block_step_kernel<1, 1, 384, 1, GeoBend1>;
    if (pair && D == 1 && threads <= 288)
        return mat == 1 ? block_step_kernel<1, 1, 288, 2, GeoRT> : block_step_kernel<0, 1, 288, 2, GeoRT>;
    return threads <= 384 ? pick_nt<384, 1>(mat, D)
         : threads <= 448 ? pick_nt<448, 1>(mat, D) : pick_nt<512, 1>(mat, D);
}

constexpr int SMEM_MAX = 227 * 1024;
constexpr int THREADS_MAX = 512;

// one lane per group of four z cells and row; the slab lanes (groups with z
// CPML) in warps of their own
static int threads_for(int ni, int ns, int R) {
    return (ni * R + 31) / 32 * 32 + (ns * R + 31) / 32 * 32;
}

}  // namespace blk
}  // namespace wfb

using namespace wfb;
using namespace wfb::blk;

static int block_check_args(const fdtd_step_args &a, const char *where) {
    if (a.nx <= 0 || a.ny <= 0 || a.nz <= 0 || !a.step || !a.coeff_e || !a.coeff_h) {
        set_error("%s: invalid grid or null pointer", where);
        return FDTD_ERR_ARG;
    }
    for (int k = 0; k < 2; ++k)
        if (!a.E[k] || !a.H[k] || !a.psi_e[k] || !a.psi_h[k]) {
            set_error("%s: null field or CPML buffer", where);
            return FDTD_ERR_ARG;
        }
    if (a.packed != FDTD_PSI_SLAB || !fz_eligible(a) || a.pitch_z < a.nz) {
        set_error("%s: needs the slab CPML layout, pitch_z %% 4 == 0, nz <= pitch_z <= 248, "
                  "psi_rz %% 4 == 0 and 16-byte aligned buffers", where);
        return FDTD_ERR_ARG;
    }
    const int maxdim = a.nx > a.ny ? (a.nx > a.nz ? a.nx : a.nz) : (a.ny > a.nz ? a.ny : a.nz);
    if (a.clen < maxdim) {
        set_error("%s: coefficient length %d < largest dimension %d", where, a.clen, maxdim);
        return FDTD_ERR_ARG;
    }
    if (a.material_kind == 1) {
        if (!a.material || !a.material_table || a.material_count < 1 || a.material_count > 256) {
            set_error("%s: uint8 material needs a table of 1..256 entries", where);
            return FDTD_ERR_ARG;
        }
    } else if (a.material_kind != 0 || !a.inv_eps) {
        set_error("%s: material_kind must be 0 (inv_eps) or 1 (uint8 index)", where);
        return FDTD_ERR_ARG;
    }
    if (a.source_x >= 0 && (!a.src_e || !a.src_h || !a.waves_e || !a.waves_h)) {
        set_error("%s: source plane without profiles or waves", where);
        return FDTD_ERR_ARG;
    }
    return 0;
}

extern "C" int fdtd_step_block_prepare(const fdtd_step_args *args, int depth,
                                       fdtd_block_plan *plan) {
    if (!args || !plan || (depth != 1 && depth != 2)) {
        set_error("fdtd_step_block_prepare: invalid arguments (depth 1 or 2)");
        return FDTD_ERR_ARG;
    }
    fdtd_step_args a = *args;
    if (a.pitch_z <= 0) a.pitch_z = a.nz;
    if (a.material_pitch <= 0) a.material_pitch = a.nz;
    int rc = block_check_args(a, "fdtd_step_block_prepare");
    if (rc) return rc;
    const int P = a.pitch_z, G = P / 4;
    if (G > FDTD_BLOCK_GROUPS_MAX) {
        set_error("fdtd_step_block_prepare: %d z groups exceed %d", G, FDTD_BLOCK_GROUPS_MAX);
        return FDTD_ERR_ARG;
    }
    // the z coefficients decide which groups of four z cells carry CPML
    const int nzc = a.nz;
    float4 *zc = new (std::nothrow) float4[2 * (size_t)nzc];
    if (!zc) {
        set_error("fdtd_step_block_prepare: host allocation failed");
        return FDTD_ERR_CUDA;
    }
    cudaError_t err = cudaMemcpy(zc, (const float4 *)a.coeff_e + 2 * (size_t)a.clen,
                                 sizeof(float4) * nzc, cudaMemcpyDeviceToHost);
    if (err == cudaSuccess)
        err = cudaMemcpy(zc + nzc, (const float4 *)a.coeff_h + 2 * (size_t)a.clen,
                         sizeof(float4) * nzc, cudaMemcpyDeviceToHost);
    if (err != cudaSuccess) {
        delete[] zc;
        set_error("fdtd_step_block_prepare: %s", cudaGetErrorString(err));
        return FDTD_ERR_CUDA;
    }
    int ni = 0, ns = 0;
    unsigned char plain[FDTD_BLOCK_GROUPS_MAX], slabs[FDTD_BLOCK_GROUPS_MAX];
    for (int g = 0; g < G; ++g) {
        bool special = false;
        for (int j = 4 * g; j < 4 * g + 4 && j < nzc; ++j)
            for (int f = 0; f < 2; ++f) {
                const float4 c = zc[f * nzc + j];
                special |= c.x != 0.0f || c.z != 1.0f;
            }
        if (special)
            slabs[ns++] = (unsigned char)g;
        else
            plain[ni++] = (unsigned char)g;
    }
    delete[] zc;
    const int S = a.stages > 0 ? a.stages : 2;
    if (S < 2 || S > 4) {
        set_error("fdtd_step_block_prepare: 2..4 stages");
        return FDTD_ERR_ARG;
    }
    int ty = a.tile_y;
    if (ty <= 0) {
        // the tallest tile whose block fits the shared-memory limit and 384
        // threads (168 registers each), else 512 threads
        ty = 0;
        for (int cap = 384; cap <= THREADS_MAX && ty == 0; cap += THREADS_MAX - 384)
            for (int cand = 32; cand >= 1; --cand) {
                const Layout L = layout(depth, cand, P, a.psi_rz, S, a.material_kind, ni);
                if (threads_for(ni, ns, L.R) <= cap && L.smem_bytes <= SMEM_MAX) {
                    ty = cand;
                    break;
                }
            }
    }
    const Layout L = layout(depth, ty > 0 ? ty : 1, P, a.psi_rz, S, a.material_kind, ni);
    const int threads = threads_for(ni, ns, L.R);
    if (ty < 1 || threads > THREADS_MAX || L.smem_bytes > SMEM_MAX || L.R + 1 > 256) {
        set_error("fdtd_step_block_prepare: a tile of %d rows does not fit (%d threads, %d bytes)",
                  ty, threads, L.smem_bytes);
        return FDTD_ERR_ARG;
    }
    memset(plan, 0, sizeof(*plan));
    // two blocks per SM when a depth-1 block fits twice (registers capped at 96)
    plan->pair_blocks = depth == 1 && threads <= 288 && 2 * L.smem_bytes <= SMEM_MAX ? 1 : 0;
    plan->depth = depth;
    plan->tile_y = ty;
    plan->stages = S;
    plan->rows = L.R;
    plan->threads = threads;
    plan->groups_plain = ni;
    plan->groups_slab = ns;
    for (int j = 0; j < ni; ++j) plan->group[j] = plain[j];
    for (int j = 0; j < ns; ++j) plan->group[ni + j] = slabs[j];
    plan->scratch_block_bytes =
        depth == 2 ? (long long)2 * 2 * 4 * L.R * P * (long long)sizeof(float) : 0;
    int dev = 0;
    err = cudaGetDevice(&dev);
    int blocks = 0, sms = 0;
    Kernel k = pick(a.material_kind, depth, threads, plan->pair_blocks, L);
    if (err == cudaSuccess)
        err = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_MAX);
    if (err == cudaSuccess)
        err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, threads, L.smem_bytes);
    if (err == cudaSuccess) err = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (err != cudaSuccess) {
        set_error("fdtd_step_block_prepare: %s", cudaGetErrorString(err));
        return FDTD_ERR_CUDA;
    }
    plan->device = dev;
    plan->blocks_per_sm = blocks;
    plan->sms = sms;
    return 0;
}

extern "C" int fdtd_step_block(const fdtd_step_args *args, const fdtd_block_plan *plan,
                               const fdtd_block_extra *extra, void *stream) {
    if (!args || !plan || (plan->depth != 1 && plan->depth != 2)) {
        set_error("fdtd_step_block: invalid arguments");
        return FDTD_ERR_ARG;
    }
    fdtd_step_args a = *args;
    if (a.pitch_z <= 0) a.pitch_z = a.nz;
    if (a.material_pitch <= 0) a.material_pitch = a.nz;
    int rc = block_check_args(a, "fdtd_step_block");
    if (rc) return rc;
    const int D = plan->depth, P = a.pitch_z, RZ = a.psi_rz;
    const int ni = plan->groups_plain, ns = plan->groups_slab;
    if (ni < 0 || ns < 0 || ni + ns != P / 4 || plan->tile_y < 1 || plan->stages < 2 ||
        plan->stages > 4) {
        set_error("fdtd_step_block: the plan does not match these arguments (pitch %d)", P);
        return FDTD_ERR_ARG;
    }
    a.tile_y = plan->tile_y;
    const int tiles = (a.ny + a.tile_y - 1) / a.tile_y;
    if (a.schedule) {
        if (a.schedule_blocks < 1 || a.chunk_x < 1) {
            set_error("fdtd_step_block: a schedule needs schedule_blocks >= 1 and chunk_x >= its "
                      "longest entry");
            return FDTD_ERR_ARG;
        }
    } else if (a.chunk_x <= 0) {
        // about one wave of the resident blocks
        const int want = (plan->sms > 0 ? plan->sms : 148) * (plan->blocks_per_sm > 0 ? plan->blocks_per_sm : 1);
        const int chunks = (want + tiles - 1) / tiles;
        a.chunk_x = (a.nx + chunks - 1) / chunks;
    }
    const int blocks = a.schedule ? a.schedule_blocks : tiles * ((a.nx + a.chunk_x - 1) / a.chunk_x);
    Layout L = layout(D, a.tile_y, P, RZ, plan->stages, a.material_kind, ni);
    if (threads_for(ni, ns, L.R) != plan->threads || L.smem_bytes > SMEM_MAX) {
        set_error("fdtd_step_block: the plan does not match these arguments (%d bytes)",
                  L.smem_bytes);
        return FDTD_ERR_ARG;
    }
    Params prm;
    memset(&prm, 0, sizeof(prm));
    prm.a = a;
    prm.L = L;
    prm.xoff = 0;
    prm.yoff = (long long)2 * a.psi_rx * a.ny * P;
    prm.zoff = prm.yoff + (long long)2 * a.psi_ry * a.nx * P;
    prm.ni = ni;
    prm.ns = ns;
    prm.ts = (ns * L.R + 31) / 32 * 32;
    prm.segments = extra && extra->segments > 0 ? extra->segments : 1;
    prm.interior_blocks = extra ? extra->interior_blocks : 0;
    if (prm.interior_blocks < 0 || prm.interior_blocks > blocks) {
        set_error("fdtd_step_block: interior_blocks %d outside 0..%d", prm.interior_blocks, blocks);
        return FDTD_ERR_ARG;
    }
    if (prm.segments > 1 && !a.schedule) {
        set_error("fdtd_step_block: several segments per block need a schedule");
        return FDTD_ERR_ARG;
    }
    for (int j = 0; j < ni + ns; ++j) prm.group[j] = plan->group[j];
    {
        // Warps run on the SM's four schedulers by warp index mod 4.  The
        // slab warps (first) carry the longest work between two barriers, so
        // the plain warps that share their schedulers get the plain lanes
        // with the least work: the rows that skip phases (halo rows and the
        // padding lanes past the last row).
        const int nplain = (threads_for(ni, ns, L.R) - prm.ts) / 32, sw = prm.ts / 32;
        int work[16], order[16];
        for (int w = 0; w < nplain && w < 16; ++w) {
            work[w] = 0;
            for (int l = 0; l < 32; ++l) {
                const int u = 32 * w + l, r = u / ni;
                if (r >= L.R) continue;
                int ph = 1 + (r < L.R - 1);
                if (D == 2) ph += (r >= 1 && r < L.R - 1) + (r >= 1 && r < L.R - 2);
                work[w] = work[w] > ph ? work[w] : ph;
            }
            order[w] = w;
        }
        for (int i = 0; i < nplain && i < 16; ++i)  // lightest first
            for (int j = i + 1; j < nplain && j < 16; ++j)
                if (work[order[j]] < work[order[i]]) {
                    const int t = order[i];
                    order[i] = order[j];
                    order[j] = t;
                }
        bool slab_sched[4] = {false, false, false, false};
        for (int w = 0; w < sw; ++w) slab_sched[w & 3] = true;
        int next = 0;
        for (int pass = 0; pass < 2; ++pass)  // slab schedulers' warps first
            for (int w = 0; w < nplain && w < 16; ++w)
                if (slab_sched[(sw + w) & 3] == (pass == 0)) prm.warp_rows[w] = (unsigned char)order[next++];
    }
    if (D == 2) {
        if (!extra || !extra->scratch || ((uintptr_t)extra->scratch & 15) ||
            extra->scratch_bytes < plan->scratch_block_bytes * blocks) {
            set_error("fdtd_step_block: depth 2 needs a 16-byte aligned scratch of "
                      "scratch_block_bytes per block (%lld bytes)",
                      plan->scratch_block_bytes * blocks);
            return FDTD_ERR_ARG;
        }
        prm.scratch = extra->scratch;
        prm.scratch_block = plan->scratch_block_bytes / (long long)sizeof(float);
        prm.nsnap = extra->nsnap;
        if (prm.nsnap < 0 || prm.nsnap > FDTD_SNAP_BOXES_MAX ||
            (prm.nsnap > 0 && (!extra->snap_e || !extra->snap_h))) {
            set_error("fdtd_step_block: 0..%d snapshot boxes with both snapshot fields",
                      FDTD_SNAP_BOXES_MAX);
            return FDTD_ERR_ARG;
        }
        prm.snap_e = extra->snap_e;
        prm.snap_h = extra->snap_h;
        for (int b = 0; b < prm.nsnap; ++b)
            for (int j = 0; j < 6; ++j) prm.snap[b][j] = extra->snap_box[b][j];
    }
    rc = get_encoder();
    if (rc) return rc;
    Maps maps;
    const cuuint64_t nz = a.nz, ny = a.ny, nx = a.nx, pz = P;
    cuuint64_t fdims[4] = {nz, ny, nx, 3};
    cuuint64_t fstr[3] = {pz * 4, pz * ny * 4, pz * ny * nx * 4};
    cuuint32_t hbox[4] = {(cuuint32_t)L.HB, (cuuint32_t)(L.R + 1), 1, 3};
    cuuint32_t ebox[4] = {(cuuint32_t)L.RW, (cuuint32_t)L.R, 1, 3};
    for (int j = 0; j < 2; ++j) {
        if ((rc = encode(&maps.H[j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.H[j], fdims, fstr, hbox)))
            return rc;
        if ((rc = encode(&maps.E[j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.E[j], fdims, fstr, ebox)))
            return rc;
    }
    cuuint64_t mdims[3] = {nz, ny, nx};
    cuuint32_t mbox[3] = {(cuuint32_t)L.MB, (cuuint32_t)L.R, 1};
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
    if (RZ > 0) {
        const cuuint64_t rz = RZ;
        cuuint64_t zdims[4] = {rz, ny, nx, 2};
        cuuint64_t zstr[3] = {rz * 4, rz * ny * 4, rz * ny * nx * 4};
        cuuint32_t zbox[4] = {(cuuint32_t)RZ, (cuuint32_t)L.R, 1, 2};
        for (int j = 0; j < 2; ++j) {
            if ((rc = encode(&maps.PZE[j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.psi_e[j] + prm.zoff,
                             zdims, zstr, zbox)))
                return rc;
            if ((rc = encode(&maps.PZH[j], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, a.psi_h[j] + prm.zoff,
                             zdims, zstr, zbox)))
                return rc;
        }
    } else {
        maps.PZE[0] = maps.PZE[1] = maps.PZH[0] = maps.PZH[1] = maps.M;  // never loaded
    }
    Kernel k = pick(a.material_kind, D, plan->threads, plan->pair_blocks, L);
    cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, L.smem_bytes);
    k<<<(unsigned)blocks, (unsigned)plan->threads, L.smem_bytes, (cudaStream_t)stream>>>(maps, prm);
    return launch_status("fdtd_step_block");
}
