/*
 * CPU oracle for the uniform-grid Yee/CPML FDTD path of warp-fdtd.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is a plain-C restatement of the
 * reference's Warp kernels, used as the checker by tests/, by
 * __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The product
 * (warp_fdtd_b200/) never links, loads or calls it.
 *
 * Every function follows one reference kernel, cited by file:line within the
 * warp-fdtd project.  Arrays use the reference layout: a field is (3, n) float32
 * with n = nx*ny*nz and flat index i = (x*ny + y)*nz + z (z fastest).  Every
 * 2-D array is passed with its own column count so that the small "dummy"
 * arrays the reference tests pass (e.g. (3, 1)) are addressed exactly as the
 * reference addresses them.
 *
 * Floating point: the file is compiled with -ffp-contract=off and without
 * -ffast-math, so every expression rounds exactly as written, operand order
 * following the reference source.  The CUDA kernels are built with the same
 * rule (--fmad=false), which makes the two bitwise comparable.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

/* liboracle64.so is this file compiled with -DORACLE_F64: every float of the
 * restatement (fields, coefficients, psi, weights, scalars) becomes double,
 * the float64 run the float32 path's rounding error is measured against.
 * (The f-suffixed literals are exact in both.) */
#ifdef ORACLE_F64
#define float double
#endif

typedef long long i64;

/* kernels.py:8-26 `sample`: three components at (x, y, z), zero outside the
 * grid, or wrapped when periodic != 0. */
static inline void sample3(const float *f, i64 cols, int x, int y, int z, int nx,
                           int ny, int nz, int periodic, float out[3]) {
    if (periodic) {
        x = (x + nx) % nx;
        y = (y + ny) % ny;
        z = (z + nz) % nz;
    }
    if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) {
        out[0] = out[1] = out[2] = 0.0f;
        return;
    }
    i64 i = ((i64)x * ny + y) * nz + z;
    out[0] = f[i];
    out[1] = f[cols + i];
    out[2] = f[2 * cols + i];
}

/* kernels.py:29-47 `cpml` (full storage) and kernels.py:50-74 `cpml_packed`.
 * coeff is (3, clen, cw) with cw = 3 (a, b, 1/kappa) or 4 (+ plane rank). */
static inline float cpml_apply(float d, float *psi, i64 psi_cols, const float *coeff,
                               int clen, int cw, int packed, int axis, int position,
                               int slot, i64 i, int nx, int ny, int nz) {
    const float *c = coeff + ((i64)axis * clen + position) * cw;
    if (c[0] != 0.0f) {
        i64 index = i;
        if (packed) {
            i64 plane = (i64)(int)c[3];
            i64 nyz = (i64)ny * nz;
            index = plane * nyz + i % nyz;
            if (axis == 1)
                index = plane * nx * nz + (i / nyz) * nz + i % nz;
            else if (axis == 2)
                index = plane * nx * ny + i / nz;
        }
        float *ps = psi + (i64)slot * psi_cols + index;
        float p = c[1] * (*ps) + c[0] * d;
        *ps = p;
        return c[2] * d + p;
    }
    return c[2] * d;
}

/* kernels.py:77-142 `make_update(electric, packed)`: one Yee half-step.
 * f is updated in place from the other field g; psi holds the six CPML
 * auxiliary fields of f; source/waves inject the plane source at x ==
 * source_x; hprev receives the old H when (not electric) and t >= save_h_from.
 */
int oracle_update(int electric, int packed, float *f, const float *g, i64 fg_cols,
                  const float *inv_eps, float *psi, i64 psi_cols, const float *coeff,
                  int clen, const float *source, i64 source_cols, const float *waves,
                  i64 waves_cols, const int *step, float *hprev, i64 hprev_cols,
                  int save_h_from, int nx, int ny, int nz, int source_x, float courant,
                  int periodic) {
    const int cw = packed ? 4 : 3;
    const i64 n = (i64)nx * ny * nz;
    const int t = step[0];
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; ++i) {
        int z = (int)(i % nz);
        int y = (int)((i / nz) % ny);
        int x = (int)(i / ((i64)ny * nz));
        float v[3], a[3], b[3], c[3], dx[3], dy[3], dz[3];
        sample3(g, fg_cols, x, y, z, nx, ny, nz, periodic, v);
        if (electric) {
            sample3(g, fg_cols, x - 1, y, z, nx, ny, nz, periodic, a);
            sample3(g, fg_cols, x, y - 1, z, nx, ny, nz, periodic, b);
            sample3(g, fg_cols, x, y, z - 1, nx, ny, nz, periodic, c);
            for (int k = 0; k < 3; ++k) {
                dx[k] = v[k] - a[k];
                dy[k] = v[k] - b[k];
                dz[k] = v[k] - c[k];
            }
        } else {
            sample3(g, fg_cols, x + 1, y, z, nx, ny, nz, periodic, a);
            sample3(g, fg_cols, x, y + 1, z, nx, ny, nz, periodic, b);
            sample3(g, fg_cols, x, y, z + 1, nx, ny, nz, periodic, c);
            for (int k = 0; k < 3; ++k) {
                dx[k] = a[k] - v[k];
                dy[k] = b[k] - v[k];
                dz[k] = c[k] - v[k];
            }
        }
        float dxz = cpml_apply(dx[2], psi, psi_cols, coeff, clen, cw, packed, 0, x, 0, i, nx, ny, nz);
        float dxy = cpml_apply(dx[1], psi, psi_cols, coeff, clen, cw, packed, 0, x, 1, i, nx, ny, nz);
        float dyx = cpml_apply(dy[0], psi, psi_cols, coeff, clen, cw, packed, 1, y, 2, i, nx, ny, nz);
        float dyz = cpml_apply(dy[2], psi, psi_cols, coeff, clen, cw, packed, 1, y, 3, i, nx, ny, nz);
        float dzy = cpml_apply(dz[1], psi, psi_cols, coeff, clen, cw, packed, 2, z, 4, i, nx, ny, nz);
        float dzx = cpml_apply(dz[0], psi, psi_cols, coeff, clen, cw, packed, 2, z, 5, i, nx, ny, nz);
        float curl[3] = {dyz - dzy, dzx - dxz, dxy - dyx};
        float old[3] = {f[i], f[fg_cols + i], f[2 * fg_cols + i]};
        float value[3];
        if (electric) {
            float ie = inv_eps[i];
            for (int k = 0; k < 3; ++k) {
                float s = courant * curl[k];
                s = s * ie;
                value[k] = old[k] + s;
            }
            if (x == source_x) {
                i64 s = (i64)y * nz + z;
                float u = source[2 * source_cols + s] * waves[2 * waves_cols + t];
                u = u * courant;
                u = u * ie;
                value[1] = value[1] + u;
                float w = source[1 * source_cols + s] * waves[1 * waves_cols + t];
                w = w * courant;
                w = w * ie;
                value[2] = value[2] - w;
            }
        } else {
            for (int k = 0; k < 3; ++k) {
                float s = courant * curl[k];
                value[k] = old[k] - s;
            }
            if (t >= save_h_from) {
                hprev[i] = old[0];
                hprev[hprev_cols + i] = old[1];
                hprev[2 * hprev_cols + i] = old[2];
            }
            if (x == source_x) {
                i64 s = (i64)y * nz + z;
                float u = source[2 * source_cols + s] * waves[2 * waves_cols + t];
                u = u * courant;
                value[1] = value[1] - u;
                float w = source[1 * source_cols + s] * waves[1 * waves_cols + t];
                w = w * courant;
                value[2] = value[2] + w;
            }
        }
        f[i] = value[0];
        f[fg_cols + i] = value[1];
        f[2 * fg_cols + i] = value[2];
    }
    return 0;
}

/* detectors.py:10-23 `ht`: temporal average of H(n+1/2) and H(n-1/2). */
static inline void ht3(const float *h, const float *prev, i64 cols, int x, int y, int z,
                       int nx, int ny, int nz, float out[3]) {
    float a[3], b[3];
    sample3(h, cols, x, y, z, nx, ny, nz, 0, a);
    sample3(prev, cols, x, y, z, nx, ny, nz, 0, b);
    for (int k = 0; k < 3; ++k) out[k] = 0.5f * (a[k] + b[k]);
}

/* detectors.py:26-62 `colocate`: E and H averaged to the Ez point, H also
 * time-centred.  The sums are evaluated left to right as written there. */
void oracle_colocate(const float *e, const float *h, const float *prev, i64 cols, int x,
                     int y, int z, int nx, int ny, int nz, float ec[3], float hc[3]) {
    float e0[3], ex[3], ey[3], ez[3], exz[3], eyz[3];
    sample3(e, cols, x, y, z, nx, ny, nz, 0, e0);
    sample3(e, cols, x - 1, y, z, nx, ny, nz, 0, ex);
    sample3(e, cols, x, y - 1, z, nx, ny, nz, 0, ey);
    sample3(e, cols, x, y, z + 1, nx, ny, nz, 0, ez);
    sample3(e, cols, x - 1, y, z + 1, nx, ny, nz, 0, exz);
    sample3(e, cols, x, y - 1, z + 1, nx, ny, nz, 0, eyz);
    ec[0] = 0.25f * (((e0[0] + ex[0]) + ez[0]) + exz[0]);
    ec[1] = 0.25f * (((e0[1] + ey[1]) + ez[1]) + eyz[1]);
    ec[2] = e0[2];
    float h0[3], hx[3], hy[3], hxy[3], hz[3], hxz[3], hyz[3], hxyz[3];
    ht3(h, prev, cols, x, y, z, nx, ny, nz, h0);
    ht3(h, prev, cols, x - 1, y, z, nx, ny, nz, hx);
    ht3(h, prev, cols, x, y - 1, z, nx, ny, nz, hy);
    ht3(h, prev, cols, x - 1, y - 1, z, nx, ny, nz, hxy);
    ht3(h, prev, cols, x, y, z + 1, nx, ny, nz, hz);
    ht3(h, prev, cols, x - 1, y, z + 1, nx, ny, nz, hxz);
    ht3(h, prev, cols, x, y - 1, z + 1, nx, ny, nz, hyz);
    ht3(h, prev, cols, x - 1, y - 1, z + 1, nx, ny, nz, hxyz);
    hc[0] = 0.5f * (h0[0] + hy[0]);
    hc[1] = 0.5f * (h0[1] + hx[1]);
    hc[2] = 0.125f * ((((((h0[2] + hx[2]) + hy[2]) + hxy[2]) + hz[2]) + hxz[2]) + hyz[2] + hxyz[2]);
}

/* Plane sample of one detector cell: colocated (exact) or the raw Yee
 * components, detectors.py:95-98. */
static inline void plane_sample(const float *e, const float *h, const float *prev, i64 cols,
                                int x, int y, int z, int nx, int ny, int nz, int exact,
                                float ee[3], float hh[3]) {
    if (exact) {
        oracle_colocate(e, h, prev, cols, x, y, z, nx, ny, nz, ee, hh);
    } else {
        sample3(e, cols, x, y, z, nx, ny, nz, 0, ee);
        sample3(h, cols, x, y, z, nx, ny, nz, 0, hh);
    }
}

/* detectors.py:65-106 `record`, phasor branch, generalised to K frequencies
 * with float64 accumulators: phasor[k, c, i] (re, im) += w[k, t] * field_c.
 * The fp32 weight and the fp32 colocated sample are promoted to double before
 * the product; the sum runs in time order, as each step calls this once.
 * weights is (K, wsteps, 2) float32; phasor is (K, 6, count, 2) float64. */
int oracle_record_phasor(const float *e, const float *h, const float *prev, i64 cols,
                         int t, const float *weights, int nfreq, i64 wsteps,
                         double *phasor, int nx, int ny, int nz, int x0, int y0, int z0,
                         int sx, int sy, int sz, int exact) {
    const i64 count = (i64)sx * sy * sz;
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < count; ++i) {
        int x = x0 + (int)(i / ((i64)sy * sz));
        int y = y0 + (int)((i / sz) % sy);
        int z = z0 + (int)(i % sz);
        float ee[3], hh[3];
        plane_sample(e, h, prev, cols, x, y, z, nx, ny, nz, exact, ee, hh);
        for (int k = 0; k < nfreq; ++k) {
            double wr = weights[((i64)k * wsteps + t) * 2];
            double wi = weights[((i64)k * wsteps + t) * 2 + 1];
            if (wr == 0.0 && wi == 0.0) continue;
            for (int c = 0; c < 6; ++c) {
                double v = c < 3 ? (double)ee[c] : (double)hh[c - 3];
                double *p = phasor + (((i64)k * 6 + c) * count + i) * 2;
                p[0] = p[0] + wr * v;
                p[1] = p[1] + wi * v;
            }
        }
    }
    return 0;
}

/* The same phasor branch in the reference's own float32 arithmetic
 * (complex64 accumulators as vec2), used to state the float64 accumulators'
 * effect against the reference's storage. phasor is (6, count, 2) float32. */
int oracle_record_phasor_f32(const float *e, const float *h, const float *prev, i64 cols,
                             int t, const float *weights, float *phasor, int nx, int ny,
                             int nz, int x0, int y0, int z0, int sx, int sy, int sz,
                             int exact) {
    const i64 count = (i64)sx * sy * sz;
    float wr = weights[2 * (i64)t], wi = weights[2 * (i64)t + 1];
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < count; ++i) {
        int x = x0 + (int)(i / ((i64)sy * sz));
        int y = y0 + (int)((i / sz) % sy);
        int z = z0 + (int)(i % sz);
        float ee[3], hh[3];
        plane_sample(e, h, prev, cols, x, y, z, nx, ny, nz, exact, ee, hh);
        for (int c = 0; c < 6; ++c) {
            float v = c < 3 ? ee[c] : hh[c - 3];
            float *p = phasor + ((i64)c * count + i) * 2;
            p[0] = p[0] + wr * v;
            p[1] = p[1] + wi * v;
        }
    }
    return 0;
}

/* detectors.py:104-106 `record`, flux branch: the plane sum of
 * cross(E, H)[axis] * area, returned in float64 (summed in cell order).  The
 * reference adds each cell's fp32 product to its fp32 bin with an atomic; this
 * oracle sums the fp32 products in double and the caller adds the total. */
double oracle_flux_sum(const float *e, const float *h, const float *prev, i64 cols,
                       const float *area, int nx, int ny, int nz, int x0, int y0, int z0,
                       int sx, int sy, int sz, int axis, int exact) {
    const i64 count = (i64)sx * sy * sz;
    double total = 0.0;
    for (i64 i = 0; i < count; ++i) {
        int x = x0 + (int)(i / ((i64)sy * sz));
        int y = y0 + (int)((i / sz) % sy);
        int z = z0 + (int)(i % sz);
        float a[3], b[3];
        plane_sample(e, h, prev, cols, x, y, z, nx, ny, nz, exact, a, b);
        float cr;
        if (axis == 0)
            cr = a[1] * b[2] - a[2] * b[1];
        else if (axis == 1)
            cr = a[2] * b[0] - a[0] * b[2];
        else
            cr = a[0] * b[1] - a[1] * b[0];
        float power = cr * area[i];
        total += (double)power;
    }
    return total;
}

/* adjoint.py:17-43 `record_curl`: courant * curl(H) (backward differences,
 * no CPML) at every design-box voxel, written to hist[t, c, j]. */
int oracle_record_curl(const float *h, i64 cols, float *hist, i64 design_n, int t, int nx,
                       int ny, int nz, int x0, int y0, int z0, int sx, int sy, int sz,
                       float courant) {
    (void)sx;
    for (i64 j = 0; j < design_n; ++j) {
        int x = x0 + (int)(j / ((i64)sy * sz));
        int y = y0 + (int)((j / sz) % sy);
        int z = z0 + (int)(j % sz);
        float v[3], a[3], b[3], c[3];
        sample3(h, cols, x, y, z, nx, ny, nz, 0, v);
        sample3(h, cols, x - 1, y, z, nx, ny, nz, 0, a);
        sample3(h, cols, x, y - 1, z, nx, ny, nz, 0, b);
        sample3(h, cols, x, y, z - 1, nx, ny, nz, 0, c);
        float dx[3], dy[3], dz[3];
        for (int k = 0; k < 3; ++k) {
            dx[k] = v[k] - a[k];
            dy[k] = v[k] - b[k];
            dz[k] = v[k] - c[k];
        }
        float curl[3] = {dy[2] - dz[1], dz[0] - dx[2], dx[1] - dy[0]};
        for (int k = 0; k < 3; ++k)
            hist[((i64)t * 3 + k) * design_n + j] = courant * curl[k];
    }
    return 0;
}

/* adjoint.py:46-88 `prepare`: transpose of the field scaling and of the CPML
 * recurrence.  q is the adjoint of f, psi the adjoint CPML state, d (6, n)
 * receives the adjoint of the six (CPML-filtered) differences. */
int oracle_prepare(const float *q, const float *eps, float *psi, const float *coeff,
                   int clen, float *d, int nx, int ny, int nz, float courant,
                   int electric) {
    const i64 n = (i64)nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; ++i) {
        int x = (int)(i / ((i64)ny * nz));
        int y = (int)((i / nz) % ny);
        int z = (int)(i % nz);
        float factor = -courant;
        if (electric) factor = courant * eps[i];
        float v[3] = {factor * q[i], factor * q[n + i], factor * q[2 * n + i]};
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
    return 0;
}

/* adjoint.py:91-104 `read`. */
static inline float read_d(const float *d, i64 n, int slot, int x, int y, int z, int nx,
                           int ny, int nz) {
    if (x < 0 || y < 0 || z < 0 || x >= nx || y >= ny || z >= nz) return 0.0f;
    return d[(i64)slot * n + ((i64)x * ny + y) * nz + z];
}

/* adjoint.py:107-162 `gather`: q += D^T d, and with from_h the design-box
 * inner product grad[j] += sum_c hist[t, c, j] * q_c.  This restatement keeps
 * grad in float32 like the reference (grad_is_f64 = 0) or in float64. */
int oracle_gather(float *q, const float *d, const float *hist, i64 design_n, void *grad,
                  int grad_is_f64, int t, int nx, int ny, int nz, int x0, int y0, int z0,
                  int sx, int sy, int sz, int from_h) {
    const i64 n = (i64)nx * ny * nz;
    const int delta = from_h ? -1 : 1;
#pragma omp parallel for schedule(static)
    for (i64 i = 0; i < n; ++i) {
        int x = (int)(i / ((i64)ny * nz));
        int y = (int)((i / nz) % ny);
        int z = (int)(i % nz);
        float v[3];
        v[0] = (read_d(d, n, 2, x, y + delta, z, nx, ny, nz) - d[2 * n + i]) +
               (read_d(d, n, 5, x, y, z + delta, nx, ny, nz) - d[5 * n + i]);
        v[1] = (read_d(d, n, 1, x + delta, y, z, nx, ny, nz) - d[1 * n + i]) +
               (read_d(d, n, 4, x, y, z + delta, nx, ny, nz) - d[4 * n + i]);
        v[2] = (read_d(d, n, 0, x + delta, y, z, nx, ny, nz) - d[0 * n + i]) +
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
        if (from_h && x >= x0 && x < x0 + sx && y >= y0 && y < y0 + sy && z >= z0 &&
            z < z0 + sz) {
            i64 j = ((i64)(x - x0) * sy + (y - y0)) * sz + (z - z0);
            const float *hh = hist + (i64)t * 3 * design_n;
            if (grad_is_f64) {
                double *g = (double *)grad;
                g[j] = g[j] + (((double)hh[j] * value[0] + (double)hh[design_n + j] * value[1]) +
                               (double)hh[2 * design_n + j] * value[2]);
            } else {
                float *g = (float *)grad;
                g[j] = g[j] + ((hh[j] * value[0] + hh[design_n + j] * value[1]) +
                               hh[2 * design_n + j] * value[2]);
            }
        }
    }
    return 0;
}

/* adjoint.py:165-178 `add` (bounds-checked scatter). */
static inline void add_q(float *q, i64 n, int c, int x, int y, int z, int nx, int ny, int nz,
                         float value) {
    if (x >= 0 && y >= 0 && z >= 0 && x < nx && y < ny && z < nz)
        q[(i64)c * n + ((i64)x * ny + y) * nz + z] += value;
}

/* adjoint.py:181-223 `inject`: transpose of the colocation, scattering the
 * real part of source * w[t] with the 1/4 and 1/16 weights.  source is
 * (6, count, 2) float32, weights (steps, 2).  Sequential scatter order. */
int oracle_inject(float *qe, float *qh, const float *source, const float *weights, int t,
                  int nx, int ny, int nz, int x0, int y0, int z0, int sx, int sy, int sz,
                  int old_h_only) {
    const i64 n = (i64)nx * ny * nz;
    const i64 count = (i64)sx * sy * sz;
    float w0 = weights[2 * (i64)t], w1 = weights[2 * (i64)t + 1];
    if (!(fabsf(w0) + fabsf(w1) > 0.0f)) return 0;
    for (i64 i = 0; i < count; ++i) {
        int x = x0 + (int)(i / ((i64)sy * sz));
        int y = y0 + (int)((i / sz) % sy);
        int z = z0 + (int)(i % sz);
        float v[6];
        for (int c = 0; c < 6; ++c) {
            const float *a = source + ((i64)c * count + i) * 2;
            v[c] = a[0] * w0 - a[1] * w1;
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
    return 0;
}

/* adjoint.py:472-490 `write_design`: eps[box] = plane[x, y] for all z. */
int oracle_write_design(const float *plane, float *eps, int nx, int ny, int nz, int x0,
                        int y0, int z0, int sx, int sy, int sz) {
    (void)nx;
    for (int x = 0; x < sx; ++x)
        for (int y = 0; y < sy; ++y)
            for (int z = 0; z < sz; ++z)
                eps[((i64)(x0 + x) * ny + y0 + y) * nz + z0 + z] = plane[(i64)x * sy + y];
    return 0;
}

/* Whole forward step of solver.py:194-237 for the CPU baseline timing:
 * update_e, update_h (no detectors), repeated `steps` times from step0. */
int oracle_run_steps(float *E, float *H, const float *inv_eps, float *psi_e, float *psi_h,
                     const float *coeff_e, const float *coeff_h, int clen,
                     const float *src_e, const float *src_h, const float *waves_e,
                     const float *waves_h, i64 waves_cols, int step0, int steps, int nx,
                     int ny, int nz, int source_x, float courant) {
    const i64 n = (i64)nx * ny * nz;
    float dummy[3] = {0, 0, 0};
    for (int s = 0; s < steps; ++s) {
        int t = step0 + s;
        oracle_update(1, 0, E, H, n, inv_eps, psi_e, n, coeff_e, clen, src_h, (i64)ny * nz,
                      waves_h, waves_cols, &t, dummy, 1, 1 << 30, nx, ny, nz, source_x,
                      courant, 0);
        oracle_update(0, 0, H, E, n, inv_eps, psi_h, n, coeff_h, clen, src_e, (i64)ny * nz,
                      waves_e, waves_cols, &t, dummy, 1, 1 << 30, nx, ny, nz, source_x,
                      courant, 0);
    }
    return 0;
}

int oracle_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
