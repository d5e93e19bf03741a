// Fused reverse step of the exact adjoint.  The reference runs each half of a
// reverse step as two full-grid passes with the d buffer (6 n floats) between
// them (adjoint.py:388-414): prepare (adjoint.py:46-88, the transpose of the
// field scaling and the CPML recurrence) writes d, then gather
// (adjoint.py:107-162, the transpose of the curl differences) reads d at the
// cell and its -/+1 neighbours.  Here one pass per half recomputes the d
// values a cell needs -- its own six and one pair at each of its x, y and z
// neighbours -- from the same inputs with the same expressions, so the result
// is bitwise the reference sequence's while d never touches memory.
//
// The CPML state is ping-ponged (read buffer step & 1, write the other): a
// neighbour's d needs that neighbour's psi before this step's update, which
// another block may be writing.  Each cell still updates its own psi exactly
// once per half step.
#include "common.cuh"

namespace wfb {

// prepare's pair of d slots (2*axis, 2*axis+1) at cell c (adjoint.py:60-86):
// v = factor * q with factor = courant * eps[c] (electric) or -courant;
// q1 = -v[a], q2 = v[b], a = axis+1, b = axis+2 (mod 3); d = k * q (+ CPML).
// With psi_out the updated psi of c is written (the cell's own update).
// co = (a, b, 1/kappa, unused): one 16-byte load per pair.
template <bool ELECTRIC>
__device__ __forceinline__ void d_pair(const float *__restrict__ q,
                                       const float *__restrict__ eps,
                                       const float *__restrict__ psi_in, float *psi_out,
                                       const float4 *__restrict__ coeff, int clen, i64 n, i64 c,
                                       int pos, int axis, float courant, float &d1, float &d2) {
    const float factor = ELECTRIC ? courant * eps[c] : -courant;
    const int a = (axis + 1) % 3, b = (axis + 2) % 3;
    const float q1 = -(factor * q[(i64)a * n + c]);
    const float q2 = factor * q[(i64)b * n + c];
    const float4 co = coeff[axis * clen + pos];
    d1 = co.z * q1;
    d2 = co.z * q2;
    if (co.x != 0.0f) {
        const float p1 = psi_in[(i64)(2 * axis) * n + c] + q1;
        const float p2 = psi_in[(i64)(2 * axis + 1) * n + c] + q2;
        d1 = d1 + co.x * p1;
        d2 = d2 + co.x * p2;
        if (psi_out) {
            psi_out[(i64)(2 * axis) * n + c] = co.y * p1;
            psi_out[(i64)(2 * axis + 1) * n + c] = co.y * p2;
        }
    }
}

// One half of a reverse step over every cell.  FROM_H (first half): q_dst =
// qE, q_src = qH, magnetic scaling, psi = the H state, neighbours at -1, the
// design gradient accumulated; otherwise (second half): q_dst = qH, q_src =
// the updated qE, electric scaling, psi = the E state, neighbours at +1,
// differences negated.
template <bool FROM_H>
__global__ void __launch_bounds__(256, 8) reverse_half_kernel(float *__restrict__ q_dst, const float *__restrict__ q_src,
                                    const float *__restrict__ eps, float *psi0, float *psi1,
                                    const float4 *__restrict__ coeff, int clen,
                                    const int *__restrict__ step, const float *__restrict__ hist,
                                    double *__restrict__ grad,
                                    const int *__restrict__ hist_step, int nx, int ny, int nz,
                                    float courant, int x0, int y0, int z0, int sx, int sy,
                                    int sz) {
    constexpr bool ELECTRIC = !FROM_H;
    const i64 n = (i64)nx * ny * nz;
    // one x plane per grid row: 32-bit (y, z) decomposition within the plane
    const int x = blockIdx.y;
    const int yz = blockIdx.x * blockDim.x + threadIdx.x;
    if (yz >= ny * nz) return;
    const int y = yz / nz;
    const int z = yz - y * nz;
    const i64 i = (i64)x * ny * nz + yz;
    const int s = step[0] & 1;
    const float *psi_in = s ? psi1 : psi0;
    float *psi_out = s ? psi0 : psi1;
    constexpr int delta = FROM_H ? -1 : 1;

    float d[6];
    d_pair<ELECTRIC>(q_src, eps, psi_in, psi_out, coeff, clen, n, i, x, 0, courant, d[0], d[1]);
    d_pair<ELECTRIC>(q_src, eps, psi_in, psi_out, coeff, clen, n, i, y, 1, courant, d[2], d[3]);
    d_pair<ELECTRIC>(q_src, eps, psi_in, psi_out, coeff, clen, n, i, z, 2, courant, d[4], d[5]);
    // neighbour pairs (adjoint.py:91-104 `read`: zero outside the grid).  The
    // pairs are evaluated unconditionally at a clamped neighbour (so every
    // load can issue early) and replaced by exactly zero outside the grid.
    float nx0, nx1, ny2, ny3, nz4, nz5;
    const int xn = x + delta, yn = y + delta, zn = z + delta;
    const bool xin = xn >= 0 && xn < nx, yin = yn >= 0 && yn < ny, zin = zn >= 0 && zn < nz;
    d_pair<ELECTRIC>(q_src, eps, psi_in, nullptr, coeff, clen, n,
                     xin ? i + (i64)delta * ny * nz : i, xin ? xn : x, 0, courant, nx0, nx1);
    d_pair<ELECTRIC>(q_src, eps, psi_in, nullptr, coeff, clen, n, yin ? i + (i64)delta * nz : i,
                     yin ? yn : y, 1, courant, ny2, ny3);
    d_pair<ELECTRIC>(q_src, eps, psi_in, nullptr, coeff, clen, n, zin ? i + delta : i,
                     zin ? zn : z, 2, courant, nz4, nz5);
    if (!xin) nx0 = nx1 = 0.0f;
    if (!yin) ny2 = ny3 = 0.0f;
    if (!zin) nz4 = nz5 = 0.0f;
    // gather (adjoint.py:118-150), same operand order
    float v[3];
    v[0] = (ny2 - d[2]) + (nz5 - d[5]);
    v[1] = (nx1 - d[1]) + (nz4 - d[4]);
    v[2] = (nx0 - d[0]) + (ny3 - d[3]);
    if (!FROM_H) {
        v[0] = -v[0];
        v[1] = -v[1];
        v[2] = -v[2];
    }
    const float value[3] = {q_dst[i] + v[0], q_dst[n + i] + v[1], q_dst[2 * n + i] + v[2]};
    q_dst[i] = value[0];
    q_dst[n + i] = value[1];
    q_dst[2 * n + i] = value[2];
    if (FROM_H && grad && x >= x0 && x < x0 + sx && y >= y0 && y < y0 + sy && z >= z0 &&
        z < z0 + sz) {
        const i64 dn = (i64)sx * sy * sz;
        const i64 j = ((i64)(x - x0) * sy + (y - y0)) * sz + (z - z0);
        const float *hh = hist + (i64)hist_step[0] * 3 * dn;
        grad[j] = grad[j] + (((double)hh[j] * value[0] + (double)hh[dn + j] * value[1]) +
                             (double)hh[2 * dn + j] * value[2]);
    }
}

}  // namespace wfb

using namespace wfb;

extern "C" int fdtd_reverse_half(int from_h, float *q_dst, const float *q_src, const float *eps,
                                 float *psi0, float *psi1, const float *coeff, int clen,
                                 const int *step, const float *hist, double *grad,
                                 const int *hist_step, int nx, int ny, int nz, float courant,
                                 int x0, int y0, int z0, int sx, int sy, int sz, void *stream) {
    const i64 n = (i64)nx * ny * nz;
    if (n <= 0 || !q_dst || !q_src || !psi0 || !psi1 || !coeff || !step || psi0 == psi1 ||
        ((uintptr_t)coeff & 15) ||
        clen < (nx > ny ? (nx > nz ? nx : nz) : (ny > nz ? ny : nz)) || (!from_h && !eps) ||
        (from_h && grad && (!hist || !hist_step || sx < 1 || sy < 1 || sz < 1 || x0 < 0 ||
                            y0 < 0 || z0 < 0 || x0 + sx > nx || y0 + sy > ny || z0 + sz > nz))) {
        set_error("fdtd_reverse_half: invalid arguments");
        return FDTD_ERR_ARG;
    }
    if (nx > 65535 || (i64)ny * nz > 0x7fffffffLL) {
        set_error("fdtd_reverse_half: nx <= 65535 and ny*nz < 2^31 required");
        return FDTD_ERR_ARG;
    }
    const dim3 blocks((unsigned)(((i64)ny * nz + 255) / 256), (unsigned)nx);
    cudaStream_t s = (cudaStream_t)stream;
    if (from_h)
        reverse_half_kernel<true><<<blocks, 256, 0, s>>>(q_dst, q_src, eps, psi0, psi1,
                                                         (const float4 *)coeff, clen, step, hist, grad, hist_step, nx,
                                                         ny, nz, courant, x0, y0, z0, sx, sy, sz);
    else
        reverse_half_kernel<false><<<blocks, 256, 0, s>>>(q_dst, q_src, eps, psi0, psi1,
                                                          (const float4 *)coeff, clen, step, nullptr, nullptr, nullptr,
                                                          nx, ny, nz, courant, 0, 0, 0, 0, 0, 0);
    return launch_status("fdtd_reverse_half");
}
