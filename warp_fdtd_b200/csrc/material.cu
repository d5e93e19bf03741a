// Design-to-material map (warp_fdtd/material.py) and its hand-written reverse
// mode.  The reference differentiates the map with a Warp Tape
// (material.py:78-102); here the adjoint of each kernel is written out, and the
// smoothing adjoint gathers per target pixel so its sums are deterministic.
#include <mutex>

#include "common.cuh"

namespace wfb {

// material.py:12-25 `smooth`: clamp-extended correlation, dx outer, dy inner.
__global__ void smooth_kernel(const float *__restrict__ p, const float *__restrict__ w,
                              int radius, float *__restrict__ out, int px, int py) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= px * py) return;
    int x = idx / py, y = idx % py;
    const int k = 2 * radius + 1;
    float total = 0.0f;
    for (int dx = -radius; dx <= radius; ++dx) {
        int ix = min(max(x + dx, 0), px - 1);
        for (int dy = -radius; dy <= radius; ++dy) {
            int iy = min(max(y + dy, 0), py - 1);
            total = total + p[ix * py + iy] * w[(dx + radius) * k + dy + radius];
        }
    }
    out[idx] = total;
}

// Adjoint of smooth_kernel: p_grad[u, v] += sum of g[x, y] * w[dx, dy] over
// every (x, y, dx, dy) whose clamped sample lands on (u, v).
__global__ void smooth_adjoint_kernel(const float *__restrict__ g, const float *__restrict__ w,
                                      int radius, float *__restrict__ p_grad, int px, int py) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= px * py) return;
    int u = idx / py, v = idx % py;
    const int k = 2 * radius + 1;
    float total = 0.0f;
    for (int dx = -radius; dx <= radius; ++dx) {
        // x such that clamp(x + dx) == u
        int xlo = u - dx, xhi = u - dx;
        if (u == 0) xlo = -1 << 20;
        if (u == px - 1) xhi = 1 << 20;
        xlo = max(xlo, 0);
        xhi = min(xhi, px - 1);
        for (int x = xlo; x <= xhi; ++x) {
            for (int dy = -radius; dy <= radius; ++dy) {
                int ylo = v - dy, yhi = v - dy;
                if (v == 0) ylo = -1 << 20;
                if (v == py - 1) yhi = 1 << 20;
                ylo = max(ylo, 0);
                yhi = min(yhi, py - 1);
                const float wv = w[(dx + radius) * k + dy + radius];
                for (int y = ylo; y <= yhi; ++y) total = total + g[x * py + y] * wv;
            }
        }
    }
    p_grad[idx] = p_grad[idx] + total;
}

// material.py:28-32 `project`.
__device__ __forceinline__ float project(float r, float beta) {
    float th = tanhf(0.5f * beta);
    return (th + tanhf(beta * (r - 0.5f))) / (2.0f * th);
}

__device__ __forceinline__ float project_grad(float r, float beta) {
    float th = tanhf(0.5f * beta);
    float u = tanhf(beta * (r - 0.5f));
    return beta * (1.0f - u * u) / (2.0f * th);
}

struct Neigh {
    int xm, xp, ym, yp;
};

__device__ __forceinline__ Neigh neighbours(int x, int y, int px, int py) {
    Neigh n;
    n.xm = max(x - 1, 0);
    n.xp = min(x + 1, px - 1);
    n.ym = max(y - 1, 0);
    n.yp = min(y + 1, py - 1);
    return n;
}

// material.py:35-55 `subpixel`.
__global__ void subpixel_kernel(const float *__restrict__ rho, float *__restrict__ out,
                                int px, int py, float beta, float eps_lo, float contrast) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= px * py) return;
    int x = idx / py, y = idx % py;
    Neigh nb = neighbours(x, y, px, py);
    float gx = (rho[nb.xp * py + y] - rho[nb.xm * py + y]) / (float)(nb.xp - nb.xm);
    float gy = (rho[x * py + nb.yp] - rho[x * py + nb.ym]) / (float)(nb.yp - nb.ym);
    float norm2 = gx * gx + gy * gy;
    float r = rho[idx];
    float value = project(r, beta);
    if (norm2 > 0.0f) {
        float norm = sqrtf(norm2);
        float d = (0.5f - r) / (0.55f * norm);
        if (fabsf(d) < 1.0f) {
            float fill = 0.5f - 0.9375f * d + 0.625f * d * d * d - 0.1875f * d * d * d * d * d;
            float lo = project(r - 0.55f * norm * fill, beta);
            float hi = project(r + 0.55f * norm * (1.0f - fill), beta);
            value = (1.0f - fill) * lo + fill * hi;
        }
    }
    out[idx] = 1.0f / (eps_lo + contrast * value);
}

// Reverse mode of subpixel_kernel for one output pixel: the adjoints of r,
// gx, gy are scattered onto the five pixels they read.
__global__ void subpixel_adjoint_kernel(const float *__restrict__ rho,
                                        const float *__restrict__ g, float *__restrict__ grad,
                                        int px, int py, float beta, float eps_lo,
                                        float contrast) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= px * py) return;
    int x = idx / py, y = idx % py;
    Neigh nb = neighbours(x, y, px, py);
    float sx = 1.0f / (float)(nb.xp - nb.xm);
    float sy = 1.0f / (float)(nb.yp - nb.ym);
    float gx = (rho[nb.xp * py + y] - rho[nb.xm * py + y]) / (float)(nb.xp - nb.xm);
    float gy = (rho[x * py + nb.yp] - rho[x * py + nb.ym]) / (float)(nb.yp - nb.ym);
    float norm2 = gx * gx + gy * gy;
    float r = rho[idx];
    float value = project(r, beta);
    float a_r = 0.0f, a_gx = 0.0f, a_gy = 0.0f;  // adjoints filled below
    // out = 1 / (eps_lo + c * value) -> d out / d value
    float dv = 0.0f;
    bool smoothed = false;
    float norm = 0.0f, d = 0.0f, fill = 0.0f, alo = 0.0f, ahi = 0.0f, lo = 0.0f, hi = 0.0f;
    if (norm2 > 0.0f) {
        norm = sqrtf(norm2);
        d = (0.5f - r) / (0.55f * norm);
        if (fabsf(d) < 1.0f) {
            smoothed = true;
            fill = 0.5f - 0.9375f * d + 0.625f * d * d * d - 0.1875f * d * d * d * d * d;
            alo = r - 0.55f * norm * fill;
            ahi = r + 0.55f * norm * (1.0f - fill);
            lo = project(alo, beta);
            hi = project(ahi, beta);
            value = (1.0f - fill) * lo + fill * hi;
        }
    }
    float den = eps_lo + contrast * value;
    dv = -contrast / (den * den) * g[idx];
    if (!smoothed) {
        a_r = dv * project_grad(r, beta);
    } else {
        float d_lo = dv * (1.0f - fill);
        float d_hi = dv * fill;
        float d_fill = dv * (hi - lo);
        float plo = project_grad(alo, beta) * d_lo;  // adjoint of alo
        float phi = project_grad(ahi, beta) * d_hi;  // adjoint of ahi
        // alo = r - 0.55 n f ; ahi = r + 0.55 n (1 - f)
        a_r = plo + phi;
        float d_norm = -0.55f * fill * plo + 0.55f * (1.0f - fill) * phi;
        d_fill = d_fill - 0.55f * norm * plo - 0.55f * norm * phi;
        // fill(d)
        float d_d = d_fill * (-0.9375f + 1.875f * d * d - 0.9375f * d * d * d * d);
        // d = (0.5 - r) / (0.55 n)
        a_r = a_r - d_d / (0.55f * norm);
        d_norm = d_norm - d_d * d / norm;
        // n = sqrt(gx^2 + gy^2)
        a_gx = d_norm * gx / norm;
        a_gy = d_norm * gy / norm;
    }
    atomicAdd(grad + idx, a_r);
    if (a_gx != 0.0f) {
        atomicAdd(grad + nb.xp * py + y, a_gx * sx);
        atomicAdd(grad + nb.xm * py + y, -a_gx * sx);
    }
    if (a_gy != 0.0f) {
        atomicAdd(grad + x * py + nb.yp, a_gy * sy);
        atomicAdd(grad + x * py + nb.ym, -a_gy * sy);
    }
}

// Scratch of fdtd_material_forward_noalloc: one static array per device that
// loads the library, shared by every call of that entry point.
static __device__ __align__(256) float g_material_scratch[FDTD_MATERIAL_NOALLOC_MAX];

// Device address of g_material_scratch on the current device, looked up once
// per device (the host-side symbol is only a stand-in, never a device pointer).
static int material_scratch_address(float **out) {
    static std::mutex lock;
    static float *cached[64] = {};
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) {
        set_error("fdtd_material_forward_noalloc: cudaGetDevice: %s", cudaGetErrorString(err));
        return FDTD_ERR_CUDA;
    }
    if (dev < 0 || dev >= 64) {
        set_error("fdtd_material_forward_noalloc: device index %d out of range", dev);
        return FDTD_ERR_ARG;
    }
    std::lock_guard<std::mutex> guard(lock);
    if (!cached[dev]) {
        void *ptr = nullptr;
        err = cudaGetSymbolAddress(&ptr, g_material_scratch);
        if (err != cudaSuccess || !ptr) {
            set_error("fdtd_material_forward_noalloc: cudaGetSymbolAddress: %s",
                      cudaGetErrorString(err));
            return FDTD_ERR_CUDA;
        }
        cached[dev] = (float *)ptr;
    }
    *out = cached[dev];
    return FDTD_OK;
}

}  // namespace wfb

using namespace wfb;

extern "C" {

int fdtd_material_smooth(const float *p, const float *weights, int radius, float *out,
                         int px, int py, void *stream) {
    if (!p || !weights || !out || px < 1 || py < 1 || radius < 0) {
        set_error("fdtd_material_smooth: invalid arguments");
        return FDTD_ERR_ARG;
    }
    int n = px * py;
    smooth_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(p, weights, radius, out,
                                                                     px, py);
    return launch_status("fdtd_material_smooth");
}

int fdtd_material_smooth_adjoint(const float *g, const float *weights, int radius,
                                 float *p_grad, int px, int py, void *stream) {
    if (!g || !weights || !p_grad || px < 1 || py < 1 || radius < 0) {
        set_error("fdtd_material_smooth_adjoint: invalid arguments");
        return FDTD_ERR_ARG;
    }
    int n = px * py;
    smooth_adjoint_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        g, weights, radius, p_grad, px, py);
    return launch_status("fdtd_material_smooth_adjoint");
}

int fdtd_material_subpixel(const float *rho, float *out, int px, int py, float beta,
                           float eps_lo, float contrast, void *stream) {
    if (!rho || !out || px < 2 || py < 2 || !(beta > 0.0f)) {
        set_error("fdtd_material_subpixel: invalid arguments");
        return FDTD_ERR_ARG;
    }
    int n = px * py;
    subpixel_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(rho, out, px, py, beta,
                                                                       eps_lo, contrast);
    return launch_status("fdtd_material_subpixel");
}

int fdtd_material_subpixel_adjoint(const float *rho, const float *g, float *rho_grad,
                                   int px, int py, float beta, float eps_lo,
                                   float contrast, void *stream) {
    if (!rho || !g || !rho_grad || px < 2 || py < 2 || !(beta > 0.0f)) {
        set_error("fdtd_material_subpixel_adjoint: invalid arguments");
        return FDTD_ERR_ARG;
    }
    int n = px * py;
    subpixel_adjoint_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        rho, g, rho_grad, px, py, beta, eps_lo, contrast);
    return launch_status("fdtd_material_subpixel_adjoint");
}

int fdtd_material_forward(const float *p, const float *weights, int radius, float *scratch,
                          float *out, int px, int py, float beta, float eps_lo,
                          float contrast, void *stream) {
    if (!scratch) {
        set_error("fdtd_material_forward: null scratch");
        return FDTD_ERR_ARG;
    }
    int rc = fdtd_material_smooth(p, weights, radius, scratch, px, py, stream);
    if (rc) return rc;
    return fdtd_material_subpixel(scratch, out, px, py, beta, eps_lo, contrast, stream);
}

int fdtd_material_forward_noalloc(const float *p, const float *weights, int radius,
                                  float *out, int px, int py, float beta, float eps_lo,
                                  float contrast, void *stream) {
    if (!p || !weights || !out || px < 2 || py < 2 || radius < 0 || !(beta > 0.0f)) {
        set_error("fdtd_material_forward_noalloc: invalid arguments");
        return FDTD_ERR_ARG;
    }
    if ((long long)px * py > FDTD_MATERIAL_NOALLOC_MAX) {
        set_error("fdtd_material_forward_noalloc: %d x %d pixels exceed the built-in scratch "
                  "of %d floats; use fdtd_material_forward with caller scratch",
                  px, py, FDTD_MATERIAL_NOALLOC_MAX);
        return FDTD_ERR_ARG;
    }
    float *scratch = nullptr;
    int rc = material_scratch_address(&scratch);
    if (rc) return rc;
    const int n = px * py;
    smooth_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(p, weights, radius,
                                                                     scratch, px, py);
    rc = launch_status("fdtd_material_forward_noalloc (smooth)");
    if (rc) return rc;
    subpixel_kernel<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(scratch, out, px, py,
                                                                       beta, eps_lo, contrast);
    return launch_status("fdtd_material_forward_noalloc (subpixel)");
}

int fdtd_material_backward(const float *p, const float *weights, int radius, const float *g,
                           float *scratch, float *p_grad, int px, int py, float beta,
                           float eps_lo, float contrast, void *stream) {
    if (!scratch || !p_grad || !g || px < 2 || py < 2) {
        set_error("fdtd_material_backward: invalid arguments");
        return FDTD_ERR_ARG;
    }
    const size_t n = (size_t)px * py;
    float *rho = scratch, *g_rho = scratch + n;
    int rc = fdtd_material_smooth(p, weights, radius, rho, px, py, stream);
    if (rc) return rc;
    cudaError_t err = cudaMemsetAsync(g_rho, 0, n * sizeof(float), (cudaStream_t)stream);
    if (err == cudaSuccess) err = cudaMemsetAsync(p_grad, 0, n * sizeof(float), (cudaStream_t)stream);
    if (err != cudaSuccess) {
        set_error("fdtd_material_backward: clearing the accumulators: %s", cudaGetErrorString(err));
        return FDTD_ERR_CUDA;
    }
    rc = fdtd_material_subpixel_adjoint(rho, g, g_rho, px, py, beta, eps_lo, contrast, stream);
    if (rc) return rc;
    return fdtd_material_smooth_adjoint(g_rho, weights, radius, p_grad, px, py, stream);
}

}  // extern "C"
