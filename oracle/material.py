"""NumPy restatement of the reference's material map (material.py:12-55).

TEST INFRASTRUCTURE ONLY (checker for warp_fdtd_b200.material).  float64
arithmetic; the float32 CUDA map is compared against it with a tolerance."""

import numpy as np


def weights(radius=9, sigma=3.0):
    xy = np.arange(-radius, radius + 1, dtype=np.float32)
    w = np.exp(-(xy[:, None] ** 2 + xy[None, :] ** 2) / np.float32(2 * sigma * sigma)).astype(np.float32)
    return w / w.sum()


def smooth(p, w):
    """material.py:12-25 with clamped edges."""
    r = (w.shape[0] - 1) // 2
    px, py = p.shape
    pad = np.pad(p.astype(np.float64), r, mode="edge")
    out = np.zeros((px, py))
    for dx in range(-r, r + 1):
        for dy in range(-r, r + 1):
            out += pad[r + dx:r + dx + px, r + dy:r + dy + py] * w[dx + r, dy + r]
    return out


def project(r, beta):
    """material.py:28-32."""
    return (np.tanh(0.5 * beta) + np.tanh(beta * (r - 0.5))) / (2.0 * np.tanh(0.5 * beta))


def subpixel(rho, beta, eps_lo=1.0, contrast=11.25):
    """material.py:35-55."""
    px, py = rho.shape
    out = np.zeros_like(rho, dtype=np.float64)
    for x in range(px):
        xm, xp = max(x - 1, 0), min(x + 1, px - 1)
        for y in range(py):
            ym, yp = max(y - 1, 0), min(y + 1, py - 1)
            gx = (rho[xp, y] - rho[xm, y]) / (xp - xm)
            gy = (rho[x, yp] - rho[x, ym]) / (yp - ym)
            norm2 = gx * gx + gy * gy
            r = rho[x, y]
            value = project(r, beta)
            if norm2 > 0:
                norm = np.sqrt(norm2)
                d = (0.5 - r) / (0.55 * norm)
                if abs(d) < 1:
                    fill = 0.5 - 0.9375 * d + 0.625 * d ** 3 - 0.1875 * d ** 5
                    lo = project(r - 0.55 * norm * fill, beta)
                    hi = project(r + 0.55 * norm * (1 - fill), beta)
                    value = (1 - fill) * lo + fill * hi
            out[x, y] = 1.0 / (eps_lo + contrast * value)
    return out


def material(p, beta, eps_lo=1.0, contrast=11.25, radius=9, sigma=3.0):
    return subpixel(smooth(p, weights(radius, sigma)), beta, eps_lo, contrast)
