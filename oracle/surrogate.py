"""CPU oracle of the CNN surrogate (test infrastructure only).

A NumPy restatement of the encoder-decoder that warp_fdtd_b200's CUDA
surrogate kernels run, forward and hand-written backward, used by the tests
as the checker.  The surrogate has no counterpart in the reference (the
reference optimises designs with the adjoint alone), so parity is against
this oracle and, for the backward, against finite differences of the oracle
itself in float64.

Two arithmetic modes:
* ``bf16=True`` rounds exactly where the CUDA path stores bf16: the network
  input, every convolution output (after bias and ReLU), every pooled map,
  the weights fed to the tensor cores, and the ReLU-masked output gradients
  that the backward GEMMs read.  Products accumulate in float32 (the tensor
  cores' accumulator), so results agree with the GPU up to float32
  summation order and the occasional bf16 rounding flip that it causes.
* ``bf16=False`` with ``dtype=np.float64``: the exact network, for the
  finite-difference check of the backward.

Architecture (levels l = 0..3 at H/2^l; c_l = base * 2^l):
  e0a 1->c0, e0b c0->c0 | pool | e1a c0->c1, e1b c1->c1 | pool |
  e2a c1->c2, e2b c2->c2 | pool | bott c2->c3 ; transmission head: global
  mean of bott -> linear c3->nwav ; decoder: up(bott)++e2b -> d2 (c3+c2->c2),
  up(d2)++e1b -> d1 (c2+c1->c1), up(d1)++e0b -> d0 (c1+c0->c0) ; gradient
  head: 1x1 c0->1.  Every 3x3 convolution is followed by ReLU; pooling is the
  2x2 mean, upsampling nearest.
"""

import numpy as np


def round_bf16(x):
    """float32 -> nearest bf16 (ties to even) -> float32."""
    x = np.ascontiguousarray(x, np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).reshape(x.shape)


def architecture(base=32):
    c0, c1, c2, c3 = base, 2 * base, 4 * base, 8 * base
    return [("e0a", 1, c0, 0), ("e0b", c0, c0, 0), ("e1a", c0, c1, 1), ("e1b", c1, c1, 1),
            ("e2a", c1, c2, 2), ("e2b", c2, c2, 2), ("bott", c2, c3, 3),
            ("d2", c3 + c2, c2, 2), ("d1", c2 + c1, c1, 1), ("d0", c1 + c0, c0, 0)]


def im2col(x, H, W):
    """x (B*H*W, C) NHWC -> (B*H*W, 9*C), column tap*C + c, tap = (dy+1)*3 + (dx+1)."""
    P, C = x.shape
    B = P // (H * W)
    xi = x.reshape(B, H, W, C)
    pad = np.zeros((B, H + 2, W + 2, C), x.dtype)
    pad[:, 1:-1, 1:-1] = xi
    cols = [pad[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W] for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    return np.concatenate(cols, axis=-1).reshape(P, 9 * C)


def col2im(dcol, H, W, C):
    """Adjoint of im2col."""
    P = dcol.shape[0]
    B = P // (H * W)
    d = dcol.reshape(B, H, W, 9, C)
    pad = np.zeros((B, H + 2, W + 2, C), dcol.dtype)
    tap = 0
    for dy in (-1, 0, 1):
        for dx in (-1, 0, 1):
            pad[:, 1 + dy:1 + dy + H, 1 + dx:1 + dx + W] += d[:, :, :, tap]
            tap += 1
    return pad[:, 1:-1, 1:-1].reshape(P, C)


def pool(x, H, W):
    P, C = x.shape
    B = P // (H * W)
    v = x.reshape(B, H // 2, 2, W // 2, 2, C)
    return (0.25 * ((v[:, :, 0, :, 0] + v[:, :, 0, :, 1]) + (v[:, :, 1, :, 0] + v[:, :, 1, :, 1]))
            ).reshape(-1, C)


def pool_backward(dy, H, W):
    """H, W: the input (large) map."""
    P, C = dy.shape
    B = P // ((H // 2) * (W // 2))
    g = 0.25 * dy.reshape(B, H // 2, 1, W // 2, 1, C)
    return np.broadcast_to(g, (B, H // 2, 2, W // 2, 2, C)).reshape(-1, C).astype(dy.dtype)


def upsample(x, H, W):
    """H, W: the small map."""
    P, C = x.shape
    B = P // (H * W)
    v = x.reshape(B, H, 1, W, 1, C)
    return np.broadcast_to(v, (B, H, 2, W, 2, C)).reshape(-1, C).copy()


def upsample_backward(dy, H, W):
    P, C = dy.shape
    B = P // (4 * H * W)
    v = dy.reshape(B, H, 2, W, 2, C)
    return ((v[:, :, 0, :, 0] + v[:, :, 0, :, 1]) + (v[:, :, 1, :, 0] + v[:, :, 1, :, 1])
            ).reshape(-1, C)


class OracleSurrogate:
    """Parameters: dict name -> array; conv layers hold "<name>.w" (cout, 9*cin)
    and "<name>.b" (cout); heads "thead.w" (nwav, c3), "thead.b" (nwav),
    "ghead.w" (c0,), "ghead.b" (1,)."""

    def __init__(self, params, size, nwav=8, base=32, bf16=True, dtype=np.float32):
        self.H, self.W = size
        self.nwav = nwav
        self.base = base
        self.bf16 = bf16
        self.dtype = dtype
        self.p = {k: np.asarray(v, dtype) for k, v in params.items()}
        self.convs = architecture(base)

    def r(self, x):
        return round_bf16(x) if self.bf16 else np.asarray(x, self.dtype)

    def _conv(self, name, x, h, w):
        col = im2col(x, h, w)
        wt = self.r(self.p[name + ".w"])
        z = (col @ wt.T).astype(self.dtype) + self.p[name + ".b"]
        return self.r(np.maximum(z, 0)), col

    def forward(self, density):
        """density (B, H, W) -> (T (B, nwav), g (B, H, W)); keeps the tape."""
        B = density.shape[0]
        H, W = self.H, self.W
        c0, c1, c2, c3 = (self.base << l for l in range(4))
        t = {}
        x0 = self.r(np.asarray(density, self.dtype).reshape(-1, 1))
        t["x0"] = x0
        sizes = [(H >> l, W >> l) for l in range(4)]
        t["e0a"], t["col.e0a"] = self._conv("e0a", x0, *sizes[0])
        t["e0b"], t["col.e0b"] = self._conv("e0b", t["e0a"], *sizes[0])
        t["pool0"] = self.r(pool(t["e0b"], *sizes[0]))
        t["e1a"], t["col.e1a"] = self._conv("e1a", t["pool0"], *sizes[1])
        t["e1b"], t["col.e1b"] = self._conv("e1b", t["e1a"], *sizes[1])
        t["pool1"] = self.r(pool(t["e1b"], *sizes[1]))
        t["e2a"], t["col.e2a"] = self._conv("e2a", t["pool1"], *sizes[2])
        t["e2b"], t["col.e2b"] = self._conv("e2b", t["e2a"], *sizes[2])
        t["pool2"] = self.r(pool(t["e2b"], *sizes[2]))
        t["bott"], t["col.bott"] = self._conv("bott", t["pool2"], *sizes[3])
        npix = sizes[3][0] * sizes[3][1]
        feat = t["bott"].reshape(B, npix, c3).astype(self.dtype).sum(axis=1) / self.dtype(npix)
        t["feat"] = feat
        T = (feat @ self.p["thead.w"].T).astype(self.dtype) + self.p["thead.b"]
        t["cat2"] = np.concatenate([upsample(t["bott"], *sizes[3]), t["e2b"]], axis=1)
        t["d2"], t["col.d2"] = self._conv("d2", t["cat2"], *sizes[2])
        t["cat1"] = np.concatenate([upsample(t["d2"], *sizes[2]), t["e1b"]], axis=1)
        t["d1"], t["col.d1"] = self._conv("d1", t["cat1"], *sizes[1])
        t["cat0"] = np.concatenate([upsample(t["d1"], *sizes[1]), t["e0b"]], axis=1)
        t["d0"], t["col.d0"] = self._conv("d0", t["cat0"], *sizes[0])
        g = (t["d0"] @ self.p["ghead.w"]).astype(self.dtype) + self.p["ghead.b"][0]
        self.tape = t
        self.B = B
        return T, g.reshape(B, H, W)

    def set_tape(self, acts, B):
        """Replace the forward tape by given activations (float32 (P, C) arrays
        for x0, e0a, e0b, pool0, e1a, e1b, pool1, e2a, e2b, pool2, bott, feat,
        d2, d1, d0), so that backward() runs on exactly those values."""
        H, W = self.H, self.W
        sizes = [(H >> l, W >> l) for l in range(4)]
        t = {k: np.asarray(v, self.dtype) for k, v in acts.items()}
        t["cat2"] = np.concatenate([upsample(t["bott"], *sizes[3]), t["e2b"]], axis=1)
        t["cat1"] = np.concatenate([upsample(t["d2"], *sizes[2]), t["e1b"]], axis=1)
        t["cat0"] = np.concatenate([upsample(t["d1"], *sizes[1]), t["e0b"]], axis=1)
        inputs = {"e0a": "x0", "e0b": "e0a", "e1a": "pool0", "e1b": "e1a", "e2a": "pool1",
                  "e2b": "e2a", "bott": "pool2", "d2": "cat2", "d1": "cat1", "d0": "cat0"}
        for name, _, _, lev in self.convs:
            t["col." + name] = im2col(t[inputs[name]], *sizes[lev])
        self.tape = t
        self.B = B

    def _conv_backward(self, name, dy, h, w, cin, grads, need_dx=True):
        t = self.tape
        m = np.where(t[name] > 0, dy, 0).astype(self.dtype)
        grads[name + ".b"] = m.sum(axis=0)
        dz = self.r(m)
        grads[name + ".w"] = (dz.T @ t["col." + name]).astype(self.dtype)
        if not need_dx:
            return None
        wt = self.r(self.p[name + ".w"])
        dcol = (dz @ wt).astype(self.dtype)
        return col2im(dcol, h, w, cin)

    def backward(self, dT, dg):
        """Gradients of sum(dT * T) + sum(dg * g) w.r.t. every parameter."""
        t = self.tape
        B = self.B
        H, W = self.H, self.W
        c0, c1, c2, c3 = (self.base << l for l in range(4))
        sizes = [(H >> l, W >> l) for l in range(4)]
        dT = np.asarray(dT, self.dtype)
        dg = np.asarray(dg, self.dtype).reshape(-1)
        grads = {}
        grads["ghead.w"] = (dg @ t["d0"]).astype(self.dtype)
        grads["ghead.b"] = np.array([dg.sum()], self.dtype)
        d_d0 = np.outer(dg, self.p["ghead.w"]).astype(self.dtype)
        d_cat0 = self._conv_backward("d0", d_d0, *sizes[0], c1 + c0, grads)
        d_d1 = upsample_backward(d_cat0[:, :c1], *sizes[1])
        d_cat1 = self._conv_backward("d1", d_d1, *sizes[1], c2 + c1, grads)
        d_d2 = upsample_backward(d_cat1[:, :c2], *sizes[2])
        d_cat2 = self._conv_backward("d2", d_d2, *sizes[2], c3 + c2, grads)
        d_b = upsample_backward(d_cat2[:, :c3], *sizes[3])
        grads["thead.w"] = (dT.T @ t["feat"]).astype(self.dtype)
        grads["thead.b"] = dT.sum(axis=0)
        npix = sizes[3][0] * sizes[3][1]
        gfeat = (dT @ self.p["thead.w"]).astype(self.dtype) / self.dtype(npix)
        d_b = d_b + np.repeat(gfeat, npix, axis=0)
        d_pool2 = self._conv_backward("bott", d_b, *sizes[3], c2, grads)
        d_e2b = d_cat2[:, c3:] + pool_backward(d_pool2, *sizes[2])
        d_e2a = self._conv_backward("e2b", d_e2b, *sizes[2], c2, grads)
        d_pool1 = self._conv_backward("e2a", d_e2a, *sizes[2], c1, grads)
        d_e1b = d_cat1[:, c2:] + pool_backward(d_pool1, *sizes[1])
        d_e1a = self._conv_backward("e1b", d_e1b, *sizes[1], c1, grads)
        d_pool0 = self._conv_backward("e1a", d_e1a, *sizes[1], c0, grads)
        d_e0b = d_cat0[:, c1:] + pool_backward(d_pool0, *sizes[0])
        d_e0a = self._conv_backward("e0b", d_e0b, *sizes[0], c0, grads)
        self._conv_backward("e0a", d_e0a, *sizes[0], 1, grads, need_dx=False)
        return grads

    def loss(self, T, g, T_target, g_target, w_T=1.0, w_g=1.0):
        """w_T * mean((T - T*)^2) + w_g * mean((g - g*)^2) and its output gradients."""
        dT = np.asarray(T, np.float64) - T_target
        dg = np.asarray(g, np.float64) - g_target
        L = w_T * np.mean(dT ** 2) + w_g * np.mean(dg ** 2)
        return L, (w_T * 2 * dT / dT.size).astype(self.dtype), (w_g * 2 * dg / dg.size).astype(
            self.dtype)


def init_params(seed=0, base=32, nwav=8):
    """He-normal convolution weights, zero biases, small heads."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, cin, cout, _ in architecture(base):
        p[name + ".w"] = (rng.standard_normal((cout, 9 * cin)) * np.sqrt(2.0 / (9 * cin))).astype(
            np.float32)
        p[name + ".b"] = np.zeros(cout, np.float32)
    c3 = 8 * base
    p["thead.w"] = (rng.standard_normal((nwav, c3)) / np.sqrt(c3)).astype(np.float32)
    p["thead.b"] = np.zeros(nwav, np.float32)
    p["ghead.w"] = (rng.standard_normal(base) / np.sqrt(base)).astype(np.float32)
    p["ghead.b"] = np.zeros(1, np.float32)
    return p
