"""CNN surrogate of a density-parameterised design problem, on the B200's
tensor cores.

A 4-level encoder-decoder (base 32 channels, about 1.16 M parameters for the
default widths) maps a design density map (H, W) to the modal transmission at
`nwav` wavelengths and to the map of the transmission's gradient with respect
to the density.  It has no counterpart in the reference, which optimises with
the exact adjoint alone (warp_fdtd/adjoint.py); here it proposes design
updates that a full FDTD forward accepts or rejects (design_loop.py).

Storage is bf16 (weights fed to the tensor cores, activations, the ReLU-masked
output gradients), accumulation float32, master weights and optimiser state
float32.  Every 3 x 3 convolution runs as conv-as-GEMM through fdtd_sg_gemm
(tcgen05.mma with the accumulator in tensor memory):
  forward      out[P, Cout]  = im2col(x)[P, 9 Cin] . W[Cout, 9 Cin]^T (+ bias, ReLU, bf16)
  input grad   dcol[P, 9 Cin] = dz[P, Cout] . Wt[9 Cin, Cout]^T, then col2im
  weight grad  dWt[9 Cin, Cout] = col^T[9 Cin, P] . dz^T[Cout, P]^T, split over P
The layer order, shapes and rounding points are those of oracle/surrogate.py.
Nothing here falls back to the CPU: every launch goes through the CUDA
library and raises if it is missing.
"""

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import SgGemmArgs

BF16 = torch.bfloat16
F32 = torch.float32
SCRATCH_ROWS = 1024  # FDTD_SG_SCRATCH_ROWS: partial-sum rows of the column reductions


def architecture(base=32):
    """(name, cin, cout, level) of the 3 x 3 convolutions, in forward order."""
    c0, c1, c2, c3 = base, 2 * base, 4 * base, 8 * base
    return [("e0a", 1, c0, 0), ("e0b", c0, c0, 0), ("e1a", c0, c1, 1), ("e1b", c1, c1, 1),
            ("e2a", c1, c2, 2), ("e2b", c2, c2, 2), ("bott", c2, c3, 3),
            ("d2", c3 + c2, c2, 2), ("d1", c2 + c1, c1, 1), ("d0", c1 + c0, c0, 0)]


def ptr(t):
    """Device pointer of a CUDA tensor that is contiguous or a row-strided 2-D
    view with unit stride along its last axis (a channel slice of an NHWC
    buffer); None -> NULL."""
    if t is None:
        return None
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise ValueError("surrogate kernels take CUDA tensors only")
    if not t.is_contiguous() and not (t.dim() == 2 and t.stride(1) == 1):
        raise ValueError("surrogate kernels take contiguous or row-strided 2-D tensors")
    return t.data_ptr()


def _round8(n):
    return (n + 7) // 8 * 8


def _s(stream):
    return ctypes.c_void_p(stream.cuda_stream if stream is not None else
                           torch.cuda.current_stream().cuda_stream)


def gemm(A, B, C, M, N, K, lda, ldb, ldc, bias=None, relu=False, accumulate=False, splits=1,
         split_stride=0, stream=None, layout=0):
    """C[M, N] = A[M, K] . B[N, K]^T through fdtd_sg_gemm (A, B bf16 tensors or
    views; C float32 or bf16; layout 0 = 128-byte swizzled operand tiles, 1 =
    interleaved core matrices).  Returns the number of K splits used."""
    a = SgGemmArgs()
    a.A, a.lda, a.B, a.ldb = ptr(A), lda, ptr(B), ldb
    a.C, a.ldc, a.c_bf16 = ptr(C), ldc, int(C.dtype == BF16)
    a.bias = ptr(bias)
    a.M, a.N, a.K = M, N, K
    a.splits, a.split_stride = splits, split_stride
    a.accumulate, a.relu, a.layout = int(accumulate), int(relu), int(layout)
    _lib.call("fdtd_sg_gemm", ctypes.byref(a), _s(stream))
    return _lib.load().fdtd_sg_gemm_splits(ctypes.byref(a)) if splits > 1 else 1


def gemm_splits(M, N, K, splits):
    a = SgGemmArgs()
    a.M, a.N, a.K, a.splits = M, N, K, splits
    return _lib.load().fdtd_sg_gemm_splits(ctypes.byref(a))


def status(reset=True):
    """1 if a GEMM's bounded wait ran out since the last reset, else 0."""
    out = ctypes.c_int(0)
    _lib.call("fdtd_sg_status", ctypes.byref(out), int(reset))
    return out.value


class Surrogate:
    """The network, its parameters and Adam state on one GPU.

    params_numpy()/load_params() exchange parameters as the oracle's dict
    ("<layer>.w" (cout, 9 cin), "<layer>.b", "thead.w" (nwav, c3), "thead.b",
    "ghead.w" (c0,), "ghead.b" (1,))."""

    def __init__(self, size=(80, 80), nwav=8, base=32, device="cuda:0", seed=0, params=None):
        H, W = (int(v) for v in size)
        if H % 8 or W % 8 or H < 8 or W < 8:
            raise ValueError("the surrogate needs H and W multiples of 8 (three 2x2 pools)")
        self.H, self.W, self.nwav, self.base = H, W, int(nwav), int(base)
        self.device = torch.device(device)
        self.convs = architecture(self.base)
        # flat float32 parameters: every conv's w then b, then the heads
        self.slots = {}
        off = 0
        for name, cin, cout, _ in self.convs:
            self.slots[name + ".w"] = (off, (cout, 9 * cin))
            off += cout * 9 * cin
            self.slots[name + ".b"] = (off, (cout,))
            off += cout
        c0, c3 = self.base, 8 * self.base
        for name, shape in (("thead.w", (self.nwav, c3)), ("thead.b", (self.nwav,)),
                            ("ghead.w", (c0,)), ("ghead.b", (1,))):
            self.slots[name] = (off, shape)
            off += int(np.prod(shape))
        self.count = off
        z = dict(dtype=F32, device=self.device)
        self.params = torch.zeros(off, **z)
        self.grads = torch.zeros(off, **z)
        self.m = torch.zeros(off, **z)
        self.v = torch.zeros(off, **z)
        self.adam_step = 0
        # bf16 operand copies: wb [cout, ldw] (forward B), wt [9 cin, cout] (input-grad B)
        self.wb, self.wt = {}, {}
        for name, cin, cout, _ in self.convs:
            self.wb[name] = torch.zeros((cout, _round8(9 * cin)), dtype=BF16, device=self.device)
            self.wt[name] = torch.zeros((9 * cin, cout), dtype=BF16, device=self.device)
        self._bufs = {}
        self._splits = {}  # (layer, batch) -> K splits of its weight-gradient GEMM
        if params is None:
            params = default_init(seed, self.base, self.nwav)
        self.load_params(params)

    # ------------------------------------------------------------ parameters
    def view(self, name, t=None):
        off, shape = self.slots[name]
        t = self.params if t is None else t
        return t[off:off + int(np.prod(shape))].view(shape)

    def load_params(self, params):
        for name, (off, shape) in self.slots.items():
            v = np.asarray(params[name], np.float32)
            if v.shape != shape:
                raise ValueError(f"{name}: expected {shape}, got {v.shape}")
            self.view(name).copy_(torch.from_numpy(v))
        self._cast()

    def params_numpy(self):
        return {name: self.view(name).cpu().numpy().copy() for name in self.slots}

    def grads_numpy(self):
        return {name: self.view(name, self.grads).cpu().numpy().copy() for name in self.slots}

    def _cast(self, stream=None):
        with torch.cuda.device(self.device):
            self._cast_launch(stream)

    def _cast_launch(self, stream=None):
        for name, cin, cout, _ in self.convs:
            _lib.call("fdtd_sg_cast_weights", ptr(self.view(name + ".w")), cout, 9 * cin,
                      ptr(self.wb[name]), self.wb[name].shape[1], ptr(self.wt[name]), _s(stream))

    # ------------------------------------------------------------ buffers
    def _buffers(self, B):
        bufs = self._bufs.get(B)
        if bufs is not None:
            return bufs
        dev = self.device
        H, W = self.H, self.W
        c = [self.base << l for l in range(4)]
        P = [B * (H >> l) * (W >> l) for l in range(4)]
        bf = lambda *s: torch.zeros(s, dtype=BF16, device=dev)  # noqa: E731
        f = lambda *s: torch.zeros(s, dtype=F32, device=dev)  # noqa: E731
        b = {"B": B, "P": P}
        b["x0"] = bf(P[0], 1)
        b["e0a"], b["e1a"], b["e2a"] = bf(P[0], c[0]), bf(P[1], c[1]), bf(P[2], c[2])
        # concatenation buffers: [up | skip]; the skip conv writes its slice
        b["cat0"], b["cat1"], b["cat2"] = (bf(P[0], c[1] + c[0]), bf(P[1], c[2] + c[1]),
                                           bf(P[2], c[3] + c[2]))
        b["pool0"], b["pool1"], b["pool2"] = bf(P[1], c[0]), bf(P[2], c[1]), bf(P[3], c[2])
        b["bott"] = bf(P[3], c[3])
        b["d2"], b["d1"], b["d0"] = bf(P[2], c[2]), bf(P[1], c[1]), bf(P[0], c[0])
        b["feat"] = f(B, c[3])
        b["T"] = f(B, self.nwav)
        b["g"] = f(P[0])
        for name, cin, cout, lev in self.convs:
            b["col." + name] = bf(P[lev], _round8(9 * cin))
        # backward
        b["dT"], b["dg"] = f(B, self.nwav), f(P[0])
        b["d_d0"] = f(P[0], c[0])
        b["d_cat0"], b["d_cat1"], b["d_cat2"] = (f(P[0], c[1] + c[0]), f(P[1], c[2] + c[1]),
                                                 f(P[2], c[3] + c[2]))
        b["d_d1"], b["d_d2"], b["d_b"] = f(P[1], c[1]), f(P[2], c[2]), f(P[3], c[3])
        b["d_pool2"], b["d_pool1"], b["d_pool0"] = f(P[3], c[2]), f(P[2], c[1]), f(P[1], c[0])
        b["d_e2a"], b["d_e1a"], b["d_e0a"] = f(P[2], c[2]), f(P[1], c[1]), f(P[0], c[0])
        maxz = max(P[lev] * cout for _, _, cout, lev in self.convs)
        maxcol = max(P[lev] * 9 * cin for _, cin, _, lev in self.convs)
        b["dz"] = torch.zeros(maxz, dtype=BF16, device=dev)
        b["dzT"] = torch.zeros(max(cout * _round8(P[lev]) for _, _, cout, lev in self.convs),
                               dtype=BF16, device=dev)
        b["colT"] = torch.zeros(max(9 * cin * _round8(P[lev]) for _, cin, _, lev in self.convs),
                                dtype=BF16, device=dev)
        b["dcol"] = torch.zeros(maxcol, dtype=F32, device=dev)
        part = 0
        for name, cin, cout, lev in self.convs:
            s = self._wgrad_splits(9 * cin, cout, P[lev])
            self._splits[(name, B)] = s
            part = max(part, s * 9 * cin * cout)
        b["part"] = f(part)
        b["scratch"] = f(SCRATCH_ROWS * max(c[3], 1))
        b["loss_T"] = f((B * self.nwav + 255) // 256)
        b["loss_g"] = f((P[0] + 255) // 256)
        self._bufs[B] = b
        return b

    @staticmethod
    def _wgrad_splits(M, N, K):
        tiles = ((M + 127) // 128) * ((N + 127) // 128 if N > 64 else 1)
        want = max(1, (2 * 148 + tiles - 1) // tiles)
        return gemm_splits(M, N, K, want)

    # ------------------------------------------------------------ forward
    def _conv(self, b, name, x, ldx, out, ldo, stream):
        cin, cout, lev = next((ci, co, l) for n, ci, co, l in self.convs if n == name)
        h, w = self.H >> lev, self.W >> lev
        col = b["col." + name]
        P = b["P"][lev]
        _lib.call("fdtd_sg_im2col", ptr(x), ldx, b["B"], h, w, cin, ptr(col), col.shape[1],
                  _s(stream))
        gemm(col, self.wb[name], out, P, cout, 9 * cin, col.shape[1], self.wb[name].shape[1], ldo,
             bias=self.view(name + ".b"), relu=True, stream=stream)

    def forward(self, density, stream=None):
        """density (B, H, W) float32 on the device -> (T (B, nwav), g (B, H, W)),
        float32 views of internal buffers (valid until the next call)."""
        with torch.cuda.device(self.device):
            return self._forward(density, stream)

    def _forward(self, density, stream=None):
        if density.shape[1:] != (self.H, self.W):
            raise ValueError(f"expected (B, {self.H}, {self.W}) densities")
        density = density.to(device=self.device, dtype=F32).contiguous()
        B = density.shape[0]
        b = self._buffers(B)
        c0, c1, c2, c3 = (self.base << l for l in range(4))
        H, W = self.H, self.W
        s = _s(stream)
        call = _lib.call
        call("fdtd_sg_to_bf16", ptr(density), ptr(b["x0"]), b["P"][0], s)
        cat0, cat1, cat2 = b["cat0"], b["cat1"], b["cat2"]
        self._conv(b, "e0a", b["x0"], 1, b["e0a"], c0, stream)
        self._conv(b, "e0b", b["e0a"], c0, cat0[:, c1:], c1 + c0, stream)
        call("fdtd_sg_pool", ptr(cat0[:, c1:]), c1 + c0, B, H, W, c0, ptr(b["pool0"]), c0, s)
        self._conv(b, "e1a", b["pool0"], c0, b["e1a"], c1, stream)
        self._conv(b, "e1b", b["e1a"], c1, cat1[:, c2:], c2 + c1, stream)
        call("fdtd_sg_pool", ptr(cat1[:, c2:]), c2 + c1, B, H // 2, W // 2, c1, ptr(b["pool1"]),
             c1, s)
        self._conv(b, "e2a", b["pool1"], c1, b["e2a"], c2, stream)
        self._conv(b, "e2b", b["e2a"], c2, cat2[:, c3:], c3 + c2, stream)
        call("fdtd_sg_pool", ptr(cat2[:, c3:]), c3 + c2, B, H // 4, W // 4, c2, ptr(b["pool2"]),
             c2, s)
        self._conv(b, "bott", b["pool2"], c2, b["bott"], c3, stream)
        h3, w3 = H // 8, W // 8
        call("fdtd_sg_gap_linear", ptr(b["bott"]), c3, B, h3 * w3, c3, ptr(self.view("thead.w")),
             ptr(self.view("thead.b")), self.nwav, ptr(b["feat"]), ptr(b["T"]), s)
        call("fdtd_sg_upsample", ptr(b["bott"]), c3, B, h3, w3, c3, ptr(cat2), c3 + c2, s)
        self._conv(b, "d2", cat2, c3 + c2, b["d2"], c2, stream)
        call("fdtd_sg_upsample", ptr(b["d2"]), c2, B, H // 4, W // 4, c2, ptr(cat1), c2 + c1, s)
        self._conv(b, "d1", cat1, c2 + c1, b["d1"], c1, stream)
        call("fdtd_sg_upsample", ptr(b["d1"]), c1, B, H // 2, W // 2, c1, ptr(cat0), c1 + c0, s)
        self._conv(b, "d0", cat0, c1 + c0, b["d0"], c0, stream)
        call("fdtd_sg_head", ptr(b["d0"]), c0, b["P"][0], c0, ptr(self.view("ghead.w")),
             ptr(self.view("ghead.b")), ptr(b["g"]), s)
        self._last_B = B
        return b["T"], b["g"].view(B, H, W)

    def activations(self):
        """The last forward's stored activations as float32 NumPy (P, C) arrays
        (the skips are the concatenation buffers' skip slices)."""
        b = self._bufs[self._last_B]
        c0, c1, c2, c3 = (self.base << l for l in range(4))
        names = ["x0", "e0a", "pool0", "e1a", "pool1", "e2a", "pool2", "bott", "d2", "d1", "d0",
                 "feat"]
        out = {k: b[k].float().cpu().numpy() for k in names}
        out["e0b"] = b["cat0"][:, c1:].float().cpu().numpy()
        out["e1b"] = b["cat1"][:, c2:].float().cpu().numpy()
        out["e2b"] = b["cat2"][:, c3:].float().cpu().numpy()
        return out

    # ------------------------------------------------------------ backward
    def _conv_backward(self, b, name, dy, lddy, y, ldy, dx, lddx, stream, need_dx=True):
        cin, cout, lev = next((ci, co, l) for n, ci, co, l in self.convs if n == name)
        h, w = self.H >> lev, self.W >> lev
        P = b["P"][lev]
        s = _s(stream)
        dz = b["dz"][:P * cout].view(P, cout)
        _lib.call("fdtd_sg_relu_backward", ptr(dy), lddy, ptr(y), ldy, P, cout, ptr(dz), cout,
                  ptr(self.view(name + ".b", self.grads)), ptr(b["scratch"]), s)
        if need_dx:
            dcol = b["dcol"][:P * 9 * cin].view(P, 9 * cin)
            gemm(dz, self.wt[name], dcol, P, 9 * cin, cout, cout, cout, 9 * cin, stream=stream)
            _lib.call("fdtd_sg_col2im", ptr(dcol), 9 * cin, b["B"], h, w, cin, ptr(dx), lddx, 0, s)
        # weight gradient over the pixels, K split across blocks
        Pp = _round8(P)
        col = b["col." + name]
        colT = b["colT"][:9 * cin * Pp].view(9 * cin, Pp)
        dzT = b["dzT"][:cout * Pp].view(cout, Pp)
        _lib.call("fdtd_sg_transpose", ptr(col), col.shape[1], P, 9 * cin, ptr(colT), Pp, s)
        _lib.call("fdtd_sg_transpose", ptr(dz), cout, P, cout, ptr(dzT), Pp, s)
        splits = self._splits[(name, b["B"])]
        stride = 9 * cin * cout
        used = gemm(colT, dzT, b["part"], 9 * cin, cout, P, Pp, Pp, cout, splits=splits,
                    split_stride=stride, stream=stream)
        _lib.call("fdtd_sg_splitk_reduce", ptr(b["part"]), used, stride, 9 * cin, cout, cout,
                  ptr(self.view(name + ".w", self.grads)), 9 * cin, 1, s)

    def backward(self, dT=None, dg=None, stream=None):
        """Parameter gradients (into self.grads) of sum(dT * T) + sum(dg * g) for
        the last forward; dT, dg default to the loss gradients left by loss()."""
        with torch.cuda.device(self.device):
            return self._backward(dT, dg, stream)

    def _backward(self, dT=None, dg=None, stream=None):
        B = self._last_B
        b = self._bufs[B]
        if dT is not None:
            b["dT"].copy_(dT.reshape(b["dT"].shape))
        if dg is not None:
            b["dg"].copy_(dg.reshape(b["dg"].shape))
        c0, c1, c2, c3 = (self.base << l for l in range(4))
        H, W = self.H, self.W
        s = _s(stream)
        call = _lib.call
        g = self.grads
        cat0, cat1, cat2 = b["cat0"], b["cat1"], b["cat2"]
        dc0, dc1, dc2 = b["d_cat0"], b["d_cat1"], b["d_cat2"]
        call("fdtd_sg_head_backward", ptr(b["dg"]), ptr(b["d0"]), c0, b["P"][0], c0,
             ptr(self.view("ghead.w")), ptr(b["d_d0"]), c0, ptr(self.view("ghead.w", g)),
             ptr(self.view("ghead.b", g)), ptr(b["scratch"]), s)
        self._conv_backward(b, "d0", b["d_d0"], c0, b["d0"], c0, dc0, c1 + c0, stream)
        call("fdtd_sg_upsample_backward", ptr(dc0), c1 + c0, B, H // 2, W // 2, c1,
             ptr(b["d_d1"]), c1, 0, s)
        self._conv_backward(b, "d1", b["d_d1"], c1, b["d1"], c1, dc1, c2 + c1, stream)
        call("fdtd_sg_upsample_backward", ptr(dc1), c2 + c1, B, H // 4, W // 4, c2,
             ptr(b["d_d2"]), c2, 0, s)
        self._conv_backward(b, "d2", b["d_d2"], c2, b["d2"], c2, dc2, c3 + c2, stream)
        h3, w3 = H // 8, W // 8
        call("fdtd_sg_upsample_backward", ptr(dc2), c3 + c2, B, h3, w3, c3, ptr(b["d_b"]), c3, 0,
             s)
        call("fdtd_sg_gap_linear_backward", ptr(b["dT"]), ptr(b["feat"]),
             ptr(self.view("thead.w")), B, h3 * w3, c3, self.nwav, ptr(self.view("thead.w", g)),
             ptr(self.view("thead.b", g)), ptr(b["d_b"]), c3, 1, s)
        self._conv_backward(b, "bott", b["d_b"], c3, b["bott"], c3, b["d_pool2"], c2, stream)
        call("fdtd_sg_pool_backward", ptr(b["d_pool2"]), c2, B, H // 4, W // 4, c2,
             ptr(dc2[:, c3:]), c3 + c2, 1, s)
        self._conv_backward(b, "e2b", dc2[:, c3:], c3 + c2, cat2[:, c3:], c3 + c2, b["d_e2a"], c2,
                            stream)
        self._conv_backward(b, "e2a", b["d_e2a"], c2, b["e2a"], c2, b["d_pool1"], c1, stream)
        call("fdtd_sg_pool_backward", ptr(b["d_pool1"]), c1, B, H // 2, W // 2, c1,
             ptr(dc1[:, c2:]), c2 + c1, 1, s)
        self._conv_backward(b, "e1b", dc1[:, c2:], c2 + c1, cat1[:, c2:], c2 + c1, b["d_e1a"], c1,
                            stream)
        self._conv_backward(b, "e1a", b["d_e1a"], c1, b["e1a"], c1, b["d_pool0"], c0, stream)
        call("fdtd_sg_pool_backward", ptr(b["d_pool0"]), c0, B, H, W, c0, ptr(dc0[:, c1:]),
             c1 + c0, 1, s)
        self._conv_backward(b, "e0b", dc0[:, c1:], c1 + c0, cat0[:, c1:], c1 + c0, b["d_e0a"], c0,
                            stream)
        self._conv_backward(b, "e0a", b["d_e0a"], c0, b["e0a"], c0, None, 0, stream,
                            need_dx=False)
        return self.grads

    # ------------------------------------------------------------ training
    def loss(self, T_target, g_target, w_T=1.0, w_g=1.0, stream=None, value=True):
        """Squared-error loss of the last forward against targets (device
        tensors (B, nwav) and (B, H, W)); leaves the output gradients for
        backward().  Returns the loss as a float (one device sync) when value."""
        b = self._bufs[self._last_B]
        with torch.cuda.device(self.device):
            s = _s(stream)
            nT, ng = b["T"].numel(), b["g"].numel()
            self._loss_launch(b, s, T_target, g_target, w_T, w_g, nT, ng)
        if not value:
            return None
        return float(w_T * b["loss_T"].sum().item() / nT + w_g * b["loss_g"].sum().item() / ng)

    def _loss_launch(self, b, s, T_target, g_target, w_T, w_g, nT, ng):
        _lib.call("fdtd_sg_mse", ptr(b["T"]), ptr(T_target.contiguous()), nT, w_T / nT,
                  ptr(b["dT"]), ptr(b["loss_T"]), s)
        _lib.call("fdtd_sg_mse", ptr(b["g"]), ptr(g_target.contiguous()), ng, w_g / ng,
                  ptr(b["dg"]), ptr(b["loss_g"]), s)

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, stream=None):
        self.adam_step += 1
        with torch.cuda.device(self.device):
            _lib.call("fdtd_sg_adam", ptr(self.params), ptr(self.grads), ptr(self.m),
                      ptr(self.v), self.count, lr, b1, b2, eps, self.adam_step, _s(stream))
            self._cast(stream)

    def train_step(self, density, T_target, g_target, lr=1e-3, w_T=1.0, w_g=1.0, value=False):
        self.forward(density)
        L = self.loss(T_target, g_target, w_T, w_g, value=value)
        self.backward()
        self.adam(lr)
        return L

    def fit(self, densities, T, g, steps, batch=32, lr=1e-3, w_T=1.0, w_g=1.0, seed=0,
            log_every=0):
        """Adam on random minibatches of a device-resident data set."""
        n = densities.shape[0]
        gen = torch.Generator(device="cpu").manual_seed(seed)
        losses = []
        for it in range(steps):
            idx = torch.randint(0, n, (min(batch, n),), generator=gen).to(self.device)
            value = bool(log_every) and (it % log_every == 0 or it == steps - 1)
            L = self.train_step(densities[idx], T[idx], g[idx], lr, w_T, w_g, value=value)
            if value:
                losses.append((it, L))
        return losses

    @torch.no_grad()
    def predict(self, density):
        """(T, g) for a (B, H, W) or (H, W) density, as new float32 tensors."""
        single = density.dim() == 2
        d = density[None] if single else density
        T, g = self.forward(d)
        T, g = T.clone(), g.clone()
        return (T[0], g[0]) if single else (T, g)


def default_init(seed=0, base=32, nwav=8):
    """He-normal convolution weights, zero biases, 1/sqrt(fan-in) heads."""
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


def train_flops(size, base=32, batch=1):
    """Algorithmic FLOPs of one training step (forward, input and weight
    gradients of every 3 x 3 convolution, 2 per multiply-add; the layer
    without an input gradient counted once less), for `batch` designs."""
    H, W = size
    total = 0
    for name, cin, cout, lev in architecture(base):
        mac = batch * (H >> lev) * (W >> lev) * 9 * cin * cout
        total += 2 * mac * (2 if name == "e0a" else 3)
    return total


def main(argv=None):
    """Time training steps of the surrogate on synthetic designs:
    python -m warp_fdtd_b200.surrogate [--batch 32] [--size 80 80] [--steps 50]"""
    import argparse
    import json

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--size", type=int, nargs=2, default=(80, 80))
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    a = ap.parse_args(argv)
    size = tuple(a.size)
    net = Surrogate(size, 8)
    gen = torch.Generator(device="cpu").manual_seed(0)
    x = torch.rand((a.batch,) + size, generator=gen).cuda()
    T = torch.rand((a.batch, 8), generator=gen).cuda()
    g = torch.randn((a.batch,) + size, generator=gen).cuda()
    for _ in range(a.warmup):
        net.train_step(x, T, g)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.steps):
        net.train_step(x, T, g)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / a.steps
    flops = train_flops(size, net.base, a.batch)
    print(json.dumps(dict(workload=f"surrogate_train_{size[0]}x{size[1]}_b{a.batch}",
                          train_step_ms=ms, designs_per_s=a.batch / ms * 1e3,
                          tflops=flops / ms / 1e9, flops_per_step=flops,
                          params=net.count, wait_status=status())))


if __name__ == "__main__":
    main()
