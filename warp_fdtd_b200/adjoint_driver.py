"""Drop-in for warp_fdtd/adjoint.py's `Adjoint`: exact discrete adjoint gradient.

The reverse sweep is the reference's exact transpose (adjoint.py:388-414):
per reverse step inject(old E/H) -> prepare(qh) -> gather(qe, grad) ->
prepare(qe) -> gather(qh) -> inject(old H) -> retreat, with the reference's
kernels' arithmetic (fdtd_inject / fdtd_prepare / fdtd_gather).  What changes:

* The forward runs on the fused B200 path and saves the full state (E, H and
  both CPML states) every `checkpoint_every` steps instead of storing the
  design-box curl for every step (adjoint.py:258-260 keeps
  steps x 3 x design_n floats, 8.06 GB for the 20 nm bend).  The reverse sweep
  walks the segments backwards; each segment is first recomputed from its
  checkpoint with the curl history recorded for that segment only
  (checkpoint_every x 3 x design_n floats).  checkpoint_every >= steps gives
  the reference's single full history.
* The design-gradient inner product accumulates in float64 (fdtd_gather with
  a float64 grad).
* The design box and the material map are parameters (the reference hard-wires
  the 20 nm bend's 80 x 80 x 20 box, adjoint.py:234-257); `strict=True` keeps
  the reference's guard.
* `TransmissionLoss` wraps the gradient as a torch.autograd.Function.
"""

import numpy as np
import torch

from . import _lib
from . import adjoint as kernels
from ._lib import ptr
from .detectors import measurements
from .material import Material
from .solver import Solver, cpml_coefficients


class Adjoint(Solver):
    def __init__(self, case, box=None, checkpoint_every=256, strict=False, device="cuda:0",
                 graph_steps=64, material_kwargs=None, fused_reverse=True):
        # single steps (the design-box history and the checkpoints need every
        # step's fields in the parity buffers)
        super().__init__(case, device=device, graph_steps=graph_steps, material="f32",
                         time_block=1)
        settings = self.meta["settings"]
        if strict:
            if (
                self.shape != (200, 200, 75)
                or settings["spacing_nm"] != 20
                or settings.get("parameterization") != "smooth"
            ):
                raise ValueError("Adjoint driver currently supports the 20 nm smooth bend only")
            required = {"time_fs": 200, "pml_cells": 10, "domain_um": 4, "voxel_nm": 20,
                        "scene": "bend"}
            if any(settings.get(k) != v for k, v in required.items()) or settings.get(
                "pad_domain", False
            ):
                raise ValueError("Adjoint driver requires the unpadded 200 fs reference geometry")
        if box is None:
            if self.shape != (200, 200, 75):
                raise ValueError("A design box (x0, y0, z0, sx, sy, sz) is required")
            box = (100, 20, 30, 80, 80, 20)  # adjoint.py:256
        self.box = tuple(int(v) for v in box)
        x0, y0, z0, sx, sy, sz = self.box
        if min(x0, y0, z0) < 0 or x0 + sx > self.shape[0] or y0 + sy > self.shape[1] or \
                z0 + sz > self.shape[2] or min(sx, sy, sz) < 1:
            raise ValueError("Design box outside the grid")
        self.design_n = sx * sy * sz
        self.material_kwargs = dict(material_kwargs or {})
        K = int(checkpoint_every)
        if K < 2:
            raise ValueError("checkpoint_every must be >= 2")
        K = min(K, self.steps)
        K += K & 1  # even: checkpoints land on parity-0 buffers
        self.checkpoint_every = K
        # one segment: the forward itself records the history, so the reverse
        # sweep needs no recomputation (the reference's storage scheme)
        self.history_in_forward = K >= self.steps
        self._history_fresh = False
        dev = self.device
        f32 = dict(dtype=torch.float32, device=dev)
        n = self.n
        self.history = torch.empty((K, 3, self.design_n), **f32)
        self.qe = torch.zeros((3, n), **f32)
        self.qh = torch.zeros((3, n), **f32)
        self.psie = torch.zeros((6, n), **f32)
        self.psih = torch.zeros((6, n), **f32)
        self.d = torch.empty((6, n), **f32)
        # fused reverse halves (fdtd_reverse_half): the CPML state ping-pongs
        self.fused_reverse = bool(fused_reverse)
        self.psie2 = torch.zeros((6, n), **f32) if self.fused_reverse else None
        self.psih2 = torch.zeros((6, n), **f32) if self.fused_reverse else None
        self._inject_planes = None  # fused path: all planes' injections in one launch
        self.grad = torch.zeros(self.design_n, dtype=torch.float64, device=dev)
        self.reverse_step = torch.zeros(1, dtype=torch.int32, device=dev)
        self.hist_step = torch.zeros(1, dtype=torch.int32, device=dev)
        # fused path: both counters advanced by one launch
        self._counters = torch.tensor([self.reverse_step.data_ptr(), self.hist_step.data_ptr()],
                                      dtype=torch.int64, device=dev)
        self._coeff3 = {f: torch.from_numpy(cpml_coefficients(self.meta, self.data, self.shape, f)).to(dev)
                        for f in "EH"}
        # the fused halves read (a, b, 1/kappa, 0) as one float4
        self._coeff4 = {f: torch.nn.functional.pad(c, (0, 1)).contiguous()
                        for f, c in self._coeff3.items()}
        self.adjoint_sources = []
        self.reverse_graphs = {}
        self.recompute_graphs = {}
        self.checkpoints = {}
        self.design_material = None

    # ------------------------------------------------------------ forward
    def _snapshot(self):
        return tuple(t.clone() for t in (self._E[0], self._H[0], self._psi_e[0], self._psi_h[0]))

    def _restore(self, snap):
        for dst, src in zip((self._E[0], self._H[0], self._psi_e[0], self._psi_h[0]), snap):
            dst.copy_(src)

    def _after_update(self, stream):
        if self.history_in_forward:
            x0, y0, z0, sx, sy, sz = self.box
            _lib.call("fdtd_record_curl_pp", ptr(self._H[0]), ptr(self._H[1]), self._pitch,
                      ptr(self.step), ptr(self.hist_step), ptr(self.history), *self.shape, x0,
                      y0, z0, sx, sy, sz, float(self.courant), stream)
            _lib.call("fdtd_advance", ptr(self.hist_step), 1, stream)

    def run(self, sync=True):
        """Forward trajectory with detectors, saving a state checkpoint every
        `checkpoint_every` steps (at step counts that are multiples of it);
        with a single segment the design-box history is recorded instead.
        Everything is enqueued on the current stream; sync=False returns
        without waiting for the device (batch.BatchAdjoint overlaps
        instances that way)."""
        K = self.checkpoint_every
        self.checkpoints = {}
        self._history_fresh = False
        if self.history_in_forward:
            self.hist_step.fill_(self._issued)
        with torch.cuda.device(self.device):
            if self.graphs and (K % self.graph_steps == 0 or self.history_in_forward):
                for c in range(self.steps // self.graph_steps):
                    start = c * self.graph_steps
                    if start % K == 0 and start > 0:
                        self.checkpoints[start] = self._snapshot()
                    self.graphs[self.graph_steps].replay()
                tail = self.steps % self.graph_steps
                start = self.steps - tail
                if tail:
                    if start % K == 0 and start > 0:
                        self.checkpoints[start] = self._snapshot()
                    self.graphs[tail].replay()
                self._issued = self.steps
                for m in self.monitors:
                    m._folded = self.steps
            else:
                while self._issued < self.steps:
                    if self._issued % K == 0 and self._issued > 0:
                        self.checkpoints[self._issued] = self._snapshot()
                    self.launch_step()
            self._history_fresh = self.history_in_forward
            if sync:
                torch.cuda.synchronize(self.device)

    def _recompute_step(self, stream):
        self._step_kernel(stream)
        x0, y0, z0, sx, sy, sz = self.box
        _lib.call("fdtd_record_curl_pp", ptr(self._H[0]), ptr(self._H[1]), self._pitch,
                  ptr(self.step), ptr(self.hist_step), ptr(self.history), *self.shape, x0, y0, z0,
                  sx, sy, sz, float(self.courant), stream)
        _lib.call("fdtd_advance", ptr(self.step), 1, stream)
        _lib.call("fdtd_advance", ptr(self.hist_step), 1, stream)

    def _recompute(self, start, length):
        """Re-run steps [start, start + length) from the checkpoint at `start`,
        recording courant * curl(H) in the design box (adjoint.py:17-43)."""
        if start == 0:
            for group in (self._E, self._H, self._psi_e, self._psi_h):
                group[0].zero_()
        else:
            self._restore(self.checkpoints[start])
        self.step.fill_(start)
        self.hist_step.zero_()
        g = self.recompute_graphs.get(length)
        if g is None:
            stream = _lib.stream_handle(self.device)
            for _ in range(length):
                self._recompute_step(stream)
            return
        g.replay()

    # ------------------------------------------------------------ reverse
    def prepare_sources(self):
        """adjoint.py:329-366: adjoint plane sources from the modal overlaps
        (factors P_out / P_in^2 for mode_in, -1 / P_in for mode_out), written
        in place into existing buffers so captured graphs stay valid."""
        previous = self.adjoint_sources
        monitors = {m.name: m for m in self.monitors}
        pin = monitors["mode_in"].power(self)
        pout = monitors["mode_out"].power(self)
        if not np.isfinite(pin) or pin <= 0 or not np.isfinite(pout):
            raise ValueError("Finite modal powers and positive incident power required")
        self.adjoint_sources = []
        for name, factor in [("mode_in", pout / pin ** 2), ("mode_out", -1 / pin)]:
            m = monitors[name]
            ph = m.phasors()
            em = self.data[name + "/_mode_E"][0]
            hm = self.data[name + "/_mode_H"][0]
            axis = m.axis
            a = (axis + 1) % 3
            b = (axis + 2) % 3
            qe = np.zeros_like(em)
            qh = np.zeros_like(hm)
            qe[a] = hm[b].conj() / 4
            qe[b] = -hm[a].conj() / 4
            qh[b] = em[a].conj() / 4
            qh[a] = -em[b].conj() / 4
            coeff = np.concatenate((qe, qh)) * m.area_numpy[None]
            beta = np.sum(coeff * ph)
            source = (2 * factor * beta.conjugate() * coeff).reshape(6, -1).astype(np.complex64)
            host = torch.from_numpy(np.ascontiguousarray(
                np.stack((source.real, source.imag), axis=-1), np.float32))
            if previous:
                old_monitor, v = previous[len(self.adjoint_sources)]
                if old_monitor.name != m.name:
                    raise ValueError("Changing detector layout requires new graphs")
                v.copy_(host)
            else:
                v = host.to(self.device)
            self.adjoint_sources.append((m, v))

    def _planes(self):
        """The adjoint sources as fdtd_inject_plane entries (their buffers are
        updated in place by prepare_sources, so the entries stay valid)."""
        key = tuple((id(m), v.data_ptr()) for m, v in self.adjoint_sources)
        if self._inject_planes is None or self._inject_planes[0] != key:
            arr = (_lib.InjectPlane * len(self.adjoint_sources))()
            for pl, (m, v) in zip(arr, self.adjoint_sources):
                sy, sz = (int(d) for d in m.shape[1:])
                pl.source, pl.weights = ptr(v), ptr(m.weights[0])
                pl.x0, pl.y0, pl.z0 = (int(c) for c in m.lo)
                pl.sx, pl.sy, pl.sz = int(v.shape[1]) // (sy * sz), sy, sz
            self._inject_planes = (key, arr)
        return self._inject_planes[1]

    def inject(self, old):
        if self.fused_reverse and 1 <= len(self.adjoint_sources) <= 8:
            planes = self._planes()
            _lib.call("fdtd_inject_many", ptr(self.qe), ptr(self.qh), planes, len(planes),
                      ptr(self.reverse_step), *self.shape, int(old),
                      _lib.stream_handle(self.device))
            return
        for m, v in self.adjoint_sources:
            kernels.inject(self.qe, self.qh, v, m.weights[0], self.reverse_step, *self.shape,
                           *m.lo, *m.shape[1:], old)

    def reverse_one(self):
        """adjoint.py:388-414 with the float64 gradient and a segment-relative
        history index.  With fused_reverse each prepare + gather pair is one
        pass (fdtd_reverse_half), bitwise the same values."""
        self.inject(0)
        if self.fused_reverse:
            stream = _lib.stream_handle(self.device)
            clen = int(self._coeff4["H"].shape[1])
            _lib.call("fdtd_reverse_half", 1, ptr(self.qe), ptr(self.qh), ptr(self.eps),
                      ptr(self.psih), ptr(self.psih2), ptr(self._coeff4["H"]), clen,
                      ptr(self.reverse_step), ptr(self.history), ptr(self.grad),
                      ptr(self.hist_step), *self.shape, self.courant, *self.box, stream)
            _lib.call("fdtd_reverse_half", 0, ptr(self.qh), ptr(self.qe), ptr(self.eps),
                      ptr(self.psie), ptr(self.psie2), ptr(self._coeff4["E"]), clen,
                      ptr(self.reverse_step), None, None, None, *self.shape, self.courant,
                      0, 0, 0, 0, 0, 0, stream)
            self.inject(1)
            _lib.call("fdtd_advance_many", ptr(self._counters), 2, -1, stream)
            return
        common = [*self.shape, self.courant]
        kernels.prepare(self.qh, self.eps, self.psih, self._coeff3["H"], self.d, *common, 0)
        args = [self.d, self.history, self.grad, self.hist_step, *self.shape, *self.box]
        kernels.gather(self.qe, *args, 1)
        kernels.prepare(self.qe, self.eps, self.psie, self._coeff3["E"], self.d, *common, 1)
        kernels.gather(self.qh, *args, 0)
        self.inject(1)
        stream = _lib.stream_handle(self.device)
        _lib.call("fdtd_advance", ptr(self.reverse_step), -1, stream)
        _lib.call("fdtd_advance", ptr(self.hist_step), -1, stream)

    def reset_reverse(self):
        for a in (self.qe, self.qh, self.psie, self.psih, self.grad, self.psie2, self.psih2):
            if a is not None:
                a.zero_()
        self.reverse_step.fill_(self.steps - 1)
        torch.cuda.synchronize(self.device)

    def _segments(self):
        K = self.checkpoint_every
        return [(s, min(K, self.steps - s)) for s in range(0, self.steps, K)]

    def compile_reverse(self):
        """Capture the recompute and reverse sequences of each segment length."""
        with torch.cuda.device(self.device):
            for _, length in self._segments():
                if length in self.reverse_graphs:
                    continue
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, capture_error_mode="relaxed"):
                    for _ in range(length):
                        self.reverse_one()
                self.reverse_graphs[length] = g
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, capture_error_mode="relaxed"):
                    s = _lib.stream_handle(self.device)
                    for _ in range(length):
                        self._recompute_step(s)
                self.recompute_graphs[length] = g
        self.reset_reverse()

    def backward(self, sync=True):
        """Reverse sweep over all segments, last first, enqueued on the current
        stream (sync=False: no wait for the device at the end)."""
        with torch.cuda.device(self.device):
            for start, length in reversed(self._segments()):
                if not (self._history_fresh and start == 0 and length == self.steps):
                    self._recompute(start, length)
                self.reverse_step.fill_(start + length - 1)
                self.hist_step.fill_(length - 1)
                g = self.reverse_graphs.get(length)
                if g is None:
                    for _ in range(length):
                        self.reverse_one()
                else:
                    g.replay()
            self._history_fresh = False
            if sync:
                torch.cuda.synchronize(self.device)

    # ------------------------------------------------------------ design
    def set_design(self, parameters):
        """adjoint.py:441-451: material map of the parameters, extruded in z
        into the design box."""
        x0, y0, z0, sx, sy, sz = self.box
        params = np.asarray(parameters, np.float32).reshape(sx, sy)
        beta = self.material_kwargs.get("beta", self.meta.get("beta", 50.0))
        kw = {k: v for k, v in self.material_kwargs.items() if k != "beta"}
        self.design_material = Material(params, beta, device=self.device, **kw)
        kernels.write_design(self.design_material.inv_eps, self.eps, *self.shape, *self.box)
        self.refresh_material()
        return self.design_material

    def voxel_gradient(self):
        x0, y0, z0, sx, sy, sz = self.box
        return self.grad.reshape(sx, sy, sz).sum(dim=2).cpu().numpy()

    def differentiate(self, parameters):
        """-modal transmission and its gradient with respect to the parameters
        (adjoint.py:453-469)."""
        material = self.set_design(parameters)
        if not self.graphs:
            self.compile()
        self.reset()
        self.run()
        self.prepare_sources()
        if not self.reverse_graphs:
            self.compile_reverse()
        self.reset_reverse()
        self.backward()
        voxel = self.voxel_gradient()
        gradient = material.pullback(voxel.astype(np.float32))
        return -measurements(self)["modal_transmission"], gradient


class TransmissionLoss(torch.autograd.Function):
    """loss = -T(params) through the checkpointed adjoint: forward runs the
    solver, backward returns dloss/dparams scaled by the incoming gradient."""

    @staticmethod
    def forward(ctx, params, adjoint):
        loss, grad = adjoint.differentiate(params.detach().cpu().numpy())
        ctx.save_for_backward(torch.as_tensor(grad, dtype=params.dtype, device=params.device))
        return torch.tensor(loss, dtype=params.dtype, device=params.device)

    @staticmethod
    def backward(ctx, upstream):
        (grad,) = ctx.saved_tensors
        return upstream * grad, None
