"""Many independent solvers advanced together on one GPU.

`BatchSolver` takes solvers of uneven grids (designs, domains) and runs their
trajectories together.  Two modes:

* streams (default): each instance's own step graphs (Solver.compile) replay
  on its own CUDA stream, round-robin, forked from and joined to the caller's
  stream, so the instances' kernels run side by side;
* fused (`fused=True`, grids on the full-z path with the same row pitch, z
  slab width, material kind and trajectory length): every step is ONE launch
  of the full-z kernel over all grids (fdtd_step_batch) with a cost-balanced
  schedule of (grid, tile, plane run) blocks across the whole batch, then each
  grid's detectors and one launch advancing every step counter; steps are
  captured in CUDA graphs of `graph_steps` steps.  On a B200 with 16 and 48
  grids of 180-340 x 180-340 x 116 cells it ran 59 and 62 Gcell/s against 69
  for the streams (its kernel reads each grid's parameters at run time).

Every instance keeps its own buffers, detectors and counters; results equal
running each solver alone, bit for bit.  `autotune=True` tunes each instance's
launch shape first (Solver.autotune; stream mode).
"""

import ctypes

import numpy as np
import torch

from . import _lib
from ._lib import ptr
from .schedule import batch_schedule


class BatchSolver:
    def __init__(self, solvers, autotune=False, fused=False):
        self.solvers = list(solvers)
        if not self.solvers:
            raise ValueError("BatchSolver needs at least one solver")
        devices = {s.device for s in self.solvers}
        if len(devices) != 1:
            raise ValueError("All solvers of a batch must share one device")
        self.device = devices.pop()
        self.fused = bool(fused) and self._fusable()
        if autotune and not self.fused:
            for s in self.solvers:
                s.autotune()
        self.streams = [torch.cuda.Stream(self.device) for _ in self.solvers]
        self.graphs = {}
        self.compiled = False
        self._issued = 0
        if self.fused:
            self._prepare()

    # ------------------------------------------------------------ fused mode
    def _fusable(self):
        s0 = self.solvers[0]
        key = lambda s: (s._psi_layout, s._pitch, s._psi_r[2], s.material_kind,
                         s.shape[2] == s._pitch, s.steps, s.graph_steps, s.stages)
        return s0._psi_layout == 2 and all(key(s) == key(s0) for s in self.solvers)

    def _prepare(self):
        solvers = self.solvers
        a0 = solvers[0]._step_args()
        _lib.call("fdtd_step_defaults", ctypes.byref(a0))
        ty = int(a0.tile_y)
        grids = [(s.shape, s._coeff_step["E"].cpu().numpy(), s._coeff_step["H"].cpu().numpy())
                 for s in solvers]
        weights = solvers[0].schedule_weights
        slots, runs = None, None
        a0.schedule = None
        for _ in range(3):  # the longest run sizes shared memory, hence occupancy
            blocks, sms = ctypes.c_int(0), ctypes.c_int(0)
            _lib.call("fdtd_step_occupancy", ctypes.byref(a0), ctypes.byref(blocks),
                      ctypes.byref(sms))
            if blocks.value * sms.value == slots:
                break
            slots = blocks.value * sms.value
            runs = batch_schedule(grids, ty, slots, *weights)
            a0.chunk_x = int((runs[:, 3] - runs[:, 2]).max())
        chunk = int((runs[:, 3] - runs[:, 2]).max())
        for s in solvers:
            s.set_tile(ty, 0, chunk, s.stages)
        n = len(solvers)
        args = (_lib.StepArgs * n)(*[s._args for s in solvers])
        nbytes = int(_lib.load().fdtd_batch_workspace_bytes(n))
        self._workspace = torch.empty(nbytes + 64, dtype=torch.uint8, device=self.device)
        base = self._workspace.data_ptr()
        self._ws = base + (-base) % 64
        self._plan = _lib.BatchPlan()
        _lib.call("fdtd_batch_prepare", args, n, self._ws, nbytes, ctypes.byref(self._plan))
        self._schedule = torch.from_numpy(np.ascontiguousarray(runs)).to(self.device)
        self._blocks = int(runs.shape[0])
        self._steps = torch.tensor([s.step.data_ptr() for s in solvers], dtype=torch.int64,
                                   device=self.device)

    def close(self):
        """Free the batch's slots in the library's grid-parameter table."""
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.count > 0:
            _lib.call("fdtd_batch_release", ctypes.byref(plan))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def launch_step(self):
        """One step of every grid: the batched fused launch, each grid's
        detectors, the counters."""
        stream = _lib.stream_handle(self.device)
        _lib.call("fdtd_step_batch", ctypes.byref(self._plan), self._ws, ptr(self._schedule),
                  self._blocks, stream)
        for s in self.solvers:
            for m in s.monitors:
                m.launch(s)
        _lib.call("fdtd_advance_many", ptr(self._steps), len(self.solvers), 1, stream)
        for s in self.solvers:
            s._issued += 1
            for m in s.monitors:
                if m.is_phasor and (s._issued % m.batch == 0 or s._issued == s.steps):
                    m.fold(s, s._issued)
        self._issued += 1

    def _set_issued(self, start):
        self._issued = start
        for s in self.solvers:
            s._issued = start
            for m in s.monitors:
                m._folded = start

    # ------------------------------------------------------------ both modes
    def compile(self):
        """Capture the step graphs; returns the seconds taken."""
        import time

        if not self.fused:
            total = sum(s.compile() for s in self.solvers)
            self.compiled = True
            return total
        start = time.perf_counter()
        s0 = self.solvers[0]
        with torch.cuda.device(self.device):
            self.launch_step()
            torch.cuda.synchronize(self.device)
            self.reset()
            for length in {s0.graph_steps, s0.steps % s0.graph_steps} - {0}:
                offset = 0 if length == s0.graph_steps else s0.steps - length
                self._set_issued(offset)
                g = torch.cuda.CUDAGraph()
                with torch.cuda.graph(g, capture_error_mode="relaxed"):
                    for _ in range(length):
                        self.launch_step()
                self.graphs[length] = g
            self.reset()
        self.compiled = True
        return time.perf_counter() - start

    def reset(self):
        for s in self.solvers:
            s.reset()
        self._issued = 0

    def run(self):
        """Advance every instance through its whole trajectory."""
        if not self.compiled:
            self.compile()
        if any(s._issued != 0 for s in self.solvers):
            raise ValueError("BatchSolver.run starts every instance from reset()")
        with torch.cuda.device(self.device):
            if self.fused:
                s0 = self.solvers[0]
                for _ in range(s0.steps // s0.graph_steps):
                    self.graphs[s0.graph_steps].replay()
                tail = s0.steps % s0.graph_steps
                if tail:
                    self.graphs[tail].replay()
                self._set_issued(s0.steps)
            else:
                self._run_streams()
            torch.cuda.synchronize(self.device)

    def _run_streams(self):
        main = torch.cuda.current_stream(self.device)
        fork = torch.cuda.Event()
        fork.record(main)
        plans = []
        for s, st in zip(self.solvers, self.streams):
            st.wait_event(fork)
            plans.append([s.steps // s.graph_steps, s.steps % s.graph_steps])
        # round-robin graph replays, one per instance per round
        while any(p[0] for p in plans):
            for s, st, p in zip(self.solvers, self.streams, plans):
                if p[0]:
                    with torch.cuda.stream(st):
                        s.graphs[s.graph_steps].replay()
                    p[0] -= 1
        for s, st, p in zip(self.solvers, self.streams, plans):
            if p[1]:
                with torch.cuda.stream(st):
                    s.graphs[p[1]].replay()
            s._issued = s.steps
            for m in s.monitors:
                m._folded = s.steps
        for st in self.streams:
            done = torch.cuda.Event()
            done.record(st)
            main.wait_event(done)
