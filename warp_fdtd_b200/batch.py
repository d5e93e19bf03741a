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
        """Free the batch's slots in the library's grid-parameter table, once
        the device has finished every launch that reads them (a batch run with
        launches still queued, for instance after graph replays without a
        synchronise, would otherwise read a later batch's parameters)."""
        plan = getattr(self, "_plan", None)
        if plan is not None and plan.count > 0:
            torch.cuda.synchronize(self.device)
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
                m.launch(s, s._ord(s._E), s._ord(s._H))
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
            plans.append(list(s._replays()))
        # round-robin graph replays, one per instance per round
        while any(plans):
            for s, st, p in zip(self.solvers, self.streams, plans):
                if p:
                    with torch.cuda.stream(st):
                        p.pop(0).replay()
        for s in self.solvers:
            s._issued = s.steps
            s._rel ^= s._final_flip
            for m in s.monitors:
                m._folded = s.steps
        for st in self.streams:
            done = torch.cuda.Event()
            done.record(st)
            main.wait_event(done)


class BatchAdjoint:
    """Gradients of many independent design problems (adjoint_driver.Adjoint
    instances of uneven grids) computed side by side on one GPU.

    Per call of differentiate(parameters): every instance's material map is
    set, then all forward trajectories run at once, each instance's captured
    step graphs replaying on its own stream (forked from and joined to the
    caller's).  The adjoint plane sources are formed on the host (one device
    synchronisation), then all reverse sweeps run at once the same way, with
    their recomputation and reverse graphs.  Each instance keeps its own
    buffers, counters and graphs, so the losses equal single runs bit for bit
    and the gradients equal them up to the float32 atomics of the adjoint
    source injection."""

    def __init__(self, adjoints):
        self.adjoints = list(adjoints)
        if not self.adjoints:
            raise ValueError("BatchAdjoint needs at least one Adjoint")
        devices = {a.device for a in self.adjoints}
        if len(devices) != 1:
            raise ValueError("All adjoints of a batch must share one device")
        self.device = devices.pop()
        self.streams = [torch.cuda.Stream(self.device) for _ in self.adjoints]

    def _each_on_its_stream(self, fn):
        caller = torch.cuda.current_stream(self.device)
        for a, s in zip(self.adjoints, self.streams):
            s.wait_stream(caller)
            with torch.cuda.stream(s):
                fn(a)
        for s in self.streams:
            caller.wait_stream(s)

    def differentiate(self, parameters):
        """[(-T, dT/dp)] per instance, as Adjoint.differentiate returns."""
        from .detectors import measurements

        if len(parameters) != len(self.adjoints):
            raise ValueError("one parameter array per instance required")
        with torch.cuda.device(self.device):
            materials = []
            for a, p in zip(self.adjoints, parameters):
                materials.append(a.set_design(p))
                if not a.graphs:
                    a.compile()
                a.reset()
            self._each_on_its_stream(lambda a: a.run(sync=False))
            torch.cuda.synchronize(self.device)
            for a in self.adjoints:
                a.prepare_sources()
                if not a.reverse_graphs:
                    a.compile_reverse()
                a.reset_reverse()
            self._each_on_its_stream(lambda a: a.backward(sync=False))
            torch.cuda.synchronize(self.device)
        out = []
        for a, m in zip(self.adjoints, materials):
            gradient = m.pullback(a.voxel_gradient().astype(np.float32))
            out.append((-measurements(a)["modal_transmission"], gradient))
        return out


def _uneven_bends(root, count, seed, steps, spacing_nm=25.0):
    """Seeded uneven 90-degree bends: interior sides drawn from 4-8 um (160-320
    cells at 25 nm), 2.4 um tall (96 cells), 10-cell CPML, radius 1.5 um, and a
    design box of 1.5-3 um square over the arc, extruded through the core."""
    from . import scene

    rng = np.random.default_rng(seed)
    out = []
    dx = spacing_nm * 1e-3
    for i in range(count):
        lx, ly = (float(v) for v in rng.uniform(4.0, 8.0, 2))
        side = float(rng.uniform(1.5, 3.0))
        radius = 1.5
        case = scene.bend_case(root / f"bend{i}", spacing_nm=spacing_nm,
                               interior_um=(lx, ly, 2.4), pml=10, steps=steps,
                               radius_um=radius, nwav=1)
        x_turn = lx - 1.5 - radius
        cx, cy = x_turn + radius * 0.7071, 1.5 + radius * (1 - 0.7071)  # arc midpoint
        n = max(8, int(round(side / dx)))
        x0 = 10 + int(round(cx / dx)) - n // 2
        y0 = 10 + int(round(cy / dx)) - n // 2
        nz = 96 + 20
        sz = max(1, int(round(0.22 / dx)))
        box = (max(10, x0), max(10, y0), nz // 2 - sz // 2, n, n, sz)
        out.append((case, box))
    return out


def main(argv=None):
    """Forward + adjoint of seeded uneven bend instances, one after another and
    batched (BatchAdjoint):
    python -m warp_fdtd_b200.batch [--instances 8] [--steps 600] [--seed 1]"""
    import argparse
    import json
    import tempfile
    import time
    from pathlib import Path

    from .adjoint_driver import Adjoint
    from .detectors import attach

    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--instances", type=int, default=8)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--checkpoint-every", type=int, default=256)
    a = ap.parse_args(argv)
    with tempfile.TemporaryDirectory(prefix="wfb_batch_") as tmp:
        specs = _uneven_bends(Path(tmp), a.instances, a.seed, a.steps)
        adjs = []
        for case, box in specs:
            adj = Adjoint(case, box=box, checkpoint_every=a.checkpoint_every,
                          material_kwargs=dict(beta=8.0, eps_lo=2.085, contrast=10.025))
            attach(adj)
            adjs.append(adj)
        rng = np.random.default_rng(a.seed)
        params = [rng.uniform(0, 1, (adj.box[3], adj.box[4])).astype(np.float32)
                  for adj in adjs]
        for adj, p in zip(adjs, params):  # graphs and warm-up
            adj.differentiate(p)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        single = [adj.differentiate(p) for adj, p in zip(adjs, params)]
        torch.cuda.synchronize()
        t_single = time.perf_counter() - t0
        batch = BatchAdjoint(adjs)
        batch.differentiate(params)
        t0 = time.perf_counter()
        batched = batch.differentiate(params)
        torch.cuda.synchronize()
        t_batch = time.perf_counter() - t0
        cells = sum(int(np.prod(adj.shape)) * adj.steps for adj in adjs)
        rel = max(float(np.linalg.norm(g1 - g0) / max(float(np.linalg.norm(g0)), 1e-300))
                  for (_, g0), (_, g1) in zip(single, batched))
        print(json.dumps(dict(
            instances=a.instances, steps=a.steps, grids=[list(adj.shape) for adj in adjs],
            boxes=[list(adj.box) for adj in adjs], cell_updates=cells,
            one_after_another_s=t_single, batched_s=t_batch, speedup=t_single / t_batch,
            losses_equal=all(l0 == l1 for (l0, _), (l1, _) in zip(single, batched)),
            transmissions=[-l for l, _ in single], gradient_max_rel_l2=rel)))


if __name__ == "__main__":
    main()
