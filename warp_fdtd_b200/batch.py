"""Many independent solvers advanced together on one GPU.

`BatchSolver` takes solvers of uneven grids (designs, domains) and runs their
trajectories side by side: each instance's captured step graphs (Solver.compile)
replay on its own CUDA stream, forked from and joined back to the caller's
stream, and the host issues the replays round-robin, so instances too small
to fill the GPU alone share it.  Every instance keeps its own buffers,
detectors and schedule; results are those of running each solver alone, bit
for bit.  `autotune=True` tunes each instance's launch shape first
(Solver.autotune).
"""

import torch


class BatchSolver:
    def __init__(self, solvers, autotune=False):
        self.solvers = list(solvers)
        if not self.solvers:
            raise ValueError("BatchSolver needs at least one solver")
        devices = {s.device for s in self.solvers}
        if len(devices) != 1:
            raise ValueError("All solvers of a batch must share one device")
        self.device = devices.pop()
        if autotune:
            for s in self.solvers:
                s.autotune()
        self.streams = [torch.cuda.Stream(self.device) for _ in self.solvers]
        self.compiled = False

    def compile(self):
        """Capture every instance's step graphs; returns the seconds taken."""
        total = sum(s.compile() for s in self.solvers)
        self.compiled = True
        return total

    def reset(self):
        for s in self.solvers:
            s.reset()

    def run(self):
        """Advance every instance through its whole trajectory."""
        if not self.compiled:
            self.compile()
        if any(s._issued != 0 for s in self.solvers):
            raise ValueError("BatchSolver.run starts every instance from reset()")
        with torch.cuda.device(self.device):
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
            torch.cuda.synchronize(self.device)
