"""Benchmark: the 20 nm silicon bend forward (324 x 324 x 144 cells, 4000 steps).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One bench step is one complete forward trajectory of the bend workload
(reset + 4000 Yee steps, two per launch of the time-blocked kernel, + the
5-wavelength modal detectors at the input and output planes), i.e.
6.05e10 cell-updates.  The metric is Gcell-updates/s over the whole job.
Under torchrun (N > 1) every rank runs its own independent replica of the
workload on its GPU (the path does not shard; there is no collective in the
data path) and `value` is the sum over ranks of cell-updates divided by the
maximum over ranks of the device time.

Printed on rank 0: one JSON line with the contract's keys plus `roofline`
(the time-blocked step kernel against the measured HBM copy bandwidth, 49
algorithmic bytes per cell-update, two cell-updates per launch, and its DRAM
traffic measured by ncu on this grid), `cpu_baseline` (the CPU oracle on this host's cores on
a bounded sample of the same grid), `e2e` (the same metric through the public
Solver API with the material grid uploaded from pinned host memory and the
detector phasors read back every step), `clocks` and `gpu_launches`.

`--impl reference` times the reference's CPU path on this host: warp-lang
(the reference's runtime) is not installable here, so the arm runs the CPU
restatement of the reference kernels (oracle/, C + OpenMP, all host threads)
on a bounded sample of the same workload per step.
"""

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOADS = {
    # name: (interior_um, time_steps)
    "bend20": ((6.0, 6.0, 2.4), 4000),
    # profiling case of the same kernel: 174 x 174 x 144 cells (fields 4 x 70 MB > L2)
    "bend20-small": ((3.0, 3.0, 2.4), 200),
}
WORKLOAD = "bend20nm_324x324x144_4000steps_5lambda"
METRIC = "Gcell-updates/s (20 nm bend forward)"
BYTES_PER_CELL = 49  # read E, H (24 B) + write E, H (24 B) + 1 B material index


def workload_config(workload, shape, time_steps, world):
    """The `config` object of both arms' JSON lines."""
    cells = int(np.prod(shape))
    return {"workload": WORKLOAD if workload == "bend20" and time_steps == 4000
            else f"{workload}_{list(shape)}_{time_steps}steps",
            "grid": list(shape), "time_steps": int(time_steps), "cells": cells,
            "materials": "uint8 index (SiO2 2.085, Si 12.11)",
            "detectors": "mode_in (read forward and backward), mode_out x 5 "
                         "wavelengths (float64 DFT)",
            "pulse": "Hann, 200 fs, 1.55 um",
            "l2": f"inputs larger than L2 (fields 4 x {cells * 12 / 1e6:.0f} MB ping-pong)",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU"}


def workload_shape(workload, time_steps=None):
    """Grid and step count of a bench workload (20 nm cells, 12-cell CPML)."""
    interior, steps = WORKLOADS[workload]
    return tuple(int(round(v * 1e-6 / 20e-9)) + 24 for v in interior), time_steps or steps


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def bundle_dir(workload="bend20", time_steps=None):
    base = Path(os.environ.get("FDTD_BENCH_CACHE", tempfile.gettempdir())) / "warp_fdtd_b200_bench"
    interior, steps = WORKLOADS[workload]
    return base / f"{workload}_{time_steps or steps}"


def make_bundle(workload="bend20", time_steps=None):
    from warp_fdtd_b200 import scene

    interior, steps = WORKLOADS[workload]
    d = bundle_dir(workload, time_steps)
    if not (d / "manifest.json").exists():
        d.parent.mkdir(parents=True, exist_ok=True)
        tmp = d.with_name(d.name + f".tmp{os.getpid()}")
        scene.bend_case(tmp, interior_um=interior, steps=time_steps or steps)
        try:
            os.replace(tmp, d)
        except OSError:
            pass  # another rank won the race
    return d


class ClockSampler:
    """nvidia-smi clock / throttle sampling while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(backend="nccl"):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE): each
    rank binds its own GPU; with world > 1 a process group of `backend`
    (nccl on GPUs, gloo for the host-only tests) carries the timing
    reductions, never field data (replicas)."""
    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist

        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
    elif backend == "nccl":
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _reduce(value, world, op):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def reduce_max(value, world):
    """Max over ranks (the job's time is its slowest rank's)."""
    import torch.distributed as dist

    return _reduce(value, world, dist.ReduceOp.MAX) if world > 1 else value


def reduce_sum(value, world):
    """Sum over ranks (the job's cell-updates)."""
    import torch.distributed as dist

    return _reduce(value, world, dist.ReduceOp.SUM) if world > 1 else value


def cpu_sample(case, time_steps, warmup_steps=0):
    """The CPU oracle's fused update on the full grid: `warmup_steps` untimed
    steps (first touch of the field pages), then `time_steps` timed ones, in
    this process; returns (Gcell-updates/s, threads, seconds)."""
    from oracle import cpu as ocpu
    from oracle.model import OracleSolver

    o = OracleSolver(case)
    L = ocpu.lib()
    nx, ny, nz = o.shape

    def run(step0, count):
        L.oracle_run_steps(o.E, o.H, o.eps, o.psi_e, o.psi_h, o.coeffs["E"], o.coeffs["H"],
                           o.coeffs["E"].shape[1], o.sources["E"], o.sources["H"], o.waves["E"],
                           o.waves["H"], o.steps, step0, count, nx, ny, nz, int(o.source_x),
                           float(o.courant))

    run(0, warmup_steps)
    start = time.perf_counter()
    run(warmup_steps, time_steps)
    sec = time.perf_counter() - start
    return o.n * time_steps / sec / 1e9, ocpu.num_threads(), sec


def cpu_sample_fresh(case, time_steps, warmup_steps=2):
    """cpu_sample in a fresh Python process (no torch, no CUDA context, no
    other thread pool in it): both bench arms time the CPU path this way, so
    their figures agree."""
    code = ("import json, sys; sys.path.insert(0, sys.argv[1]); import bench; "
            "print(json.dumps(bench.cpu_sample(sys.argv[2], int(sys.argv[3]), int(sys.argv[4]))))")
    out = subprocess.run([sys.executable, "-c", code, str(ROOT), str(case), str(time_steps),
                          str(warmup_steps)], check=True, capture_output=True, text=True)
    rate, cores, sec = json.loads(out.stdout.strip().splitlines()[-1])
    return rate, cores, sec


def run_reference(args, world, rank):
    """Reference arm: the CPU restatement of the reference kernels (oracle)."""
    if rank != 0:
        return
    case = make_bundle(args.workload, args.time_steps)
    sample_steps = args.cpu_steps
    for _ in range(args.warmup):
        cpu_sample_fresh(case, min(sample_steps, 10))
    rates, secs, cores = [], [], 1
    for _ in range(args.steps):
        r, cores, s = cpu_sample_fresh(case, sample_steps)
        rates.append(r)
        secs.append(s)
    value = statistics.median(rates)
    sample = (f"{sample_steps} of 4000 time steps on the full 324x324x144 grid per step "
              f"({statistics.median(secs):.1f} s), E+H updates with CPML and source "
              "(oracle/fdtd_oracle.c, OpenMP), each in a fresh process after 2 untimed steps")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Gcell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * statistics.median(secs), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args.workload, *workload_shape(args.workload, args.time_steps),
                                  world),
        "cpu_baseline": {"value": value, "unit": "Gcell-updates/s", "cores": cores,
                         "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "warp-lang is not installed here; the reference's CPU path is timed as its "
                "C restatement",
    }
    print(json.dumps(line), flush=True)


def surrogate_train_rate(steps=20, warmup=3, device="cuda:0"):
    """The CNN surrogate's training step (32 designs of 80 x 80, the 20 nm
    bend's design box) timed with CUDA events, against the measured bf16 peak."""
    import torch

    from warp_fdtd_b200.surrogate import Surrogate, status, train_flops

    size, batch = (80, 80), 32
    net = Surrogate(size, 8, device=device)
    gen = torch.Generator(device="cpu").manual_seed(0)
    x = torch.rand((batch,) + size, generator=gen).to(device)
    T = torch.rand((batch, 8), generator=gen).to(device)
    g = torch.randn((batch,) + size, generator=gen).to(device)
    for _ in range(warmup):
        net.train_step(x, T, g)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        net.train_step(x, T, g)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    flops = train_flops(size, net.base, batch)
    peaks = ROOT / "MEASURED_PEAKS.json"
    peak = json.loads(peaks.read_text())["bf16_tflops"] if peaks.exists() else 1590.0
    tflops = flops / ms / 1e9
    return {"workload": f"CNN surrogate training step, {batch} designs of {size[0]}x{size[1]}, "
                        f"{net.count} parameters, bf16 tcgen05 GEMMs",
            "train_step_ms": ms, "designs_per_s": batch / ms * 1e3, "tflops": tflops,
            "peak_tflops": peak, "frac": tflops / peak, "wait_status": status()}


def run_ours(args, world, rank, local):
    import torch

    from warp_fdtd_b200 import _lib
    from warp_fdtd_b200.detectors import attach, measurements
    from warp_fdtd_b200.solver import Solver

    case = make_bundle(args.workload, args.time_steps)
    s = Solver(case, device=f"cuda:{local}", graph_steps=64)
    attach(s)
    s.compile()
    stream = torch.cuda.current_stream()
    cells = s.n * s.steps

    for _ in range(args.warmup):
        s.reset()
        s.run()
    barrier(world)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.reset()
        s.run()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    clock_info = clocks.stop()
    ms_local = e0.elapsed_time(e1)
    ms = reduce_max(ms_local, world)
    total_cells = reduce_sum(float(cells * args.steps), world)
    value = total_cells / (ms / 1e3) / 1e9
    meas = measurements(s)
    # per step: the fused step, the staged planes' shared recorder (or one
    # recorder per monitor), the counter; per trajectory: each staged
    # monitor's folds (every `batch` steps and at the end)
    planes, grouped = s._staged_planes()
    own = sum(1 for m in s.monitors if m.shared is None and id(m) not in grouped)
    recorders_per_step = own + 1  # the grouped recorder also advances the counter
    pairs, singles = s.step_launches()
    s.reset()
    merged = bool(pairs) and own == 0 and s._pair_staging()  # one staging launch per pair
    recorder_launches = recorders_per_step * (singles + (pairs if merged else 2 * pairs))
    folds = sum(-(-s.steps // m.batch) for m in s.monitors if m.is_phasor and m.shared is None)

    # dominant kernel alone: average duration of the step kernel the
    # trajectory runs (two time steps per launch at time_block 2) over 200
    # launches on the launching stream
    s.reset()
    kernel_name, updates = "fz_step_kernel (fdtd_step_fused, one step)", 1
    launch = lambda: _lib.call("fdtd_step_fused", s._args, stream.cuda_stream)
    if s.time_block == 2:
        info, extra = s._block[2], s._pair_extra()
        kernel_name, updates = "block_step_kernel (fdtd_step_block, two steps per launch)", 2
        launch = lambda: _lib.call("fdtd_step_block", ctypes.byref(info["args"][s._rel]),
                                   ctypes.byref(info["plan"]), ctypes.byref(extra),
                                   stream.cuda_stream)
    elif s.time_block == 1:
        kernel_name = "block_step_kernel (fdtd_step_block, one step per launch)"
        launch = lambda: s._step_kernel(stream.cuda_stream)
    for _ in range(5):
        launch()
    k0 = torch.cuda.Event(enable_timing=True)
    k1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    k0.record(stream)
    nk = 200
    for _ in range(nk):
        launch()
    k1.record(stream)
    torch.cuda.synchronize()
    kernel_ms = k0.elapsed_time(k1) / nk
    achieved = BYTES_PER_CELL * s.n * updates / (kernel_ms / 1e3) / 1e9
    peak, peak_kind = load_peaks()
    # DRAM bytes of one launch of this kernel on this grid, from an ncu
    # capture of the benchmark itself (null for any other kernel or grid)
    traffic = None
    tfile = ROOT / "profiles" / "block_step_bend20_traffic.json"
    if tfile.exists() and args.workload == "bend20" and s.time_block == 2:
        try:
            rec = json.loads(tfile.read_text())
            if rec.get("grid") == list(s.shape) and rec.get("cell_updates_per_launch") == 2:
                traffic = rec.get("bytes_per_launch")
        except (ValueError, OSError):
            traffic = None

    # end to end through the public API: material upload from pinned host memory,
    # full trajectory, phasor read-back and the host modal overlap, every step
    host_mat = torch.empty(s.material.numel(), dtype=torch.uint8, pin_memory=True)
    host_mat.copy_(s.material.cpu())
    phasor_bytes = sum(m.phasor.numel() * 8 for m in s.monitors if m.shared is None)
    e2e_steps = max(1, min(args.steps, 3))
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        s.material.copy_(host_mat, non_blocking=True)
        s.reset()
        s.run()
        meas = measurements(s)
    torch.cuda.synchronize()
    e2e_sec = reduce_max(time.perf_counter() - t0, world)
    e2e_value = reduce_sum(float(cells * e2e_steps), world) / e2e_sec / 1e9

    try:
        surrogate = surrogate_train_rate(device=f"cuda:{local}")
    except Exception as exc:  # the FDTD line is still reported
        surrogate = {"error": f"{type(exc).__name__}: {exc}"}

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        rate, cores, sec = cpu_sample_fresh(case, args.cpu_steps)
        cpu = {"value": rate, "unit": "Gcell-updates/s", "cores": cores, "kind": "port",
               "sample": f"{args.cpu_steps} of 4000 time steps on the full 324x324x144 grid "
                         f"({sec:.1f} s, after 2 untimed steps), CPU oracle E+H updates with "
                         "CPML and source, in a fresh process"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": workload_config(args.workload, s.shape, s.steps, world),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": kernel_name, "cell_updates_per_launch": updates,
                         "kernel_ms": kernel_ms, "bytes_per_cell": BYTES_PER_CELL,
                         "peak_kind": f"{peak_kind} (copy bandwidth)"},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "Gcell-updates/s",
                    "h2d_bytes_per_step": int(host_mat.numel()),
                    "d2h_bytes_per_step": int(phasor_bytes)},
            "gpu_launches": int((pairs + singles + recorder_launches + folds) * args.steps),
            "clocks": clock_info,
            "modal_transmission_1550nm": meas.get("modal_transmission_spectrum", [None] * 3)[2],
            "surrogate_train": surrogate,
        }
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--skip-cpu", action="store_true", help="omit the CPU baseline sample")
    ap.add_argument("--cpu-steps", type=int, default=20,
                    help="time steps of the CPU sample (both arms; 4000 = the whole trajectory)")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="bend20",
                    help="bend20 is the benchmark; bend20-small is for profiling captures")
    ap.add_argument("--time-steps", type=int, default=None,
                    help="override the trajectory length (profiling only)")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup()
    try:
        run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
