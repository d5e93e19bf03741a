"""Adjoint timing and validation, the B200 counterpart of the reference's
warp_fdtd/gradient_benchmark.py.

Default (`--case` a gradient bundle such as tests/golden/gradient20, the
reference's 20 nm bend with its 80 x 80 x 20 design box): the checks of
gradient_benchmark.py:16-165 --
* material parity: Material(p0, beta) against the bundle's inv_permittivity
  in the design box (gradient_benchmark.py:26-31);
* timed repetitions of forward (with checkpoints) and reverse sweep
  (:37-56);
* the gradient against the committed Warp and FDTDX gradients, relative L2
  and cosine (:58-68; the files sit next to the bundle);
* central differences along the normalised gradient at h = 0.03, 0.01,
  0.003 (:111-133);
* a changed-design replay that checks the adjoint source buffers keep their
  addresses (captured graphs stay valid) and its own difference check
  (:140-162).

`--config3`: the gradient on the 20 nm 90-degree bend of the forward
benchmark (324 x 324 x 144 cells, 4000 steps).  The 125 x 125 x 11 design box
sits over the arc.  Densities are seeded uniform in [0, 1]; the material map
is a 19 x 19 Gaussian filter (sigma 3 cells = 60 nm), tanh projection
beta = 8, and eps linear from 2.085 to 12.11.  Checkpoints every 256 steps
(`--checkpoint-every`; at or above the step count the forward records the
whole design-box history and the reverse sweep recomputes nothing); the
gradient is checked against central differences (h = 1e-3) on 16 seeded
pixels from the upper quartile of |gradient|.

    python -m warp_fdtd_b200.gradient_benchmark [--case DIR] [--reps 2] [--out result.json]
    python -m warp_fdtd_b200.gradient_benchmark --config3 [--out result.json]
"""

import argparse
import json
import tempfile
import time
from pathlib import Path

import numpy as np
import torch

from .adjoint_driver import Adjoint
from .detectors import attach, measurements
from .material import Material


def _rel(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _cos(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))


def _transmission(adj, p):
    adj.set_design(p)
    adj.reset()
    adj.run()
    return float(measurements(adj)["modal_transmission"])


def _timed(adj, reps):
    """(total, forward, backward) seconds of `reps` evaluations after one
    untimed one; the gradient transfer and the material pullback included."""
    out = []
    for rep in range(reps + 1):
        adj.reset()
        adj.reset_reverse()
        torch.cuda.synchronize(adj.device)
        t0 = time.perf_counter()
        adj.run()
        t1 = time.perf_counter()
        adj.prepare_sources()
        adj.backward()
        voxel = adj.voxel_gradient()
        adj.design_material.pullback(voxel.astype(np.float32))
        t2 = time.perf_counter()
        if rep:
            out.append((t2 - t0, t1 - t0, t2 - t1))
    return out


def _tune(adj):
    """Time the fused step's launch shapes on this grid (before any graph is
    captured) and keep the fastest; returns {shape: ms}."""
    try:
        timings = adj.autotune(tiles=[2, 3, 4, 5, 6, 8, 10, 12, 14, 16])
    except ValueError as exc:  # not the full-z path: keep the defaults
        return {"skipped": str(exc)}
    return {f"tile {k[0]}, stages {k[1]}, weights {k[2]}": v for k, v in timings.items()}


def reference_case(case, reps=2, checkpoint_every=256, tune=False):
    case = Path(case)
    adj = Adjoint(case, checkpoint_every=checkpoint_every)
    attach(adj)
    tuned = _tune(adj) if tune else None
    p0 = np.asarray(adj.data["parameters/p0"])[..., 0]
    x0, y0, z0, sx, sy, sz = adj.box
    beta = adj.meta.get("beta", 50.0)
    material = Material(p0, beta, device=adj.device)
    projected = material.inv_eps.cpu().numpy()
    reference = np.asarray(adj.data["inv_permittivity"])[0, x0:x0 + sx, y0:y0 + sy, z0]
    res = dict(case=str(case), shape=list(adj.shape), time_steps=adj.steps,
               box=list(adj.box), material_max_absolute_error=float(
                   np.max(np.abs(projected - reference))),
               launch_shape=dict(tile_y=adj.tile[0], stages=adj.stages, autotune=tuned))
    loss, grad = adj.differentiate(p0)  # builds the graphs
    times = _timed(adj, reps)
    res.update(seconds=[t[0] for t in times], forward_seconds=[t[1] for t in times],
               backward_seconds=[t[2] for t in times],
               median_seconds=float(np.median([t[0] for t in times])),
               measurements=measurements(adj), history_bytes=int(adj.history.numel() * 4),
               checkpoint_every=adj.checkpoint_every)
    grad = np.asarray(grad, np.float64)
    for name, key in (("warp_gradient.npz", "gradient"), ("fdtdx_gradient.npz", "g0")):
        f = case / name
        if f.exists():
            ref = np.load(f)[key]
            ref = ref[..., 0] if ref.ndim == 3 else ref
            res[name.split("_")[0]] = dict(relative_l2=_rel(grad, ref), cosine=_cos(grad, ref))
    # central differences along the normalised gradient (loss = -T)
    direction = grad / np.linalg.norm(grad)
    analytic = float(np.sum(grad * direction))
    fd = []
    for h in (0.03, 0.01, 0.003):
        vals = [-_transmission(adj, p0 + sign * h * direction) for sign in (1, -1)]
        finite = (vals[0] - vals[1]) / (2 * h)
        fd.append(dict(step=h, analytic=analytic, finite_difference=finite,
                       relative_error=abs(finite - analytic) / abs(analytic)))
    res["finite_difference"] = fd
    # changed design: same graphs, source buffers updated in place
    changed = np.clip(p0 - 0.2 * direction, 0, 1)
    ptrs = [v.data_ptr() for _, v in adj.adjoint_sources]
    closs, cgrad = adj.differentiate(changed)
    preserved = [v.data_ptr() for _, v in adj.adjoint_sources] == ptrs
    cgrad = np.asarray(cgrad, np.float64)
    cdir = cgrad / np.linalg.norm(cgrad)
    canalytic = float(np.sum(cgrad * cdir))
    cvals = [-_transmission(adj, changed + sign * 0.01 * cdir) for sign in (1, -1)]
    cfd = (cvals[0] - cvals[1]) / 0.02
    res["changed_design"] = dict(loss=closs, analytic=canalytic, finite_difference=cfd,
                                 relative_error=abs(cfd - canalytic) / abs(canalytic),
                                 source_buffer_pointers_preserved=preserved)
    res["passed"] = bool(
        np.isfinite(grad).all() and res.get("warp", {}).get("relative_l2", 0) < 0.01
        and res.get("fdtdx", {}).get("cosine", 1) > 0.999
        and min(r["relative_error"] for r in fd) < 0.01 and preserved
        and res["changed_design"]["relative_error"] < 0.01)
    return res


def config3(reps=1, workdir=None, pixels=16, h=1e-3, checkpoint_every=256, tune=False):
    from . import scene

    if workdir is None:
        with tempfile.TemporaryDirectory(prefix="wfb_config3_") as tmp:
            return config3(reps, tmp, pixels, h, checkpoint_every, tune)
    workdir = Path(workdir)
    case = scene.bend_case(workdir / "bend20", steps=4000)
    box = (145, 54, 67, 125, 125, 11)
    material_kwargs = dict(beta=8.0, eps_lo=2.085, contrast=12.11 - 2.085, radius=9, sigma=3.0)
    adj = Adjoint(case, box=box, checkpoint_every=checkpoint_every,
                  material_kwargs=material_kwargs)
    attach(adj)
    tuned = _tune(adj) if tune else None
    p = np.random.default_rng(0).uniform(0, 1, (125, 125)).astype(np.float32)
    loss, grad = adj.differentiate(p)
    times = _timed(adj, reps)
    res = dict(case="bend 20 nm, 324 x 324 x 144, 4000 steps", box=list(box),
               material=material_kwargs, design_seed=0, loss=loss,
               seconds=[t[0] for t in times], forward_seconds=[t[1] for t in times],
               backward_seconds=[t[2] for t in times],
               cell_updates=int(np.prod(adj.shape)) * adj.steps,
               history_bytes=int(adj.history.numel() * 4),
               checkpoint_every=adj.checkpoint_every,
               launch_shape=dict(tile_y=adj.tile[0], stages=adj.stages, autotune=tuned))
    g = np.asarray(grad, np.float64).ravel()
    rng = np.random.default_rng(16)
    top = np.flatnonzero(np.abs(g) >= np.quantile(np.abs(g), 0.75))
    chosen = rng.choice(top, pixels, replace=False)
    fd = []
    for j in chosen:
        pp, pm = p.ravel().copy(), p.ravel().copy()
        pp[j] += h
        pm[j] -= h
        fd.append(-(_transmission(adj, pp.reshape(p.shape)) -
                    _transmission(adj, pm.reshape(p.shape))) / (2 * h))
    fd = np.array(fd)
    err = np.abs(fd - g[chosen]) / np.abs(g[chosen])
    res.update(fd_pixels=[int(j) for j in chosen], fd=fd.tolist(),
               adjoint=g[chosen].tolist(), fd_relative_l2=_rel(fd, g[chosen]),
               fd_median_relative_error=float(np.median(err)))
    res["passed"] = bool(res["fd_relative_l2"] < 0.02)
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--case", default=str(Path(__file__).resolve().parent.parent / "tests" /
                                          "golden" / "gradient20"))
    ap.add_argument("--reps", type=int, default=2)
    ap.add_argument("--config3", action="store_true")
    ap.add_argument("--checkpoint-every", type=int, default=256,
                    help="steps per checkpoint segment; >= the step count keeps the whole "
                         "design-box history and skips the recomputation")
    ap.add_argument("--autotune", action="store_true",
                    help="time the fused step's launch shapes on the grid first")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    if a.reps < 1:
        ap.error("--reps must be positive")
    res = (config3(reps=a.reps, checkpoint_every=a.checkpoint_every, tune=a.autotune)
           if a.config3 else reference_case(a.case, a.reps, a.checkpoint_every, a.autotune))
    text = json.dumps(res, indent=2)
    if a.out:
        Path(a.out).write_text(text + "\n")
    print(text, flush=True)
    if not res["passed"]:
        raise SystemExit("gradient check failed")


if __name__ == "__main__":
    main()
