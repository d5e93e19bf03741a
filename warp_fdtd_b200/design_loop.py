"""Surrogate-proposed inverse design against the plain adjoint loop.

The design problem is the adjoint driver's (adjoint_driver.Adjoint, the
reference's warp_fdtd/adjoint.py:231-469): maximise the fundamental-mode
transmission T(p) at the source wavelength over the density p in [0, 1] of
the design box, p -> material map -> FDTD -> modal overlap.  The modal
monitors also record T at `nwav` more wavelengths across a band, which the
surrogate learns as its first output.

Both loops take the same normalised ascent step from the same seeded start,
p <- clip(p + step * d / max|d|, 0, 1):

* plain adjoint loop: d = dT/dp from Adjoint.differentiate (one forward and
  one checkpointed reverse sweep per iteration); T of each iterate comes from
  the same call.
* surrogate-extrapolated loop (extrapolate_loop): each iteration is the
  adjoint step from p followed by k steps along the CNN's predicted gradient
  map; a full FDTD forward accepts the extrapolated design only if its T
  beats T(p), otherwise the loop keeps the plain adjoint step.
* surrogate-proposed loop (surrogate_loop): d = the CNN's predicted gradient map at p.  The
  proposal q is judged by a full FDTD forward and accepted only if T(q) > T(p).
  On rejection the loop falls back to the exact method: differentiate at p,
  take the adjoint step, measure T of the result with a full forward, and
  fine-tune the surrogate on the new (p, spectrum, gradient) triple.

Every accepted design has an FDTD-measured T; the time to reach T >= target is
measured on the host clock around the whole loop (solver, adjoint, surrogate
inference and fine-tuning, host transfers), after a warm-up that builds the
solver's CUDA graphs.

    python -m warp_fdtd_b200.design_loop --case <bundle> --out result.json
"""

import argparse
import json
import time

import numpy as np
import torch

from .adjoint_driver import Adjoint
from .detectors import attach, measurements
from .surrogate import Surrogate

C0 = 299792458.0


class DesignProblem:
    """An Adjoint solver on `case` with modal monitors at the source frequency
    (index 0, the objective) and at `nwav` wavelengths across `band`."""

    def __init__(self, case, box=None, nwav=8, band=(1.50e-6, 1.60e-6), checkpoint_every=256,
                 device="cuda:0", material_kwargs=None):
        self.adj = Adjoint(case, box=box, checkpoint_every=checkpoint_every, device=device,
                           material_kwargs=material_kwargs)
        src = next(o for o in self.adj.meta["objects"] if o["class"] == "ModePlaneSource")
        self.wavelengths = np.linspace(band[0], band[1], nwav)
        freqs = [float(src["frequency_hz"])] + [C0 / w for w in self.wavelengths]
        for obj in self.adj.meta["objects"]:
            if obj["class"] == "ModeOverlapDetector":
                profiles = self.adj.data[obj["name"] + "/_mode_E"].shape[0]
                if profiles != 1:
                    raise ValueError("DesignProblem needs bundles with one mode profile per "
                                     "modal detector (used at every wavelength)")
                obj["frequencies_hz"] = freqs
        attach(self.adj)
        x0, y0, z0, sx, sy, sz = self.adj.box
        self.shape = (sx, sy)
        self.nwav = nwav
        self.forwards = 0
        self.adjoints = 0

    def _measure(self):
        m = measurements(self.adj)
        spectrum = np.asarray(m["modal_transmission_spectrum"][1:], np.float64)
        return float(m["modal_transmission"]), spectrum

    def transmission(self, p):
        """Full FDTD forward: (T, T spectrum)."""
        a = self.adj
        a.set_design(p)
        if not a.graphs:
            a.compile()
        a.reset()
        a.run()
        self.forwards += 1
        return self._measure()

    def differentiate(self, p):
        """(T, T spectrum, dT/dp) through the exact checkpointed adjoint."""
        loss, grad = self.adj.differentiate(p)
        self.adjoints += 1
        T, spectrum = self._measure()
        return T, spectrum, -np.asarray(grad, np.float32)


def ascent(p, d, step):
    scale = float(np.max(np.abs(d)))
    if not np.isfinite(scale) or scale == 0:
        return p.copy()
    return np.clip(p + step * d / scale, 0.0, 1.0).astype(np.float32)


def adjoint_loop(problem, p0, target=0.9, iters=100, step=0.1, record=None):
    """The plain adjoint loop; returns (p, history).  record(p, spectrum, g)
    receives every triple (data generation uses it)."""
    p = np.asarray(p0, np.float32).copy()
    hist = []
    t0 = time.perf_counter()
    for it in range(iters):
        T, spectrum, g = problem.differentiate(p)
        hist.append(dict(it=it, T=T, t=time.perf_counter() - t0, kind="adjoint"))
        if record is not None:
            record(p, spectrum, g)
        if T >= target:
            break
        p = ascent(p, g, step)
    return p, hist


class Dataset:
    """(density, spectrum, gradient) triples kept on the host; tensors()
    uploads them with the gradients divided by g_scale, the RMS gradient of
    the data present at the first call (or the value given), kept fixed so
    later additions are scaled alike."""

    def __init__(self, shape, nwav, device="cuda:0", g_scale=None):
        self.shape, self.nwav, self.device = shape, nwav, torch.device(device)
        self.p, self.T, self.g = [], [], []
        self.g_scale = g_scale

    def add(self, p, spectrum, g):
        self.p.append(np.asarray(p, np.float32).copy())
        self.T.append(np.asarray(spectrum, np.float32).copy())
        self.g.append(np.asarray(g, np.float32).copy())

    def __len__(self):
        return len(self.p)

    def tensors(self, last=None):
        sl = slice(-last, None) if last else slice(None)
        if self.g_scale is None:
            self.g_scale = float(np.sqrt(np.mean(np.square(np.stack(self.g)))))
        P = torch.from_numpy(np.stack(self.p[sl])).to(self.device)
        T = torch.from_numpy(np.stack(self.T[sl])).to(self.device)
        G = torch.from_numpy(np.stack(self.g[sl]) / self.g_scale).to(self.device)
        return P, T, G

    def save(self, path, n_train=None):
        np.savez_compressed(path, p=np.stack(self.p), T=np.stack(self.T), g=np.stack(self.g),
                            n_train=np.int64(len(self) if n_train is None else n_train))

    @classmethod
    def load(cls, path, device="cuda:0"):
        """(data set, number of training triples) from save()."""
        f = np.load(path)
        d = cls(f["p"].shape[1:], f["T"].shape[1], device)
        for p, T, g in zip(f["p"], f["T"], f["g"]):
            d.add(p, T, g)
        return d, int(f["n_train"])


def generate(problem, seeds, steps, step=0.1, data=None):
    """Triples from short plain-adjoint trajectories started at the seeded
    uniform densities `seeds` (never the evaluation seed)."""
    data = data or Dataset(problem.shape, problem.nwav, problem.adj.device)
    for s in seeds:
        p0 = np.random.default_rng(s).uniform(0, 1, problem.shape).astype(np.float32)
        adjoint_loop(problem, p0, target=2.0, iters=steps, step=step, record=data.add)
    return data


def surrogate_loop(problem, net, p0, data, target=0.9, iters=100, step=0.1, finetune_steps=30,
                   lr=3e-4, window=64):
    """The surrogate-proposed loop; returns (p, history)."""
    p = np.asarray(p0, np.float32).copy()
    hist = []
    t0 = time.perf_counter()
    T, _ = problem.transmission(p)
    hist.append(dict(it=0, T=T, t=time.perf_counter() - t0, kind="start"))
    for it in range(1, iters):
        if T >= target:
            break
        _, ghat = net.predict(torch.from_numpy(p).to(net.device))
        q = ascent(p, ghat.cpu().numpy(), step)
        Tq, _ = problem.transmission(q)
        if Tq > T:
            p, T, kind = q, Tq, "surrogate"
        else:
            _, spectrum, g = problem.differentiate(p)
            data.add(p, spectrum, g)
            finetune(net, data, finetune_steps, lr, window, seed=it)
            p = ascent(p, g, step)
            T, _ = problem.transmission(p)
            kind = "adjoint"
        hist.append(dict(it=it, T=T, t=time.perf_counter() - t0, kind=kind))
    return p, hist


def extrapolate_loop(problem, net, p0, data, target=0.9, iters=100, step=0.1, k=1,
                     finetune_steps=15, lr=3e-4, window=64):
    """Surrogate-extrapolated adjoint loop; returns (p, history).

    Each iteration differentiates at the current design p (exact T and dT/dp;
    the triple fine-tunes the surrogate) and takes the adjoint step to p1; the
    surrogate then extrapolates k more steps along its predicted gradient, and
    a full FDTD forward judges the result q: accepted when T(q) > T(p), else
    the loop continues from p1 exactly as the plain adjoint loop would."""
    p = np.asarray(p0, np.float32).copy()
    hist = []
    t0 = time.perf_counter()
    for it in range(iters):
        T, spectrum, g = problem.differentiate(p)
        hist.append(dict(it=it, T=T, t=time.perf_counter() - t0, kind="adjoint"))
        if T >= target:
            break
        data.add(p, spectrum, g)
        finetune(net, data, finetune_steps, lr, window, seed=it)
        p1 = ascent(p, g, step)
        q = p1
        for _ in range(k):
            _, ghat = net.predict(torch.from_numpy(q).to(net.device))
            q = ascent(q, ghat.cpu().numpy(), step)
        Tq, _ = problem.transmission(q)
        accepted = Tq > T
        hist.append(dict(it=it, T=Tq, t=time.perf_counter() - t0,
                         kind="surrogate" if accepted else "rejected"))
        if accepted and Tq >= target:
            break
        p = q if accepted else p1
    return p, hist


def finetune(net, data, steps, lr, window, newest=8, batch=32, seed=0):
    """Adam steps on minibatches that always hold the newest triple (`newest`
    copies) next to random triples of the last `window`: the surrogate follows
    the exact gradients of the current trajectory."""
    P, T, G = data.tensors(last=window)
    n = P.shape[0]
    gen = torch.Generator(device="cpu").manual_seed(seed)
    for _ in range(steps):
        rest = torch.randint(0, n, (max(batch - newest, 1),), generator=gen)
        idx = torch.cat([torch.full((newest,), n - 1, dtype=torch.long), rest]).to(net.device)
        net.train_step(P[idx], T[idx], G[idx], lr)


def time_to(hist, target):
    """Time of the first verified design with T >= target (rejected proposals
    are not designs the loop holds)."""
    for h in hist:
        if h["T"] >= target and h["kind"] != "rejected":
            return h["t"]
    return None


def cosine(a, b):
    a, b = np.ravel(a).astype(np.float64), np.ravel(b).astype(np.float64)
    return float(a @ b / max(np.linalg.norm(a) * np.linalg.norm(b), 1e-300))


def held_out_cosine(net, data, idx):
    out = []
    for i in idx:
        _, ghat = net.predict(torch.from_numpy(data.p[i]).to(net.device))
        out.append(cosine(ghat.cpu().numpy(), data.g[i]))
    return float(np.mean(out))


def run(case, box=None, target=0.9, iters=100, steps=(0.1,), starts=(0,),
        train_seeds=range(1, 9), traj_steps=16, held_out_seeds=(100,), held_out_steps=8,
        train_steps=1500, batch=32, lr=1e-3, finetune_steps=30, data_step=0.1, device="cuda:0",
        log=print, data_path=None, save_data=None,
        loops=("adjoint", "extrapolate", "propose")):
    """Data generation (or a saved data set), training, then every loop at
    every step size from every seeded start (uniform densities of seed s).
    Each surrogate loop starts from the same trained network and data set."""
    problem = DesignProblem(case, box=box, device=device)
    shape = problem.shape
    # warm-up: CUDA graphs of the forward and reverse sweeps
    problem.differentiate(np.full(shape, 0.5, np.float32))
    torch.cuda.synchronize()
    res = dict(case=str(case), shape=list(problem.adj.shape), time_steps=problem.adj.steps,
               design=list(shape), target=target, iters=iters, runs={})

    t0 = time.perf_counter()
    if data_path:
        data, n_train = Dataset.load(data_path, device)
        res["data_from"] = str(data_path)
    else:
        data = generate(problem, list(train_seeds), traj_steps, data_step)
        n_train = len(data)
        generate(problem, list(held_out_seeds), held_out_steps, data_step, data)
        if save_data:
            data.save(save_data, n_train)
    res["data_seconds"] = time.perf_counter() - t0
    res["train_triples"], res["held_out_triples"] = n_train, len(data) - n_train
    log(f"data: {len(data)} triples in {res['data_seconds']:.1f} s")

    net = Surrogate(shape, problem.nwav, device=device, seed=0)
    held = list(range(n_train, len(data)))
    res["held_out_cosine_untrained"] = held_out_cosine(net, data, held)
    P, T, G = data.tensors()
    t0 = time.perf_counter()
    losses = net.fit(P[:n_train], T[:n_train], G[:n_train], steps=train_steps, batch=batch, lr=lr,
                     log_every=max(train_steps // 10, 1))
    torch.cuda.synchronize()
    res["train_seconds"] = time.perf_counter() - t0
    res["train_loss"] = losses
    res["held_out_cosine_trained"] = held_out_cosine(net, data, held)
    Tp, _ = net.predict(P[n_train:])
    res["held_out_spectrum_rmse"] = float(torch.sqrt(torch.mean((Tp - T[n_train:]) ** 2)))
    log(f"trained in {res['train_seconds']:.1f} s; held-out gradient cosine "
        f"{res['held_out_cosine_untrained']:.3f} -> {res['held_out_cosine_trained']:.3f}")

    trained = net.params_numpy()
    for start in starts:
        p_start = np.random.default_rng(start).uniform(0, 1, shape).astype(np.float32)
        for step in steps:
            for name in loops:
                problem.forwards = problem.adjoints = 0
                if name == "adjoint":
                    _, h = adjoint_loop(problem, p_start, target, iters, step)
                else:
                    run_net = Surrogate(shape, problem.nwav, device=device, params=trained)
                    run_data = Dataset(shape, problem.nwav, device, data.g_scale)
                    for i in range(n_train):
                        run_data.add(data.p[i], data.T[i], data.g[i])
                    if name == "extrapolate":
                        _, h = extrapolate_loop(problem, run_net, p_start, run_data, target,
                                                iters, step, k=1)
                    elif name == "propose":
                        _, h = surrogate_loop(problem, run_net, p_start, run_data, target, iters,
                                              step, finetune_steps)
                    else:
                        raise ValueError(f"unknown loop {name!r}")
                key = f"{name}_step{step}_start{start}"
                res["runs"][key] = dict(
                    loop=name, step=step, start=start, history=h,
                    time_to_target=time_to(h, target),
                    best=max(x["T"] for x in h if x["kind"] != "rejected"),
                    forwards=problem.forwards, adjoints=problem.adjoints,
                    accepted=sum(x["kind"] == "surrogate" for x in h))
                r = res["runs"][key]
                log(f"{key}: time to {target} {r['time_to_target']}, best T {r['best']:.4f}, "
                    f"{r['adjoints']} adjoint + {r['forwards']} forward runs, "
                    f"{r['accepted']} surrogate steps kept")
    return res


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--case", required=True)
    ap.add_argument("--box", type=int, nargs=6, default=None)
    ap.add_argument("--target", type=float, default=0.9)
    ap.add_argument("--iters", type=int, default=100)
    ap.add_argument("--steps", type=float, nargs="+", default=[0.1],
                    help="ascent step sizes (max-norm) to run every loop at")
    ap.add_argument("--starts", type=int, nargs="+", default=[0],
                    help="seeds of the uniform-density starting designs")
    ap.add_argument("--train-seeds", type=int, default=8)
    ap.add_argument("--traj-steps", type=int, default=16)
    ap.add_argument("--held-out-steps", type=int, default=8)
    ap.add_argument("--train-steps", type=int, default=1500)
    ap.add_argument("--out", default=None)
    ap.add_argument("--data", default=None, help="saved data set (Dataset.save) to train on")
    ap.add_argument("--save-data", default=None)
    ap.add_argument("--loops", nargs="+", default=["adjoint", "extrapolate", "propose"],
                    choices=["adjoint", "extrapolate", "propose"])
    a = ap.parse_args(argv)
    res = run(a.case, a.box, a.target, a.iters, tuple(a.steps), tuple(a.starts),
              range(1, 1 + a.train_seeds), a.traj_steps, held_out_steps=a.held_out_steps,
              train_steps=a.train_steps, data_path=a.data, save_data=a.save_data,
              loops=a.loops)
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f)
    print(json.dumps({k: v for k, v in res.items() if k not in ("runs", "train_loss")}))
    print(json.dumps({k: {kk: vv for kk, vv in r.items() if kk != "history"}
                      for k, r in res["runs"].items()}))


if __name__ == "__main__":
    main()
