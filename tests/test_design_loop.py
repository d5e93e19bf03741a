"""Host logic of the design loops on CPU: a fake design problem with an
analytic transmission stands in for the FDTD solver and its adjoint, and a
fake network for the surrogate, so the acceptance rules, histories and data
handling are checked without a GPU."""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from warp_fdtd_b200 import design_loop as dl  # noqa: E402


class FakeProblem:
    """T(p) = 1 - mean((p - p*)^2) with its exact gradient; counts calls."""

    def __init__(self, shape=(8, 8), nwav=3, seed=0):
        self.shape, self.nwav = shape, nwav
        self.target = np.random.default_rng(seed).uniform(0.3, 0.7, shape).astype(np.float32)
        self.forwards = self.adjoints = 0

        class _Adj:
            device = torch.device("cpu")

        self.adj = _Adj()

    def _T(self, p):
        return float(1.0 - np.mean((p - self.target) ** 2))

    def transmission(self, p):
        self.forwards += 1
        T = self._T(p)
        return T, np.full(self.nwav, T)

    def differentiate(self, p):
        self.adjoints += 1
        T = self._T(p)
        return T, np.full(self.nwav, T), (-2.0 * (p - self.target) / p.size).astype(np.float32)


class FakeNet:
    """predict() returns a fixed gradient map (`sign` * the true gradient at
    the start design, or its negative): proposals that help or hurt."""

    def __init__(self, problem, sign=1.0):
        self.device = torch.device("cpu")
        self.problem, self.sign = problem, sign
        self.steps = 0

    def predict(self, density):
        p = density.cpu().numpy()
        g = -2.0 * (p - self.problem.target) / p.size
        return torch.zeros(self.problem.nwav), torch.from_numpy(self.sign * g)

    def train_step(self, P, T, G, lr):
        assert P.shape[0] == T.shape[0] == G.shape[0]
        self.steps += 1


def test_ascent_normalises_and_clips():
    p = np.full((4, 4), 0.95, np.float32)
    d = np.zeros((4, 4), np.float32)
    d[0, 0], d[1, 1] = 2.0, -1.0
    q = dl.ascent(p, d, 0.1)
    assert q[0, 0] == 1.0  # 0.95 + 0.1 clipped
    assert np.isclose(q[1, 1], 0.95 - 0.05)
    assert np.array_equal(dl.ascent(p, np.zeros_like(p), 0.1), p)


def test_time_to_skips_rejected_designs():
    hist = [dict(T=0.2, t=1.0, kind="adjoint"), dict(T=0.95, t=2.0, kind="rejected"),
            dict(T=0.91, t=3.0, kind="surrogate")]
    assert dl.time_to(hist, 0.9) == 3.0
    assert dl.time_to(hist, 0.99) is None


def test_adjoint_loop_stops_at_target_and_records_triples():
    prob = FakeProblem()
    seen = []
    p0 = np.zeros(prob.shape, np.float32)
    _, hist = dl.adjoint_loop(prob, p0, target=0.95, iters=50, step=0.05,
                              record=lambda p, s, g: seen.append(p.copy()))
    assert hist[-1]["T"] >= 0.95 and all(h["T"] < 0.95 for h in hist[:-1])
    assert len(seen) == len(hist) == prob.adjoints and prob.forwards == 0


@pytest.mark.parametrize("sign", [1.0, -1.0])
def test_extrapolate_loop_keeps_only_verified_improvements(sign):
    prob = FakeProblem(seed=1)
    net = FakeNet(prob, sign)
    data = dl.Dataset(prob.shape, prob.nwav, device="cpu")
    p0 = np.zeros(prob.shape, np.float32)
    _, hist = dl.extrapolate_loop(prob, net, p0, data, target=2.0, iters=6, step=0.05,
                                  finetune_steps=2)
    kinds = [h["kind"] for h in hist]
    assert kinds[::2] == ["adjoint"] * 6
    for before, judged in zip(hist[::2], hist[1::2]):
        assert (judged["kind"] == "surrogate") == (judged["T"] > before["T"])
    if sign > 0:  # the true gradient direction always helps on this concave T
        assert kinds[1::2] == ["surrogate"] * 6
    else:  # the reversed direction never does
        assert kinds[1::2] == ["rejected"] * 6
    assert len(data) == 6 and net.steps == 12
    assert prob.adjoints == 6 and prob.forwards == 6


def test_surrogate_loop_falls_back_to_the_adjoint_step():
    prob = FakeProblem(seed=2)
    net = FakeNet(prob, -1.0)  # every proposal is rejected
    data = dl.Dataset(prob.shape, prob.nwav, device="cpu")
    p0 = np.zeros(prob.shape, np.float32)
    _, hist = dl.surrogate_loop(prob, net, p0, data, target=2.0, iters=5, step=0.05,
                                finetune_steps=1)
    assert [h["kind"] for h in hist] == ["start"] + ["adjoint"] * 4
    assert all(a["T"] <= b["T"] for a, b in zip(hist, hist[1:]))
    assert prob.adjoints == 4 and prob.forwards == 1 + 4 * 2


def test_dataset_round_trip(tmp_path):
    d = dl.Dataset((4, 6), 3, device="cpu")
    rng = np.random.default_rng(0)
    for _ in range(5):
        d.add(rng.uniform(0, 1, (4, 6)), rng.uniform(0, 1, 3), rng.standard_normal((4, 6)))
    P, T, G = d.tensors()
    assert P.shape == (5, 4, 6) and T.shape == (5, 3) and G.shape == (5, 4, 6)
    assert np.isclose(float(torch.sqrt(torch.mean(G ** 2))), 1.0, rtol=1e-5)
    d.save(tmp_path / "d.npz", n_train=3)
    e, n_train = dl.Dataset.load(tmp_path / "d.npz", device="cpu")
    assert n_train == 3 and len(e) == 5
    assert np.array_equal(np.stack(e.p), np.stack(d.p).astype(np.float32))
    P2, _, _ = e.tensors(last=2)
    assert torch.equal(P2, P[-2:])
