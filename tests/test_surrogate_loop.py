"""The surrogate search loop on the host with stand-ins for the FDTD problem and the
network (no GPU): a smooth transmission landscape with its exact gradient, and a
surrogate that is either exact or corrupted. A corrupted surrogate misses the verified
transmission change by more than the tolerance, so every round falls back (and the loop
still climbs on the exact-gradient steps); an exact surrogate is trusted."""
import numpy as np
import torch

from beamz_b200.surrogate.topo import SurrogateSearch, active_learning

N = 24


class FakeProblem:
    """T(rho) = 1 - mean((rho - target)^2): one 'wavelength', maximum 1 at the target."""

    def __init__(self):
        g = torch.Generator().manual_seed(3)
        self.target = torch.rand(N, N, generator=g, dtype=torch.float64) * 0.6 + 0.2
        self.n_freq = 1
        self.kw = {"region": (0, 0, N, N)}
        self.grad_calls = 0
        self.forward_designs = 0
        self.fdtd_designs = 0

    def T(self, rho):
        rho = torch.as_tensor(np.asarray(rho), dtype=torch.float64)
        return 1.0 - ((rho - self.target) ** 2).mean(dim=(1, 2))

    def transmission(self, rho):
        self.forward_designs += len(rho)
        self.fdtd_designs += len(rho)
        return self.T(rho).numpy()[:, None]

    def value_and_grad(self, rho):
        self.grad_calls += 1
        self.fdtd_designs += len(rho)
        rho_t = torch.as_tensor(np.asarray(rho), dtype=torch.float64)
        return self.T(rho_t).numpy(), (-2.0 * (rho_t - self.target) / (N * N)).numpy()


class FakeNet:
    """The surrogate interface the loop uses. exact=True predicts the true T (and its
    gradient); exact=False returns corrupted predictions: uniform noise in [0, 5)."""

    def __init__(self, problem, exact):
        self.p, self.exact = problem, exact
        self.dev = torch.device("cpu")
        self.y_scale = torch.ones(1)
        self._x = None
        self.gen = torch.Generator().manual_seed(11)
        self.adam_steps = 0

    def forward(self, rho, keep=False):
        self._x = rho.double()
        if self.exact:
            return self.p.T(rho.double()).float()[:, None]
        return torch.rand((len(rho), 1), generator=self.gen) * 5.0

    def backward(self, d_out, want_input_grad=False):
        x = self._x
        g = -2.0 * (x - self.p.target) / (N * N) if self.exact else torch.randn(x.shape, dtype=torch.float64)
        return (g * d_out.double()[:, :1, None]).float() if want_input_grad else None

    def zero_grad(self):
        pass

    def adam_step(self, lr=1e-3, **kw):
        self.adam_steps += 1


def _start():
    return np.full((N, N), 0.5)


def test_corrupted_surrogate_falls_back_every_round():
    prob = FakeProblem()
    search = SurrogateSearch(prob, FakeNet(prob, exact=False), n_candidates=96, n_verify=8, n_anchor=4, tol=1e-2)
    t0 = float(prob.T(_start()[None])[0])
    hist, _, best = search.run(_start(), rounds=5)
    assert all(r["fallback"] for r in search.log)
    assert all(r["surrogate_err"] > 1e-2 for r in search.log)
    assert all(r["step_err"] is None or r["step_err"] > 1e-2 for r in search.log)
    assert prob.grad_calls == 1 + 5  # the first direction plus one exact gradient per round
    assert hist[-1] > t0 and all(b >= a for a, b in zip(hist, hist[1:]))


def test_exact_surrogate_is_trusted():
    prob = FakeProblem()
    search = SurrogateSearch(prob, FakeNet(prob, exact=True), n_candidates=96, n_verify=8, n_anchor=4, tol=1e-2)
    hist, _, best = search.run(_start(), rounds=4)
    assert all(r["surrogate_err"] < 1e-6 for r in search.log)
    assert all(r["step_err"] is None or r["step_err"] < 1e-6 for r in search.log)
    trusted = [r for r in search.log if not r["fallback"]]
    assert trusted, search.log
    assert prob.grad_calls == 1 + len(search.log)
    assert hist[-1] > hist[0]


def test_without_surrogate_is_a_batched_line_search():
    prob = FakeProblem()
    search = SurrogateSearch(prob, FakeNet(prob, exact=True), n_candidates=96, n_verify=8, n_anchor=4,
                             use_surrogate=False)
    hist, _, _ = search.run(_start(), rounds=3)
    assert prob.grad_calls == 1 + 3 and prob.forward_designs == 3 * 12
    assert hist[-1] > hist[0]


def test_search_stops_at_the_target_without_a_further_gradient():
    """Once the verified T reaches the target the loop ends: no exact gradient is taken
    at the final design (the plain ascent takes none there either)."""
    prob = FakeProblem()
    t0 = float(prob.T(_start()[None])[0])
    search = SurrogateSearch(prob, FakeNet(prob, exact=True), n_candidates=96, n_verify=8, n_anchor=4)
    hist, _, _ = search.run(_start(), rounds=10, target=t0 + 1e-9)
    assert len(search.log) == 1 and hist[-1] >= t0 + 1e-9
    assert prob.grad_calls == 1


def test_active_learning_fine_tunes_on_its_own_proposals():
    """Searches from each start (no target): with a corrupted surrogate every round falls
    back and fine-tunes the network (3 Adam steps per round); the FDTD count is the
    verified batches plus one gradient per round and the initial one per start."""
    prob = FakeProblem()
    net = FakeNet(prob, exact=False)
    starts = np.stack([_start(), np.full((N, N), 0.3)])
    st = active_learning(prob, net, starts, rounds=3, n_candidates=96, n_verify=8, n_anchor=4)
    assert net.adam_steps == 2 * 3 * 3
    assert st["fdtd_designs"] == 2 * 3 * (8 + 4) + 2 * (1 + 3)
    assert len(st["best_T"]) == 2 and st["seconds"] >= 0
