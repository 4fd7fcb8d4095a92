"""Surrogate-assisted topology optimisation on the batched FDTD.

The design problem is the topology workload with a pulsed source: a 120 x 120 density
region in a 600 x 400 grid, objective = mean over five wavelengths of the fundamental
mode transmission T_f = |a_f|^2 / |a_f(straight guide)|^2 at the output monitor.

* ``TransmissionProblem`` evaluates T for a batch of densities with one batched FDTD
  forward (``AdjointFDTD2D``), and the exact gradient of the mean transmission with
  the batched adjoint.
* ``make_dataset`` draws smoothed random densities and labels them with batched FDTD.
* ``train`` fits the FNO surrogate (bf16 kernels, f32 accumulation) on them.
* ``SurrogateSearch`` runs the loop: the surrogate proposes candidates around the
  current design (steps along its own input gradient plus smooth perturbations), the
  best-ranked are verified by one batched FDTD forward, and the best verified one is
  kept if it improves; whenever the surrogate misses the verified transmission by more
  than ``tol`` (or proposes nothing better), that round takes a plain exact-adjoint
  step instead and the verified samples are added to the surrogate's training set.
* ``plain_adjoint`` is the baseline: the same ascent with the exact adjoint gradient,
  one design per FDTD call.
"""
from __future__ import annotations

import time

import numpy as np
import torch
import torch.nn.functional as F

from .. import workloads as W
from ..optimization.adjoint import AdjointFDTD2D
from .fno import FNO2d

_KEYS = ("eps_base", "sigma", "dx", "dt", "n_steps", "sources", "monitor", "mode_profile", "frequency", "region")


def smooth(rho: torch.Tensor, radius: int = 1) -> torch.Tensor:
    """Box blur with replicated edges, (B, n, n) -> (B, n, n)."""
    k = 2 * radius + 1
    x = F.pad(rho[:, None], (radius,) * 4, mode="replicate")
    return F.avg_pool2d(x, k, stride=1)[:, 0]


def densities(seeds, r: int = 120, sigma: float = 3.0) -> np.ndarray:
    """Smoothed random densities: uniform [0, 1] (torch generator seeded per design,
    as the topology workload draws them), Gaussian-filtered with ``sigma`` cells, then
    contrast-stretched to mean 0.5, standard deviation 0.25 and clipped to [0, 1]
    (the filtered fields alone have a standard deviation near 0.03)."""
    from scipy.ndimage import gaussian_filter

    out = np.empty((len(seeds), r, r), dtype=np.float32)
    for i, s in enumerate(seeds):
        f = gaussian_filter(torch.rand((r, r), generator=torch.Generator().manual_seed(int(s)),
                                       dtype=torch.float64).numpy(), sigma=sigma)
        f = (f - f.mean()) / max(f.std(), 1e-12)
        out[i] = np.clip(0.5 + 0.25 * f, 0.0, 1.0)
    return out


class TransmissionProblem:
    def __init__(self, n_steps=8000, precision="fp32", checkpoint_every=500, max_batch=64):
        kw = W.surrogate_2d(n_designs=1, n_steps=n_steps)
        self.kw = kw
        self.base = {k: kw[k] for k in _KEYS}
        self.eps_lo, self.eps_hi = kw["eps_lo"], kw["eps_hi"]
        self.precision, self.K, self.max_batch = precision, checkpoint_every, max_batch
        self.n_freq = len(np.atleast_1d(kw["frequency"]))
        self.weights = np.ones(self.n_freq)
        self._probs: dict[int, AdjointFDTD2D] = {}
        self.fdtd_designs = 0  # designs simulated (forward runs; an adjoint step counts one)
        self.fdtd_seconds = 0.0
        ref = self._problem(1)
        ref.forward(self.eps(kw["rho_straight"][None]), keep_checkpoints=False)
        self.ref_power = ref.power[0].copy()
        self.weights = 1.0 / (self.n_freq * self.ref_power)  # J = mean_f T_f
        for p in self._probs.values():
            p.c_f = self.weights.copy()

    def eps(self, rho):
        return self.eps_lo + np.asarray(rho, dtype=np.float64) * (self.eps_hi - self.eps_lo)

    def _problem(self, B):
        p = self._probs.get(B)
        if p is None:
            p = AdjointFDTD2D(**self.base, n_designs=B, precision=self.precision, checkpoint_every=self.K,
                              weights=self.weights)
            self._probs[B] = p
        return p

    def transmission(self, rho) -> np.ndarray:
        """T (B, n_freq) for densities rho (B, r, r) by batched FDTD forward runs."""
        rho = np.asarray(rho)
        out = np.empty((len(rho), self.n_freq))
        t0 = time.perf_counter()
        for i in range(0, len(rho), self.max_batch):
            chunk = rho[i:i + self.max_batch]
            p = self._problem(len(chunk))
            p.forward(self.eps(chunk), keep_checkpoints=False)
            out[i:i + len(chunk)] = p.power / self.ref_power[None, :]
        torch.cuda.synchronize()
        self.fdtd_seconds += time.perf_counter() - t0
        self.fdtd_designs += len(rho)
        return out

    def value_and_grad(self, rho):
        """Mean transmission (B,) and its exact gradient with respect to rho (B, r, r)."""
        rho = np.asarray(rho)
        t0 = time.perf_counter()
        p = self._problem(len(rho))
        J, g = p.value_and_grad(self.eps(rho))
        torch.cuda.synchronize()
        self.fdtd_seconds += time.perf_counter() - t0
        self.fdtd_designs += len(rho)
        return J, g * (self.eps_hi - self.eps_lo)


def make_dataset(problem: TransmissionProblem, n_samples: int, seed0: int = 10000, batch: int = 64):
    """(rho (n, r, r) float32, T (n, n_freq) float32) labelled by batched FDTD."""
    r = problem.kw["region"][2]
    rho = densities(range(seed0, seed0 + n_samples), r)
    T = np.empty((n_samples, problem.n_freq), dtype=np.float32)
    for i in range(0, n_samples, batch):
        T[i:i + batch] = problem.transmission(rho[i:i + batch])
    return rho, T


def train(net: FNO2d, rho: np.ndarray, T: np.ndarray, epochs: int = 20, batch: int = 64, lr: float = 2e-3,
          seed: int = 0, log=None) -> list[float]:
    """MSE fit of T with Adam and a cosine learning-rate decay; returns per-epoch losses."""
    rng = np.random.default_rng(seed)
    n = len(rho)
    rho_d = torch.as_tensor(rho, device=net.dev)
    T_d = torch.as_tensor(T, device=net.dev)
    steps = epochs * ((n + batch - 1) // batch)
    k, losses = 0, []
    for ep in range(epochs):
        perm = torch.as_tensor(rng.permutation(n), device=net.dev)
        tot = 0.0
        for i in range(0, n, batch):
            idx = perm[i:i + batch]
            out = net.forward(rho_d[idx], keep=True)
            err = out - T_d[idx]
            tot += float((err ** 2).sum())
            net.zero_grad()
            net.backward(2.0 * err / err.numel())
            net.adam_step(lr=lr * 0.5 * (1 + np.cos(np.pi * k / steps)))
            k += 1
        losses.append(tot / (n * T.shape[1]))
        if log:
            log(f"epoch {ep}: mse {losses[-1]:.3e}")
    return losses


def _ascend(rho: torch.Tensor, g: torch.Tensor, step) -> torch.Tensor:
    g = g / g.abs().amax(dim=(1, 2), keepdim=True).clamp_min(1e-30)
    step = torch.as_tensor(step, dtype=rho.dtype, device=rho.device).reshape(-1, 1, 1)
    return smooth(rho + step * g, 1).clamp(0.0, 1.0)


def plain_adjoint(problem: TransmissionProblem, rho0: np.ndarray, iterations: int, step: float = 0.05):
    """Exact-adjoint ascent on one design (the per-design baseline). Returns the
    mean-transmission history (value before each step, then the final value), seconds."""
    rho = torch.as_tensor(rho0[None], dtype=torch.float64)
    hist = []
    t0 = time.perf_counter()
    for _ in range(iterations):
        J, g = problem.value_and_grad(rho.numpy())
        hist.append(float(J[0]))
        rho = _ascend(rho, torch.as_tensor(g), step)
    hist.append(float(problem.transmission(rho.numpy()).mean()))
    return hist, time.perf_counter() - t0, rho[0].numpy()


class SurrogateSearch:
    def __init__(self, problem: TransmissionProblem, net: FNO2d, n_candidates=256, n_verify=16, tol=1e-2,
                 adjoint_step=0.05, seed=0):
        self.problem, self.net = problem, net
        self.n_cand, self.n_verify, self.tol = n_candidates, n_verify, tol
        self.adjoint_step = adjoint_step
        self.gen = torch.Generator(device=net.dev).manual_seed(seed)
        self.rho_new, self.T_new = [], []  # verified samples collected for fine-tuning
        self.log = []

    def _predict(self, rho: torch.Tensor) -> torch.Tensor:
        return torch.cat([self.net.forward(rho[i:i + 256].float()) for i in range(0, len(rho), 256)])

    def _proposals(self, rho: torch.Tensor) -> torch.Tensor:
        """n_candidates densities around rho (r, r): steps along the surrogate's gradient
        of the mean transmission (log-spaced sizes) plus smooth random perturbations."""
        x = rho[None].float()
        self.net.forward(x, keep=True)
        g = self.net.backward(torch.full((1, self.problem.n_freq), 1.0 / self.problem.n_freq, device=self.net.dev),
                              want_input_grad=True)
        self.net.zero_grad()
        n = self.n_cand
        steps = torch.logspace(-2.3, -0.5, n, device=self.net.dev)
        noise = smooth(torch.randn(n, *rho.shape, generator=self.gen, device=self.net.dev), 3)
        noise = noise / noise.abs().amax(dim=(1, 2), keepdim=True)
        amp = torch.rand(n, 1, 1, generator=self.gen, device=self.net.dev) * 0.08
        gg = g.double().expand(n, -1, -1) / g.abs().max().clamp_min(1e-30)
        cand = rho[None] + steps.double()[:, None, None] * gg + amp.double() * noise.double()
        return smooth(cand, 1).clamp(0.0, 1.0)

    def _finetune(self, steps=20, lr=5e-4):
        if not self.rho_new:
            return
        rho = torch.as_tensor(np.concatenate(self.rho_new), dtype=torch.float32, device=self.net.dev)
        T = torch.as_tensor(np.concatenate(self.T_new), dtype=torch.float32, device=self.net.dev)
        for _ in range(steps):
            idx = torch.randint(0, len(rho), (min(64, len(rho)),), generator=self.gen, device=self.net.dev)
            out = self.net.forward(rho[idx], keep=True)
            err = out - T[idx]
            self.net.zero_grad()
            self.net.backward(2.0 * err / err.numel())
            self.net.adam_step(lr=lr)

    def run(self, rho0: np.ndarray, rounds: int, target: float | None = None):
        """Optimise from rho0; stops after ``rounds`` or once the verified mean transmission
        reaches ``target``. Returns (best mean T history per round, seconds, best rho)."""
        dev = self.net.dev
        rho = torch.as_tensor(rho0, dtype=torch.float64, device=dev)
        best = float(self.problem.transmission(rho[None].cpu().numpy()).mean())
        hist = [best]
        t0 = time.perf_counter()
        for rnd in range(rounds):
            cand = self._proposals(rho)
            pred = self._predict(cand).mean(dim=1)
            top = torch.topk(pred, self.n_verify).indices
            chosen = cand[top]
            T_true = self.problem.transmission(chosen.cpu().numpy())
            t_true = T_true.mean(axis=1)
            err = float(np.abs(pred[top].double().cpu().numpy() - t_true).max())
            self.rho_new.append(chosen.float().cpu().numpy())
            self.T_new.append(T_true.astype(np.float32))
            k = int(np.argmax(t_true))
            improved = t_true[k] > best
            if improved:
                best, rho = float(t_true[k]), chosen[k]
            fallback = err > self.tol or not improved
            if fallback:
                J, g = self.problem.value_and_grad(rho[None].cpu().numpy())
                nxt = _ascend(rho[None].cpu(), torch.as_tensor(g), self.adjoint_step)
                t_next = float(self.problem.transmission(nxt.numpy()).mean())
                if t_next > best:
                    best, rho = t_next, nxt[0].to(dev)
                self._finetune()
            self.log.append(dict(round=rnd, best=best, surrogate_err=err, fallback=bool(fallback)))
            hist.append(best)
            if target is not None and best >= target:
                break
        return hist, time.perf_counter() - t0, rho.cpu().numpy()
