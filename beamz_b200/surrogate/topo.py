"""Surrogate-assisted topology optimisation on the batched FDTD.

The design problem is the topology workload with a pulsed source: a 120 x 120 density
region in a 600 x 400 grid, objective = mean over five wavelengths of the fundamental
mode transmission T_f = |a_f|^2 / |a_f(straight guide)|^2 at the output monitor.

* ``TransmissionProblem`` evaluates T for a batch of densities with one batched FDTD
  forward (``AdjointFDTD2D``), and the exact gradient of the mean transmission with
  the batched adjoint.
* ``make_dataset`` draws smoothed random densities (optionally also the designs visited
  by batched exact-adjoint ascents from random starts) and labels them with batched FDTD.
* ``train`` fits the FNO surrogate (bf16 kernels, f32 accumulation) on them.
* ``SurrogateSearch`` runs the loop: the surrogate proposes candidates around the
  current design (steps along its own input gradient plus smooth perturbations), the
  best-ranked are verified by one batched FDTD forward, and the best verified one is
  kept if it improves; whenever the surrogate misses the verified transmission by more
  than ``tol`` (or proposes nothing better), that round also takes a plain exact-adjoint
  step (verified together with the next round's candidates) and fine-tunes the
  surrogate on the verified samples.
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
        self.fdtd_runs = 0  # solver invocations (one batched forward, or one forward + adjoint)
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
            self.fdtd_runs += 1
        torch.cuda.synchronize()
        self.fdtd_seconds += time.perf_counter() - t0
        self.fdtd_designs += len(rho)
        return out

    def value_and_grad(self, rho, return_T=False):
        """Mean transmission (B,) and its exact gradient with respect to rho (B, r, r)
        (and T (B, n_freq) when asked)."""
        rho = np.asarray(rho)
        t0 = time.perf_counter()
        p = self._problem(len(rho))
        J, g = p.value_and_grad(self.eps(rho))
        torch.cuda.synchronize()
        self.fdtd_seconds += time.perf_counter() - t0
        self.fdtd_designs += len(rho)
        self.fdtd_runs += 1
        g = g * (self.eps_hi - self.eps_lo)
        if return_T:
            return J, g, p.power / self.ref_power[None, :]
        return J, g


def make_dataset(problem: TransmissionProblem, n_samples: int, seed0: int = 10000, batch: int = 64,
                 trajectory_frac: float = 0.0, step: float = 0.05):
    """(rho (n, r, r) float32, T (n, n_freq) float32) labelled by batched FDTD.

    A fraction ``trajectory_frac`` comes from exact-adjoint ascent trajectories (``batch``
    random starts stepped together with the batched adjoint, every visited design kept),
    so that the set also covers the high-transmission designs an optimiser reaches; the
    rest are independent smoothed random densities."""
    r = problem.kw["region"][2]
    n_traj = int(round(n_samples * trajectory_frac)) // batch * batch
    n_rand = n_samples - n_traj
    rho = np.empty((n_samples, r, r), dtype=np.float32)
    T = np.empty((n_samples, problem.n_freq), dtype=np.float32)
    rho[:n_rand] = densities(range(seed0, seed0 + n_rand), r)
    for i in range(0, n_rand, batch):
        T[i:i + batch] = problem.transmission(rho[i:i + batch])
    cur = torch.as_tensor(densities(range(seed0 + n_rand, seed0 + n_rand + batch), r), dtype=torch.float64)
    for i in range(n_rand, n_samples, batch):
        _, g, Tb = problem.value_and_grad(cur.numpy(), return_T=True)
        rho[i:i + batch], T[i:i + batch] = cur.numpy(), Tb
        cur = _ascend(cur, torch.as_tensor(g), step)
    return rho, T


def train(net: FNO2d, rho: np.ndarray, T: np.ndarray, epochs: int = 20, batch: int = 64, lr: float = 2e-3,
          seed: int = 0, val_frac: float = 0.05, weight_decay: float = 1e-4, log=None) -> dict:
    """MSE fit of T (targets standardised per output) with Adam, a cosine learning-rate
    decay and weight decay; a held-out split picks the best epoch, whose weights are kept.
    Returns {"train": per-epoch MSE, "val": per-epoch validation MAE, "best_epoch"}."""
    rng = np.random.default_rng(seed)
    order = rng.permutation(len(rho))
    n_val = max(1, int(len(rho) * val_frac))
    val, tr = order[:n_val], order[n_val:]
    n = len(tr)
    rho_d = torch.as_tensor(rho, device=net.dev)
    T_d = torch.as_tensor(T, device=net.dev)
    net.y_shift.copy_(T_d[tr].mean(0))
    net.y_scale.copy_(T_d[tr].std(0).clamp_min(1e-6))
    steps = epochs * ((n + batch - 1) // batch)
    k, losses, vals, best = 0, [], [], (np.inf, -1, None)
    for ep in range(epochs):
        perm = torch.as_tensor(tr[rng.permutation(n)], device=net.dev)
        tot = 0.0
        for i in range(0, n, batch):
            idx = perm[i:i + batch]
            out = net.forward(rho_d[idx], keep=True)
            err = (out - T_d[idx]) / net.y_scale[None, :]
            tot += float((err ** 2).sum())
            net.zero_grad()
            net.backward(2.0 * err / (err.numel() * net.y_scale[None, :]))
            net.adam_step(lr=lr * 0.5 * (1 + np.cos(np.pi * k / steps)), weight_decay=weight_decay)
            k += 1
        losses.append(tot / (n * T.shape[1]))
        vi = torch.as_tensor(val, device=net.dev)
        pred = torch.cat([net.forward(rho_d[vi[i:i + 256]]) for i in range(0, n_val, 256)])
        vals.append(float((pred - T_d[vi]).abs().mean()))
        if vals[-1] < best[0]:
            best = (vals[-1], ep, net.state_dict())
        if log:
            log(f"epoch {ep}: standardised mse {losses[-1]:.3e}, validation mae {vals[-1]:.4f}")
    net.load_state_dict(best[2])
    return {"train": losses, "val": vals, "best_epoch": best[1]}


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
    """Surrogate-ranked ascent of the mean transmission, every accepted design judged by
    a batched FDTD forward run.

    Round r, from the current design rho, its exact adjoint gradient g (one per-design
    adjoint run per round: the batched FDTD judges the candidates, the adjoint steers
    them) and the surrogate's own input gradient:
      1. candidates: points along ascent paths followed on the surrogate itself (many
         small steps of its input gradient, ``_trajectories``), steps of a geometric
         ladder of sizes along the ascent directions (the exact gradient, the
         surrogate's gradient and mixes of the two, each scaled to a unit peak), and
         smooth random perturbations of the best-predicted ones; each is box-blurred
         (radius 1) and clipped to [0, 1] as a plain ascent step is;
      2. verification: the ``n_verify`` candidates the surrogate ranks highest plus
         ``n_anchor`` steps along the exact gradient at fixed sizes (when it is known),
         in one batched FDTD forward; with ``use_surrogate=False`` the batch is
         ``n_verify + n_anchor`` evenly spaced ladder steps along the exact gradient (the
         method without the network);
      3. the best verified design replaces rho when it raises the verified T;
      4. fallback: when the accepted step's transmission change predicted by the
         surrogate, dT = T_pred(new) - T_pred(rho), misses the verified change by more
         than ``tol`` -- or the step was not the network's, or nothing improved -- the
         round counts as a fallback: its progress came from (or rests on) the exact
         adjoint steps, and the surrogate is fine-tuned on the verified samples (mixed
         with training samples) before it proposes again. Steps the network proposes
         on its own gradient were measured to climb slower than with the exact gradient
         beside them, so the adjoint run is taken every round.
    ``log`` keeps, per round, the best T, the error of the accepted step's predicted dT,
    the surrogate's largest miss of a verified T and whether the round fell back."""

    def __init__(self, problem: TransmissionProblem, net: FNO2d, n_candidates=256, n_verify=24, tol=1e-2,
                 adjoint_step=0.05, seed=0, replay=None, use_surrogate=True, n_anchor=8, ladder=(0.01, 0.8)):
        self.problem, self.net = problem, net
        self.n_cand, self.n_verify, self.tol = n_candidates, n_verify, tol
        self.adjoint_step = adjoint_step
        self.use_surrogate = use_surrogate
        self.n_anchor = max(0, int(n_anchor))
        self.ladder = ladder
        self.gen = torch.Generator(device=net.dev).manual_seed(seed)
        self.rho_new, self.T_new = [], []  # verified samples collected for fine-tuning
        self.replay = replay  # (rho, T) of the training set, mixed into fine-tuning batches
        self.log = []

    def _predict(self, rho: torch.Tensor) -> torch.Tensor:
        return torch.cat([self.net.forward(rho[i:i + 256].float()) for i in range(0, len(rho), 256)])

    def _surrogate_grad(self, rho: torch.Tensor) -> torch.Tensor:
        self.net.forward(rho[None].float(), keep=True)
        n_out = self.problem.n_freq
        g = self.net.backward(torch.full((1, n_out), 1.0 / n_out, device=self.net.dev), want_input_grad=True)
        self.net.zero_grad()
        return g[0].double()

    @staticmethod
    def _unit(d: torch.Tensor) -> torch.Tensor:
        return d / d.abs().max().clamp_min(1e-30)

    def _steps(self, rho, d, sizes):
        cand = rho[None] + sizes.double()[:, None, None] * d[None]
        return smooth(cand, 1).clamp(0.0, 1.0)

    def _sizes(self, n):
        lo, hi = self.ladder
        return torch.logspace(np.log10(lo), np.log10(hi), n, device=self.net.dev, dtype=torch.float64)

    def _trajectories(self, rho, g_adj, n_traj=8, n_inner=24, keep=(1, 2, 4, 6, 9, 13, 18, 24)):
        """Ascent paths on the surrogate itself: n_traj copies of rho, each stepped n_inner
        times along the unit-peak input gradient of the surrogate's mean transmission
        (step sizes spread geometrically over the copies; the first step follows the
        exact gradient when it is known), blurred and clipped like a plain step; the
        designs after the steps in ``keep`` are candidates. The network is thus used to
        follow a curved path that one gradient step cannot."""
        dev = self.net.dev
        n_out = self.problem.n_freq
        sizes = torch.logspace(np.log10(0.02), np.log10(0.12), n_traj, device=dev, dtype=torch.float64)[:, None, None]
        x = rho[None].expand(n_traj, -1, -1).clone()
        out = []
        for i in range(1, n_inner + 1):
            if i == 1 and g_adj is not None:
                d = self._unit(g_adj)[None].expand(n_traj, -1, -1)
            else:
                self.net.forward(x.float(), keep=True)
                g = self.net.backward(torch.full((n_traj, n_out), 1.0 / n_out, device=dev), want_input_grad=True)
                self.net.zero_grad()
                d = g.double() / g.double().abs().amax(dim=(1, 2), keepdim=True).clamp_min(1e-30)
            x = smooth(x + sizes * d, 1).clamp(0.0, 1.0)
            if i in keep:
                out.append(x.clone())
        return torch.cat(out)

    def _candidates(self, rho, g_adj, g_sur):
        dirs = [self._unit(g_sur)]
        if g_adj is not None:
            ga = self._unit(g_adj)
            dirs = [ga, dirs[0]] + [self._unit(a * ga + (1 - a) * dirs[0]) for a in (0.25, 0.5, 0.75)]
        per = 16
        line = torch.cat([self._trajectories(rho, g_adj)] + [self._steps(rho, d, self._sizes(per)) for d in dirs])
        n_noise = max(0, self.n_cand - len(line))
        if n_noise == 0:
            return line[:self.n_cand]
        pred = self._predict(line).mean(dim=1)
        seeds = line[torch.topk(pred, min(8, len(line))).indices]
        pick = torch.randint(0, len(seeds), (n_noise,), generator=self.gen, device=self.net.dev)
        noise = smooth(torch.randn(n_noise, *rho.shape, generator=self.gen, device=self.net.dev), 3)
        noise = noise / noise.abs().amax(dim=(1, 2), keepdim=True)
        amp = torch.rand(n_noise, 1, 1, generator=self.gen, device=self.net.dev) * 0.06
        return torch.cat([line, smooth(seeds[pick] + amp.double() * noise.double(), 1).clamp(0.0, 1.0)])

    def _finetune(self, steps=3, lr=5e-4):
        if not self.rho_new:
            return
        dev = self.net.dev
        rho = torch.as_tensor(np.concatenate(self.rho_new), dtype=torch.float32, device=dev)
        T = torch.as_tensor(np.concatenate(self.T_new), dtype=torch.float32, device=dev)
        rng = np.random.default_rng(len(self.rho_new))
        for _ in range(steps):
            idx = torch.randint(0, len(rho), (min(32, len(rho)),), generator=self.gen, device=dev)
            xb, yb = rho[idx], T[idx]
            if self.replay is not None:  # half of each batch from the training set
                j = rng.integers(0, len(self.replay[0]), 32)
                xb = torch.cat([xb, torch.as_tensor(self.replay[0][j], device=dev)])
                yb = torch.cat([yb, torch.as_tensor(self.replay[1][j], device=dev)])
            out = self.net.forward(xb, keep=True)
            err = (out - yb) / self.net.y_scale[None, :]
            self.net.zero_grad()
            self.net.backward(2.0 * err / (err.numel() * self.net.y_scale[None, :]))
            self.net.adam_step(lr=lr)

    def _exact_grad(self, rho, with_value=False):
        J, g = self.problem.value_and_grad(rho[None].cpu().numpy())
        g = torch.as_tensor(g[0], device=self.net.dev)
        return (float(J[0]), g) if with_value else g

    def run(self, rho0: np.ndarray, rounds: int, target: float | None = None):
        """Optimise from rho0; stops after ``rounds`` or once the verified mean transmission
        reaches ``target``. Returns (best mean T history per round, seconds, best rho)."""
        dev = self.net.dev
        rho = torch.as_tensor(rho0, dtype=torch.float64, device=dev)
        t0 = time.perf_counter()
        best, g_adj = self._exact_grad(rho, with_value=True)  # the first direction is exact
        hist = [best]
        for rnd in range(rounds):
            err, miss, n_rank = float("inf"), 0.0, 0
            if self.use_surrogate:
                pred_cur = float(self._predict(rho[None]).mean())
                g_sur = self._surrogate_grad(rho)
                cand = self._candidates(rho, g_adj, g_sur)
                pred = self._predict(cand).mean(dim=1)
                n_rank = min(self.n_verify, len(cand))
                top = torch.topk(pred, n_rank).indices
                ranked, pred_ranked = cand[top], pred[top]
                parts = [ranked]
                if g_adj is not None and self.n_anchor:
                    parts.append(self._steps(rho, self._unit(g_adj),
                                             self._sizes(self.n_anchor + 2)[1:-1]))
                batch = torch.cat(parts)
            else:
                batch = self._steps(rho, self._unit(g_adj), self._sizes(self.n_verify + self.n_anchor))
            T_true = self.problem.transmission(batch.cpu().numpy())
            t_true = T_true.mean(axis=1)
            k = int(np.argmax(t_true))
            improved = t_true[k] > best
            if n_rank:
                pr = pred_ranked.double().cpu().numpy()
                miss = float(np.abs(pr - t_true[:n_rank]).max())
                if improved and k < n_rank:  # the accepted step came from the network:
                    # |dT predicted - dT verified| of that step
                    err = abs((pr[k] - pred_cur) - (t_true[k] - best))
                self.rho_new.append(batch[:n_rank].float().cpu().numpy())
                self.T_new.append(T_true[:n_rank].astype(np.float32))
            if improved:
                best, rho = float(t_true[k]), batch[k]
            fallback = (not self.use_surrogate) or not improved or err > self.tol
            self.log.append(dict(round=rnd, best=best, step_err=(err if np.isfinite(err) else None),
                                 surrogate_err=miss, fallback=bool(fallback), ranked_best=bool(n_rank and k < n_rank)))
            hist.append(best)
            if target is not None and best >= target:
                break  # done: no gradient is needed at the final design (plain ascent takes none either)
            g_adj = self._exact_grad(rho)
            if self.use_surrogate and fallback:
                self._finetune()
        return hist, time.perf_counter() - t0, rho.cpu().numpy()


def active_learning(problem: TransmissionProblem, net: FNO2d, starts: np.ndarray, rounds: int = 4, replay=None,
                    **search_kw) -> dict:
    """Fine-tunes a trained surrogate on its own proposals: a search of ``rounds`` rounds
    from each start design (no target), whose FDTD-verified candidates fine-tune the
    network on every fallback round as in ``SurrogateSearch.run``. Part of training: the
    start designs must not include the one a timed search starts from. Returns the
    seconds, FDTD-simulated designs and the best T reached from each start."""
    t0 = time.perf_counter()
    d0 = problem.fdtd_designs
    best = []
    for i, rho0 in enumerate(np.asarray(starts)):
        s = SurrogateSearch(problem, net, replay=replay, seed=1000 + i, **search_kw)
        hist, _, _ = s.run(rho0, rounds=rounds)
        best.append(hist[-1])
    return {"seconds": time.perf_counter() - t0, "fdtd_designs": problem.fdtd_designs - d0, "best_T": best}
