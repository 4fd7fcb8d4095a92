"""Fourier neural operator over a square design density, on the library's bf16 kernels.

Maps a density rho (B, n, n) in [0, 1] to n_out values (transmission at n_out
wavelengths). Layout: activations are channels-first [B][C][P] (P = n*n pixels,
x fastest), bf16; accumulation is f32 everywhere; master weights are f32 with bf16
copies for the kernels.

Layers (the 2D FNO of Li et al. 2021 with a pooled head):
  lift      V0 = W0 [rho, x/n, y/n] + b0                       (C x 3 pointwise)
  Fourier   V' = act(W V + b + IDFT(R * DFT(V)))               (act = GELU except last)
  head      T  = Q2 mean_p(GELU(Q1 V + q1)) + q2
DFT/IDFT are one GEMM each against fixed bf16 bases over the kept modes
(ky in [-m, m), kx in [0, m): 2m*m complex modes = 4m^2 real columns), so the
spectral transform runs on the tensor cores; R is a complex C x C matrix per mode.
Backward is written out layer by layer with the same kernels (no autograd).
"""
from __future__ import annotations

import math

import numpy as np
import torch

from .. import _native as nat

BF16 = torch.bfloat16


def spectral_bases(n: int, modes: int):
    """Forward basis F [P][2K] (cos, -sin of each mode) and inverse basis G [2K][P]
    (Hermitian weights w = 1 for kx = 0 else 2, divided by P), float64."""
    ky = np.concatenate([np.arange(modes), np.arange(n - modes, n)])
    kx = np.arange(modes)
    KY, KX = np.meshgrid(ky, kx, indexing="ij")
    KY, KX = KY.ravel(), KX.ravel()  # K = 2m*m modes
    y, x = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    th = 2 * np.pi * (np.outer(y.ravel(), KY) + np.outer(x.ravel(), KX)) / n  # [P][K]
    F = np.empty((n * n, 2 * len(KY)))
    F[:, 0::2] = np.cos(th)
    F[:, 1::2] = -np.sin(th)
    w = np.where(KX == 0, 1.0, 2.0) / (n * n)
    G = np.empty((2 * len(KY), n * n))
    G[0::2] = (w[:, None] * np.cos(th.T))
    G[1::2] = (-w[:, None] * np.sin(th.T))
    return F, G


class _Param:
    def __init__(self, value: torch.Tensor):
        self.w = value.float().contiguous()
        self.h = self.w.to(BF16)
        self.g = torch.zeros_like(self.w)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)


def _p(t: torch.Tensor) -> int:
    return t.data_ptr() if t is not None else None


class FNO2d:
    def __init__(self, n=120, width=32, modes=16, layers=4, head=64, n_out=5, seed=0, device=None):
        self.dev = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.n, self.C, self.modes, self.L, self.Hd, self.n_out = n, width, modes, layers, head, n_out
        self.P = n * n
        self.K = 2 * modes * modes
        F, G = spectral_bases(n, modes)
        self.F = torch.as_tensor(F, dtype=torch.float32).to(self.dev).to(BF16)
        self.G = torch.as_tensor(G, dtype=torch.float32).to(self.dev).to(BF16)
        # transposed copies: every large GEMM then reads its B operand K-contiguous
        self.FT = self.F.t().contiguous()  # [2K][P]
        self.GT = self.G.t().contiguous()  # [P][2K]
        gen = torch.Generator().manual_seed(seed)
        C, Hd = width, head

        def rnd(*shape, scale):
            return (torch.randn(*shape, generator=gen, dtype=torch.float64) * scale).to(self.dev)

        self.params = {"W0": _Param(rnd(C, 3, scale=1 / math.sqrt(3))), "b0": _Param(rnd(C, scale=0.0))}
        for l in range(layers):
            self.params[f"W{l + 1}"] = _Param(rnd(C, C, scale=1 / math.sqrt(C)))
            self.params[f"b{l + 1}"] = _Param(rnd(C, scale=0.0))
            # the forward basis is unnormalised and the inverse carries 1/P, so R ~ 1/C keeps
            # the spectral branch at the scale of the pointwise one
            r = torch.randn(self.K, C, C, 2, generator=gen, dtype=torch.float64) / C
            self.params[f"R{l + 1}"] = _Param(r.to(self.dev))
        self.params["Q1"] = _Param(rnd(Hd, C, scale=1 / math.sqrt(C)))
        self.params["q1"] = _Param(rnd(Hd, scale=0.0))
        self.params["Q2"] = _Param(rnd(n_out, Hd, scale=1 / math.sqrt(Hd)))
        self.params["q2"] = _Param(rnd(n_out, scale=0.0))
        # outputs are y = raw * y_scale + y_shift (targets standardised for training)
        self.y_scale = torch.ones(n_out, device=self.dev)
        self.y_shift = torch.zeros(n_out, device=self.dev)
        self.step_count = 0
        self._acts = None
        self.flops = 0.0  # tensor-core FLOPs issued (2*M*N*K per GEMM), for throughput reports

    # ---- kernel helpers ---------------------------------------------------------------
    @staticmethod
    def _stream() -> int:
        return torch.cuda.current_stream().cuda_stream

    def _gemm(self, M, N, K, A, lda, B, ldb, *, batch=1, sa=0, sb=0, ta=0, tb=0, outf=None, outh=None, ldc=None,
              sc=0, cadd=None, cadd_h=None, ldadd=0, sadd=0, bias_m=None, bias_n=None, act=0, pre=None, atomic=0,
              splitk=1, alpha=1.0):
        g = nat.Gemm()
        g.M, g.N, g.K, g.batch, g.splitk, g.act = M, N, K, batch, splitk, act
        g.ta, g.tb, g.atomic = ta, tb, atomic
        g.A, g.lda, g.sa, g.B, g.ldb, g.sb = _p(A), lda, sa, _p(B), ldb, sb
        g.alpha = alpha
        g.cadd, g.cadd_h, g.ldadd, g.sadd = _p(cadd), _p(cadd_h), ldadd, sadd
        g.bias_m, g.bias_n = _p(bias_m), _p(bias_n)
        g.outf, g.outh = _p(outf), _p(outh)
        g.ldc, g.sc = (N if ldc is None else ldc), sc
        g.pre, g.ldpre, g.spre = _p(pre), (N if ldc is None else ldc), sc
        nat.gemm(g, self._stream())
        self.flops += 2.0 * M * N * K * batch

    @staticmethod
    def _split(M, N):
        """K splits giving about one CTA of 128 x 256 output tiles per SM (the TMA GEMM
        holds one CTA per SM)."""
        return max(1, min(16, 148 // max(1, ((M + 127) // 128) * ((N + 255) // 256))))

    def _dft(self, V, B):
        """U = V [B*C x P] @ F [P x 2K] (split over P, f32 atomics) -> bf16."""
        BC, K2 = B * self.C, 2 * self.K
        acc = torch.zeros((BC, K2), dtype=torch.float32, device=self.dev)
        self._gemm(BC, K2, self.P, V, self.P, self.FT, self.P, tb=1, outf=acc, atomic=1, splitk=self._split(BC, K2))
        out = torch.empty((BC, K2), dtype=BF16, device=self.dev)
        nat.to_bf16(acc.data_ptr(), out.data_ptr(), acc.numel(), self._stream())
        return out

    def _dft_t(self, D, B):
        """D [B*C x P] @ G^T -> bf16 [B*C x 2K] (gradient through the inverse transform)."""
        BC, K2 = B * self.C, 2 * self.K
        acc = torch.zeros((BC, K2), dtype=torch.float32, device=self.dev)
        self._gemm(BC, K2, self.P, D, self.P, self.G, self.P, tb=1, outf=acc, atomic=1, splitk=self._split(BC, K2))
        out = torch.empty((BC, K2), dtype=BF16, device=self.dev)
        nat.to_bf16(acc.data_ptr(), out.data_ptr(), acc.numel(), self._stream())
        return out

    def _inputs(self, rho: torch.Tensor) -> torch.Tensor:
        B, n = rho.shape[0], self.n
        c = (torch.arange(n, device=self.dev, dtype=torch.float32) + 0.5) / n
        X = torch.empty((B, 3, n, n), dtype=torch.float32, device=self.dev)
        X[:, 0] = rho.to(self.dev, torch.float32)
        X[:, 1] = c[None, None, :]
        X[:, 2] = c[None, :, None]
        return X.reshape(B, 3, self.P).to(BF16).contiguous()

    # ---- forward ------------------------------------------------------------------------
    def forward(self, rho, keep=False) -> torch.Tensor:
        """Predictions (B, n_out) float32 for densities rho (B, n, n)."""
        p, C, P, Hd = self.params, self.C, self.P, self.Hd
        B = rho.shape[0]
        X = self._inputs(rho)
        V = torch.empty((B, C, P), dtype=BF16, device=self.dev)
        self._gemm(C, P, 3, p["W0"].h, 3, X, P, batch=B, sb=3 * P, outh=V, sc=C * P, bias_m=p["b0"].w)
        acts = {"X": X, "V": [V], "U": [], "pre": []}
        for l in range(1, self.L + 1):
            U = self._dft(V, B)
            O = torch.empty_like(U)
            nat.spectral_mix(U.data_ptr(), p[f"R{l}"].h.data_ptr(), O.data_ptr(), B, C, C, self.K, self._stream())
            # the spectral branch in bf16 (half the bytes of the write and of its read-back)
            S = torch.empty((B * C, P), dtype=BF16, device=self.dev)
            self._gemm(B * C, P, 2 * self.K, O, 2 * self.K, self.GT, 2 * self.K, tb=1, outh=S)
            act = 1 if l < self.L else 0
            pre = torch.empty((B, C, P), dtype=BF16, device=self.dev) if act else None
            Vn = torch.empty((B, C, P), dtype=BF16, device=self.dev)
            self._gemm(C, P, C, p[f"W{l}"].h, C, V, P, batch=B, sb=C * P, outh=Vn, sc=C * P, cadd_h=S, ldadd=P,
                       sadd=C * P, bias_m=p[f"b{l}"].w, act=act, pre=pre)
            del S
            acts["U"].append(U)
            acts["pre"].append(pre)
            acts["V"].append(Vn)
            V = Vn
        Hh = torch.empty((B, Hd, P), dtype=BF16, device=self.dev)
        preh = torch.empty_like(Hh)
        self._gemm(Hd, P, C, p["Q1"].h, C, V, P, batch=B, sb=C * P, outh=Hh, sc=Hd * P, bias_m=p["q1"].w, act=1,
                   pre=preh)
        pooled = torch.empty((B, Hd), dtype=torch.float32, device=self.dev)
        nat.row_mean(Hh.data_ptr(), pooled.data_ptr(), B * Hd, P, 1.0 / P, self._stream())
        pooled_h = pooled.to(BF16)
        out = torch.empty((B, self.n_out), dtype=torch.float32, device=self.dev)
        self._gemm(B, self.n_out, Hd, pooled_h, Hd, p["Q2"].h, Hd, tb=1, outf=out, bias_n=p["q2"].w)
        out = out * self.y_scale[None, :] + self.y_shift[None, :]
        if keep:
            acts.update(preh=preh, pooled_h=pooled_h, B=B)
            self._acts = acts
        else:
            self._acts = None
        return out

    # ---- backward -----------------------------------------------------------------------
    def backward(self, d_out: torch.Tensor, want_input_grad=False):
        """Accumulates parameter gradients (.g) for d loss / d out (B, n_out) of the last
        forward(keep=True); returns d loss / d rho (B, n, n) float32 if asked."""
        a = self._acts
        if a is None:
            raise RuntimeError("backward needs forward(..., keep=True)")
        p, C, P, Hd, B = self.params, self.C, self.P, self.Hd, a["B"]
        st = self._stream()
        split = lambda k: max(1, min(16, k // 2048))  # noqa: E731
        dO = (d_out.float() * self.y_scale[None, :]).contiguous()
        dOh = dO.to(BF16)
        p["q2"].g += dO.sum(0)
        self._gemm(self.n_out, Hd, B, dOh, self.n_out, a["pooled_h"], Hd, ta=1, outf=p["Q2"].g, atomic=1)
        dpool = torch.empty((B, Hd), dtype=torch.float32, device=self.dev)
        self._gemm(B, Hd, self.n_out, dOh, self.n_out, p["Q2"].h, Hd, outf=dpool)
        dH = torch.empty((B, Hd, P), dtype=BF16, device=self.dev)
        nat.row_broadcast(dpool.data_ptr(), dH.data_ptr(), B * Hd, P, 1.0 / P, st)
        nat.gelu_bwd(dH.data_ptr(), a["preh"].data_ptr(), dH.data_ptr(), dH.numel(), st)
        nat.chan_sum(dH.data_ptr(), p["q1"].g.data_ptr(), B, Hd, P, st)
        V = a["V"][-1]
        self._gemm(Hd, C, P, dH, P, V, P, tb=1, batch=B, sa=Hd * P, sb=C * P, outf=p["Q1"].g, sc=0, atomic=1,
                   splitk=split(P))
        dV = torch.empty((B, C, P), dtype=BF16, device=self.dev)
        self._gemm(C, P, Hd, p["Q1"].h, C, dH, P, ta=1, batch=B, sb=Hd * P, outh=dV, sc=C * P)
        del dH
        for l in range(self.L, 0, -1):
            pre = a["pre"][l - 1]
            if pre is not None:
                nat.gelu_bwd(dV.data_ptr(), pre.data_ptr(), dV.data_ptr(), dV.numel(), st)
            nat.chan_sum(dV.data_ptr(), p[f"b{l}"].g.data_ptr(), B, C, P, st)
            Vin = a["V"][l - 1]
            self._gemm(C, C, P, dV, P, Vin, P, tb=1, batch=B, sa=C * P, sb=C * P, outf=p[f"W{l}"].g, sc=0, atomic=1,
                       splitk=split(P))
            dOm = self._dft_t(dV, B)
            dU = torch.empty_like(dOm)
            nat.spectral_mix_bwd(dOm.data_ptr(), a["U"][l - 1].data_ptr(), p[f"R{l}"].h.data_ptr(), dU.data_ptr(),
                                 p[f"R{l}"].g.data_ptr(), B, C, C, self.K, st)
            dVs = torch.empty((B * C, P), dtype=BF16, device=self.dev)
            self._gemm(B * C, P, 2 * self.K, dU, 2 * self.K, self.F, 2 * self.K, tb=1, outh=dVs)
            dVn = torch.empty((B, C, P), dtype=BF16, device=self.dev)
            self._gemm(C, P, C, p[f"W{l}"].h, C, dV, P, ta=1, batch=B, sb=C * P, outh=dVn, sc=C * P, cadd_h=dVs,
                       ldadd=P, sadd=C * P)
            dV = dVn
        nat.chan_sum(dV.data_ptr(), p["b0"].g.data_ptr(), B, C, P, st)
        self._gemm(C, 3, P, dV, P, a["X"], P, tb=1, batch=B, sa=C * P, sb=3 * P, outf=p["W0"].g, sc=0, atomic=1,
                   splitk=split(P))
        if not want_input_grad:
            return None
        dX = torch.empty((B, 3, P), dtype=torch.float32, device=self.dev)
        self._gemm(3, P, C, p["W0"].h, 3, dV, P, ta=1, batch=B, sb=C * P, outf=dX, sc=3 * P)
        return dX[:, 0].reshape(B, self.n, self.n)

    # ---- optimiser ----------------------------------------------------------------------
    def zero_grad(self):
        for q in self.params.values():
            q.g.zero_()

    def adam_step(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8, weight_decay=0.0):
        self.step_count += 1
        for q in self.params.values():
            nat.adam(q.w.data_ptr(), q.g.data_ptr(), q.m.data_ptr(), q.v.data_ptr(), q.h.data_ptr(), q.w.numel(), lr,
                     b1, b2, eps, self.step_count, weight_decay, self._stream())

    def state_dict(self) -> dict:
        sd = {k: q.w.detach().cpu().clone() for k, q in self.params.items()}
        sd["_y_scale"], sd["_y_shift"] = self.y_scale.cpu().clone(), self.y_shift.cpu().clone()
        return sd

    def load_state_dict(self, sd: dict):
        for k, v in sd.items():
            if k == "_y_scale":
                self.y_scale.copy_(v.to(self.dev))
            elif k == "_y_shift":
                self.y_shift.copy_(v.to(self.dev))
            else:
                q = self.params[k]
                q.w.copy_(v.to(q.w.device))
                q.h.copy_(q.w.to(BF16))


def bench_step(batch: int = 64, steps: int = 10, warmup: int = 3) -> float:
    """Milliseconds per training step (forward, backward, Adam) of the default FNO on
    ``batch`` random 120 x 120 densities, timed with CUDA events."""
    net = FNO2d()
    rho = torch.rand((batch, 120, 120), device=net.dev)

    def step():
        out = net.forward(rho, keep=True)
        net.backward(2 * (out - 0.5) / out.numel())
        net.adam_step()

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record()
    for _ in range(steps):
        step()
    b.record()
    torch.cuda.synchronize()
    return a.elapsed_time(b) / max(1, steps)


def bench_mixing(reps: int = 20) -> list:
    """The 1x1 channel-mixing GEMMs of the default FNO at batch 64 (120 x 120 pixels)
    through bz_gemm_bf16 with engine 0 (the tcgen05 mixing kernel) and engine 1
    (mma.sync): microseconds per launch (CUDA events over ``reps`` back-to-back launches,
    operands and outputs of 120-300 MB, above the 126 MB L2) and the algorithmic bytes
    per second (activations read, f32 term read, pre-activation and output written)."""
    dev = torch.device("cuda")
    B, P = 64, 120 * 120
    st = torch.cuda.current_stream().cuda_stream
    rows = []
    # (M, K, ta, fused): the forward layer (f32 term, bias, pre-activation, GELU), the head's
    # first layer, the head's transposed layer in the backward, a transposed layer with
    # the f32 term (backward through a Fourier layer)
    for M, K, ta, fused in ((32, 32, 0, True), (64, 32, 0, True), (32, 64, 1, False), (32, 32, 1, True)):
        W = torch.randn(M, K, device=dev).to(BF16)
        Wd = (W.t() if ta else W).contiguous()
        X = torch.randn(B, K, P, device=dev).to(BF16)
        add = torch.randn(B, M, P, device=dev) if fused else None
        bias = torch.randn(M, device=dev)
        outh = torch.empty(B, M, P, device=dev, dtype=BF16)
        pre = torch.empty_like(outh) if fused else None
        row = {"M": M, "K": K, "ta": ta, "fused": fused}
        for engine in (0, 1):
            g = nat.Gemm()
            g.M, g.N, g.K, g.batch, g.splitk, g.act, g.ta, g.tb, g.atomic = M, P, K, B, 1, int(fused), ta, 0, 0
            g.engine = engine
            g.A, g.lda, g.sa = Wd.data_ptr(), (M if ta else K), 0
            g.B, g.ldb, g.sb = X.data_ptr(), P, K * P
            g.alpha = 1.0
            if fused:
                g.cadd, g.ldadd, g.sadd = add.data_ptr(), P, M * P
                g.bias_m = bias.data_ptr()
                g.pre, g.ldpre, g.spre = pre.data_ptr(), P, M * P
            g.outh, g.ldc, g.sc = outh.data_ptr(), P, M * P
            for _ in range(3):
                nat.gemm(g, st)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                nat.gemm(g, st)
            b.record()
            torch.cuda.synchronize()
            us = a.elapsed_time(b) / reps * 1e3
            nbytes = B * P * (2 * K + 2 * M + (6 * M if fused else 0))
            row["tcgen05_us" if engine == 0 else "mma_sync_us"] = round(us, 1)
            row["tcgen05_gbs" if engine == 0 else "mma_sync_gbs"] = round(nbytes / us / 1e3)
        rows.append(row)
    return rows
