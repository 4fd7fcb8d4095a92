"""Surrogate kernels on the GPU.

* bz_gemm_bf16 against an f32 matmul of the same bf16 operands: relative L2 error
  <= 1e-5 for f32 outputs (accumulation order only), <= 8e-3 for bf16 outputs;
  every transpose combination, batch sharing, epilogue terms and split-K atomics.
* The FNO (bf16 activations and weights, f32 accumulation) against the float64
  oracle (oracle/fno_ref.py) with the same master weights: outputs within 3e-2
  relative L2; parameter and input gradients (explicit backward) within 6e-2
  relative L2 of the oracle's autograd.
"""
import numpy as np
import pytest
import torch

from oracle import fno_ref

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = torch.as_tensor(a).double().cpu(), torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / max(float(b.norm()), 1e-300))


@pytest.mark.parametrize("ta,tb", [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize("M,N,K", [(37, 45, 70), (200, 30, 64), (24, 300, 19), (130, 260, 96)])
def test_gemm_matches_f32_matmul(bz, ta, tb, M, N, K):
    from beamz_b200 import _native as nat

    g = torch.Generator().manual_seed(M * 7 + N + K)
    batch = 3
    A = torch.randn(batch, M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(batch, K, N, generator=g).to(torch.bfloat16)
    add = torch.randn(batch, M, N, generator=g)
    bm, bn = torch.randn(M, generator=g), torch.randn(N, generator=g)
    want = torch.bmm(A.float(), B.float()) * 0.5 + add + bm[None, :, None] + bn[None, None, :]
    dev = "cuda"
    Ad = (A.transpose(1, 2) if ta else A).contiguous().to(dev)
    Bd = (B.transpose(1, 2) if tb else B).contiguous().to(dev)
    outf = torch.empty(batch, M, N, device=dev)
    outh = torch.empty(batch, M, N, device=dev, dtype=torch.bfloat16)
    pre = torch.empty_like(outh)
    p = nat.Gemm()
    p.M, p.N, p.K, p.batch, p.splitk, p.act, p.ta, p.tb, p.atomic = M, N, K, batch, 1, 0, ta, tb, 0
    p.A, p.lda, p.sa = Ad.data_ptr(), (M if ta else K), M * K
    p.B, p.ldb, p.sb = Bd.data_ptr(), (K if tb else N), K * N
    p.alpha = 0.5
    addd, bmd, bnd = add.to(dev), bm.to(dev), bn.to(dev)
    p.cadd, p.ldadd, p.sadd = addd.data_ptr(), N, M * N
    p.bias_m, p.bias_n = bmd.data_ptr(), bnd.data_ptr()
    p.outf, p.outh, p.ldc, p.sc = outf.data_ptr(), outh.data_ptr(), N, M * N
    p.pre, p.ldpre, p.spre = pre.data_ptr(), N, M * N
    nat.gemm(p, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert rel(outf, want) <= 1e-5
    assert rel(outh.float(), want) <= 8e-3
    # GELU epilogue and split-K atomic accumulation over a shared output
    p.act = 1
    nat.gemm(p, torch.cuda.current_stream().cuda_stream)
    assert rel(outf, fno_ref.gelu(want.double())) <= 1e-5
    assert rel(pre.float(), want) <= 8e-3
    acc = torch.zeros(M, N, device=dev)
    q = nat.Gemm.from_buffer_copy(p)
    q.act, q.cadd, q.bias_m, q.bias_n, q.outh, q.pre = 0, None, None, None, None, None
    q.alpha, q.atomic, q.splitk, q.outf, q.sc = 1.0, 1, 3, acc.data_ptr(), 0
    nat.gemm(q, torch.cuda.current_stream().cuda_stream)
    assert rel(acc, torch.bmm(A.float(), B.float()).sum(0)) <= 1e-5


def _small_fno(bz, seed=0):
    from beamz_b200.surrogate.fno import FNO2d

    return FNO2d(n=24, width=8, modes=4, layers=3, head=16, n_out=5, seed=seed)


def _oracle_params(net):
    return {k: q.w.detach().double().cpu().clone().requires_grad_(True) for k, q in net.params.items()}


def test_fno_forward_and_gradients_match_float64_oracle(bz):
    net = _small_fno(bz)
    g = torch.Generator().manual_seed(3)
    rho = torch.rand(4, 24, 24, generator=g, dtype=torch.float64)
    target = torch.rand(4, 5, generator=g, dtype=torch.float64)
    out = net.forward(rho.cuda(), keep=True)
    params = _oracle_params(net)
    rho_r = rho.clone().requires_grad_(True)
    ref = fno_ref.forward(params, rho_r, 24, 4, 3)
    assert rel(out, ref.detach()) <= 3e-2
    loss = ((ref - target) ** 2).sum()
    loss.backward()
    d_out = 2 * (ref.detach() - target)
    net.zero_grad()
    d_rho = net.backward(d_out.float().cuda(), want_input_grad=True)
    for k, q in net.params.items():
        assert rel(q.g, params[k].grad) <= 6e-2, (k, rel(q.g, params[k].grad))
    assert rel(d_rho, rho_r.grad) <= 6e-2


def test_fno_training_reduces_loss(bz):
    """A few hundred Adam steps on a smooth functional of the density."""
    net = _small_fno(bz, seed=1)
    g = torch.Generator().manual_seed(4)
    rho = torch.rand(64, 24, 24, generator=g)
    w = torch.linspace(0.2, 1.0, 5)
    target = (rho.mean(dim=(1, 2))[:, None] * w[None, :] + 0.1 * rho[:, :12].mean(dim=(1, 2))[:, None]).cuda()
    losses = []
    for it in range(300):
        out = net.forward(rho.cuda(), keep=True)
        err = out - target
        losses.append(float((err ** 2).mean()))
        net.zero_grad()
        net.backward(2 * err / err.numel())
        net.adam_step(lr=3e-3)
    assert losses[-1] < 0.05 * losses[0], (losses[0], losses[-1])


def test_transmission_problem_and_search_loop(bz):
    """The pulsed five-wavelength problem (shortened to 3000 steps): batched FDTD
    transmissions agree with single-design runs and with the adjoint's objective; the
    search loop keeps its best verified design monotone and counts its FDTD designs."""
    from beamz_b200.surrogate.fno import FNO2d
    from beamz_b200.surrogate.topo import SurrogateSearch, TransmissionProblem, densities

    prob = TransmissionProblem(n_steps=3000)
    rho = densities([10000, 10001, 10002])
    T3 = prob.transmission(rho)
    T1 = np.concatenate([prob.transmission(rho[i:i + 1]) for i in range(3)])
    np.testing.assert_allclose(T3, T1, rtol=1e-5)
    assert np.all(T3 >= 0) and np.all(T3 < 1.5)
    T_ref = prob.transmission(prob.kw["rho_straight"][None])
    np.testing.assert_allclose(T_ref, 1.0, rtol=1e-5)
    J, g = prob.value_and_grad(rho[:2])
    np.testing.assert_allclose(J, T3[:2].mean(axis=1), rtol=1e-4)
    assert g.shape == (2, 120, 120) and np.abs(g).max() > 0
    net = FNO2d(width=16, modes=8, layers=2, head=32)
    search = SurrogateSearch(prob, net, n_candidates=32, n_verify=4, n_anchor=2)
    before = prob.fdtd_designs
    hist, secs, best = search.run(rho[0], rounds=2)
    assert all(b >= a for a, b in zip(hist, hist[1:]))
    assert prob.fdtd_designs - before >= 1 + 2 * 4
    assert best.shape == (120, 120) and best.min() >= 0 and best.max() <= 1


@pytest.mark.parametrize("M,N,K,batch,split", [(128, 256, 64, 1, 1), (300, 600, 200, 2, 1), (256, 512, 1000, 1, 3),
                                                (333, 700, 520, 1, 1)])
def test_tcgen05_gemm_matches_mma_sync_and_f32(bz, M, N, K, batch, split):
    """The tcgen05/TMEM kernels (A row-major, B stored [N][K]; engine 0 = TMA-fed for
    batch 1, engine 2 = register-staged) against the mma.sync kernel (engine 1) and an
    f32 matmul of the same bf16 operands: relative L2 <= 1e-5."""
    from beamz_b200 import _native as nat

    g = torch.Generator().manual_seed(M + N + K)
    A = torch.randn(batch, M, K, generator=g).to(torch.bfloat16)
    Bt = torch.randn(batch, N, K, generator=g).to(torch.bfloat16)  # stored [N][K]
    add = torch.randn(batch, M, N, generator=g)
    want = torch.bmm(A.float(), Bt.float().transpose(1, 2))
    dev = "cuda"
    Ad, Bd, addd = A.to(dev), Bt.to(dev), add.to(dev)
    outs = {}
    nat.gemm_error(reset=True)
    for engine in (0, 1, 2):
        p = nat.Gemm()
        p.M, p.N, p.K, p.batch, p.act, p.ta, p.tb, p.engine = M, N, K, batch, 0, 0, 1, engine
        p.A, p.lda, p.sa = Ad.data_ptr(), K, M * K
        p.B, p.ldb, p.sb = Bd.data_ptr(), K, N * K
        p.alpha = 1.0
        if split == 1:
            out = torch.empty(batch, M, N, device=dev)
            p.splitk, p.atomic, p.cadd, p.ldadd, p.sadd = 1, 0, addd.data_ptr(), N, M * N
        else:
            out = torch.zeros(batch, M, N, device=dev)
            p.splitk, p.atomic = split, 1
        p.outf, p.ldc, p.sc = out.data_ptr(), N, M * N
        nat.gemm(p, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        outs[engine] = out
    assert nat.gemm_error(reset=True) == 0
    ref = want + (add if split == 1 else 0)
    for engine in (0, 2):
        assert rel(outs[engine], ref) <= 1e-5, engine
        assert rel(outs[engine], outs[1]) <= 1e-5, engine


@pytest.mark.parametrize("K,M", [(32, 32), (32, 64), (64, 32), (64, 64)])
@pytest.mark.parametrize("ta", [0, 1])
@pytest.mark.parametrize("N", [14400, 200])
def test_tcgen05_channel_mixing_matches_mma_sync_and_f32(bz, K, M, ta, N):
    """The tcgen05 channel-mixing kernel (engine 0: a weight shared by the batch times
    pixel-contiguous activations, X the MN-major operand by TMA) against the mma.sync
    kernel (engine 1) and an f32 matmul of the same bf16 operands, with every epilogue
    term (f32 add, both biases, pre-activation copy, GELU, f32 and bf16 outputs);
    N = 200 leaves a partial 128-pixel tile and a fully out-of-range TMA box."""
    from beamz_b200 import _native as nat

    g = torch.Generator().manual_seed(K * 1000 + M * 10 + ta + N)
    batch = 3
    W = torch.randn(M, K, generator=g).to(torch.bfloat16)
    X = torch.randn(batch, K, N, generator=g).to(torch.bfloat16)
    add = torch.randn(batch, M, N, generator=g)
    bm, bn = torch.randn(M, generator=g), torch.randn(N, generator=g)
    lin = torch.einsum("mk,bkn->bmn", W.float(), X.float()) * 0.5 + add + bm[None, :, None] + bn[None, None, :]
    dev = "cuda"
    Wd = (W.t() if ta else W).contiguous().to(dev)
    Xd, addd, bmd, bnd = X.to(dev), add.to(dev), bm.to(dev), bn.to(dev)
    res = {}
    nat.gemm_error(reset=True)
    for engine in (0, 1):
        outf = torch.empty(batch, M, N, device=dev)
        outh = torch.empty(batch, M, N, device=dev, dtype=torch.bfloat16)
        pre = torch.empty_like(outh)
        p = nat.Gemm()
        p.M, p.N, p.K, p.batch, p.splitk, p.act, p.ta, p.tb, p.atomic = M, N, K, batch, 1, 1, ta, 0, 0
        p.engine = engine
        p.A, p.lda, p.sa = Wd.data_ptr(), (M if ta else K), 0
        p.B, p.ldb, p.sb = Xd.data_ptr(), N, K * N
        p.alpha = 0.5
        p.cadd, p.ldadd, p.sadd = addd.data_ptr(), N, M * N
        p.bias_m, p.bias_n = bmd.data_ptr(), bnd.data_ptr()
        p.outf, p.outh, p.ldc, p.sc = outf.data_ptr(), outh.data_ptr(), N, M * N
        p.pre, p.ldpre, p.spre = pre.data_ptr(), N, M * N
        nat.gemm(p, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        res[engine] = (outf, outh, pre)
    assert nat.gemm_error(reset=True) == 0
    want = fno_ref.gelu(lin.double())
    outf, outh, pre = res[0]
    assert rel(outf, want) <= 1e-5
    assert rel(outh.float(), want) <= 8e-3
    assert rel(pre.float(), lin) <= 8e-3
    assert rel(outf, res[1][0]) <= 1e-5


@pytest.mark.parametrize("B,ci,co,nk", [(64, 32, 32, 512), (5, 8, 8, 30), (19, 12, 20, 37)])
def test_spectral_mixing_kernels_match_complex_products(bz, B, ci, co, nk):
    """bz_spectral_mix / bz_spectral_mix_bwd against complex float64 products of the same
    bf16 values: O = sum_c U W, dU = sum_o dO conj(W), dW += sum_b dO conj(U). Shapes
    cover mode counts that leave a partial group of four modes, batches that leave a
    partial chunk, and channel counts that are not powers of two."""
    from beamz_b200 import _native as nat

    g = torch.Generator().manual_seed(B * 100 + ci + co + nk)
    U = torch.randn(B, ci, nk, 2, generator=g).to(torch.bfloat16)
    W = (torch.randn(nk, ci, co, 2, generator=g) / ci ** 0.5).to(torch.bfloat16)
    dO = torch.randn(B, co, nk, 2, generator=g).to(torch.bfloat16)
    dW0 = torch.randn(nk, ci, co, 2, generator=g)
    cU = torch.view_as_complex(U.double().contiguous())
    cW = torch.view_as_complex(W.double().contiguous())
    cG = torch.view_as_complex(dO.double().contiguous())
    want_O = torch.einsum("bck,kco->bok", cU, cW)
    want_dU = torch.einsum("bok,kco->bck", cG, cW.conj())
    want_dW = dW0.double() + torch.view_as_real(torch.einsum("bok,bck->kco", cG, cU.conj()))
    dev = "cuda"
    Ud, Wd, dOd = U.to(dev), W.to(dev), dO.to(dev)
    O = torch.empty(B, co, nk, 2, dtype=torch.bfloat16, device=dev)
    dU = torch.empty(B, ci, nk, 2, dtype=torch.bfloat16, device=dev)
    dW = dW0.to(dev)
    st = torch.cuda.current_stream().cuda_stream
    nat.spectral_mix(Ud.data_ptr(), Wd.data_ptr(), O.data_ptr(), B, ci, co, nk, st)
    nat.spectral_mix_bwd(dOd.data_ptr(), Ud.data_ptr(), Wd.data_ptr(), dU.data_ptr(), dW.data_ptr(), B, ci, co, nk,
                         st)
    torch.cuda.synchronize()
    assert rel(O.double(), torch.view_as_real(want_O)) <= 8e-3
    assert rel(dU.double(), torch.view_as_real(want_dU)) <= 8e-3
    assert rel(dW, want_dW) <= 1e-5


@pytest.mark.parametrize("B,C,P", [(4, 8, 576), (3, 5, 37)])
def test_elementwise_surrogate_kernels(bz, B, C, P):
    """GELU backward, per-channel sums and the per-row broadcast against torch on the same
    bf16 values; P = 576 takes the 16-byte paths, P = 37 the scalar ones."""
    from beamz_b200 import _native as nat

    g = torch.Generator().manual_seed(B + C + P)
    dy = torch.randn(B, C, P, generator=g).to(torch.bfloat16)
    pre = torch.randn(B, C, P, generator=g).to(torch.bfloat16)
    rows = torch.randn(B * C, generator=g)
    pre64 = pre.double().requires_grad_(True)
    fno_ref.gelu(pre64).backward(dy.double())
    dev, st = "cuda", torch.cuda.current_stream().cuda_stream
    dyd, pred = dy.to(dev), pre.to(dev)
    dx = torch.empty_like(dyd)
    nat.gelu_bwd(dyd.data_ptr(), pred.data_ptr(), dx.data_ptr(), dx.numel(), st)
    sums = torch.full((C,), 0.5, device=dev)
    nat.chan_sum(dyd.data_ptr(), sums.data_ptr(), B, C, P, st)
    bc = torch.empty(B * C, P, dtype=torch.bfloat16, device=dev)
    rows_d = rows.to(dev)
    nat.row_broadcast(rows_d.data_ptr(), bc.data_ptr(), B * C, P, 0.25, st)
    torch.cuda.synchronize()
    assert rel(dx.float(), pre64.grad) <= 8e-3
    assert rel(sums, 0.5 + dy.double().sum(dim=(0, 2))) <= 1e-5
    assert torch.equal(bc.cpu(), (rows * 0.25).to(torch.bfloat16)[:, None].expand(B * C, P))


@pytest.mark.parametrize("M,N,K", [(32, 32, 14400), (64, 32, 1000), (32, 64, 4096)])
def test_tcgen05_weight_gradient_matches_mma_sync_and_f32(bz, M, N, K):
    """The tcgen05 weight-gradient kernel (engine 0: outf += sum_b A[b] B[b]^T with both
    operands pixel-contiguous) against the mma.sync kernel (engine 1, split-K 3) and an
    f32 sum of the same bf16 values, accumulating onto a nonzero output; K = 1000 leaves
    a partial 64-pixel item."""
    from beamz_b200 import _native as nat

    g = torch.Generator().manual_seed(M + N + K)
    batch = 5
    A = torch.randn(batch, M, K, generator=g).to(torch.bfloat16)
    Bm = torch.randn(batch, N, K, generator=g).to(torch.bfloat16)
    init = torch.randn(M, N, generator=g)
    want = init.double() + 0.5 * torch.einsum("bmk,bnk->mn", A.double(), Bm.double())
    dev = "cuda"
    Ad, Bd = A.to(dev), Bm.to(dev)
    outs = {}
    nat.gemm_error(reset=True)
    for engine in (0, 1):
        out = init.to(dev)
        p = nat.Gemm()
        p.M, p.N, p.K, p.batch, p.splitk, p.act, p.ta, p.tb, p.atomic = M, N, K, batch, 3, 0, 0, 1, 1
        p.engine = engine
        p.A, p.lda, p.sa = Ad.data_ptr(), K, M * K
        p.B, p.ldb, p.sb = Bd.data_ptr(), K, N * K
        p.alpha = 0.5
        p.outf, p.ldc, p.sc = out.data_ptr(), N, 0
        nat.gemm(p, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        outs[engine] = out
    assert nat.gemm_error(reset=True) == 0
    assert rel(outs[0], want) <= 1e-5
    assert rel(outs[0], outs[1]) <= 1e-5


@pytest.mark.parametrize("K,M,N", [(32, 32, 14400), (32, 64, 200)])
def test_channel_mixing_with_bf16_term(bz, K, M, N):
    """The mixing kernel and the mma.sync kernel with the added term given in bf16
    (cadd_h), as the surrogate passes its spectral branch: against f32 of the same values."""
    from beamz_b200 import _native as nat

    g = torch.Generator().manual_seed(K + M + N)
    batch = 3
    W = torch.randn(M, K, generator=g).to(torch.bfloat16)
    X = torch.randn(batch, K, N, generator=g).to(torch.bfloat16)
    add = torch.randn(batch, M, N, generator=g).to(torch.bfloat16)
    want = torch.einsum("mk,bkn->bmn", W.float(), X.float()) + add.float()
    dev = "cuda"
    Wd, Xd, addd = W.to(dev), X.to(dev), add.to(dev)
    for engine in (0, 1):
        outh = torch.empty(batch, M, N, device=dev, dtype=torch.bfloat16)
        p = nat.Gemm()
        p.M, p.N, p.K, p.batch, p.splitk, p.act, p.ta, p.tb, p.atomic = M, N, K, batch, 1, 0, 0, 0, 0
        p.engine = engine
        p.A, p.lda, p.sa = Wd.data_ptr(), K, 0
        p.B, p.ldb, p.sb = Xd.data_ptr(), N, K * N
        p.alpha = 1.0
        p.cadd_h, p.ldadd, p.sadd = addd.data_ptr(), N, M * N
        p.outh, p.ldc, p.sc = outh.data_ptr(), N, M * N
        nat.gemm(p, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        assert rel(outh.float(), want) <= 8e-3, engine


def test_tma_gemm_plain_bf16_output(bz):
    """The TMA-fed tcgen05 GEMM storing bf16 only (16-byte stores per 8 columns, the
    surrogate's inverse transform): against f32 of the same bf16 operands, with a partial
    last column tile."""
    from beamz_b200 import _native as nat

    M, N, K = 256, 600, 192
    g = torch.Generator().manual_seed(11)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    Bt = torch.randn(N, K, generator=g).to(torch.bfloat16)
    want = A.float() @ Bt.float().t()
    dev = "cuda"
    Ad, Bd = A.to(dev), Bt.to(dev)
    outh = torch.empty(M, N, device=dev, dtype=torch.bfloat16)
    p = nat.Gemm()
    p.M, p.N, p.K, p.batch, p.splitk, p.act, p.ta, p.tb, p.atomic, p.engine = M, N, K, 1, 1, 0, 0, 1, 0, 0
    p.A, p.lda, p.B, p.ldb = Ad.data_ptr(), K, Bd.data_ptr(), K
    p.alpha = 1.0
    p.outh, p.ldc = outh.data_ptr(), N
    nat.gemm_error(reset=True)
    nat.gemm(p, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert nat.gemm_error(reset=True) == 0
    assert rel(outh.float(), want) <= 8e-3


def test_fno_with_tcgen05_spectral_gemms_matches_oracle(bz):
    """n = 64, 8 modes, width 32, batch 8: the DFT GEMMs (M = 256, N = 256, K = 4096)
    and their inverses run on the tcgen05 kernel."""
    from beamz_b200 import _native as nat
    from beamz_b200.surrogate.fno import FNO2d

    net = FNO2d(n=64, width=32, modes=8, layers=2, head=16, n_out=5, seed=2)
    g = torch.Generator().manual_seed(5)
    rho = torch.rand(8, 64, 64, generator=g, dtype=torch.float64)
    target = torch.rand(8, 5, generator=g, dtype=torch.float64)
    out = net.forward(rho.cuda(), keep=True)
    params = _oracle_params(net)
    rho_r = rho.clone().requires_grad_(True)
    ref = fno_ref.forward(params, rho_r, 64, 8, 2)
    assert rel(out, ref.detach()) <= 3e-2
    ((ref - target) ** 2).sum().backward()
    net.zero_grad()
    d_rho = net.backward((2 * (ref.detach() - target)).float().cuda(), want_input_grad=True)
    for k, q in net.params.items():
        assert rel(q.g, params[k].grad) <= 6e-2, (k, rel(q.g, params[k].grad))
    assert rel(d_rho, rho_r.grad) <= 6e-2
    assert nat.gemm_error(reset=True) == 0


def test_surrogate_search_reaches_plain_adjoint_transmission(bz):
    """A reduced surrogate run (the 8000-step problem, 8192 FDTD-labelled samples of
    which half come from batched exact-adjoint ascents, 15 epochs). From the same start,
    the surrogate search reaches the final mean transmission of a 15-iteration plain
    per-design adjoint ascent within 1e-3 with fewer solver runs (a batched forward of
    the verified candidates and one adjoint run per round, against one forward + adjoint
    run per plain iteration), and in less wall time than the same search without the
    network (exact-gradient steps only). The wall time against the plain ascent is
    printed, not asserted: it varies between runs around parity (see the C5 bench line)."""
    from beamz_b200.surrogate.fno import FNO2d
    from beamz_b200.surrogate.topo import SurrogateSearch, TransmissionProblem, densities, make_dataset
    from beamz_b200.surrogate.topo import plain_adjoint, train

    prob = TransmissionProblem(n_steps=8000)
    rho, T = make_dataset(prob, 8192, trajectory_frac=0.5)
    net = FNO2d()
    train(net, rho, T, epochs=15)
    rho0 = densities([1234])[0]
    plain_adjoint(prob, rho0, 2)  # warm both problem sizes up
    r0 = prob.fdtd_runs
    hist_p, sec_p, _ = plain_adjoint(prob, rho0, 15)
    runs_p = prob.fdtd_runs - r0
    target = hist_p[-1] - 1e-3
    res = {}
    for use in (True, False):
        search = SurrogateSearch(prob, net, replay=(rho, T), use_surrogate=use)
        r0 = prob.fdtd_runs
        hist, sec, _ = search.run(rho0, rounds=30, target=target)
        res[use] = (hist[-1], sec, prob.fdtd_runs - r0, len(hist) - 1)
    print(f"plain: T {hist_p[-1]:.4f} in {sec_p:.3f} s, {runs_p} solver runs; surrogate: T {res[True][0]:.4f} in "
          f"{res[True][1]:.3f} s, {res[True][2]} runs, {res[True][3]} rounds; without network: T {res[False][0]:.4f} "
          f"in {res[False][1]:.3f} s, {res[False][2]} runs; wall-time ratio plain / surrogate "
          f"{sec_p / res[True][1]:.2f}")
    T_s, sec_s, runs_s, _ = res[True]
    assert T_s >= target
    assert runs_s < runs_p
    assert sec_s < res[False][1] and res[False][0] >= target
