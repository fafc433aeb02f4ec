"""Device Newton driver and the warm-start MLP kernels.

* BF16 tensor-core GEMM vs float64 products of the same BF16 inputs
  (tolerance 1e-5 relative: FP32 accumulation);
* MLP forward / backward vs the CPU oracle (oracle/mlp.py) with BF16
  rounding at the same points (tolerance 2e-3 relative);
* Newton + golden-section line search reaches the 1e-6 relative gradient
  tolerance on p-Laplace and Ginzburg-Landau, with the energy matching the
  CPU oracle's energy at the returned point.
"""

import numpy as np
import pytest
import torch

from oracle import mlp as omlp
from oracle.assembler import OracleAssembler
from fenics_nonlinear_energies_b200 import meshes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(64, 64, 32), (200, 96, 40), (1, 7, 300), (513, 257, 129), (8192, 256, 256),
                                   (300, 3, 256), (5, 33, 12), (130, 32, 0)])
@pytest.mark.parametrize("transA", [False, True])
@pytest.mark.parametrize("transB", [False, True])
def test_gemm_bf16(M, N, K, transA, transB):
    from fenics_nonlinear_energies_b200.warmstart import gemm

    g = torch.Generator().manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16)
    B = torch.randn(K, N, generator=g).to(torch.bfloat16)
    ref = A.double() @ B.double()
    Ad = (A.t().contiguous() if transA else A).cuda()
    Bd = (B.t().contiguous() if transB else B).cuda()
    sam, sak = (1, M) if transA else (K, 1)
    sbk, sbn = (1, K) if transB else (N, 1)
    C = torch.full((M, N), 3.0, dtype=torch.float32, device="cuda")
    gemm(Ad, sam, sak, Bd, sbk, sbn, M, N, K, C, beta=0.5)
    got = C.double().cpu() - 1.5
    assert (got - ref).abs().max() <= 1e-5 * ref.abs().max() + 1e-5


def test_gemm_wait_timeout_is_reported():
    """The tensor-core GEMM's MMA-completion wait, set to give up at once:
    fne_gemm_check_status reports FNE_ETIMEOUT (then cleared), and with the
    default bound restored the next product is exact again."""
    from fenics_nonlinear_energies_b200 import _lib
    from fenics_nonlinear_energies_b200.warmstart import gemm

    A = torch.randn(256, 64).to(torch.bfloat16)
    B = torch.randn(64, 128).to(torch.bfloat16)
    C = torch.zeros(256, 128, dtype=torch.float32, device="cuda")
    _lib.check(_lib.lib.fne_gemm_set_wait_limit(0))
    try:
        gemm(A.cuda(), 64, 1, B.cuda(), 128, 1, 256, 128, 64, C)
        torch.cuda.synchronize()
        assert _lib.lib.fne_gemm_check_status() == _lib.FNE_ETIMEOUT
        assert _lib.lib.fne_gemm_check_status() == _lib.FNE_OK
    finally:
        _lib.check(_lib.lib.fne_gemm_set_wait_limit(-1))
    gemm(A.cuda(), 64, 1, B.cuda(), 128, 1, 256, 128, 64, C)
    torch.cuda.synchronize()
    assert _lib.lib.fne_gemm_check_status() == _lib.FNE_OK
    ref = A.double() @ B.double()
    assert (C.double().cpu() - ref).abs().max() <= 1e-5 * ref.abs().max()


def test_mlp_forward_backward_match_oracle():
    from fenics_nonlinear_energies_b200.warmstart import BF16, NodalMLP

    mlp = NodalMLP((12, 64, 64, 64, 3), seed=3)
    rng = np.random.default_rng(0)
    X = rng.standard_normal((333, 12)).astype(np.float32)
    T = rng.standard_normal((333, 3)).astype(np.float32)
    Y = mlp.forward(torch.as_tensor(X, device="cuda").to(BF16), keep=True)
    W = [w.cpu().numpy() for w in mlp.W]
    b = [v.cpu().numpy() for v in mlp.b]
    Y_ref, saved = omlp.forward(W, b, X)
    assert np.abs(Y.cpu().numpy() - Y_ref).max() <= 2e-3 * np.abs(Y_ref).max()
    dY = (2.0 / Y.numel()) * (Y - torch.as_tensor(T, device="cuda"))
    gW, gb = mlp.backward(dY)
    dY_ref = (2.0 / Y_ref.size) * (Y_ref - T)
    gW_ref, gb_ref = omlp.backward(W, saved, dY_ref)
    for l in range(4):
        assert np.abs(gW[l].cpu().numpy() - gW_ref[l]).max() <= 2e-2 * np.abs(gW_ref[l]).max()
        assert np.abs(gb[l].cpu().numpy() - gb_ref[l]).max() <= 2e-2 * np.abs(gb_ref[l]).max()


def test_mlp_training_reduces_loss():
    from fenics_nonlinear_energies_b200.warmstart import train_mlp

    rng = np.random.default_rng(1)
    F = rng.uniform(-1, 1, (4096, 12)).astype(np.float32)
    T = np.stack([np.sin(2 * F[:, 0]) * F[:, 3], F[:, 1] * F[:, 2], np.cos(F[:, 4])], 1).astype(np.float32)
    mlp, hist = train_mlp(F, T, width=128, epochs=60, batch=1024, lr=2e-3)
    assert hist[-1] < 0.05 * hist[0]


@pytest.mark.parametrize("family", ["plaplace", "gl"])
def test_newton_converges(family):
    from fenics_nonlinear_energies_b200.assembler import GLCudaAssembler, PLaplaceCudaAssembler
    from fenics_nonlinear_energies_b200.newton import newton

    if family == "plaplace":
        params, u0 = meshes.plaplace_problem(n=32, seed=0)
        asm = PLaplaceCudaAssembler(params)
        ref = OracleAssembler("plaplace", params)
    else:
        params, u0 = meshes.gl_problem(n=32, seed=0)
        asm = GLCudaAssembler(params)
        ref = OracleAssembler("gl", params)
    x, info = newton(asm, torch.as_tensor(u0, device="cuda"), tolg_rel=1e-6)
    assert info["converged"], info["message"]
    xs = x.cpu().numpy()
    assert abs(info["energy"] - ref.energy_fn(xs)) <= 1e-10 * max(1.0, abs(info["energy"]))
    assert np.linalg.norm(ref.gradient_fn(xs)) <= 1.01e-6 * info["grad_norm0"]
    assert info["energy"] < ref.energy_fn(u0)


def test_learned_warm_start_cuts_newton_iterations():
    """Train on solver-generated load-path solutions of a small twisted beam and
    compare, on a held-out path, the Newton iterations from the MLP prediction
    with those from the plain previous-step start (same 1e-6 gradient tolerance
    and energy; a rejected prediction is charged both solves)."""
    from fenics_nonlinear_energies_b200 import warmstart_experiment as wx

    res = wx.run(nx=32, ny=3, nz=3, train_paths=6, test_paths=1, steps=12, epochs=60, seed=3, log=lambda *_: None)
    t = res["test"]
    assert t["accepted_steps"] >= t["steps"] - 1
    assert t["learned_newton_its"] <= 0.85 * t["plain_newton_its"], t
