"""Learned Newton warm start for load paths (no counterpart in the reference).

A small MLP over nodal features predicts the next load step's displacement
increment.  The forward and backward passes run on the project's own
kernels (``csrc/fne_mlp.cu``: BF16 tensor-core GEMMs with FP32 accumulation,
fused bias + SiLU, SiLU backward, bias-gradient sums and Adam on FP32 master
weights).  The prediction is only a starting point: Newton from it must
reach the same gradient tolerance and energy as the plain previous-step
start, otherwise the plain start is used (``run_load_path``).
"""

from __future__ import annotations

import math
import time

import numpy as np
import torch

from fenics_nonlinear_energies_b200 import _lib, meshes
from fenics_nonlinear_energies_b200._lib import check, lib
from fenics_nonlinear_energies_b200.newton import newton

BF16 = torch.bfloat16


def _stream():
    return torch.cuda.current_stream().cuda_stream


def gemm(A, sam, sak, B, sbk, sbn, M, N, K, C, beta=0.0):
    """``C[M, N] = A(M, K) B(K, N) (+ beta C)`` through ``fne_gemm_bf16``."""
    check(lib.fne_gemm_bf16(M, N, K, A.data_ptr(), sam, sak, B.data_ptr(), sbk, sbn, C.data_ptr(), N, float(beta),
                            _stream()))
    return C


class NodalMLP:
    """``dims = (d_in, 256, 256, 256, d_out)``: 4 linear layers, SiLU between them."""

    def __init__(self, dims, seed=0, device="cuda"):
        self.dims = tuple(int(d) for d in dims)
        g = torch.Generator().manual_seed(seed)
        self.W, self.b, self.W16 = [], [], []
        for din, dout in zip(self.dims[:-1], self.dims[1:]):
            w = torch.randn(dout, din, generator=g, dtype=torch.float32) * math.sqrt(2.0 / din)
            self.W.append(w.to(device))
            self.b.append(torch.zeros(dout, dtype=torch.float32, device=device))
        for w in self.W:
            w16 = torch.empty(w.shape, dtype=BF16, device=device)
            check(lib.fne_mlp_cast_bf16(w.numel(), w.data_ptr(), w16.data_ptr(), _stream()))
            self.W16.append(w16)
        self.m = [torch.zeros_like(p) for p in self.W + self.b]
        self.v = [torch.zeros_like(p) for p in self.W + self.b]
        self.step = 0
        self.n_layers = len(self.W)
        self.kernel_launches = 0

    # -- forward -------------------------------------------------------------
    def forward(self, X16, keep=False):
        """``X16`` (N, d_in) BF16 -> FP32 (N, d_out).  ``keep`` saves what backward needs."""
        N = X16.shape[0]
        h16 = X16
        saved = []
        out = None
        for l in range(self.n_layers):
            din, dout = self.dims[l], self.dims[l + 1]
            Z = torch.empty(N, dout, dtype=torch.float32, device=X16.device)
            gemm(h16, din, 1, self.W16[l], 1, din, N, dout, din, Z)
            last = l == self.n_layers - 1
            if last:
                out = torch.empty_like(Z)
                check(lib.fne_mlp_bias_act(N, dout, Z.data_ptr(), self.b[l].data_ptr(), 0, out.data_ptr(), None,
                                           _stream()))
            else:
                nxt = torch.empty(N, dout, dtype=BF16, device=X16.device)
                check(lib.fne_mlp_bias_act(N, dout, Z.data_ptr(), self.b[l].data_ptr(), 1, None, nxt.data_ptr(),
                                           _stream()))
            self.kernel_launches += 2
            if keep:
                saved.append((h16, Z))
            if not last:
                h16 = nxt
        if keep:
            self._saved = saved
        return out

    # -- backward ------------------------------------------------------------
    def backward(self, dY):
        """Gradients of the parameters for ``dL/dY = dY`` (FP32, shape (N, d_out))."""
        N = dY.shape[0]
        gW, gb = [None] * self.n_layers, [None] * self.n_layers
        dH = dY.contiguous()
        for l in reversed(range(self.n_layers)):
            din, dout = self.dims[l], self.dims[l + 1]
            h16, Z = self._saved[l]
            act = 0 if l == self.n_layers - 1 else 1
            dZ32 = torch.empty(N, dout, dtype=torch.float32, device=dY.device)
            dZ16 = torch.empty(N, dout, dtype=BF16, device=dY.device)
            check(lib.fne_mlp_act_bwd(N * dout, Z.data_ptr(), dH.data_ptr(), act, dZ32.data_ptr(), dZ16.data_ptr(),
                                      _stream()))
            gW[l] = torch.empty(dout, din, dtype=torch.float32, device=dY.device)
            gemm(dZ16, 1, dout, h16, din, 1, dout, din, N, gW[l])            # dZ^T H
            gb[l] = torch.empty(dout, dtype=torch.float32, device=dY.device)
            check(lib.fne_mlp_colsum(N, dout, dZ32.data_ptr(), gb[l].data_ptr(), _stream()))
            self.kernel_launches += 3
            if l > 0:
                dH = torch.empty(N, din, dtype=torch.float32, device=dY.device)
                gemm(dZ16, dout, 1, self.W16[l], din, 1, N, din, dout, dH)   # dZ W
                self.kernel_launches += 1
        return gW, gb

    def adam_step(self, gW, gb, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        params = self.W + self.b
        grads = gW + gb
        for i, (p, g) in enumerate(zip(params, grads)):
            p16 = self.W16[i] if i < self.n_layers else None
            check(lib.fne_mlp_adam(p.numel(), p.data_ptr(), g.data_ptr(), self.m[i].data_ptr(), self.v[i].data_ptr(),
                                   lr, b1, b2, eps, self.step, p16.data_ptr() if p16 is not None else None, _stream()))
            self.kernel_launches += 1

    def state(self):
        return {"dims": self.dims, "W": [w.cpu() for w in self.W], "b": [b.cpu() for b in self.b]}


# ---------------------------------------------------------------------------
# nodal features of the twisted hyperelastic beam
# ---------------------------------------------------------------------------
N_FEATURES = 12


class BeamFeatures:
    """Feature / target scaling for one beam mesh (free nodes, in free-DOF order).

    Features of a free node at step k (before solving step k+1):
      X / (L, w, w)              reference position (3)
      u_k / w                    current displacement (3)
      (u_k - u_{k-1}) / w        last increment (3)
      dtheta_{k+1}, theta_k / (2 pi), E / 20    load-path descriptors (3)
    Target: (u_{k+1} - u_k) / w.
    """

    def __init__(self, params):
        free = np.asarray(params["freedofs"], dtype=np.int64)
        self.nodes = free[0::3] // 3
        X = np.asarray(params["nodes2coord"], dtype=np.float64)[self.nodes]
        self.L = float(np.ptp(np.asarray(params["nodes2coord"])[:, 0]))
        self.w = float(np.ptp(np.asarray(params["nodes2coord"])[:, 1]))
        self.Xs = X / np.array([self.L, self.w, self.w])
        self.X = X

    def features(self, u_k, u_km1, dtheta, theta, E):
        n = self.X.shape[0]
        f = np.empty((n, N_FEATURES), dtype=np.float32)
        f[:, 0:3] = self.Xs
        f[:, 3:6] = u_k / self.w
        f[:, 6:9] = (u_k - u_km1) / self.w
        f[:, 9] = dtheta
        f[:, 10] = theta / (2.0 * math.pi)
        f[:, 11] = E / 20.0
        return f

    def target(self, u_k, u_kp1):
        return ((u_kp1 - u_k) / self.w).astype(np.float32)


def mlp_predict(mlp, feats_np):
    X16 = torch.as_tensor(feats_np, device="cuda").to(BF16).contiguous()
    return mlp.forward(X16).cpu().numpy().astype(np.float64)


# ---------------------------------------------------------------------------
# load paths
# ---------------------------------------------------------------------------
def make_beam(nx, ny, nz, E):
    params, y0 = meshes.he_beam_problem(nx=nx, ny=ny, nz=nz, E=E)
    return params, y0


def run_load_path(params, theta_total, steps, *, predictor=None, features=None, E=10.0, newton_kw=None,
                  record=False):
    """Rotate the right face in ``steps`` equal increments up to ``theta_total``.

    Each step starts Newton from the previous solution (plain start) or, when
    ``predictor`` is given, from ``u_k + predictor(features)``.  A prediction
    is accepted only if Newton from it converges to the same gradient
    tolerance and an energy within 1e-8 (relative) of the plain start's
    solve; otherwise the plain start is used and both iteration counts are
    charged.  Returns per-step records (and the solutions when ``record``).
    """
    from fenics_nonlinear_energies_b200.assembler import HECudaAssembler
    from fenics_nonlinear_energies_b200.newton import DeviceCG

    kw = dict(tolg_rel=1e-6, linesearch_tol=1e-3, ksp_rtol=1e-2, ksp_max_it=2000, maxit=200)
    kw.update(newton_kw or {})
    asm = HECudaAssembler(params)
    kw["cg"] = DeviceCG.for_assembler(asm)
    lay = asm.layout
    free = np.asarray(params["freedofs"], dtype=np.int64)
    X_free = np.asarray(params["u_0_ref"], dtype=np.float64)[free]
    perm = np.asarray(lay.perm)

    def to_dev(y_free):       # free-DOF order -> reordered device vector
        return torch.as_tensor(y_free[perm], device=asm.device)

    def to_host(x_dev):
        out = np.empty(free.size)
        out[perm] = x_dev.cpu().numpy()
        return out

    y = X_free.copy()
    y_prev = X_free.copy()
    dtheta = theta_total / steps
    recs, sols = [], [y.copy()]
    for k in range(1, steps + 1):
        theta = k * dtheta
        asm.update_dirichlet(meshes.rotate_right_face_from_reference(
            params["u_0_ref"], params["nodes2coord"], theta, params["right_nodes"]))
        t0 = time.perf_counter()
        x_plain, info_plain = newton(asm, to_dev(y), **kw)
        t_plain = time.perf_counter() - t0
        rec = {"step": k, "theta": theta, "plain_its": info_plain["iterations"],
               "plain_converged": info_plain["converged"], "plain_message": info_plain["message"],
               "energy": info_plain["energy"], "plain_s": t_plain}
        x_use = x_plain
        if predictor is not None:
            u_k = (y - X_free).reshape(-1, 3)
            u_km1 = (y_prev - X_free).reshape(-1, 3)
            du = predictor(features.features(u_k, u_km1, dtheta, theta - dtheta, E)) * features.w
            y_pred = y + du.reshape(-1)
            x_pred, info_pred = newton(asm, to_dev(y_pred), **kw)
            t_pred = time.perf_counter() - t0 - t_plain  # prediction (features, MLP) + Newton from it
            same = (info_pred["converged"] and info_plain["converged"] and
                    abs(info_pred["energy"] - info_plain["energy"]) <= 1e-8 * max(1.0, abs(info_plain["energy"])))
            rec.update(pred_its=info_pred["iterations"], pred_converged=info_pred["converged"],
                       pred_energy=info_pred["energy"], accepted=bool(same),
                       learned_its=info_pred["iterations"] if same else
                       info_pred["iterations"] + info_plain["iterations"],
                       learned_s=t_pred if same else t_pred + t_plain)
            if same:
                x_use = x_pred
        rec["time_s"] = time.perf_counter() - t0
        recs.append(rec)
        y_prev = y
        y = to_host(x_use)
        if record:
            sols.append(y.copy())
    kw["cg"].close()
    asm.cleanup()
    return (recs, sols) if record else recs


def training_pairs(features, sols, theta_total, E):
    """(features, targets) of every step transition k -> k+1 of one solved path."""
    steps = len(sols) - 1
    dtheta = theta_total / steps
    X_free = sols[0]
    F, T = [], []
    for k in range(1, steps):
        u_k = (sols[k] - X_free).reshape(-1, 3)
        u_km1 = (sols[k - 1] - X_free).reshape(-1, 3)
        u_kp1 = (sols[k + 1] - X_free).reshape(-1, 3)
        F.append(features.features(u_k, u_km1, dtheta, k * dtheta, E))
        T.append(features.target(u_k, u_kp1))
    return np.concatenate(F), np.concatenate(T)


def train_mlp(F, T, *, width=256, epochs=200, batch=8192, lr=2e-3, seed=0, log=None):
    """Fit the MLP on all (feature, target) rows; returns the model and the loss history."""
    mlp = NodalMLP((F.shape[1], width, width, width, T.shape[1]), seed=seed)
    Fd = torch.as_tensor(F, device="cuda").to(BF16)
    Td = torch.as_tensor(T, device="cuda")
    n = Fd.shape[0]
    g = torch.Generator(device="cuda").manual_seed(seed)
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, device="cuda", generator=g)
        tot = 0.0
        for s in range(0, n, batch):
            idx = perm[s:s + batch]
            Xb, Tb = Fd.index_select(0, idx).contiguous(), Td.index_select(0, idx)
            Y = mlp.forward(Xb, keep=True)
            diff = Y - Tb
            dY = (2.0 / diff.numel()) * diff
            gW, gb = mlp.backward(dY)
            cur_lr = lr * 0.5 * (1.0 + math.cos(math.pi * ep / epochs))
            mlp.adam_step(gW, gb, lr=cur_lr)
            tot += float((diff * diff).sum())
        hist.append(tot / (n * T.shape[1]))
        if log and (ep % max(1, epochs // 10) == 0 or ep == epochs - 1):
            log(f"epoch {ep} mse {hist[-1]:.3e}")
    return mlp, hist
