"""Spectral form of the 3-D Mohr-Coulomb stress and tangent (oracle side).

Test infrastructure only.  The 3-D density is psi(eps) = F(lambda_1,
lambda_2, lambda_3, eps), where the lambda_k are the eigenvalues of
A(eps) = tensor(eps) + tiny diag(0, 1, 2) (``oracle/energies3d.py``).  A
device kernel cannot autodiff through ``eigvalsh``; it evaluates the chain
rule with the classical eigenvalue derivatives (distinct eigenvalues):

    d lambda_k / dA          = v_k v_k^T
    d2 lambda_k / dA dA[X,Y] = 2 sum_{j != k} (v_k^T X v_j)(v_j^T Y v_k) / (lambda_k - lambda_j)

    sigma = dF/deps + sum_k F_k g_k,        g_k = d lambda_k / deps
    D     = d2F/deps2 + sum_k (F_{eps k} g_k^T + g_k F_{eps k}^T)
            + sum_{k,l} F_kl g_k g_l^T + sum_k F_k H_k,  H_k = d2 lambda_k / deps2

with the partial derivatives of F (in lambda and in eps with lambda held
fixed) taken by autodiff here.  ``tests/test_oracle3d.py`` checks this
composition against the full autodiff through ``eigvalsh`` -- the same
derivative JAX takes in the reference -- so the kernel's formula is pinned
before the kernel exists.
"""

from __future__ import annotations

import numpy as np
import torch

from oracle import energies3d as E3

# d A / d eps_m for eps = [xx, yy, zz, xy, yz, xz] (engineering shears)
_DA = np.zeros((6, 3, 3))
_DA[0, 0, 0] = _DA[1, 1, 1] = _DA[2, 2, 2] = 1.0
for _m, (_i, _j) in zip((3, 4, 5), ((0, 1), (1, 2), (0, 2))):
    _DA[_m, _i, _j] = _DA[_m, _j, _i] = 0.5


def _branch_F(branch, c_bar, sin_phi, shear, bulk, lame, tiny):
    """F(lam (3,), eps (6,)) of one branch, lam = (l1, l2, l3) descending."""
    sp = torch.tensor(sin_phi, dtype=torch.float64)

    def F(lam, eps):
        l1, l2, l3 = lam[0], lam[1], lam[2]
        I1 = eps[0] + eps[1] + eps[2]
        quad = eps[0] ** 2 + eps[1] ** 2 + eps[2] ** 2 + 0.5 * (eps[3] ** 2 + eps[4] ** 2 + eps[5] ** 2)
        base = 0.5 * lame * I1 ** 2
        if branch == 0:
            return base + shear * quad
        if branch == 1:
            d_s = 4.0 * lame * sp ** 2 + 4.0 * shear * (1.0 + sp ** 2)
            f_tr = 2.0 * shear * ((1.0 + sp) * l1 - (1.0 - sp) * l3) + 2.0 * lame * sp * I1 - c_bar
            return base + shear * quad - 0.5 * f_tr ** 2 / d_s
        if branch == 2:
            d_l = 4.0 * lame * sp ** 2 + shear * (1.0 + sp) ** 2 + 2.0 * shear * (1.0 - sp) ** 2
            lam_l = (shear * ((1.0 + sp) * (l1 + l2) - 2.0 * (1.0 - sp) * l3) + 2.0 * lame * sp * I1 - c_bar) / d_l
            return base + shear * (l3 ** 2 + 0.5 * (l1 + l2) ** 2) - 0.5 * d_l * lam_l ** 2
        if branch == 3:
            d_r = 4.0 * lame * sp ** 2 + 2.0 * shear * (1.0 + sp) ** 2 + shear * (1.0 - sp) ** 2
            lam_r = (shear * (2.0 * (1.0 + sp) * l1 - (1.0 - sp) * (l2 + l3)) + 2.0 * lame * sp * I1 - c_bar) / d_r
            return base + shear * (l1 ** 2 + 0.5 * (l2 + l3) ** 2) - 0.5 * d_r * lam_r ** 2
        d_a = 4.0 * bulk * sp ** 2
        lam_a = (2.0 * bulk * sp * I1 - c_bar) / d_a
        return 0.5 * bulk * I1 ** 2 - 0.5 * d_a * lam_a ** 2

    return F


def stress_tangent_spectral(eps6, c_bar, sin_phi, shear, bulk, lame, tiny=E3.TINY, eigh=np.linalg.eigh):
    """(sigma (6,), D (6, 6), branch) at one strain by the spectral chain rule;
    ``eigh``: the symmetric eigen-decomposition used (LAPACK or ``jacobi_eigh3``)."""
    eps6 = np.asarray(eps6, dtype=np.float64)
    _, br = E3.mc_density(eps6[None], c_bar, sin_phi, shear, bulk, lame, tiny)
    br = int(br[0])
    A = np.einsum("m,mij->ij", eps6, _DA) + tiny * np.diag([0.0, 1.0, 2.0])
    w, V = eigh(A)
    order = [2, 1, 0]                       # descending: lambda_1 >= lambda_2 >= lambda_3
    lam, V = w[order], V[:, order]
    g = np.einsum("ik,mij,jk->km", V, _DA, V)            # g[k, m] = v_k^T dA_m v_k
    Hk = np.zeros((3, 6, 6))
    X = np.einsum("ik,mij,jl->klm", V, _DA, V)           # X[k, l, m] = v_k^T dA_m v_l
    for k in range(3):
        for j in range(3):
            if j != k:
                Hk[k] += 2.0 * np.outer(X[k, j], X[j, k]) / (lam[k] - lam[j])
    F = _branch_F(br, c_bar, sin_phi, shear, bulk, lame, tiny)
    lt, et = torch.tensor(lam), torch.tensor(eps6)
    (F_l, F_e) = torch.func.grad(F, argnums=(0, 1))(lt, et)
    hess = torch.func.hessian(F, argnums=(0, 1))(lt, et)
    F_ll, F_le, F_ee = hess[0][0].numpy(), hess[0][1].numpy(), hess[1][1].numpy()
    F_l, F_e = F_l.numpy(), F_e.numpy()
    sigma = F_e + g.T @ F_l
    D = F_ee + g.T @ F_le + F_le.T @ g + g.T @ F_ll @ g + np.einsum("k,kmn->mn", F_l, Hk)
    return sigma, D, br


def jacobi_eigh3(A, sweeps=6):
    """Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations
    (the textbook method: for each off-diagonal (p, q), the rotation that
    zeroes it, t = sgn(theta) / (|theta| + sqrt(theta^2 + 1)) with
    theta = (a_qq - a_pp) / (2 a_pq)), a fixed number of sweeps -- the form a
    device kernel evaluates per quadrature point without data-dependent loop
    counts.  Returns (w ascending, V) like numpy.linalg.eigh."""
    a = np.array(A, dtype=np.float64, copy=True)
    V = np.eye(3)
    for _ in range(sweeps):
        for p, q in ((0, 1), (0, 2), (1, 2)):
            apq = a[p, q]
            if apq == 0.0:
                continue
            theta = (a[q, q] - a[p, p]) / (2.0 * apq)
            # t -> 1 / (2 theta) for large theta (no overflow of theta^2)
            t = 0.5 / theta if abs(theta) > 1e100 else np.copysign(1.0, theta) / (abs(theta) + np.sqrt(theta * theta + 1.0))
            c = 1.0 / np.sqrt(t * t + 1.0)
            s = t * c
            R = np.eye(3)
            R[p, p] = R[q, q] = c
            R[p, q], R[q, p] = s, -s
            a = R.T @ a @ R
            V = V @ R
    w = np.diag(a).copy()
    order = np.argsort(w)
    return w[order], V[:, order]
