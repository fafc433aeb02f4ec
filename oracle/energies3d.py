"""3-D Mohr-Coulomb density and its strain derivatives (oracle for the 3-D slope family).

Test infrastructure only.  Restates ``src/problems/slope_stability_3d/jax/jax_energy_3d.py``:

* strain ordering ``[xx, yy, zz, xy, yz, xz]`` with engineering shears
  (``strain6_from_local_gradients``, :12-30) and the strain operator B_q
  (``strain6_matrix_from_local_gradients``, :262-286);
* principal strains ``eig_1 >= eig_2 >= eig_3`` of the tensor-shear matrix
  plus the tie-break ``tiny * diag(0, 1, 2)`` (``principal_values_from_sym6``,
  :38-70);
* the five-branch potential (elastic, smooth return, left / right edge,
  apex) with the branch chosen from the primal values
  (``mc_potential_density_3d``, :73-191), and the linear-elastic density
  (:194-211);
* element energy sum_q w_q psi_q; residual sum_q w_q B_q^T sigma_q and the
  constitutive tangent sum_q w_q B_q^T D_q B_q with sigma = dpsi/deps,
  D = d2psi/deps2 (:289-357).

Derivatives come from ``torch.func`` (float64, autodiff through
``torch.linalg.eigvalsh``) standing in for JAX's autodiff of the same
formula; the value path is plain NumPy.
"""

from __future__ import annotations

import numpy as np
import torch

TINY = 1.0e-15
BRANCHES = ("elastic", "smooth", "left", "right", "apex")


def strain6(u_e, dphix, dphiy, dphiz):
    """Strains at the quadrature points: ``u_e`` (..., 3n) interleaved (x, y, z)
    per node, basis derivatives (..., nq, n) -> (..., nq, 6)."""
    u = np.asarray(u_e, dtype=np.float64)
    ux, uy, uz = u[..., 0::3], u[..., 1::3], u[..., 2::3]
    d = lambda v, g: np.einsum("...a,...qa->...q", v, g)  # noqa: E731
    return np.stack([d(ux, dphix), d(uy, dphiy), d(uz, dphiz), d(ux, dphiy) + d(uy, dphix),
                     d(uy, dphiz) + d(uz, dphiy), d(ux, dphiz) + d(uz, dphix)], axis=-1)


def strain_operator(dphix, dphiy, dphiz):
    """B_q (..., nq, 6, 3n) with the DOF order (x, y, z) per node."""
    gx, gy, gz = (np.asarray(g, dtype=np.float64) for g in (dphix, dphiy, dphiz))
    n = gx.shape[-1]
    B = np.zeros(gx.shape[:-1] + (6, 3 * n))
    B[..., 0, 0::3] = gx
    B[..., 1, 1::3] = gy
    B[..., 2, 2::3] = gz
    B[..., 3, 0::3], B[..., 3, 1::3] = gy, gx
    B[..., 4, 1::3], B[..., 4, 2::3] = gz, gy
    B[..., 5, 0::3], B[..., 5, 2::3] = gz, gx
    return B


def _tensor(eps6, lib):
    e11, e22, e33, g12, g23, g13 = (eps6[..., k] for k in range(6))
    h12, h23, h13 = 0.5 * g12, 0.5 * g23, 0.5 * g13
    rows = [lib.stack([e11, h12, h13], -1), lib.stack([h12, e22, h23], -1), lib.stack([h13, h23, e33], -1)]
    return lib.stack(rows, -2)


def principal_values(eps6, tiny=TINY, lib=np):
    """(eig_1, eig_2, eig_3, I1) with eig_1 >= eig_2 >= eig_3 (NumPy or torch)."""
    A = _tensor(eps6, lib)
    tb = lib.asarray([0.0, 1.0, 2.0], dtype=A.dtype) if lib is np else torch.tensor([0.0, 1.0, 2.0],
                                                                                     dtype=A.dtype)
    A = A + tiny * (lib.diag_embed(tb) if lib is torch else np.diag(tb))
    ev = np.linalg.eigvalsh(A) if lib is np else torch.linalg.eigvalsh(A)
    I1 = eps6[..., 0] + eps6[..., 1] + eps6[..., 2]
    return ev[..., 2], ev[..., 1], ev[..., 0], I1


def _safe_denom(x, tiny, lib):
    sign = lib.where(x >= 0.0, 1.0, -1.0) if lib is np else torch.where(x >= 0.0, 1.0, -1.0).to(x.dtype)
    return lib.where(lib.abs(x) < tiny, sign * tiny, x)


def _pieces(eps6, c_bar, sin_phi, shear, bulk, lame, tiny, lib, with_tests=True):
    """Branch potentials and the (primal) branch tests of the 3-D density."""
    mx = np.maximum if lib is np else torch.clamp
    e = [eps6[..., k] for k in range(6)]
    quad = e[0] ** 2 + e[1] ** 2 + e[2] ** 2 + 0.5 * (e[3] ** 2 + e[4] ** 2 + e[5] ** 2)
    l1, l2, l3, I1 = principal_values(eps6, tiny, lib)
    sp = sin_phi
    f_tr = 2.0 * shear * ((1.0 + sp) * l1 - (1.0 - sp) * l3) + 2.0 * lame * sp * I1 - c_bar
    if lib is np:
        g_sl = (l1 - l2) / np.maximum(tiny, 1.0 + sp)
        g_sr = (l2 - l3) / np.maximum(tiny, 1.0 - sp)
        g_la = (l1 + l2 - 2.0 * l3) / np.maximum(tiny, 3.0 - sp)
        g_ra = (2.0 * l1 - l2 - l3) / np.maximum(tiny, 3.0 + sp)
    else:
        g_sl = (l1 - l2) / mx(1.0 + sp, min=tiny)
        g_sr = (l2 - l3) / mx(1.0 - sp, min=tiny)
        g_la = (l1 + l2 - 2.0 * l3) / mx(3.0 - sp, min=tiny)
        g_ra = (2.0 * l1 - l2 - l3) / mx(3.0 + sp, min=tiny)
    d_s = 4.0 * lame * sp ** 2 + 4.0 * shear * (1.0 + sp ** 2)
    d_l = 4.0 * lame * sp ** 2 + shear * (1.0 + sp) ** 2 + 2.0 * shear * (1.0 - sp) ** 2
    d_r = 4.0 * lame * sp ** 2 + 2.0 * shear * (1.0 + sp) ** 2 + shear * (1.0 - sp) ** 2
    d_a = 4.0 * bulk * sp ** 2
    lam_s = f_tr / _safe_denom(d_s, tiny, lib)
    lam_l = (shear * ((1.0 + sp) * (l1 + l2) - 2.0 * (1.0 - sp) * l3) + 2.0 * lame * sp * I1 - c_bar) / \
        _safe_denom(d_l, tiny, lib)
    lam_r = (shear * (2.0 * (1.0 + sp) * l1 - (1.0 - sp) * (l2 + l3)) + 2.0 * lame * sp * I1 - c_bar) / \
        _safe_denom(d_r, tiny, lib)
    lam_a = (2.0 * bulk * sp * I1 - c_bar) / _safe_denom(d_a, tiny, lib)
    base = 0.5 * lame * I1 ** 2
    psi = {
        "elastic": base + shear * quad,
        "smooth": base + shear * quad - 0.5 * d_s * lam_s ** 2,
        "left": base + shear * (l3 ** 2 + 0.5 * (l1 + l2) ** 2) - 0.5 * d_l * lam_l ** 2,
        "right": base + shear * (l1 ** 2 + 0.5 * (l2 + l3) ** 2) - 0.5 * d_r * lam_r ** 2,
        "apex": 0.5 * bulk * I1 ** 2 - 0.5 * d_a * lam_a ** 2,
    }
    if not with_tests:
        return psi, None
    tests = {k: (v.detach().cpu().numpy() if lib is torch else v) for k, v in
             dict(f_tr=f_tr, g_sl=g_sl, g_sr=g_sr, g_la=g_la, g_ra=g_ra, lam_s=lam_s, lam_l=lam_l,
                  lam_r=lam_r).items()}
    return psi, tests


def branch_index(t):
    """0 elastic, 1 smooth, 2 left edge, 3 right edge, 4 apex (first test that holds)."""
    el = t["f_tr"] <= 0.0
    s = ~el & (t["lam_s"] <= np.minimum(t["g_sl"], t["g_sr"]))
    left = ~(el | s) & (t["g_sl"] < t["g_sr"]) & (t["lam_l"] >= t["g_sl"]) & (t["lam_l"] <= t["g_la"])
    right = ~(el | s | left) & (t["g_sl"] > t["g_sr"]) & (t["lam_r"] >= t["g_sr"]) & (t["lam_r"] <= t["g_ra"])
    return np.select([el, s, left, right], [0, 1, 2, 3], default=4)


def mc_density(eps6, c_bar, sin_phi, shear, bulk, lame, tiny=TINY):
    """psi at every point (NumPy, float64) and the branch index."""
    args = [np.asarray(a, dtype=np.float64) for a in (eps6, c_bar, sin_phi, shear, bulk, lame)]
    psi, tests = _pieces(*args, tiny, np)
    br = branch_index(tests)
    return np.choose(br, [psi[k] for k in BRANCHES]), br


def elastic_density(eps6, shear, lame):
    e = np.asarray(eps6, dtype=np.float64)
    quad = (e[..., :3] ** 2).sum(-1) + 0.5 * (e[..., 3:] ** 2).sum(-1)
    return 0.5 * lame * e[..., :3].sum(-1) ** 2 + shear * quad


def mc_stress_tangent(eps6, c_bar, sin_phi, shear, bulk, lame, tiny=TINY):
    """(sigma (P, 6), D (P, 6, 6), psi (P,), branch (P,)) by autodiff of the
    selected branch potential at each point (the branch is fixed by the
    primal tests, as the reference's stop_gradient + cond does)."""
    eps = torch.as_tensor(np.asarray(eps6, dtype=np.float64).reshape(-1, 6))
    prm = [torch.as_tensor(np.broadcast_to(np.asarray(a, dtype=np.float64), eps.shape[:1]).copy())
           for a in (c_bar, sin_phi, shear, bulk, lame)]
    _, tests = _pieces(eps, *prm, tiny, torch)
    br = branch_index(tests)

    def one(e, c, s, g, k, lm, b):
        p, _ = _pieces(e[None], c[None], s[None], g[None], k[None], lm[None], tiny, torch, with_tests=False)
        stacked = torch.stack([p[name][0] for name in BRANCHES])
        return stacked[b]

    sig = np.zeros((eps.shape[0], 6))
    D = np.zeros((eps.shape[0], 6, 6))
    psi = np.zeros(eps.shape[0])
    for i in range(eps.shape[0]):
        args = (eps[i], *[a[i] for a in prm], int(br[i]))
        f = lambda e: one(e, *args[1:])  # noqa: E731
        psi[i] = float(f(args[0]))
        sig[i] = torch.func.grad(f)(args[0]).numpy()
        D[i] = torch.func.hessian(f)(args[0]).numpy()
    return sig, D, psi, br


def element_derivatives(u_e, dphix, dphiy, dphiz, qw, c_bar, sin_phi, shear, bulk, lame, tiny=TINY):
    """Energy, residual and constitutive tangent of one element (float64)."""
    eps = strain6(u_e, dphix, dphiy, dphiz)            # (nq, 6)
    B = strain_operator(dphix, dphiy, dphiz)            # (nq, 6, 3n)
    sig, D, psi, br = mc_stress_tangent(eps, c_bar, sin_phi, shear, bulk, lame, tiny)
    w = np.asarray(qw, dtype=np.float64)
    e = float(np.sum(w * psi))
    g = np.einsum("qsi,qs,q->i", B, sig, w)
    H = np.einsum("qsi,qst,qtj,q->ij", B, D, B, w)
    return e, g, H, br
