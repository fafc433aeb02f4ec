"""Element energy densities of the four families, restated from the reference (oracle).

Test infrastructure only.  Each ``*_element_energy`` follows the cited JAX
function line by line, written for float64 torch tensors so that
``torch.func.grad`` / ``torch.func.hessian`` give an autodiff independent of
the hand-written CUDA adjoints.  ``element_derivatives`` vmaps them over all
elements and returns (energy, gradient, Hessian) stacks as NumPy float64.

The one deliberate deviation: the p-Laplace density at a zero element
gradient.  JAX differentiates ``s**(p/2)`` at ``s = 0`` into ``inf * 0 = NaN``
for the Hessian; the mathematical limit for ``p > 2`` is 0.  The oracle and
the kernels both return the limit (``plaplace_limit_fixup``).
"""

from __future__ import annotations

import math

import numpy as np
import torch
from torch.func import grad, hessian, vmap

torch.set_default_dtype(torch.float64)


# --------------------------------------------------------------------------
# p-Laplace: src/problems/plaplace/jax_petsc/reordered_element_assembler.py:16-19, 38-39
# --------------------------------------------------------------------------
def plaplace_element_energy(v_e, dvx_e, dvy_e, vol_e, p):
    fx = torch.sum(v_e * dvx_e, dim=-1)
    fy = torch.sum(v_e * dvy_e, dim=-1)
    return (1.0 / p) * (fx**2 + fy**2) ** (p / 2.0) * vol_e


# --------------------------------------------------------------------------
# Ginzburg-Landau: src/problems/ginzburg_landau/jax_petsc/reordered_element_assembler.py:18-24
# --------------------------------------------------------------------------
def gl_element_energy(v_e, dvx_e, dvy_e, vol_e, ip, w, eps):
    fx = torch.sum(v_e * dvx_e, dim=-1)
    fy = torch.sum(v_e * dvy_e, dim=-1)
    grad_term = 0.5 * eps * (fx**2 + fy**2)
    nodal_vals = v_e @ ip
    potential_term = (0.25 * ((nodal_vals**2) - 1.0) ** 2) @ w
    return (grad_term + potential_term) * vol_e


# --------------------------------------------------------------------------
# Neo-Hookean: src/problems/hyperelasticity/jax_petsc/parallel_hessian_dof.py:17-52
# --------------------------------------------------------------------------
def he_element_energy(v_e, dphix_e, dphiy_e, dphiz_e, vol_e, C1, D1, use_abs_det=False):
    vx = v_e[..., 0::3]
    vy = v_e[..., 1::3]
    vz = v_e[..., 2::3]
    F11 = torch.sum(vx * dphix_e, dim=-1)
    F12 = torch.sum(vx * dphiy_e, dim=-1)
    F13 = torch.sum(vx * dphiz_e, dim=-1)
    F21 = torch.sum(vy * dphix_e, dim=-1)
    F22 = torch.sum(vy * dphiy_e, dim=-1)
    F23 = torch.sum(vy * dphiz_e, dim=-1)
    F31 = torch.sum(vz * dphix_e, dim=-1)
    F32 = torch.sum(vz * dphiy_e, dim=-1)
    F33 = torch.sum(vz * dphiz_e, dim=-1)
    I1 = F11**2 + F12**2 + F13**2 + F21**2 + F22**2 + F23**2 + F31**2 + F32**2 + F33**2
    detF = (
        F11 * (F22 * F33 - F23 * F32)
        - F12 * (F21 * F33 - F23 * F31)
        + F13 * (F21 * F32 - F22 * F31)
    )
    det = torch.abs(detF) if use_abs_det else detF
    return (C1 * (I1 - 3.0 - 2.0 * torch.log(det)) + D1 * (det - 1.0) ** 2) * vol_e


# --------------------------------------------------------------------------
# Mohr-Coulomb plane strain: src/problems/slope_stability/jax/jax_energy.py:11-142
# --------------------------------------------------------------------------
def mc_elastic_tensors(E, nu):
    """``jax_energy.py:11-30``."""
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    mu = E / (2.0 * (1.0 + nu))
    C = torch.tensor(
        [[lam + 2.0 * mu, lam, 0.0], [lam, lam + 2.0 * mu, 0.0], [0.0, 0.0, mu]],
        dtype=torch.float64,
    )
    S = torch.tensor(
        [
            [(1.0 - nu * nu) / E, -(nu * (1.0 + nu)) / E, 0.0],
            [-(nu * (1.0 + nu)) / E, (1.0 - nu * nu) / E, 0.0],
            [0.0, 0.0, 1.0 / mu],
        ],
        dtype=torch.float64,
    )
    return C, S


def mc_energy_density(strain, eps_p_old, E, nu, phi_deg, cohesion, reg):
    """``jax_energy.py:45-108`` for ONE quadrature point.

    ``lax.cond`` under ``vmap`` becomes a select over both branches; the
    plastic branch is evaluated on safe inputs where the elastic branch is
    selected (and vice versa for the line/apex choice), so the autodiff of the
    branch that is NOT taken cannot inject ``0 * NaN`` (the isotropic trial
    stress makes ``atan2(0, 0)`` non-differentiable).
    """
    C, S = mc_elastic_tensors(E, nu)
    eps_e = strain - eps_p_old
    sig_tr = C @ eps_e
    sxx, syy, txy = sig_tr[0], sig_tr[1], sig_tr[2]
    m = 0.5 * (sxx + syy)
    d = 0.5 * (sxx - syy)
    r = torch.sqrt(d * d + txy * txy + reg * reg)
    s1 = m + r
    s2 = m - r
    phi = math.radians(phi_deg)
    alpha = 1.0 + math.sin(phi)
    beta = 1.0 - math.sin(phi)
    kappa = 2.0 * cohesion * math.cos(phi)
    f_tr = alpha * s1 - beta * s2 - kappa
    elastic = f_tr <= 0.0

    psi_el = sig_tr @ eps_e - 0.5 * sig_tr @ (S @ sig_tr)

    A11, A12, A22 = float(S[0, 0]), float(S[0, 1]), float(S[1, 1])
    n1, n2 = alpha, -beta
    det = A11 * A22 - A12 * A12
    z1 = (A22 * n1 - A12 * n2) / det
    z2 = (-A12 * n1 + A11 * n2) / det
    lam_mc = (n1 * s1 + n2 * s2 - kappa) / (n1 * z1 + n2 * z2)
    s1_line = s1 - lam_mc * z1
    s2_line = s2 - lam_mc * z2
    safe_den = (alpha - beta) if abs(alpha - beta) > 1.0e-14 else 1.0
    s_apex = kappa / safe_den
    line = s1_line >= s2_line
    s1p = torch.where(line, s1_line, torch.full_like(s1_line, s_apex))
    s2p = torch.where(line, s2_line, torch.full_like(s2_line, s_apex))
    mp = 0.5 * (s1p + s2p)
    rp = 0.5 * (s1p - s2p)
    # direction of the trial stress; (1, 0) stands in where the branch is unused
    dd = torch.where(elastic, torch.ones_like(d), sxx - syy)
    tt = torch.where(elastic, torch.zeros_like(txy), 2.0 * txy)
    two_theta = torch.atan2(tt, dd)
    sig = torch.stack(
        (mp + rp * torch.cos(two_theta), mp - rp * torch.cos(two_theta), rp * torch.sin(two_theta))
    )
    psi_pl = sig @ eps_e - 0.5 * sig @ (S @ sig)
    return torch.where(elastic, psi_el, psi_pl)


def mc_elastic_density(strain, eps_p_old, E, nu):
    """``jax_energy.py:33-42``."""
    C, S = mc_elastic_tensors(E, nu)
    eps_e = strain - eps_p_old
    sig = C @ eps_e
    return sig @ eps_e - 0.5 * sig @ (S @ sig)


def mc_element_energy(u_e, B_e, w_e, epsp_e, E, nu, phi_deg, cohesion, reg=1.0e-12, elastic=False):
    """``jax_energy.py:121-142`` (and the elastic variant ``:145-157``)."""
    strain = torch.einsum("qij,j->qi", B_e, u_e)
    if elastic:
        dens = vmap(lambda s, e0: mc_elastic_density(s, e0, E, nu))(strain, epsp_e)
    else:
        dens = vmap(lambda s, e0: mc_energy_density(s, e0, E, nu, phi_deg, cohesion, reg))(
            strain, epsp_e
        )
    return torch.sum(w_e * dens)


# --------------------------------------------------------------------------
# batched derivatives
# --------------------------------------------------------------------------
def _t(a):
    return torch.as_tensor(np.asarray(a, dtype=np.float64))


def element_derivatives(family, v_elems, data, params, *, want_hessian=True, chunk=65536):
    """Return ``(e, g, H)`` float64 NumPy stacks for every element.

    ``v_elems`` is ``(E, n)``; ``data`` holds the reference's element arrays
    (``dvx, dvy, vol`` / ``dphix, dphiy, dphiz, vol`` /
    ``elem_B, quad_weight, eps_p_old``); ``params`` the scalars.
    """
    if family == "plaplace":
        p = float(params["p"])

        def f(v, dvx, dvy, vol):
            return plaplace_element_energy(v, dvx, dvy, vol, p)

        args = (data["dvx"], data["dvy"], data["vol"])
    elif family == "gl":
        ip = _t(params["ip"])
        w = _t(params["w"])
        eps = float(params["eps"])

        def f(v, dvx, dvy, vol):
            return gl_element_energy(v, dvx, dvy, vol, ip, w, eps)

        args = (data["dvx"], data["dvy"], data["vol"])
    elif family == "he":
        C1, D1 = float(params["C1"]), float(params["D1"])
        ab = bool(params.get("use_abs_det", False))

        def f(v, dx, dy, dz, vol):
            return he_element_energy(v, dx, dy, dz, vol, C1, D1, ab)

        args = (data["dphix"], data["dphiy"], data["dphiz"], data["vol"])
    elif family == "mc":
        E, nu = float(params["E"]), float(params["nu"])
        phi, c = float(params["phi_deg"]), float(params["cohesion"])
        reg = float(params.get("reg", 1.0e-12))
        el = bool(params.get("elastic", False))

        def f(v, B, w, ep):
            return mc_element_energy(v, B, w, ep, E, nu, phi, c, reg, el)

        args = (data["elem_B"], data["quad_weight"], data["eps_p_old"])
    else:
        raise ValueError(family)

    n_e = int(np.asarray(v_elems).shape[0])
    es, gs, hs = [], [], []
    fe, fg, fh = vmap(f), vmap(grad(f)), vmap(hessian(f))
    for s in range(0, n_e, chunk):
        sl = slice(s, min(n_e, s + chunk))
        v = _t(v_elems[sl])
        a = tuple(_t(x[sl]) for x in args)
        es.append(fe(v, *a).numpy())
        gs.append(fg(v, *a).numpy())
        if want_hessian:
            hs.append(fh(v, *a).numpy())
    e = np.concatenate(es) if es else np.zeros(0)
    g = np.concatenate(gs) if gs else np.zeros((0, np.asarray(v_elems).shape[1]))
    h = np.concatenate(hs) if want_hessian and hs else None
    if family == "plaplace":
        e, g, h = plaplace_limit_fixup(v_elems, data, params, e, g, h)
    return e, g, h


def plaplace_limit_fixup(v_elems, data, params, e, g, h):
    """Replace autodiff's ``0 * inf`` at a zero element gradient by the limit value."""
    v = np.asarray(v_elems, dtype=np.float64)
    fx = np.sum(v * data["dvx"], axis=1)
    fy = np.sum(v * data["dvy"], axis=1)
    zero = (fx * fx + fy * fy) == 0.0
    p = float(params["p"])
    if np.any(zero):
        g = g.copy()
        g[zero] = 0.0
        if h is not None:
            h = h.copy()
            if p > 2.0:
                h[zero] = 0.0
    return e, g, h
