"""3-D Mohr-Coulomb family (FNE_MOHR_COULOMB_3D) on the GPU against the FP64
oracle (``oracle/energies3d.py``: the reference's 3-D density restated, its
stress and tangent by torch autodiff through ``eigvalsh``).

A synthetic tetrahedral slope (P1: centroid rule; P2: the reference's
11-point rule; P4: its 24-point rule), states small enough to stay elastic
and large enough to reach the plastic branches.  Mesh sizes are chosen with the number of free
DOFs a multiple of 3: the reference's block_xyz permutation takes every
third free DOF as a node id (reordered_element_base.py:150-161), which the
layout builders restate.  Bars: FP64 mode 1e-12 relative (energy vs the
sum of |element energy| + |load term|, gradient / Hessian vs their largest
entry); FP32 mode 2e-5 (Hessian), 1e-4 (gradient), 1e-6 (energy).
"""

import numpy as np
import pytest
import torch

from fenics_nonlinear_energies_b200 import _lib, meshes
from oracle import energies3d as E3

pytestmark = pytest.mark.gpu

TOL = {"fp64": (1e-12, 1e-12, 1e-12), "fp32": (1e-6, 1e-4, 2e-5)}


def _elastic_element(u_e, dphix, dphiy, dphiz, qw, c_bar, sin_phi, shear, bulk, lame):
    """The elastic mode's element: psi = lame/2 I1^2 + mu Q (the oracle's
    elastic_density), sigma = C eps, tangent C, contracted with B_q."""
    eps = E3.strain6(u_e, dphix, dphiy, dphiz)
    B = E3.strain_operator(dphix, dphiy, dphiz)
    psi = E3.elastic_density(eps, shear, lame)
    C = np.zeros((eps.shape[0], 6, 6))
    C[:, :3, :3] = lame[:, None, None]
    for i in range(3):
        C[:, i, i] += 2.0 * shear
        C[:, 3 + i, 3 + i] = shear
    sig = np.einsum("qst,qt->qs", C, eps)
    w = np.asarray(qw)
    return (float(np.sum(w * psi)), np.einsum("qsi,qs,q->i", B, sig, w),
            np.einsum("qsi,qst,qtj,q->ij", B, C, B, w), np.zeros(eps.shape[0], dtype=np.int64))


def _oracle(p, u_free, elastic=False):
    """Energy, gradient (free DOFs) and dense Hessian (free x free) assembled
    from the oracle's element derivatives, in total-DOF order; also the
    energy's rounding scale and the branch of every point."""
    free, elems = p["freedofs"], p["elems"]
    u = p["u_0"].copy()
    u[free] = u_free
    n = u.size
    g, H = np.zeros(n), np.zeros((n, n))
    e_tot, scale, branches = 0.0, 0.0, []
    for e in range(elems.shape[0]):
        args = (p["dphix"][e], p["dphiy"][e], p["dphiz"][e], p["quad_weight"][e],
                p["c_bar"][e], p["sin_phi"][e], p["shear"][e], p["bulk"][e], p["lame"][e])
        if elastic:
            ee, ge, He, br = _elastic_element(u[elems[e]], *args)
        else:
            ee, ge, He, br = E3.element_derivatives(u[elems[e]], *args)
        e_tot += ee
        scale += abs(ee)
        np.add.at(g, elems[e], ge)
        H[np.ix_(elems[e], elems[e])] += He
        branches.append(br)
    load = float(p["force"] @ u)
    return e_tot - load, (g - p["force"])[free], H, scale + abs(load), np.concatenate(branches)


def _compare(p, precision, amp, seed, elastic=False):
    from fenics_nonlinear_energies_b200.assembler import SlopeStability3DCudaAssembler

    hd = torch.float32 if precision == "fp32" else torch.float64
    gpu = SlopeStability3DCudaAssembler(p, precision=precision, hess_dtype=hd,
                                        constitutive_mode="elastic" if elastic else "mc")
    assert gpu.info["kernel_variant"] == 11
    lay = gpu.layout
    free = np.asarray(p["freedofs"])
    rng = np.random.default_rng(seed)
    u_free = amp * rng.standard_normal(free.size)          # original free order
    e_ref, g_ref, H_ref, scale, br = _oracle(p, u_free, elastic)
    # the assembler works in the reordered numbering
    u_reord = u_free[lay.perm]
    e, g, h = gpu.eval(torch.as_tensor(u_reord, device="cuda"), 7)
    torch.cuda.synchronize()
    te, tg, th = TOL[precision]
    assert abs(float(e.item()) - e_ref) <= te * scale, (float(e.item()), e_ref)
    g_ref_reord = g_ref[lay.perm][lay.lo: lay.hi]
    gg = g[: gpu.n_owned].cpu().numpy()
    assert np.abs(gg - g_ref_reord).max() <= tg * np.abs(g_ref_reord).max()
    rev = np.empty(lay.n_free, dtype=np.int64)
    rev[lay.total_to_free_reord[free]] = free               # reordered id -> total DOF
    H_coo = H_ref[rev[lay.owned_rows], rev[lay.owned_cols]]
    hh = h.double().cpu().numpy()
    assert np.abs(hh - H_coo).max() <= th * np.abs(H_coo).max()
    # every element pair of free DOFs is in the pattern: the COO values carry all of H
    assert abs(np.abs(H_coo).sum() - np.abs(H_ref[np.ix_(free, free)]).sum()) <= 1e-9 * np.abs(H_coo).sum()
    return br


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_mc3d_p2_matches_oracle_plastic(precision):
    n = (3, 2, 2) if precision == "fp64" else (3, 2, 1)
    p = meshes.slope3d_problem(nx=n[0], ny=n[1], nz=n[2], degree=2, lam=1.5)
    br = _compare(p, precision, amp=4e-2, seed=3)
    assert (br > 0).mean() > 0.2  # the plastic branches are exercised
    assert len(set(br.tolist())) >= 3


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_mc3d_p2_matches_oracle_elastic_state(precision):
    p = meshes.slope3d_problem(nx=3, ny=2, nz=1, degree=2, lam=1.5)
    br = _compare(p, precision, amp=1e-5, seed=4)
    assert (br == 0).all()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_mc3d_p4_matches_oracle(precision):
    """P4 tetrahedra (35 nodes, the reference's 24-point rule; the node-by-node
    contraction of k_mc3d_elem_hi) against the oracle, elastic and plastic
    points mixed."""
    p = meshes.slope3d_problem(nx=3, ny=1, nz=1, degree=4, lam=1.5)
    br = _compare(p, precision, amp=2e-2, seed=9)
    assert len(set(br.tolist())) >= 2


def test_mc3d_p1_matches_oracle():
    p = meshes.slope3d_problem(nx=4, ny=2, nz=3, degree=1, lam=1.2)
    _compare(p, "fp64", amp=4e-2, seed=5)


def test_mc3d_elastic_mode_matches_oracle():
    p = meshes.slope3d_problem(nx=3, ny=2, nz=1, degree=2, lam=1.5)
    _compare(p, "fp64", amp=4e-2, seed=6, elastic=True)


def test_mc3d_separate_callbacks_and_rank_split():
    """energy_fn / gradient_fn / assemble_hessian agree with the fused pass,
    and a 2-rank split reproduces each rank's owned rows."""
    from fenics_nonlinear_energies_b200.assembler import SlopeStability3DCudaAssembler

    p = meshes.slope3d_problem(nx=3, ny=2, nz=2, degree=2, lam=1.5)
    full = SlopeStability3DCudaAssembler(p)
    u = 4e-2 * np.random.default_rng(8).standard_normal(full.layout.n_free)
    e, g, h = full.eval(torch.as_tensor(u, device="cuda"), 7)
    e, g, h = float(e.item()), g[: full.n_owned].cpu().numpy(), h.cpu().numpy()
    assert abs(full.energy_fn(u) - e) <= 1e-12 * max(1.0, abs(e))
    gg = np.zeros(full.n_owned)
    full.gradient_fn(u, gg)  # gradient-only path: rows summed by k_rowgrad, another fixed order
    np.testing.assert_allclose(gg, g, rtol=0, atol=1e-13 * np.abs(g).max())
    full.assemble_hessian(u)
    np.testing.assert_array_equal(full.owned_values.cpu().numpy(), h)

    class _Comm:
        def __init__(self, rank, size):
            self.rank, self.size = rank, size

        def Get_rank(self):
            return self.rank

        def Get_size(self):
            return self.size

    energies = 0.0
    for r in range(2):
        part = SlopeStability3DCudaAssembler(p, comm=_Comm(r, 2))
        ep, gp, hp = part.eval(torch.as_tensor(u, device="cuda"), 7)
        energies += float(ep.item())
        lo, hi = part.layout.lo, part.layout.hi
        np.testing.assert_allclose(gp[: part.n_owned].cpu().numpy(), g[lo:hi], rtol=0, atol=1e-12 * np.abs(g).max())
        keys_full = full.layout.owned_rows.astype(np.int64) * full.layout.n_free + full.layout.owned_cols
        keys_part = part.layout.owned_rows.astype(np.int64) * part.layout.n_free + part.layout.owned_cols
        order = np.argsort(keys_full)
        pos = order[np.searchsorted(keys_full[order], keys_part)]
        assert np.array_equal(keys_full[pos], keys_part)
        np.testing.assert_allclose(hp.cpu().numpy(), h[pos], rtol=0, atol=1e-12 * np.abs(h).max())
    # the element energies are split by ownership; the load term by owned rows
    assert abs(energies - e) <= 1e-11 * max(1.0, abs(e))
