"""Oracle, host layout and mesh inputs against outputs of the reference itself.

``tests/golden/reference_*.npz`` were written by ``tests/golden/make_fixtures.py``,
which runs the reference's own assembler classes and helpers (torch standing
in for JAX).  These CPU tests check, on the same inputs:

* the oracle (``oracle/``) -- energies, owned gradients and owned COO Hessian
  values of every family, one rank and every rank of 2/3-rank splits, at
  1e-12 relative; the layout arrays bit-exact;
* the host C++ layout (``fne_layout_build`` through the C ABI) bit-exact;
* this repository's mesh generators: the structured P1 geometry, the
  Neo-Hookean twist, the P2 slope generator and the P4 same-mesh builder
  reproduce the reference's arrays; Davis-B values;
* the 3-D oracle against the reference's 3-D element functions (energy,
  residual, constitutive Hessian, elastic mode) on P1 / P2 / P4 tets.
"""

from pathlib import Path

import numpy as np
import pytest

from fenics_nonlinear_energies_b200 import _lib, meshes
from oracle.assembler import OracleAssembler

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = 1e-12
LAYOUT_KEYS = ("perm", "iperm", "total_to_free_reord", "owned_rows", "owned_cols", "elem_owner")

FAMILIES = {
    # family: (fixture, oracle family, oracle kwargs, scalar keys)
    "plaplace": ("plaplace", "plaplace", {}, ("p",)),
    "gl": ("gl", "gl", {}, ("eps",)),
    "he": ("he", "he", dict(block_size=3, coordinate_key="nodes2coord", dirichlet_key="u_0_ref"), ("C1", "D1")),
    "mc_p2": ("mc_p2", "mc", dict(block_size=2), ("E", "nu", "phi_deg", "cohesion", "reg")),
    "mc_p4": ("mc_p4", "mc", dict(block_size=2), ("E", "nu", "phi_deg", "cohesion", "reg")),
}


def load(name):
    return dict(np.load(GOLDEN / f"reference_{name}.npz"))


def fixture_params(fx):
    params = {k[3:]: v for k, v in fx.items() if k.startswith("in_")}
    for k, v in fx.items():
        if k.startswith("sc_"):
            params[k[3:]] = float(v)
    return params


def splits(fx):
    out = []
    for size in (1, 2, 3):
        for r in range(size):
            if f"r{size}_{r}_energy" in fx:
                out.append((r, size))
    return out


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(1e-300, np.abs(np.asarray(b)).max())


@pytest.mark.parametrize("name", list(FAMILIES))
def test_oracle_matches_reference_outputs(name):
    fixture, fam, okw, _ = FAMILIES[name]
    fx = load(fixture)
    params = fixture_params(fx)
    u = fx["in_u"]
    for r, size in splits(fx):
        key = f"r{size}_{r}_"
        orc = OracleAssembler(fam, params, rank=r, size=size, **okw)
        if "in_dirichlet" in fx:
            orc.update_dirichlet(fx["in_dirichlet"])
        for k in LAYOUT_KEYS:
            np.testing.assert_array_equal(getattr(orc.layout, k), fx[key + k], err_msg=f"{name} {r}/{size} {k}")
        assert (orc.layout.lo, orc.layout.hi) == (int(fx[key + "lo"]), int(fx[key + "hi"]))
        np.testing.assert_array_equal(orc.local.energy_weights, fx[key + "energy_weights"])
        e, g, h = orc.all_in_one(u)
        e_ref = float(fx[key + "energy"])
        assert abs(e - e_ref) <= TOL * max(1.0, abs(e_ref)), (name, r, size, e, e_ref)
        assert rel(g, fx[key + "grad"]) <= TOL, (name, r, size)
        assert rel(h, fx[key + "hess"]) <= TOL, (name, r, size)
        np.testing.assert_array_equal(fx[key + "coo_rows"], orc.layout.owned_rows)
        np.testing.assert_array_equal(fx[key + "coo_cols"], orc.layout.owned_cols)


@pytest.mark.parametrize("name", list(FAMILIES))
def test_host_layout_matches_reference(name):
    fixture, _, okw, _ = FAMILIES[name]
    fx = load(fixture)
    params = fixture_params(fx)
    bs = okw.get("block_size", 1)
    ck = okw.get("coordinate_key", "nodes")
    dk = okw.get("dirichlet_key", "u_0")
    for r, size in splits(fx):
        key = f"r{size}_{r}_"
        lay = _lib.build_layout(freedofs=params["freedofs"], elems=params["elems"], n_total=len(params[dk]),
                                block_size=bs, coords=params[ck], rank=r, size=size, device=False)
        for k in LAYOUT_KEYS:
            np.testing.assert_array_equal(lay[k], fx[key + k], err_msg=f"{name} {r}/{size} {k}")
        assert (lay["lo"], lay["hi"]) == (int(fx[key + "lo"]), int(fx[key + "hi"]))


def test_plaplace_zero_state_energy_and_gradient():
    """The p-Laplace configuration's assembly start (u = 0): energy and gradient as the reference."""
    fx, z = load("plaplace"), load("plaplace_zero")
    orc = OracleAssembler("plaplace", fixture_params(fx))
    u = np.zeros(orc.layout.n_free)
    assert abs(orc.energy_fn(u) - float(z["energy"])) <= TOL
    np.testing.assert_allclose(orc.gradient_fn(u), z["grad"], rtol=0, atol=TOL * np.abs(z["grad"]).max())


def test_mesh_generators_reproduce_reference_inputs():
    fx = load("gl")
    params, u0 = meshes.gl_problem(n=16, seed=3)
    for k in ("nodes", "u_0", "freedofs", "elems", "dvx", "dvy", "vol", "ip", "w"):
        np.testing.assert_array_equal(params[k], fx["in_" + k], err_msg=k)
    fx = load("plaplace")
    params, _ = meshes.plaplace_problem(n=16)
    for k in ("nodes", "freedofs", "elems", "dvx", "dvy", "vol", "f"):
        np.testing.assert_array_equal(params[k], fx["in_" + k], err_msg=k)
    fx = load("he")
    params, _ = meshes.he_beam_problem(nx=6, ny=2, nz=2)
    for k in ("u_0_ref", "freedofs", "elems", "elems_scalar", "dphix", "dphiy", "dphiz", "vol", "nodes2coord"):
        np.testing.assert_array_equal(params[k], fx["in_" + k], err_msg=k)
    rotated = meshes.rotate_right_face_from_reference(params["u_0_ref"], params["nodes2coord"],
                                                      float(fx["sc_angle"]), params["right_nodes"])
    np.testing.assert_allclose(rotated, fx["in_dirichlet"], rtol=0, atol=1e-16)


def test_structured_p1_geometry_matches_reference():
    """``p1_triangle_operators`` against the reference's ``_triangle_operators``."""
    s = load("support")
    for n in (4, 16):
        nodes, elems, _ = meshes.square_p1(n, -1.0, 1.0)
        np.testing.assert_array_equal(nodes, s[f"n{n}_nodes"])
        np.testing.assert_array_equal(elems, s[f"n{n}_elems"])
        dvx, dvy, vol = meshes.p1_triangle_operators(nodes, elems)
        for mine, k in ((dvx, "dvx"), (dvy, "dvy"), (vol, "vol")):
            ref = s[f"n{n}_{k}"]
            np.testing.assert_allclose(mine, ref, rtol=0, atol=1e-15 * np.abs(ref).max(), err_msg=k)


def test_davis_b_matches_reference():
    s = load("support")
    for lam, (c, phi) in zip(s["lams"], s["davis_b"]):
        mc, mphi = meshes.davis_b_reduction(6.0, 45.0, 0.0, float(lam))
        assert (mc, mphi) == (c, phi)


@pytest.mark.parametrize("degree", [2, 4])
def test_slope_generator_matches_reference(degree):
    """The slope generator and same-mesh builder against the reference's
    ``build_case_data`` (P2) / ``_build_same_mesh_lagrange_case_data_impl``
    (P4; basix stood in by this repository's basis and rule)."""
    fx = load(f"mc_p{degree}")
    p = meshes.slope_problem(level=int(fx["sc_level"]), degree=degree, with_elem_B=True)
    for k in ("elems_scalar", "elems", "freedofs", "q_mask"):
        np.testing.assert_array_equal(p[k], fx["in_" + k], err_msg=k)
    for k in ("nodes", "quad_weight", "force", "elem_B"):
        ref = fx["in_" + k]
        # same formulas, summation order differs (matrix products vs the reference's loops)
        np.testing.assert_allclose(p[k], ref, rtol=0, atol=1e-14 * np.abs(ref).max(), err_msg=k)
    assert (p["cohesion"], p["phi_deg"]) == (float(fx["sc_cohesion"]), float(fx["sc_phi_deg"]))


@pytest.mark.parametrize("degree", [2, 4])
def test_slope_fixture_state_is_partly_plastic(degree):
    """The stored displacement drives some quadrature points off the elastic branch."""
    from oracle import energies

    fx = load(f"mc_p{degree}")
    params = fixture_params(fx)
    orc = OracleAssembler("mc", params, block_size=2)
    v = orc.v_local(fx["in_u"])[orc.local.elems_local_np]
    strain = np.einsum("eqij,ej->eqi", orc.elem_data["elem_B"], v)
    C, _ = energies.mc_elastic_tensors(params["E"], params["nu"])
    sig = np.einsum("ij,eqj->eqi", np.asarray(C), strain - orc.elem_data["eps_p_old"])
    m, d = 0.5 * (sig[..., 0] + sig[..., 1]), 0.5 * (sig[..., 0] - sig[..., 1])
    r = np.sqrt(d * d + sig[..., 2] ** 2 + params["reg"] ** 2)
    sp = np.sin(np.deg2rad(params["phi_deg"]))
    f_tr = (1 + sp) * (m + r) - (1 - sp) * (m - r) - 2 * params["cohesion"] * np.cos(np.deg2rad(params["phi_deg"]))
    frac = float(np.mean(f_tr > 0.0))
    assert 0.05 < frac < 0.95, frac


@pytest.mark.parametrize("degree", [2, 4])
def test_geometry_recovered_from_reference_elem_B(degree):
    """The element map recovered from the reference's stored ``elem_B`` /
    ``quad_weight`` (how the CUDA assembler accepts the reference's own
    problem data) rebuilds ``elem_B`` and matches the generator's map."""
    fx = load(f"mc_p{degree}")
    p = meshes.slope_problem(level=int(fx["sc_level"]), degree=degree)
    inv, det = meshes.geometry_from_elem_B(fx["in_elem_B"], fx["in_quad_weight"], p["dhat1"], p["dhat2"], p["quad_w"])
    B = meshes.slope_elem_B(dict(p, inv_jac=inv, det_j=det))
    np.testing.assert_allclose(B, fx["in_elem_B"], rtol=0, atol=1e-14 * np.abs(fx["in_elem_B"]).max())
    ref_inv = p["inv_jac"] if p["inv_jac"].ndim == 3 else np.broadcast_to(p["inv_jac"][:, None], inv.shape)
    np.testing.assert_allclose(inv, ref_inv, rtol=0, atol=1e-13 * np.abs(ref_inv).max())
    ref_det = p["det_j"] if p["det_j"].ndim == 2 else np.broadcast_to(p["det_j"][:, None], det.shape)
    np.testing.assert_allclose(det, ref_det, rtol=1e-13)


@pytest.mark.parametrize("degree", [1, 2, 4])
def test_mc3d_oracle_matches_reference_elements(degree):
    """The 3-D oracle (``oracle/energies3d.py``) against the reference's own
    3-D element functions run on the same inputs (``reference_mc3d.npz``:
    ``element_energy_3d``, ``element_residual_3d``,
    ``constitutive_element_hessian_3d`` and the elastic mode's energy and
    constitutive Hessian of ``slope_stability_3d/jax/jax_energy_3d.py``),
    P1 / P2 / P4 tets at a state that reaches every return branch: 1e-12
    relative (energy to |e|, gradient and Hessian to their largest entry)."""
    from oracle import energies3d as E3

    d = np.load(GOLDEN / "reference_mc3d.npz")
    keys = ("dphix", "dphiy", "dphiz", "quad_weight", "c_bar", "sin_phi", "shear", "bulk", "lame")
    ue = d[f"p{degree}_u_elem"]
    branches = []
    for e in range(ue.shape[0]):
        args = [d[f"p{degree}_{k}"][e] for k in keys]
        ee, ge, He, br = E3.element_derivatives(ue[e], *args)
        branches.append(br)
        er, gr, hr = float(d[f"p{degree}_energy"][e]), d[f"p{degree}_grad"][e], d[f"p{degree}_hess"][e]
        assert abs(ee - er) <= 1e-12 * abs(er), (e, ee, er)
        assert np.abs(ge - gr).max() <= 1e-12 * np.abs(gr).max(), e
        assert np.abs(He - hr).max() <= 1e-12 * np.abs(hr).max(), e
        # elastic mode: psi = lame/2 I1^2 + mu Q, tangent C (closed form)
        dphix, dphiy, dphiz, w = args[:4]
        shear, lame = args[6], args[8]
        eps = E3.strain6(ue[e], dphix, dphiy, dphiz)
        B = E3.strain_operator(dphix, dphiy, dphiz)
        C = np.zeros((eps.shape[0], 6, 6))
        C[:, :3, :3] = lame[:, None, None]
        for i in range(3):
            C[:, i, i] += 2.0 * shear
            C[:, 3 + i, 3 + i] = shear
        el_e = float(np.sum(w * E3.elastic_density(eps, shear, lame)))
        el_h = np.einsum("qsi,qst,qtj,q->ij", B, C, B, w)
        assert abs(el_e - float(d[f"p{degree}_el_energy"][e])) <= 1e-12 * abs(el_e)
        ref_h = d[f"p{degree}_el_hess"][e]
        assert np.abs(el_h - ref_h).max() <= 1e-12 * np.abs(ref_h).max()
    if degree > 1:  # the fixture states reach the plastic branches
        assert len(set(np.concatenate(branches).tolist())) >= 4
