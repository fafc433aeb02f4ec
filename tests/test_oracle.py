"""Pin the CPU oracle: reference golden vectors and finite-difference consistency.

The golden vectors are the reference's own unit tests
(``tests/test_reordered_element_base.py:12-73``).  Element values have no
numeric golden in the reference; like its ``tests/test_slope_stability_3d.py:434-523``
the oracle derivatives are checked against central finite differences.
"""

import numpy as np
import pytest
from scipy import sparse

from oracle import energies, layout as L
from oracle.assembler import OracleAssembler
from fenics_nonlinear_energies_b200 import meshes


def test_block_xyz_scalar_golden():
    coords = np.array([[1.0, 0.0], [0.0, 1.0], [0.0, 0.0], [1.0, 1.0]])
    perm = L.select_permutation("block_xyz", adjacency=sparse.eye(4, format="csr"), coords_all=coords,
                                freedofs=np.arange(4), block_size=1)
    assert perm.tolist() == [2, 1, 0, 3]


def test_block_xyz_vector_golden():
    coords = np.array([[1.0, 0.0, 0.0], [0.0, 0.0, 0.0]])
    perm = L.select_permutation("block_xyz", adjacency=sparse.eye(6, format="csr"), coords_all=coords,
                                freedofs=np.arange(6), block_size=3)
    assert perm.tolist() == [3, 4, 5, 0, 1, 2]


def test_local_vec_from_full_golden():
    v = L.local_vec_from_full(np.array([10.0, 20.0, 30.0]), np.array([-1, 0, 1, -1, 2]),
                              np.arange(5), np.array([5.0, -1.0, -1.0, 6.0, -1.0]))
    np.testing.assert_allclose(v, [5.0, 10.0, 20.0, 6.0, 30.0])


def test_ownership_ranges():
    assert [L.petsc_ownership_range(10, r, 3) for r in range(3)] == [(0, 4), (4, 7), (7, 10)]
    assert [L.petsc_ownership_range(12, r, 2, block_size=3) for r in range(2)] == [(0, 6), (6, 12)]
    np.testing.assert_array_equal(L.rank_of_dof_vec(np.arange(10), 10, 3), [0, 0, 0, 0, 1, 1, 1, 2, 2, 2])


def _fd_check(family, v_e, data, params, h=1e-7, seed=0):
    """Central FD of energy vs gradient, and of gradient vs Hessian (directional)."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal(v_e.shape)
    e, g, H = energies.element_derivatives(family, v_e, data, params)
    ep, gp, _ = energies.element_derivatives(family, v_e + h * d, data, params, want_hessian=False)
    em, gm, _ = energies.element_derivatives(family, v_e - h * d, data, params, want_hessian=False)
    dd_fd = (ep - em) / (2 * h)
    dd = np.sum(g * d, axis=1)
    np.testing.assert_allclose(dd, dd_fd, rtol=2e-4, atol=1e-8 * np.abs(dd).max())
    hv_fd = (gp - gm) / (2 * h)
    hv = np.einsum("eij,ej->ei", H, d)
    np.testing.assert_allclose(hv, hv_fd, rtol=5e-3, atol=1e-5 * np.abs(hv).max())


def test_plaplace_oracle_fd():
    params, _ = meshes.plaplace_problem(n=4)
    v = np.random.default_rng(1).random(len(params["u_0"]))
    e = params["elems"]
    _fd_check("plaplace", v[e], {k: params[k] for k in ("dvx", "dvy", "vol")}, params)


def test_gl_oracle_fd():
    params, _ = meshes.gl_problem(n=4)
    v = np.random.default_rng(2).uniform(-1, 1, len(params["u_0"]))
    e = params["elems"]
    _fd_check("gl", v[e], {k: params[k] for k in ("dvx", "dvy", "vol")}, params)


def test_he_oracle_fd():
    params, _ = meshes.he_beam_problem(nx=3, ny=1, nz=1)
    y = params["u_0_ref"] + 1e-3 * np.random.default_rng(3).standard_normal(len(params["u_0_ref"]))
    e = params["elems"]
    _fd_check("he", y[e], {k: params[k] for k in ("dphix", "dphiy", "dphiz", "vol")}, params, h=1e-7)


def test_plaplace_zero_gradient_limit():
    params, _ = meshes.plaplace_problem(n=2)
    e = params["elems"]
    v = np.zeros((len(e), 3))
    _, g, H = energies.element_derivatives("plaplace", v, {k: params[k] for k in ("dvx", "dvy", "vol")}, params)
    assert np.all(g == 0.0) and np.all(H == 0.0)


@pytest.mark.parametrize("numbering", ["x_slow", "x_fast"])
def test_oracle_assembler_consistency(numbering):
    params, _ = meshes.gl_problem(n=6, numbering=numbering)
    asm = OracleAssembler("gl", params)
    rng = np.random.default_rng(4)
    u = rng.uniform(-0.8, 0.8, asm.layout.n_free)
    d = rng.standard_normal(asm.layout.n_free)
    h = 1e-6
    g = asm.gradient_fn(u)
    fd = (asm.energy_fn(u + h * d) - asm.energy_fn(u - h * d)) / (2 * h)
    assert abs(fd - g @ d) < 1e-6 * max(1.0, abs(fd))
    vals = asm.assemble_hessian_element(u)
    A = sparse.coo_matrix((vals, (asm.layout.owned_rows, asm.layout.owned_cols)),
                          shape=(asm.layout.n_free,) * 2).tocsr()
    hv_fd = (asm.gradient_fn(u + h * d) - asm.gradient_fn(u - h * d)) / (2 * h)
    np.testing.assert_allclose(A @ d, hv_fd, rtol=1e-5, atol=1e-7)
    assert abs(A - A.T).max() < 1e-14


def test_golden_section_restatement():
    from fenics_nonlinear_energies_b200.newton import golden_section_search, repair_linesearch_interval

    calls = []

    def f(a):
        calls.append(a)
        return (a - 0.7) ** 2

    alpha, n = golden_section_search(f, -0.5, 2.0, 1e-3)
    assert abs(alpha - 0.7) < 1e-3 and n == len(calls)
    # non-finite right end is bisected back toward the centre
    g = lambda a: float("inf") if a > 1.0 else (a - 0.5) ** 2  # noqa: E731
    a, b, _, repaired = repair_linesearch_interval(g, -0.5, 2.0, center=0.0, center_value=g(0.0), tol=1e-6)
    assert repaired and a == -0.5 and 1.0 - 1e-5 < b <= 1.0


def test_mlp_oracle_bf16_rounding():
    from oracle.mlp import bf16_round

    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0], dtype=np.float32)
    np.testing.assert_array_equal(bf16_round(x), [1.0, 1.0, 1.0 + 2 ** -7, -2.5, 0.0])



@pytest.mark.parametrize("case", ["spd", "indefinite_late", "indefinite_first", "maxit", "zero_rhs"])
def test_scalar_cg_oracle(case):
    from oracle import krylov

    rng = np.random.default_rng(7)
    n = 60
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    ev = np.linspace(1.0, 50.0, n)
    if case == "indefinite_late":
        ev[:3] = [-4.0, -2.0, -1.0]
    if case == "indefinite_first":
        ev[:] = -np.linspace(1.0, 5.0, n)
    A = (Q * ev) @ Q.T
    A = 0.5 * (A + A.T)
    b = np.zeros(n) if case == "zero_rhs" else rng.standard_normal(n)
    dinv = krylov.jacobi_scaling(np.diag(A))
    rtol, maxit = (1e-10, 7) if case == "maxit" else (1e-10, 200)
    x, it, why = krylov.pcg(A, dinv, b, rtol, maxit)
    if case == "spd":
        assert why == krylov.CONVERGED and it < n + 5
        np.testing.assert_allclose(x, np.linalg.solve(A, b), rtol=1e-8, atol=1e-10)
    elif case == "indefinite_late":
        assert why == krylov.NEGATIVE_CURVATURE and it > 1 and (x @ b) > 0  # descent for the quadratic
    elif case == "indefinite_first":
        assert (it, why) == (1, krylov.NEGATIVE_CURVATURE) and np.array_equal(x, b)
    elif case == "maxit":
        assert (it, why) == (7, krylov.ITERATION_LIMIT)
    else:
        assert (it, why) == (0, krylov.ZERO_RHS) and not x.any()
    np.testing.assert_array_equal(krylov.jacobi_scaling([2.0, -4.0, 0.0, np.nan]), [0.5, 0.25, 1.0, 1.0])


def test_oracle_adopted_layout_and_restricted_rows():
    """A precomputed layout gives the same callbacks; ``restricted_rows`` equals
    the full assembly on the rows it covers (used by the full-size GPU tests)."""
    from fenics_nonlinear_energies_b200 import _lib

    p = meshes.slope_problem(level=1, degree=4, with_elem_B=True)
    full = OracleAssembler("mc", p, block_size=2)
    lay = _lib.build_layout(freedofs=p["freedofs"], elems=p["elems"], n_total=len(p["u_0"]), block_size=2,
                            coords=p["nodes"])
    lay["n_free"] = full.layout.n_free
    adopted = OracleAssembler("mc", p, block_size=2, layout=lay)
    u = 2e-3 * np.random.default_rng(4).standard_normal(full.layout.n_free)
    e0, g0, h0 = full.all_in_one(u)
    e1, g1, h1 = adopted.all_in_one(u)
    assert e0 == e1 and np.array_equal(g0, g1) and np.array_equal(h0, h1)
    rows = np.random.default_rng(5).choice(full.layout.n_free, 40, replace=False)
    g, pos, vals = full.restricted_rows(u, rows)
    np.testing.assert_allclose(g, g0[np.sort(rows)], rtol=0, atol=1e-13 * np.abs(g0).max())
    np.testing.assert_array_equal(np.sort(pos), np.flatnonzero(np.isin(full.layout.owned_rows, rows)))
    np.testing.assert_allclose(vals, h0[pos], rtol=0, atol=1e-13 * np.abs(h0).max())


@pytest.mark.parametrize("family", ["gl", "plaplace"])
def test_numba_cpu_line_matches_oracle(family):
    """The numba-parallel CPU line of the benchmark equals the oracle."""
    from oracle.cpu_fast import FastTriangleAssembler

    if family == "gl":
        params, u = meshes.gl_problem(n=24, seed=4)
    else:
        params, _ = meshes.plaplace_problem(n=24)
        u = None
    orc = OracleAssembler(family, params)
    fast = FastTriangleAssembler(orc)
    states = [u[orc.layout.perm]] if u is not None else [
        0.3 * np.random.default_rng(2).standard_normal(orc.layout.n_free), np.zeros(orc.layout.n_free)]
    for s in states:
        e0, g0, h0 = orc.all_in_one(s)
        e1, g1, h1 = fast.all_in_one(s)
        assert abs(e1 - e0) <= 1e-12 * max(1.0, abs(e0))
        np.testing.assert_allclose(g1, g0, rtol=0, atol=1e-12 * max(1e-300, np.abs(g0).max()))
        np.testing.assert_allclose(h1, h0, rtol=0, atol=1e-12 * max(1e-300, np.abs(h0).max()))
