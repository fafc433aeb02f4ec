"""Slope (Mohr-Coulomb) geometry pinned to the reference's own goldens.

Counts from ``tests/test_slope_stability_support.py:18-91`` and the Davis-B
values of ``tests/test_slope_stability_jax.py:20-24`` of the reference.
"""

import math

import numpy as np
import pytest

from fenics_nonlinear_energies_b200 import _lib, meshes
from oracle import energies, layout as L
from oracle.assembler import OracleAssembler


@pytest.mark.parametrize("level,nodes,elements,free", [
    (1, 157, 64, 260), (2, 701, 320, 1290), (3, 2721, 1300, 5220), (4, 10641, 5200, 20840)])
def test_p2_level_counts(level, nodes, elements, free):
    p = meshes.slope_problem(level=level, degree=2)
    assert p["nodes"].shape == (nodes, 2)
    assert p["elems_scalar"].shape == (elements, 6)
    assert p["elems"].shape == (elements, 12)
    assert p["freedofs"].shape == (free,)


def test_level3_qmask_sums():
    p = meshes.slope_problem(level=3, degree=2)
    assert int(p["q_mask"][:, 0].sum()) == 2580
    assert int(p["q_mask"][:, 1].sum()) == 2640


@pytest.mark.parametrize("degree,nodes,free", [(1, 2721, 5220), (2, 10641, 20840), (4, 42081, 83280)])
def test_same_mesh_counts_level4(degree, nodes, free):
    p = meshes.slope_problem(level=4, degree=degree)
    assert p["nodes"].shape == (nodes, 2)
    assert p["elems_scalar"].shape == (5200, {1: 3, 2: 6, 4: 15}[degree])
    assert p["freedofs"].shape == (free,)


def test_davis_b_golden():
    c, phi = meshes.davis_b_reduction(6.0, 45.0, 0.0, 1.0)
    assert math.isclose(c, 4.242640687119286, rel_tol=1e-14)
    assert math.isclose(phi, 35.264389682754654, rel_tol=1e-14)
    assert math.isclose(2.0 * c * math.cos(math.radians(phi)), 6.928203230275509, rel_tol=1e-14)


@pytest.mark.parametrize("n", [3, 5])
def test_gauss_jacobi_exactness(n):
    xi, w = meshes.gauss_jacobi_triangle(n)
    for i in range(2 * n):
        for j in range(2 * n - i):
            exact = math.factorial(i) * math.factorial(j) / math.factorial(i + j + 2)
            assert abs((w * xi[0] ** i * xi[1] ** j).sum() - exact) <= 1e-13 * exact


def test_p4_rule_degree9():
    """The P4 rule (the reference's make_quadrature(triangle, 9)): 19 points
    inside the triangle, positive weights, exact on every monomial of degree
    <= 9, and within rounding of Dunavant's published 15-digit table."""
    xi, w = meshes.slope_quadrature(4)
    assert xi.shape == (2, 19) and w.shape == (19,)
    assert (w > 0).all() and (xi > 0).all() and (xi.sum(0) < 1).all()
    for i in range(10):
        for j in range(10 - i):
            exact = math.factorial(i) * math.factorial(j) / math.factorial(i + j + 2)
            assert abs((w * xi[0] ** i * xi[1] ** j).sum() - exact) <= 2e-15 * exact, (i, j)
    published = [0.097135796282799, 0.489682519198738, 0.031334700227139, 0.437089591492937, 0.077827541004774,
                 0.188203535619033, 0.079647738927210, 0.044729513394453, 0.025577675658698, 0.221962989160766,
                 0.036838412054736, 0.043283539377289]
    ours = [meshes.DEG9_CENTROID_W] + [v for aw in meshes.DEG9_ORBITS_A for v in aw] + list(meshes.DEG9_ORBIT_AB)
    np.testing.assert_allclose(ours, published, rtol=0, atol=1e-15)


def test_lagrange_tabulation_partition_of_unity():
    for k in (1, 2, 4):
        xi, _ = meshes.slope_quadrature(k)
        phi, d1, d2 = meshes.lagrange_tabulate(k, xi)
        np.testing.assert_allclose(phi.sum(0), 1.0, atol=1e-13)
        np.testing.assert_allclose(d1.sum(0), 0.0, atol=1e-11)
        np.testing.assert_allclose(d2.sum(0), 0.0, atol=1e-11)
        # nodal interpolation property
        pts = meshes.lagrange_points(k).T
        np.testing.assert_allclose(meshes.lagrange_tabulate(k, pts)[0], np.eye(pts.shape[1]), atol=1e-12)


@pytest.mark.parametrize("degree", [2, 4])
def test_slope_layout_cabi_matches_oracle(degree):
    p = meshes.slope_problem(level=1, degree=degree)
    lay = _lib.build_layout(freedofs=p["freedofs"], elems=p["elems"], n_total=len(p["u_0"]), block_size=2,
                            coords=p["nodes"])
    adj = L.element_adjacency(p["elems"], p["freedofs"], len(p["u_0"]))
    perm = L.select_permutation("block_xyz", adjacency=adj, coords_all=p["nodes"], freedofs=p["freedofs"],
                                block_size=2)
    ref = L.build_global_layout(p["freedofs"], p["elems"], len(p["u_0"]), adj, perm, block_size=2)
    for k in ("perm", "owned_rows", "owned_cols", "elem_owner"):
        np.testing.assert_array_equal(lay[k], getattr(ref, k))


def test_mc_oracle_fd():
    p = meshes.slope_problem(level=1, degree=2, lam=1.3, with_elem_B=True)
    rng = np.random.default_rng(0)
    v = 0.05 * rng.standard_normal(p["elems"].shape)
    data = {k: p[k] for k in ("elem_B", "quad_weight", "eps_p_old")}
    d = rng.standard_normal(v.shape)
    h = 1e-7
    e, g, H = energies.element_derivatives("mc", v, data, p)
    ep = energies.element_derivatives("mc", v + h * d, data, p, want_hessian=False)
    em = energies.element_derivatives("mc", v - h * d, data, p, want_hessian=False)
    np.testing.assert_allclose(np.sum(g * d, 1), (ep[0] - em[0]) / (2 * h), rtol=2e-4, atol=1e-6)
    np.testing.assert_allclose(np.einsum("eij,ej->ei", H, d), (ep[1] - em[1]) / (2 * h), rtol=5e-3,
                               atol=1e-4 * np.abs(H).max())


def test_mc_oracle_gravity_load_matches_reference_rule():
    """force_a = sum_q quad_weight[e, q] * phi_a(q) * (0, -gamma), as the reference assembles it."""
    p = meshes.slope_problem(level=1, degree=2)
    asm = OracleAssembler("mc", dict(p, elem_B=meshes.slope_elem_B(p)), block_size=2)
    total = float(np.sum(p["force"][1::2]))
    area = float(np.sum(p["quad_weight"]))  # sum_q |det J_q| w_q over the elements
    assert math.isclose(total, -p["gamma"] * area, rel_tol=1e-12)
    assert asm.f_owned.size == asm.layout.hi - asm.layout.lo


@pytest.mark.parametrize("p", [1, 2, 4])
def test_tet_lagrange_tabulation(p):
    """Tetrahedral Lagrange basis: node count, the simplex_lagrange node order
    (P2 golden: vertices, then edge midpoints of (0,1), (1,2), (0,2), (1,3),
    (2,3), (0,3)), Kronecker property, partition of unity, and derivatives by
    central differences."""
    from fenics_nonlinear_energies_b200 import meshes

    counts = meshes.tet_lagrange_counts(p)
    assert len(counts) == (p + 1) * (p + 2) * (p + 3) // 6 and len(set(counts)) == len(counts)
    if p == 2:
        assert counts == [(2, 0, 0, 0), (0, 2, 0, 0), (0, 0, 2, 0), (0, 0, 0, 2), (1, 1, 0, 0), (0, 1, 1, 0),
                          (1, 0, 1, 0), (0, 1, 0, 1), (0, 0, 1, 1), (1, 0, 0, 1)]
    pts = meshes.tet_lagrange_points(p)
    phi, d1, d2, d3 = meshes.tet_lagrange_tabulate(p, pts)
    np.testing.assert_allclose(phi, np.eye(len(counts)), atol=1e-12)
    rng = np.random.default_rng(p)
    x = rng.dirichlet(np.ones(4), size=7).T[1:]          # interior points (3, 7)
    phi, d1, d2, d3 = meshes.tet_lagrange_tabulate(p, x)
    np.testing.assert_allclose(phi.sum(0), 1.0, atol=1e-12)
    for k, dk in enumerate((d1, d2, d3)):
        np.testing.assert_allclose(dk.sum(0), 0.0, atol=1e-10)
        h = 1e-6
        e = np.zeros((3, 1))
        e[k] = h
        fd = (meshes.tet_lagrange_tabulate(p, x + e)[0] - meshes.tet_lagrange_tabulate(p, x - e)[0]) / (2 * h)
        np.testing.assert_allclose(dk, fd, atol=1e-7 * max(1.0, np.abs(dk).max()))
