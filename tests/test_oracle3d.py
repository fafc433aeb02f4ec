"""CPU checks of the 3-D Mohr-Coulomb oracle (``oracle/energies3d.py``).

The reference pins its 3-D density the same way (finite differences of the
autodiff stress / tangent, ``tests/test_slope_stability_3d.py:434-523``):
elastic closed form, central differences of sigma = dpsi/deps and
D = dsigma/deps inside every branch, branch coverage, continuity of psi
across the yield surface, and an element-level check on a P1 tetrahedron.
"""

import numpy as np
import pytest

from oracle import energies3d as E3

LAME, SHEAR = 2.0e4 * 0.3 / (1.3 * 0.4), 2.0e4 / 2.6  # E = 2e4, nu = 0.3
BULK = LAME + 2.0 * SHEAR / 3.0


def _params(c_bar, sin_phi, n):
    return [np.full(n, v) for v in (c_bar, sin_phi, SHEAR, BULK, LAME)]


def test_elastic_branch_closed_form():
    rng = np.random.default_rng(0)
    eps = 1e-4 * rng.standard_normal((5, 6))
    sig, D, psi, br = E3.mc_stress_tangent(eps, *_params(1e6, 0.5, 5))
    assert (br == 0).all()
    np.testing.assert_allclose(psi, E3.elastic_density(eps, SHEAR, LAME), rtol=1e-13)
    I1 = eps[:, :3].sum(1)
    sig_ref = np.concatenate([LAME * I1[:, None] + 2 * SHEAR * eps[:, :3], SHEAR * eps[:, 3:]], axis=1)
    np.testing.assert_allclose(sig, sig_ref, rtol=1e-12, atol=1e-12 * np.abs(sig_ref).max())
    D_ref = np.zeros((6, 6))
    D_ref[:3, :3] = LAME
    D_ref += np.diag([2 * SHEAR] * 3 + [SHEAR] * 3)
    for i in range(5):
        np.testing.assert_allclose(D[i], D_ref, rtol=1e-12, atol=1e-9)


def _sample_branches(n=4000, seed=1):
    rng = np.random.default_rng(seed)
    dev = rng.standard_normal((n, 6)) * 1e-3
    vol = rng.uniform(-1.0, 4.0, size=(n, 1)) * 1e-3
    eps = dev.copy()
    eps[:, :3] += vol
    c = rng.uniform(0.1, 20.0, size=n)
    sp = rng.uniform(0.2, 0.7, size=n)
    _, br = E3.mc_density(eps, c, sp, SHEAR, BULK, LAME)
    return eps, c, sp, br


def test_every_branch_is_reached():
    _, _, _, br = _sample_branches()
    counts = np.bincount(br, minlength=5)
    assert (counts > 0).all(), counts


@pytest.mark.parametrize("branch", [1, 2, 3, 4])
def test_stress_and_tangent_by_central_differences(branch):
    eps, c, sp, br = _sample_branches()
    idx = np.flatnonzero(br == branch)[:3]
    h = 1e-8
    for i in idx:
        e0 = eps[i]
        prm = [c[i], sp[i], SHEAR, BULK, LAME]
        sig, D, psi, b = E3.mc_stress_tangent(e0[None], *prm)
        assert b[0] == branch
        ok = True
        fd_sig = np.zeros(6)
        fd_D = np.zeros((6, 6))
        for k in range(6):
            dk = np.zeros(6)
            dk[k] = h
            (pp, bp), (pm, bm) = E3.mc_density(e0 + dk, *prm), E3.mc_density(e0 - dk, *prm)
            ok &= bool(bp[()] == branch and bm[()] == branch)
            fd_sig[k] = (pp - pm) / (2 * h)
            sp_, _, _, _ = E3.mc_stress_tangent((e0 + dk)[None], *prm)
            sm_, _, _, _ = E3.mc_stress_tangent((e0 - dk)[None], *prm)
            fd_D[:, k] = (sp_[0] - sm_[0]) / (2 * h)
        if not ok:  # a difference step crossed a branch boundary
            continue
        # the apex potential is linear in I1 (zero tangent): absolute scale = the elastic modulus
        scale = LAME + 2.0 * SHEAR
        np.testing.assert_allclose(sig[0], fd_sig, rtol=2e-5, atol=2e-5 * np.abs(sig[0]).max())
        np.testing.assert_allclose(D[0], fd_D, rtol=5e-4, atol=5e-4 * np.abs(D[0]).max() + 1e-8 * scale)
        np.testing.assert_allclose(D[0], D[0].T, atol=1e-9 * max(np.abs(D[0]).max(), scale))


def test_potential_continuous_across_yield_surface():
    """psi is C1 across the elastic / plastic boundary: along a strain ray the
    values just inside and just outside agree to the step."""
    rng = np.random.default_rng(3)
    for _ in range(20):
        d = rng.standard_normal(6)
        prm = [rng.uniform(0.5, 5.0), rng.uniform(0.2, 0.6), SHEAR, BULK, LAME]
        ts = np.linspace(0.0, 5e-3, 4001)
        psi, br = E3.mc_density(ts[:, None] * d[None], *prm)
        cross = np.flatnonzero((br[:-1] == 0) & (br[1:] != 0))
        if cross.size == 0:
            continue
        j = cross[0]
        jump = abs(psi[j + 1] - psi[j])
        slope = abs(psi[j] - psi[j - 1])
        assert jump <= 3.0 * slope + 1e-12


def test_p1_tet_element_derivatives():
    X = np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [0.2, 1.1, 0.1], [0.1, 0.3, 0.9]])
    M = np.concatenate([np.ones((4, 1)), X], axis=1)
    grads = np.linalg.inv(M)[1:]                       # (3, 4): d phi_a / d x_k
    vol = abs(np.linalg.det(M)) / 6.0
    dphix, dphiy, dphiz = (grads[k][None, :] for k in range(3))
    qw = np.array([vol])
    prm = [np.array([60.0]), np.array([0.45]), np.array([SHEAR]), np.array([BULK]), np.array([LAME])]
    rng = np.random.default_rng(4)
    u = 2e-3 * rng.standard_normal(12)
    e, g, H, br = E3.element_derivatives(u, dphix, dphiy, dphiz, qw, *prm)
    assert br[0] == 2  # a return branch with a full-rank tangent at this load (left edge)
    h = 1e-8
    fd_g = np.array([(E3.element_derivatives(u + h * np.eye(12)[i], dphix, dphiy, dphiz, qw, *prm)[0] -
                      E3.element_derivatives(u - h * np.eye(12)[i], dphix, dphiy, dphiz, qw, *prm)[0]) / (2 * h)
                     for i in range(12)])
    np.testing.assert_allclose(g, fd_g, rtol=1e-5, atol=1e-5 * np.abs(g).max())
    d = rng.standard_normal(12)
    gp = E3.element_derivatives(u + h * d, dphix, dphiy, dphiz, qw, *prm)[1]
    gm = E3.element_derivatives(u - h * d, dphix, dphiy, dphiz, qw, *prm)[1]
    np.testing.assert_allclose(H @ d, (gp - gm) / (2 * h), rtol=5e-4, atol=5e-4 * np.abs(H @ d).max())
    np.testing.assert_allclose(H, H.T, atol=1e-9 * np.abs(H).max())


@pytest.mark.parametrize("branch", [0, 1, 2, 3, 4])
def test_spectral_chain_rule_matches_autodiff(branch):
    """The eigenvalue chain rule a device kernel evaluates (d lambda = v v^T,
    second derivatives with the 1/(lambda_k - lambda_j) eigenvector terms)
    against autodiff through eigvalsh, in every branch."""
    from oracle import spectral3d

    eps, c, sp, br = _sample_branches()
    idx = np.flatnonzero(br == branch)[:4]
    assert idx.size > 0
    for i in idx:
        prm = [c[i], sp[i], SHEAR, BULK, LAME]
        sig_a, D_a, _, b = E3.mc_stress_tangent(eps[i][None], *prm)
        scale = LAME + 2.0 * SHEAR
        for eigh in (np.linalg.eigh, spectral3d.jacobi_eigh3):   # LAPACK and the kernel's Jacobi sweeps
            sig_s, D_s, bs = spectral3d.stress_tangent_spectral(eps[i], *prm, eigh=eigh)
            assert b[0] == bs == branch
            np.testing.assert_allclose(sig_s, sig_a[0], rtol=1e-9, atol=1e-11 * scale * np.abs(eps[i]).max())
            np.testing.assert_allclose(D_s, D_a[0], rtol=1e-7, atol=1e-9 * scale)


def test_tet_quadrature_exactness():
    from math import factorial

    from fenics_nonlinear_energies_b200 import meshes

    for n in (2, 3, 4):
        xi, w = meshes.gauss_jacobi_tet(n)
        assert abs(w.sum() - 1.0 / 6.0) < 1e-15
        for a in range(2 * n):
            for b in range(2 * n - a):
                for c in range(2 * n - a - b):
                    exact = factorial(a) * factorial(b) * factorial(c) / factorial(a + b + c + 3)
                    assert abs(np.sum(w * xi[0] ** a * xi[1] ** b * xi[2] ** c) - exact) < 1e-15


def test_slope3d_mesh_and_assembly():
    """Synthetic P2 tet slope: counts, volume, orientation; global energy,
    gradient and Hessian assembled from the 3-D oracle, checked by central
    differences along random directions (the layout of the future family)."""
    from fenics_nonlinear_energies_b200 import meshes

    p = meshes.slope3d_problem(nx=2, ny=1, nz=1, degree=2, lam=1.5, quad_n=2)  # 8 points: enough for FD checks
    nv = 3 * 2 * 2
    assert p["elems_scalar"].shape == (12, 10)
    assert p["nodes"].shape[0] == nv + len({tuple(sorted(e)) for t in p["elems_scalar"][:, :4]
                                            for e in [(t[a], t[b]) for a, b in meshes.TET_EDGES]})
    # straight-sided slope over two x cells: H = 20 at x = 0, 15 at x = 20, 10 at x = 40
    assert abs(p["quad_weight"].sum() - 10.0 * (20.0 * 17.5 + 20.0 * 12.5)) < 1e-9
    X = p["nodes"][p["elems_scalar"][:, :4]]
    assert (np.linalg.det(np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], 1)) > 0).all()
    free, elems = p["freedofs"], p["elems"]
    prm = [p[k] for k in ("c_bar", "sin_phi", "shear", "bulk", "lame")]

    def assemble(u_free, want_h=True):
        u = p["u_0"].copy()
        u[free] = u_free
        n = u.size
        e_tot, g, H = 0.0, np.zeros(n), np.zeros((n, n)) if want_h else None
        for e in range(elems.shape[0]):
            args = (p["dphix"][e], p["dphiy"][e], p["dphiz"][e], p["quad_weight"][e], *[a[e] for a in prm])
            if want_h:
                ee, ge, He, _ = E3.element_derivatives(u[elems[e]], *args)
                H[np.ix_(elems[e], elems[e])] += He
            else:
                eps = E3.strain6(u[elems[e]], *args[:3])
                ee = float(np.sum(args[3] * E3.mc_density(eps, *[a for a in args[4:]])[0]))
                ge = 0.0
            e_tot += ee
            if want_h:
                np.add.at(g, elems[e], ge)
        e_tot -= p["force"] @ u
        return e_tot, (g - p["force"])[free], (H[np.ix_(free, free)] if want_h else None)

    rng = np.random.default_rng(7)
    u = 3e-3 * rng.standard_normal(free.size)
    e0, g0, H0 = assemble(u)
    np.testing.assert_allclose(H0, H0.T, atol=1e-9 * np.abs(H0).max())
    d = rng.standard_normal(free.size)
    h = 1e-7
    fd = (assemble(u + h * d, False)[0] - assemble(u - h * d, False)[0]) / (2 * h)
    assert abs(fd - g0 @ d) <= 1e-5 * abs(g0 @ d) + 1e-9
    gp, gm = assemble(u + h * d)[1], assemble(u - h * d)[1]
    np.testing.assert_allclose(H0 @ d, (gp - gm) / (2 * h), rtol=1e-3, atol=1e-4 * np.abs(H0 @ d).max())


def test_jacobi_eigh3_matches_lapack():
    """Fixed-sweep cyclic Jacobi on symmetric 3x3 matrices (random, repeated and
    tie-broken nearly repeated eigenvalues, diagonal) against LAPACK."""
    from oracle import spectral3d

    rng = np.random.default_rng(11)
    mats = [(lambda M: 0.5 * (M + M.T))(rng.standard_normal((3, 3))) * 10.0 ** rng.uniform(-4, 2) for _ in range(200)]
    Q = np.linalg.qr(rng.standard_normal((3, 3)))[0]
    mats += [Q @ np.diag([1e-3, 1e-3, -2e-3]) @ Q.T, Q @ np.diag([5e-4] * 3) @ Q.T,
             np.diag([3.0, 1.0, 2.0]), Q @ np.diag([1e-3, 1e-3 + 1e-15, 1e-3 + 2e-15]) @ Q.T]
    for A in mats:
        w, V = spectral3d.jacobi_eigh3(A)
        w_ref = np.linalg.eigvalsh(A)
        scale = max(np.abs(w_ref).max(), 1e-300)
        np.testing.assert_allclose(w, w_ref, rtol=0, atol=1e-14 * scale)
        np.testing.assert_allclose(V.T @ V, np.eye(3), atol=1e-13)
        np.testing.assert_allclose(V @ np.diag(w) @ V.T, A, atol=1e-13 * scale)


@pytest.fixture(scope="module")
def mc3d_host(tmp_path_factory):
    """The device header's point function compiled for the host with g++."""
    import ctypes
    import os
    import subprocess

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    d = tmp_path_factory.mktemp("mc3d")
    src = d / "shim.cpp"
    src.write_text('#include "fne_mc3d_point.cuh"\n'
                   'extern "C" double mc3d_element_p2_host(const double* u, const double* gx, const double* gy,\n'
                   '    const double* gz, const double* w, const double* prm, int nq, double tiny, double* g,\n'
                   '    double* K) { return fne::mc3d::element<10>(u, gx, gy, gz, w, prm, nq, tiny, g, K); }\n'
                   'extern "C" int mc3d_point_host(const double* e, double c, double sp, double mu, double K,\n'
                   '                               double lame, double tiny, double* psi, double* sig, double* D) {\n'
                   '  double Dm[6][6];\n'
                   '  const int br = fne::mc3d::point(e, c, sp, mu, K, lame, tiny, *psi, sig, Dm);\n'
                   '  for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) D[i * 6 + j] = Dm[i][j];\n'
                   '  return br;\n}\n')
    lib = d / "libmc3d.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I",
                    os.path.join(root, "fenics_nonlinear_energies_b200", "csrc"), str(src), "-o", str(lib)],
                   check=True)
    so = ctypes.CDLL(str(lib))
    dp = ctypes.POINTER(ctypes.c_double)
    so.mc3d_point_host.restype = ctypes.c_int
    so.mc3d_point_host.argtypes = [dp] + [ctypes.c_double] * 6 + [dp, dp, dp]

    so.mc3d_element_p2_host.restype = ctypes.c_double
    so.mc3d_element_p2_host.argtypes = [dp] * 6 + [ctypes.c_int, ctypes.c_double, dp, dp]

    def element(u, gx, gy, gz, w, prm, tiny=E3.TINY):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (u, gx, gy, gz, w, prm)]
        g = np.zeros(30)
        K = np.zeros(900)
        e = so.mc3d_element_p2_host(*[a.ctypes.data_as(dp) for a in arrs], int(arrs[4].size), tiny,
                                    g.ctypes.data_as(dp), K.ctypes.data_as(dp))
        return e, g, K.reshape(30, 30)

    def call(e, c, sp, mu, K, lame, tiny=E3.TINY):
        e = np.ascontiguousarray(e, dtype=np.float64)
        psi = np.zeros(1)
        sig = np.zeros(6)
        D = np.zeros(36)
        br = so.mc3d_point_host(e.ctypes.data_as(dp), c, sp, mu, K, lame, tiny, psi.ctypes.data_as(dp),
                                sig.ctypes.data_as(dp), D.ctypes.data_as(dp))
        return br, psi[0], sig, D.reshape(6, 6)

    call.element = element
    return call


@pytest.mark.parametrize("branch", [0, 1, 2, 3, 4])
def test_device_point_function_on_host(mc3d_host, branch):
    """fne_mc3d_point.cuh (k_mc3d_elem's per-point code: Jacobi eigen
    solve, branch potentials as quadratic forms, spectral chain rule), compiled
    for the host, against the oracle: branch, psi, sigma and D."""
    eps, c, sp, br = _sample_branches()
    idx = np.flatnonzero(br == branch)[:5]
    scale = LAME + 2.0 * SHEAR
    for i in idx:
        b, psi, sig, D = mc3d_host(eps[i], c[i], sp[i], SHEAR, BULK, LAME)
        assert b == branch
        psi_ref, _ = E3.mc_density(eps[i][None], c[i], sp[i], SHEAR, BULK, LAME)
        assert abs(psi - psi_ref[0]) <= 1e-12 * max(1.0, abs(psi_ref[0]))
        sig_a, D_a, _, _ = E3.mc_stress_tangent(eps[i][None], c[i], sp[i], SHEAR, BULK, LAME)
        np.testing.assert_allclose(sig, sig_a[0], rtol=1e-9, atol=1e-11 * scale * np.abs(eps[i]).max())
        np.testing.assert_allclose(D, D_a[0], rtol=1e-7, atol=1e-9 * scale)


def test_reference_tet_rules():
    """The reference's P1 / P2 tet rules: volume 1/6, exactness (Keast's
    11-point rule: degree 4, to the truncation of its digits), symmetric orbits."""
    from math import factorial

    from fenics_nonlinear_energies_b200 import meshes

    for deg, exact_to in ((1, 1), (2, 4)):
        xi, w = meshes.tet_quadrature_reference(deg)
        assert abs(w.sum() - 1.0 / 6.0) < 1e-14
        for a in range(exact_to + 1):
            for b in range(exact_to + 1 - a):
                for c in range(exact_to + 1 - a - b):
                    exact = factorial(a) * factorial(b) * factorial(c) / factorial(a + b + c + 3)
                    assert abs(np.sum(w * xi[0] ** a * xi[1] ** b * xi[2] ** c) - exact) < 2e-14
    xi, w = meshes.tet_quadrature_reference(2)
    bary = np.vstack([1.0 - xi.sum(0), xi])
    for k in range(1, 11):  # every point's barycentric coordinates are one of the two orbits
        s = np.sort(bary[:, k])
        assert np.allclose(s, [meshes.KEAST11_A] * 3 + [meshes.KEAST11_B], atol=1e-14) or \
            np.allclose(s, [meshes.KEAST11_D] * 2 + [meshes.KEAST11_C] * 2, atol=1e-14)


def test_device_element_function_on_host(mc3d_host):
    """fne::mc3d::element<10> (P2 tet: energy, B^T sigma, B^T D B over the
    reference's 11-point rule), host-compiled, against the oracle element."""
    from fenics_nonlinear_energies_b200 import meshes

    p = meshes.slope3d_problem(nx=2, ny=1, nz=1, degree=2, lam=1.5)
    prm = np.stack([p[k] for k in ("c_bar", "sin_phi", "shear", "bulk", "lame")], axis=-1)  # (E, nq, 5)
    rng = np.random.default_rng(21)
    for el in (0, 5, 11):
        u = 3e-3 * rng.standard_normal(30)
        args = (p["dphix"][el], p["dphiy"][el], p["dphiz"][el], p["quad_weight"][el])
        e_ref, g_ref, H_ref, br = E3.element_derivatives(u, *args, *[prm[el, :, k] for k in range(5)])
        e, g, H = mc3d_host.element(u, *args, prm[el])
        assert abs(e - e_ref) <= 1e-12 * max(1.0, abs(e_ref))
        np.testing.assert_allclose(g, g_ref, rtol=1e-9, atol=1e-10 * np.abs(g_ref).max())
        np.testing.assert_allclose(H, H_ref, rtol=1e-7, atol=1e-9 * np.abs(H_ref).max())


def test_device_point_zero_friction(mc3d_host):
    """sin_phi = 0 (Tresca limit): the apex denominator 4 K sin^2(phi) is 0
    and every return term is written as the reference writes it,
    -d/2 (n / guarded d)^2, so a zero denominator weights its term by 0.
    At sin_phi = 0 the branch tests never select the apex (the edge returns
    always hold); every branch that is reached matches the oracle."""
    rng = np.random.default_rng(11)
    n = 3000
    eps = rng.standard_normal((n, 6)) * 10 ** rng.uniform(-5, -2, size=(n, 1))
    eps[:, :3] += rng.uniform(-5, 5, size=(n, 1)) * 10 ** rng.uniform(-5, -2, size=(n, 1))
    c = 10 ** rng.uniform(-3, 1.5, size=n)
    psi_ref, br = E3.mc_density(eps, c, np.zeros(n), SHEAR, BULK, LAME)
    assert set(np.unique(br)) == {0, 1, 2, 3}
    scale = LAME + 2.0 * SHEAR
    for branch in (0, 1, 2, 3):
        for i in np.flatnonzero(br == branch)[:4]:
            b, psi, sig, D = mc3d_host(eps[i], c[i], 0.0, SHEAR, BULK, LAME)
            assert b == branch
            assert abs(psi - psi_ref[i]) <= 1e-12 * max(1.0, abs(psi_ref[i]))
            sig_a, D_a, _, _ = E3.mc_stress_tangent(eps[i][None], c[i], 0.0, SHEAR, BULK, LAME)
            np.testing.assert_allclose(sig, sig_a[0], rtol=1e-9, atol=1e-11 * scale * np.abs(eps[i]).max())
            np.testing.assert_allclose(D, D_a[0], rtol=1e-7, atol=1e-9 * scale)


@pytest.mark.parametrize("branch", [2, 3])
def test_device_point_near_degenerate_edges(mc3d_host, branch):
    """Edge returns with the two eigenvalues of the edge equal up to the
    reference's 1e-15 tie-break: the pair-summed eigenvalue curvature keeps
    D finite and symmetric, and D matches central differences of the
    oracle's stress."""
    rng = np.random.default_rng(12 + branch)
    found = 0
    for _ in range(20000):
        a, b = sorted(rng.uniform(-2e-3, 4e-3, size=2))[::-1]
        eps = np.array([a, a, b, 0.0, 0.0, 0.0]) if branch == 2 else np.array([a, b, b, 0.0, 0.0, 0.0])
        c = rng.uniform(0.1, 20.0)
        sp = rng.uniform(0.2, 0.7)
        _, br = E3.mc_density(eps[None], c, sp, SHEAR, BULK, LAME)
        if br[0] != branch:
            continue
        bb, psi, sig, D = mc3d_host(eps, c, sp, SHEAR, BULK, LAME)
        assert bb == branch
        assert np.isfinite(D).all()
        np.testing.assert_allclose(D, D.T, rtol=0, atol=1e-9 * np.abs(D).max())
        h = 1e-8 * max(1e-3, np.abs(eps).max())
        Dfd = np.zeros((6, 6))
        for m in range(6):
            ep, em = eps.copy(), eps.copy()
            ep[m] += h
            em[m] -= h
            sp_, _, _, _ = E3.mc_stress_tangent(ep[None], c, sp, SHEAR, BULK, LAME)
            sm_, _, _, _ = E3.mc_stress_tangent(em[None], c, sp, SHEAR, BULK, LAME)
            Dfd[:, m] = (sp_[0] - sm_[0]) / (2 * h)
        np.testing.assert_allclose(D, Dfd, rtol=1e-4, atol=1e-5 * np.abs(Dfd).max())
        found += 1
        if found == 3:
            break
    assert found == 3


def test_p4_tet_rule_and_mesh():
    """The P4 rule (the reference's 24-point Keast rule): weights sum to the
    volume 1/6, exact on every monomial of degree <= 6; the P4 slope mesh
    shares edge and face nodes between its tets (one hex: the 5^3 lattice)."""
    import math

    from fenics_nonlinear_energies_b200 import meshes

    xi, w = meshes.tet_quadrature_reference(4)
    assert xi.shape == (3, 24) and w.shape == (24,)
    assert (xi > 0).all() and (xi.sum(0) < 1).all()
    assert abs(w.sum() - 1.0 / 6.0) <= 1e-15
    for i in range(7):
        for j in range(7 - i):
            for k in range(7 - i - j):
                exact = math.factorial(i) * math.factorial(j) * math.factorial(k) / math.factorial(i + j + k + 3)
                assert abs((w * xi[0] ** i * xi[1] ** j * xi[2] ** k).sum() - exact) <= 1e-14 * exact
    p = meshes.slope3d_problem(nx=1, ny=1, nz=1, degree=4)
    assert p["elems_scalar"].shape == (6, 35) and p["nodes"].shape == (125, 3)
    assert p["dphix"].shape == (6, 24, 35)
    # the nodes of every element sit at its P4 lattice points
    pts = meshes.tet_lagrange_points(4)                    # (3, 35)
    for e in range(6):
        X = p["nodes"][p["elems_scalar"][e]]               # (35, 3)
        V = X[:4]
        np.testing.assert_allclose(X, V[0] + pts.T @ (V[1:] - V[0]), atol=1e-12)
    np.testing.assert_allclose(p["quad_weight"].sum(), 40.0 * 10.0 * 15.0, rtol=1e-13)


def test_device_point_function_matches_reference_elements(mc3d_host):
    """The kernels' point function (fne_mc3d_point.cuh, compiled for the host)
    contracted over P2 elements against the reference's own 3-D element
    functions (tests/golden/reference_mc3d.npz: element_energy_3d,
    element_residual_3d, constitutive_element_hessian_3d of
    slope_stability_3d/jax/jax_energy_3d.py on the same inputs): 1e-12
    relative to the energy, and to the largest gradient / Hessian entry over
    the elements (an apex element's tangent is pure rounding of cancelling
    terms, ~1e-11 against entries of ~1e4)."""
    from pathlib import Path

    d = np.load(Path(__file__).resolve().parent / "golden" / "reference_mc3d.npz")
    ue = d["p2_u_elem"]
    gs, hs = np.abs(d["p2_grad"]).max(), np.abs(d["p2_hess"]).max()
    for e in range(ue.shape[0]):
        prm = np.stack([d[f"p2_{k}"][e] for k in ("c_bar", "sin_phi", "shear", "bulk", "lame")], axis=1)
        en, g, K = mc3d_host.element(ue[e], d["p2_dphix"][e], d["p2_dphiy"][e], d["p2_dphiz"][e],
                                     d["p2_quad_weight"][e], prm)
        er, gr, hr = float(d["p2_energy"][e]), d["p2_grad"][e], d["p2_hess"][e]
        assert abs(en - er) <= 1e-12 * abs(er), (e, en, er)
        assert np.abs(g - gr).max() <= 1e-12 * gs, e
        assert np.abs(K - hr).max() <= 1e-12 * hs, e
