"""Synthetic meshes and problem dictionaries for the four energy families.

The dictionaries carry the same keys the reference's mesh loaders put into
``params`` (``src/problems/plaplace/support/mesh.py``,
``src/problems/ginzburg_landau/jax/mesh.py``,
``src/problems/hyperelasticity/support/mesh.py:19-84``), so the assemblers
take them unchanged:

* P1 triangles on a structured square grid, every cell split into
  ``(ll, lr, ul)`` and ``(ur, ul, lr)`` (the split of
  ``src/problems/plaplace_u3/support/mesh.py:150-157``: all lower triangles
  first, then all upper triangles).
* P1 tetrahedra on a structured box, every hexahedron split into the six
  Kuhn tetrahedra around its main diagonal.

Node numbering.  ``numbering="x_slow"`` (default) numbers nodes with x the
slowest coordinate, which is the order the reference's ``block_xyz``
permutation sorts into (``np.lexsort`` on (z, y, x) keys), so that
permutation becomes the identity.  ``numbering="x_fast"`` gives the
row-major numbering of the reference's structured helper; both are valid
inputs and give the same energies.
"""

from __future__ import annotations

import math

import numpy as np

# Ginzburg-Landau 3-point rule on the reference triangle, as stored in the
# reference's GL_level*.h5 files: ip[a, q] = value of the P1 basis a at point q.
GL_IP = np.array(
    [[1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0],
     [2.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0],
     [1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0]], dtype=np.float64)
GL_W = np.array([1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0], dtype=np.float64)


def _grid_ids(nx, ny, numbering):
    """ids[i, j] = node id of grid point (x index i, y index j)."""
    if numbering == "x_slow":
        return np.arange((nx + 1) * (ny + 1), dtype=np.int64).reshape(nx + 1, ny + 1)
    if numbering == "x_fast":
        return np.arange((nx + 1) * (ny + 1), dtype=np.int64).reshape(ny + 1, nx + 1).T.copy()
    raise ValueError(f"unknown numbering {numbering!r}")


def square_p1(n, lo=0.0, hi=1.0, numbering="x_slow"):
    """Structured ``n x n`` grid of P1 triangles on ``[lo, hi]^2``.

    Returns ``nodes (N, 2)``, ``elems (2 n^2, 3)`` and the boundary mask.
    """
    c = np.linspace(lo, hi, n + 1, dtype=np.float64)
    ids = _grid_ids(n, n, numbering)
    nodes = np.zeros(((n + 1) * (n + 1), 2), dtype=np.float64)
    ii, jj = np.meshgrid(np.arange(n + 1), np.arange(n + 1), indexing="ij")
    nodes[ids.ravel(), 0] = c[ii.ravel()]
    nodes[ids.ravel(), 1] = c[jj.ravel()]
    # cells in (j, i) row-major order, like the reference helper's np.nonzero
    jc, ic = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    jc, ic = jc.ravel(), ic.ravel()
    ll, lr = ids[ic, jc], ids[ic + 1, jc]
    ul, ur = ids[ic, jc + 1], ids[ic + 1, jc + 1]
    elems = np.vstack((np.column_stack((ll, lr, ul)), np.column_stack((ur, ul, lr)))).astype(np.int64)
    x, y = nodes[:, 0], nodes[:, 1]
    tol = 1e-12 * max(1.0, abs(hi - lo))
    boundary = (np.abs(x - lo) < tol) | (np.abs(x - hi) < tol) | (np.abs(y - lo) < tol) | (np.abs(y - hi) < tol)
    return nodes, elems, boundary


def p1_triangle_operators(nodes, elems):
    """Gradients of the three P1 basis functions and the triangle areas."""
    v = nodes[elems]
    x0, y0 = v[:, 0, 0], v[:, 0, 1]
    x1, y1 = v[:, 1, 0], v[:, 1, 1]
    x2, y2 = v[:, 2, 0], v[:, 2, 1]
    det = (x1 - x0) * (y2 - y0) - (x2 - x0) * (y1 - y0)
    if np.any(det <= 0.0):
        raise ValueError("non-positive triangle orientation")
    dvx = np.stack((y1 - y2, y2 - y0, y0 - y1), axis=1) / det[:, None]
    dvy = np.stack((x2 - x1, x0 - x2, x1 - x0), axis=1) / det[:, None]
    return dvx, dvy, 0.5 * det


def plaplace_problem(n=128, p=3.0, f=-10.0, numbering="x_slow", seed=None):
    """p-Laplace on the unit square; ``f`` is the constant source density.

    The load vector is ``f_i = int f phi_i`` (P1: ``f * area / 3`` per vertex),
    the discrete form of ``- int f u`` in the reference's energy.
    """
    nodes, elems, bnd = square_p1(n, 0.0, 1.0, numbering)
    dvx, dvy, vol = p1_triangle_operators(nodes, elems)
    load = np.zeros(nodes.shape[0])
    np.add.at(load, elems, np.repeat((f * vol / 3.0)[:, None], 3, axis=1))
    freedofs = np.flatnonzero(~bnd).astype(np.int64)
    params = {
        "nodes": nodes, "u_0": np.zeros(nodes.shape[0]), "freedofs": freedofs,
        "elems": elems, "dvx": dvx, "dvy": dvy, "vol": vol, "f": load, "p": float(p),
    }
    if seed is None:
        u_init = np.zeros(freedofs.size)
    else:
        u_init = np.random.default_rng(seed).random(freedofs.size)
    return params, u_init


def gl_problem(n=1024, eps=0.01, seed=0, numbering="x_slow"):
    """Ginzburg-Landau on ``[-1, 1]^2``, initial guess ``U[-0.5, 0.5]`` from ``seed``."""
    nodes, elems, bnd = square_p1(n, -1.0, 1.0, numbering)
    dvx, dvy, vol = p1_triangle_operators(nodes, elems)
    freedofs = np.flatnonzero(~bnd).astype(np.int64)
    params = {
        "nodes": nodes, "u_0": np.zeros(nodes.shape[0]), "freedofs": freedofs,
        "elems": elems, "dvx": dvx, "dvy": dvy, "vol": vol,
        "ip": GL_IP.copy(), "w": GL_W.copy(), "eps": float(eps),
    }
    u_init = np.random.default_rng(seed).uniform(-0.5, 0.5, freedofs.size)
    return params, u_init


# Kuhn split of the unit cube: the six monotone paths (0,0,0) -> (1,1,1).
_KUHN_PATHS = ((0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0))


def box_p1_tets(nx, ny, nz, lo, hi):
    """Structured box of hexes, six Kuhn tets each; nodes numbered x slowest, z fastest."""
    xs = [np.linspace(lo[d], hi[d], m + 1) for d, m in enumerate((nx, ny, nz))]
    I, J, K = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    nodes = np.column_stack((xs[0][I.ravel()], xs[1][J.ravel()], xs[2][K.ravel()]))

    def nid(i, j, k):
        return (i * (ny + 1) + j) * (nz + 1) + k

    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ci, cj, ck = ci.ravel(), cj.ravel(), ck.ravel()
    tets = []
    for path in _KUHN_PATHS:
        cur = [ci.copy(), cj.copy(), ck.copy()]
        verts = [nid(*cur)]
        for ax in path:
            cur[ax] = cur[ax] + 1
            verts.append(nid(*cur))
        tets.append(np.column_stack(verts))
    # interleave so the six tets of one hex are consecutive
    elems = np.stack(tets, axis=1).reshape(-1, 4).astype(np.int64)
    return nodes, elems


def p1_tet_operators(nodes, elems):
    """Gradients of the four P1 basis functions and the tet volumes."""
    v = nodes[elems]                                  # (E, 4, 3)
    J = np.stack((v[:, 1] - v[:, 0], v[:, 2] - v[:, 0], v[:, 3] - v[:, 0]), axis=2)  # columns
    det = np.linalg.det(J)
    invJ = np.linalg.inv(J)                           # rows = grads of lambda_1..3
    g123 = invJ                                       # (E, 3, 3): row a-1 is grad of lambda_a
    g0 = -np.sum(g123, axis=1)
    grads = np.concatenate((g0[:, None, :], g123), axis=1)   # (E, 4, 3)
    return grads[:, :, 0].copy(), grads[:, :, 1].copy(), grads[:, :, 2].copy(), np.abs(det) / 6.0


def expand_connectivity_to_dofs(elems_scalar, bs):
    """``[n0, n1, ...] -> [bs*n0, bs*n0+1, ..., bs*n1, ...]`` (the reference's DOF expansion)."""
    es = np.asarray(elems_scalar, dtype=np.int64)
    return (bs * es[:, :, None] + np.arange(bs, dtype=np.int64)[None, None, :]).reshape(es.shape[0], -1)


def neohookean_constants(E, nu):
    """``C1 = E / (4 (1 + nu))``, ``D1 = E / (6 (1 - 2 nu))``."""
    return E / (4.0 * (1.0 + nu)), E / (6.0 * (1.0 - 2.0 * nu))


def he_beam_problem(nx=160, ny=8, nz=8, E=10.0, nu=0.3, length=0.4, half_width=0.01):
    """Neo-Hookean beam ``[0, L] x [-w, w]^2``; x = 0 clamped, x = L rotated (Dirichlet).

    The unknown is the deformed position, initialised to the reference
    coordinates (``u_0_ref``).
    """
    nodes, es = box_p1_tets(nx, ny, nz, (0.0, -half_width, -half_width), (length, half_width, half_width))
    dphix, dphiy, dphiz, vol = p1_tet_operators(nodes, es)
    n_nodes = nodes.shape[0]
    left = np.abs(nodes[:, 0]) < 1e-14
    right = np.abs(nodes[:, 0] - length) < 1e-14
    free_nodes = np.flatnonzero(~(left | right))
    freedofs = (3 * free_nodes[:, None] + np.arange(3)[None, :]).ravel().astype(np.int64)
    u0 = nodes.reshape(-1).copy()
    C1, D1 = neohookean_constants(E, nu)
    params = {
        "u_0": u0.copy(), "u_0_ref": u0.copy(), "freedofs": freedofs,
        "elems": expand_connectivity_to_dofs(es, 3), "elems_scalar": es,
        "dphix": dphix, "dphiy": dphiy, "dphiz": dphiz, "vol": vol,
        "C1": float(C1), "D1": float(D1), "nodes2coord": nodes,
        "right_nodes": np.flatnonzero(right).astype(np.int64),
        "E": float(E), "nu": float(nu),
    }
    return params, u0[freedofs].copy()


def rotate_right_face_from_reference(u0_reference, nodes2coord, angle, right_nodes):
    """Rigid rotation of the right face about the beam axis (x), from the undeformed
    coordinates: ``y' = cos(a) y + sin(a) z``, ``z' = -sin(a) y + cos(a) z``
    (the map of ``src/problems/hyperelasticity/support/rotate_boundary.py:4-22``)."""
    out = np.asarray(u0_reference, dtype=np.float64).reshape(-1).copy()
    rn = np.asarray(right_nodes, dtype=np.int64)
    y0, z0 = nodes2coord[rn, 1], nodes2coord[rn, 2]
    ca, sa = math.cos(angle), math.sin(angle)
    out[3 * rn + 0] = nodes2coord[rn, 0]
    out[3 * rn + 1] = ca * y0 + sa * z0
    out[3 * rn + 2] = -sa * y0 + ca * z0
    return out


# ---------------------------------------------------------------------------
# Plane-strain slope (Mohr-Coulomb): P1 macro mesh -> same-mesh Pk Lagrange
# ---------------------------------------------------------------------------
SLOPE_LEVEL_TO_H = {1: 4.0, 2: 2.0, 3: 1.0, 4: 0.5, 5: 0.25, 6: 0.125, 7: 0.0625}
SLOPE_GEOMETRY = {"x1": 15.0, "x2": 10.0, "x3": 15.0, "y1": 10.0, "y2": 10.0}

# 7-point degree-5 rule on the reference triangle (area 1/2) with the
# 13-digit constants the reference's P2 slope operators use
# (src/problems/slope_stability/support/mesh.py:151-190).
P2_QUAD_XI = np.array([
    [0.1012865073235, 0.7974269853531, 0.1012865073235, 0.4701420641051, 0.4701420641051, 0.0597158717898,
     1.0 / 3.0],
    [0.1012865073235, 0.1012865073235, 0.7974269853531, 0.0597158717898, 0.4701420641051, 0.4701420641051,
     1.0 / 3.0]])
P2_QUAD_W = np.array([0.1259391805448, 0.1259391805448, 0.1259391805448, 0.1323941527885, 0.1323941527885,
                      0.1323941527885, 0.225]) / 2.0


def slope_counts(h, x1=15.0, x2=10.0, x3=15.0, y1=10.0, y2=10.0):
    """Cell counts of the homogeneous slope grid for mesh size ``h``."""
    nx12 = int(round((x1 + x2) / h))
    nx3 = int(round(x3 / h))
    ny1 = int(round(y1 / h))
    ny2 = int(round(y2 / h))
    return nx12, nx3, ny1, ny2


def slope_p2_mesh(h, x1=15.0, x2=10.0, x3=15.0, y1=10.0, y2=10.0):
    """P2 slope mesh with the node and element numbering of the reference's
    generator (``slope_stability/support/mesh.py:334-521``).

    Nodes live on the half-spacing grid: ``2 nx + 1`` columns for the rows of
    the lower block ``[0, x1+x2+x3] x [0, y1]``, ``2 nx12 + 1`` columns for
    the rows above it, whose right end follows the slope from ``(x1+x2, y1)``
    to ``(x1, y1+y2)``; numbered row by row from the bottom, left to right.
    Each cell (lower block first, then the upper part; rows outer, columns
    inner) gives the triangles ``(ll, lr, ul)`` and ``(ur, ul, lr)``, each
    with its vertices and then the midpoints of the edges opposite vertex
    0, 1 and 2.  Returns ``nodes (N, 2)`` and ``elems (E, 6)``."""
    nx12, nx3, ny1, ny2 = slope_counts(h, x1, x2, x3, y1, y2)
    nx = nx12 + nx3
    gx = np.concatenate((np.linspace(0.0, x1 + x2, 2 * nx12 + 1), np.linspace(x1 + x2, x1 + x2 + x3, 2 * nx3 + 1)[1:]))
    gy = np.concatenate((np.linspace(0.0, y1, 2 * ny1 + 1), np.linspace(y1, y1 + y2, 2 * ny2 + 1)[1:]))
    rows = []
    for j in range(2 * (ny1 + ny2) + 1):
        if j <= 2 * ny1:
            xs = gx
        else:
            xs = np.linspace(0.0, x1 + x2 * (y1 + y2 - gy[j]) / y2, 2 * nx12 + 1)
        rows.append(np.column_stack((xs, np.full(xs.size, gy[j]))))
    start = np.cumsum([0] + [r.shape[0] for r in rows])
    nodes = np.vstack(rows)

    def nid(i, j):
        return start[j] + i

    tris = []
    for (j0, j1, ncols) in ((0, ny1, nx), (ny1, ny1 + ny2, nx12)):
        for j in range(j0, j1):
            for i in range(ncols):
                a, b = 2 * i, 2 * j
                tris.append((nid(a, b), nid(a + 2, b), nid(a, b + 2),
                             nid(a + 1, b + 1), nid(a, b + 1), nid(a + 1, b)))
                tris.append((nid(a + 2, b + 2), nid(a, b + 2), nid(a + 2, b),
                             nid(a + 1, b + 1), nid(a + 2, b + 1), nid(a + 1, b + 2)))
    return nodes, np.asarray(tris, dtype=np.int64)


def slope_macro_mesh(h, x1=15.0, x2=10.0, x3=15.0, y1=10.0, y2=10.0):
    """Vertices and P1 triangles of the 2-D slope: the vertices of the P2 mesh
    (``slope_p2_mesh``) renumbered in their P2 order, and its triangles'
    vertex columns -- the macro mesh the reference's same-mesh Pk builder
    starts from (``slope_stability/support/mesh.py:698-708``).  A full block
    ``[0, x1+x2+x3] x [0, y1]`` under a trapezoid whose right edge runs from
    ``(x1+x2, y1)`` to ``(x1, y1+y2)``; every cell split into ``(ll, lr, ul)``
    and ``(ur, ul, lr)``; lower block first."""
    p2_nodes, p2_elems = slope_p2_mesh(h, x1, x2, x3, y1, y2)
    verts = np.unique(p2_elems[:, :3])
    new_id = np.full(p2_nodes.shape[0], -1, dtype=np.int64)
    new_id[verts] = np.arange(verts.size, dtype=np.int64)
    return p2_nodes[verts].copy(), new_id[p2_elems[:, :3]]


def lagrange_points(degree):
    """Equispaced Lagrange points on the reference triangle, ordered vertices,
    then edges (edge 0 = v1-v2, edge 1 = v0-v2, edge 2 = v0-v1, each from its
    first to its second vertex), then interior points (x fastest)."""
    k = int(degree)
    v = [(0.0, 0.0), (1.0, 0.0), (0.0, 1.0)]
    pts = list(v)
    for (a, b) in ((1, 2), (0, 2), (0, 1)):
        for t in range(1, k):
            s = t / k
            pts.append((v[a][0] + s * (v[b][0] - v[a][0]), v[a][1] + s * (v[b][1] - v[a][1])))
    for j in range(1, k):
        for i in range(1, k - j):
            pts.append((i / k, j / k))
    return np.asarray(pts, dtype=np.float64)


def lagrange_tabulate(degree, xi):
    """Values and reference gradients of the equispaced Lagrange basis at ``xi`` (2, nq)."""
    pts = lagrange_points(degree)
    k = int(degree)
    mons = [(i, j) for j in range(k + 1) for i in range(k + 1 - j)]
    V = np.array([[x ** i * y ** j for (i, j) in mons] for (x, y) in pts])
    coef = np.linalg.inv(V)  # column a = monomial coefficients of basis a
    x, y = xi[0], xi[1]
    M = np.array([x ** i * y ** j for (i, j) in mons])
    Mx = np.array([i * x ** max(i - 1, 0) * y ** j if i > 0 else 0 * x for (i, j) in mons])
    My = np.array([j * x ** i * y ** max(j - 1, 0) if j > 0 else 0 * y for (i, j) in mons])
    return coef.T @ M, coef.T @ Mx, coef.T @ My


def gauss_jacobi_triangle(n):
    """Collapsed (Duffy) Gauss-Jacobi rule with ``n*n`` points, exact to degree 2n-1
    on the reference triangle (area 1/2)."""
    from scipy.special import roots_jacobi

    a, wa = roots_jacobi(n, 1.0, 0.0)   # weight (1 - t) on [-1, 1]
    b, wb = roots_jacobi(n, 0.0, 0.0)
    s = (a + 1.0) / 2.0                  # collapsed coordinate
    t = (b + 1.0) / 2.0
    X, Y, W = [], [], []
    for i in range(n):
        for j in range(n):
            X.append(t[j] * (1.0 - s[i]))
            Y.append(s[i])
            W.append(wa[i] * wb[j] / 8.0)
    return np.array([X, Y]), np.array(W)


# Fully symmetric 19-point rule exact to degree 9 on the triangle: the centroid,
# four (a, a, 1-2a) orbits and one (a, b, 1-a-b) orbit, weights normalised to
# sum 1.  Values of Dunavant, "High degree efficient symmetrical Gaussian
# quadrature rules for the triangle", IJNME 21 (1985) 1129-1148, degree 9,
# refined to double precision by Newton's method on the moment equations of
# every monomial of degree <= 9 (the refinement moves the published 15-digit
# values by < 4e-16).  Its orbit structure (1 + 4x3 + 6 = 19 points, 12
# unknowns for 12 invariant moments) is that of the 19-point degree-9 rule of
# Xiao & Gimbutas (2010), which basix's make_quadrature(triangle, 9) -- the
# reference's P4 rule -- returns.
DEG9_CENTROID_W = 0.09713579628279883
DEG9_ORBITS_A = (  # (a, w): points (1-2a, a, a) and permutations
    (0.4896825191987376, 0.03133470022713907),
    (0.4370895914929366, 0.07782754100477428),
    (0.1882035356190327, 0.07964773892721025),
    (0.04472951339445271, 0.02557767565869803),
)
DEG9_ORBIT_AB = (0.2219629891607657, 0.03683841205473628, 0.04328353937728938)  # (a, b, w)


def triangle_rule_degree9():
    """(xi (2, 19), w (19,)) of the 19-point degree-9 rule on the reference
    triangle (area 1/2): centroid, then each (a, a, 1-2a) orbit, then the
    six points of the (a, b, 1-a-b) orbit."""
    bary, w = [(1.0 / 3.0, 1.0 / 3.0, 1.0 / 3.0)], [DEG9_CENTROID_W]
    for a, wa in DEG9_ORBITS_A:
        b = 1.0 - 2.0 * a
        bary += [(b, a, a), (a, b, a), (a, a, b)]
        w += [wa] * 3
    a, b, wab = DEG9_ORBIT_AB
    c = 1.0 - a - b
    bary += [(a, b, c), (b, a, c), (a, c, b), (c, a, b), (b, c, a), (c, b, a)]
    w += [wab] * 6
    bary = np.asarray(bary, dtype=np.float64)
    return np.stack([bary[:, 1], bary[:, 2]]), 0.5 * np.asarray(w, dtype=np.float64)


def slope_quadrature(degree):
    """The reference's triangle rule for element degree ``degree``: the
    13-digit 7-point rule for P2, the centroid for P1, the degree-9 rule for
    P4 (``make_quadrature(triangle, 2p+1)``,
    ``src/problems/slope_stability/support/mesh.py:293-296``); a collapsed
    Gauss-Jacobi rule of the same exactness for other degrees."""
    if degree == 2:
        return P2_QUAD_XI.copy(), P2_QUAD_W.copy()
    if degree == 1:
        return np.array([[1.0 / 3.0], [1.0 / 3.0]]), np.array([0.5])
    if degree == 4:
        return triangle_rule_degree9()
    return gauss_jacobi_triangle(degree + 1)  # degree 2*deg+1 exactness


def same_mesh_lagrange(macro_nodes, macro_elems, degree, decimals=12):
    """Pk nodes on every macro triangle, shared nodes merged by rounded coordinates
    in element order (the numbering rule of the reference's same-mesh builder:
    a node gets the next id when its rounded coordinates first appear, walking
    the elements and their local points in order)."""
    ref = lagrange_points(degree)
    v = macro_nodes[macro_elems]                                  # (E, 3, 2)
    lam = np.stack((1.0 - ref[:, 0] - ref[:, 1], ref[:, 0], ref[:, 1]), axis=1)  # (n_p, 3)
    pts = (lam[None, :, 0, None] * v[:, None, 0] + lam[None, :, 1, None] * v[:, None, 1]
           + lam[None, :, 2, None] * v[:, None, 2])               # (E, n_p, 2)
    flat = pts.reshape(-1, 2)
    keys = np.round(flat, decimals)
    keys[keys == 0.0] = 0.0                                       # -0.0 and 0.0 are one key
    _, first, inverse = np.unique(keys, axis=0, return_index=True, return_inverse=True)
    order = np.argsort(first, kind="stable")                      # ids by first appearance
    new_id = np.empty(order.size, dtype=np.int64)
    new_id[order] = np.arange(order.size, dtype=np.int64)
    elems = new_id[inverse.reshape(-1)].reshape(macro_elems.shape[0], ref.shape[0])
    return flat[first[order]].copy(), elems


def affine_triangle_geometry(nodes, elems_scalar):
    """Inverse Jacobian (row-major ``[dxi/dx, dxi/dy, deta/dx, deta/dy]``) and
    ``|det J|`` of the affine map of every triangle (vertices = first 3 nodes)."""
    v = nodes[elems_scalar[:, :3]]
    j11 = v[:, 1, 0] - v[:, 0, 0]
    j12 = v[:, 1, 1] - v[:, 0, 1]
    j21 = v[:, 2, 0] - v[:, 0, 0]
    j22 = v[:, 2, 1] - v[:, 0, 1]
    det = j11 * j22 - j12 * j21
    # grads = inv @ [dhat1; dhat2] with inv = [[j22, -j12], [-j21, j11]] / det
    inv = np.stack((j22 / det, -j12 / det, -j21 / det, j11 / det), axis=1)
    return inv, np.abs(det)


def isoparametric_triangle_geometry(nodes, elems_scalar, dhat1, dhat2):
    """Inverse Jacobian and ``|det J|`` at every quadrature point of the
    isoparametric map through all element nodes, ``(E, nq, 4)`` and
    ``(E, nq)``: ``J_q = [[x.dh1_q, y.dh1_q], [x.dh2_q, y.dh2_q]]`` with
    ``dhat1 / dhat2 (nq, n_p)`` the reference basis gradients -- the map of
    the reference's P2 slope operators (``slope_stability/support/mesh.py:530-567``),
    whose slope-side elements have their hypotenuse midpoint off the
    straight edge."""
    x = nodes[elems_scalar, 0]                      # (E, n_p)
    y = nodes[elems_scalar, 1]
    j11, j12 = x @ dhat1.T, y @ dhat1.T             # (E, nq)
    j21, j22 = x @ dhat2.T, y @ dhat2.T
    det = j11 * j22 - j12 * j21
    inv = np.stack((j22 / det, -j12 / det, -j21 / det, j11 / det), axis=-1)
    return inv, np.abs(det)


def geometry_from_elem_B(elem_B, quad_weight, dhat1, dhat2, quad_w):
    """Per-point ``J^-1 (E, nq, 4)`` and ``|det J| (E, nq)`` recovered from the
    reference's stored operators: ``elem_B[e, q]`` holds the physical basis
    gradients ``g = J_q^-1 [dh1; dh2]`` (rows xx: g_x at even columns, yy: g_y
    at odd columns) and ``quad_weight = |det J_q| w_q``.  ``J_q^-1`` is the
    least-squares solution over the element's nodes (exact for data that
    came from a Jacobian)."""
    gx = elem_B[:, :, 0, 0::2]                      # (E, nq, n_p)
    gy = elem_B[:, :, 1, 1::2]
    R = np.stack((dhat1, dhat2), axis=1)            # (nq, 2, n_p)
    # g = X R  with X (2x2) per (e, q):  X = g R^T (R R^T)^-1
    RRt_inv = np.linalg.inv(np.einsum("qkn,qln->qkl", R, R))
    Rp = np.einsum("qkn,qkl->qnl", R, RRt_inv)      # (nq, n_p, 2)
    ix = np.einsum("eqn,qnl->eql", gx, Rp)          # row 0 of J^-1
    iy = np.einsum("eqn,qnl->eql", gy, Rp)          # row 1
    inv = np.concatenate((ix, iy), axis=-1)
    return inv, quad_weight / quad_w[None, :]


def davis_b_reduction(c0, phi_deg, psi_deg, lam):
    """Davis-B strength reduction: reduced cohesion and friction angle (degrees)."""
    if lam <= 0.0:
        raise ValueError("lambda must be positive")
    phi, psi = math.radians(phi_deg), math.radians(psi_deg)
    c01 = c0 / lam
    phi1 = math.atan(math.tan(phi) / lam)
    psi1 = math.atan(math.tan(psi) / lam)
    beta = math.cos(phi1) * math.cos(psi1) / (1.0 - math.sin(phi1) * math.sin(psi1))
    return beta * c01, math.degrees(math.atan(beta * math.tan(phi1)))


def slope_problem(*, level=None, h=None, degree=4, E=2.0e4, nu=0.49, c0=6.0, phi_deg=45.0, psi_deg=0.0,
                  gamma=20.0, lam=1.0, with_elem_B=False):
    """Homogeneous slope, plane strain, Pk same-mesh elements, Davis-B reduced strength."""
    if h is None:
        h = SLOPE_LEVEL_TO_H[int(level)]
    if int(degree) == 2:  # the reference builds P2 with its own grid generator
        nodes, es = slope_p2_mesh(h)
    else:
        macro_nodes, macro_elems = slope_macro_mesh(h)
        nodes, es = same_mesh_lagrange(macro_nodes, macro_elems, degree)
    xi, wq = slope_quadrature(degree)
    hatp, dh1, dh2 = lagrange_tabulate(degree, xi)      # (n_p, nq)
    if int(degree) == 2:  # per-point map through all six nodes, as the reference's P2 operators
        inv, det = isoparametric_triangle_geometry(nodes, es, dh1.T, dh2.T)
    else:                 # vertex (affine) map, as the reference's Pk same-mesh operators
        inv, det = affine_triangle_geometry(nodes, es)
    n_nodes = nodes.shape[0]
    xmax = float(np.max(nodes[:, 0])) - 1.0e-9
    q_mask = np.zeros((n_nodes, 2), dtype=bool)
    q_mask[:, 0] = (nodes[:, 0] > 0.0) & (nodes[:, 1] > 0.0) & (nodes[:, 0] < xmax)
    q_mask[:, 1] = nodes[:, 1] > 0.0
    freedofs = np.arange(2 * n_nodes, dtype=np.int64).reshape(n_nodes, 2)[q_mask]
    qw = (det if det.ndim == 2 else det[:, None]) * wq[None, :]   # (E, nq)
    # gravity load f_a = sum_q w_q phi_a(q) (0, -gamma)
    force = np.zeros(2 * n_nodes)
    np.add.at(force, 2 * es + 1, -gamma * (qw @ hatp.T))
    coh, phi = davis_b_reduction(c0, phi_deg, psi_deg, lam)
    params = {
        "nodes": nodes, "elems_scalar": es, "elems": expand_connectivity_to_dofs(es, 2),
        "freedofs": freedofs, "q_mask": q_mask, "u_0": np.zeros(2 * n_nodes), "force": force,
        "inv_jac": inv, "det_j": det, "quad_xi": xi, "quad_w": wq,
        "dhat1": dh1.T.copy(), "dhat2": dh2.T.copy(), "hatp": hatp.T.copy(),   # (nq, n_p)
        "quad_weight": qw, "eps_p_old": np.zeros((es.shape[0], wq.size, 3)),
        "E": float(E), "nu": float(nu), "phi_deg": float(phi), "cohesion": float(coh),
        "c0": float(c0), "phi0_deg": float(phi_deg), "psi_deg": float(psi_deg), "gamma": float(gamma),
        "lambda": float(lam), "reg": 1.0e-12, "degree": int(degree), "h": float(h),
    }
    if with_elem_B:
        params["elem_B"] = slope_elem_B(params)
    return params


def slope_elem_B(params):
    """Reference-layout strain operators ``elem_B (E, nq, 3, 2 n_p)``:
    rows (eps_xx, eps_yy, gamma_xy), interleaved (u_x, u_y) per node."""
    inv = params["inv_jac"]
    d1, d2 = params["dhat1"], params["dhat2"]            # (nq, n_p)
    if inv.ndim == 2:  # affine: one J^-1 per element
        inv = np.broadcast_to(inv[:, None, :], (inv.shape[0], d1.shape[0], 4))
    gx = inv[:, :, 0, None] * d1[None] + inv[:, :, 1, None] * d2[None]
    gy = inv[:, :, 2, None] * d1[None] + inv[:, :, 3, None] * d2[None]
    E, nq, n_p = gx.shape
    B = np.zeros((E, nq, 3, 2 * n_p))
    B[:, :, 0, 0::2] = gx
    B[:, :, 1, 1::2] = gy
    B[:, :, 2, 0::2] = gy
    B[:, :, 2, 1::2] = gx
    return B


# ---------------------------------------------------------------------------
# Tetrahedral Lagrange elements (3-D slope family)
# ---------------------------------------------------------------------------
# Node order of src/problems/slope_stability_3d/support/simplex_lagrange.py:
# vertices, then the interior points of the edges (0,1), (1,2), (0,2), (1,3),
# (2,3), (0,3) from the first vertex towards the second, then the interior
# points of the faces (0,1,2), (0,1,3), (0,2,3), (1,2,3), then the cell
# interior.  Each node is a tuple of barycentric counts summing to p.
TET_EDGES = ((0, 1), (1, 2), (0, 2), (1, 3), (2, 3), (0, 3))
TET_FACES = ((0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3))


def _tri_interior_counts(p):
    return [(a, b, p - a - b) for a in range(p - 2, 0, -1) for b in range(p - a - 1, 0, -1) if p - a - b > 0]


def tet_lagrange_counts(p):
    """Barycentric count tuples (c0, c1, c2, c3) of the degree-p nodes, in node order."""
    p = int(p)
    if p < 1:
        raise ValueError("degree must be >= 1")
    out = [tuple(p if i == v else 0 for i in range(4)) for v in range(4)]
    for i, j in TET_EDGES:
        for k in range(1, p):
            c = [0, 0, 0, 0]
            c[i], c[j] = p - k, k
            out.append(tuple(c))
    for face in TET_FACES:
        for tri in _tri_interior_counts(p):
            c = [0, 0, 0, 0]
            for local, vertex in enumerate(face):
                c[vertex] = tri[local]
            out.append(tuple(c))
    out += [(a, b, c, p - a - b - c) for a in range(p - 3, 0, -1) for b in range(p - a - 2, 0, -1)
            for c in range(p - a - b - 1, 0, -1) if p - a - b - c > 0]
    return out


def tet_lagrange_points(p):
    """Reference coordinates (3, n_p) of the nodes: (c1, c2, c3) / p."""
    return np.array([[c[1], c[2], c[3]] for c in tet_lagrange_counts(p)], dtype=np.float64).T / float(p)


def tet_lagrange_tabulate(p, xi):
    """Values (n_p, nq) and reference derivatives d/dxi_k (3 x (n_p, nq)) of the
    degree-p basis at ``xi`` (3, nq).  Basis of node c: prod_i L_{c_i}(lambda_i)
    with L_m(l) = prod_{j<m} (p l - j) / (j + 1) (barycentric Lagrange form);
    d/dxi_k = d/dlambda_k - d/dlambda_0."""
    p = int(p)
    xi = np.asarray(xi, dtype=np.float64)
    lam = np.stack([1.0 - xi[0] - xi[1] - xi[2], xi[0], xi[1], xi[2]])   # (4, nq)

    def factor(m, l):
        val, der = np.ones_like(l), np.zeros_like(l)
        for j in range(m):
            f = (p * l - j) / (j + 1)
            der = der * f + val * (p / (j + 1))
            val = val * f
        return val, der

    counts = tet_lagrange_counts(p)
    phi = np.empty((len(counts), xi.shape[1]))
    dlam = np.empty((4, len(counts), xi.shape[1]))
    for n, c in enumerate(counts):
        vals, ders = zip(*(factor(c[i], lam[i]) for i in range(4)))
        phi[n] = vals[0] * vals[1] * vals[2] * vals[3]
        for i in range(4):
            term = ders[i]
            for j in range(4):
                if j != i:
                    term = term * vals[j]
            dlam[i, n] = term
    return phi, dlam[1] - dlam[0], dlam[2] - dlam[0], dlam[3] - dlam[0]


def gauss_jacobi_tet(n):
    """Collapsed (Stroud conical product) Gauss-Jacobi rule with ``n**3`` points,
    exact to degree 2n-1 on the reference tetrahedron (volume 1/6):
    x = a (1-b)(1-c), y = b (1-c), z = c with Jacobian (1-b)(1-c)^2."""
    from scipy.special import roots_jacobi

    tc, wc = roots_jacobi(n, 2.0, 0.0)
    tb, wb = roots_jacobi(n, 1.0, 0.0)
    ta, wa = roots_jacobi(n, 0.0, 0.0)
    c, b, a = (tc + 1.0) / 2.0, (tb + 1.0) / 2.0, (ta + 1.0) / 2.0
    pts, w = [], []
    for i in range(n):
        for j in range(n):
            for k in range(n):
                pts.append((a[k] * (1.0 - b[j]) * (1.0 - c[i]), b[j] * (1.0 - c[i]), c[i]))
                w.append(wc[i] * wb[j] * wa[k] / 64.0)
    return np.array(pts).T, np.array(w)


def slope3d_problem(nx=8, ny=2, nz=4, *, degree=2, length=40.0, width=10.0, h_left=20.0, h_right=10.0,
                    x1=15.0, x2=25.0, E=2.0e4, nu=0.3, c0=6.0, phi_deg=45.0, psi_deg=0.0, lam=1.0,
                    gamma=20.0, quad_n=None):
    """Synthetic 3-D slope: x in [0, length], y in [0, width], z in [0, H(x)] with
    H = h_left up to x1, linear to h_right at x2, h_right after; a structured
    nx x ny x nz hex grid mapped to that profile, every hex split into six
    tetrahedra (positively oriented), P1, P2 or P4 nodes in the tetrahedral
    Lagrange order of ``tet_lagrange_counts``.  Fixed: all components at
    z = 0, u_x at x = 0 and x = length, u_y at y = 0 and y = width.  Davis-B
    reduced strength at ``lam``; gravity ``gamma`` along -z.  Quadrature:
    the reference's rule for the degree (``tet_quadrature_reference``) unless
    ``quad_n`` asks for a Gauss-Jacobi rule.  Returns the element data the
    3-D density needs per element and quadrature point."""
    if degree not in (1, 2, 4):
        raise ValueError("degree must be 1, 2 or 4")
    xs = np.linspace(0.0, length, nx + 1)
    hx = np.interp(xs, [0.0, x1, x2, length], [h_left, h_left, h_right, h_right])
    nid = np.arange((nx + 1) * (ny + 1) * (nz + 1)).reshape(nx + 1, ny + 1, nz + 1)
    I, J, K = np.meshgrid(np.arange(nx + 1), np.arange(ny + 1), np.arange(nz + 1), indexing="ij")
    verts = np.stack([xs[I], width * J / ny, hx[I] * K / nz], axis=-1).reshape(-1, 3)
    kuhn = ((0, 1, 3, 7), (0, 1, 5, 7), (0, 2, 3, 7), (0, 2, 6, 7), (0, 4, 5, 7), (0, 4, 6, 7))
    tets = []
    for i in range(nx):
        for j in range(ny):
            for k in range(nz):
                c = [nid[i + (m & 1), j + ((m >> 1) & 1), k + ((m >> 2) & 1)] for m in range(8)]
                for t in kuhn:
                    v = [c[m] for m in t]
                    if np.linalg.det(verts[v[1:]] - verts[v[0]]) < 0.0:
                        v[2], v[3] = v[3], v[2]
                    tets.append(v)
    tets = np.array(tets, dtype=np.int64)
    nodes = verts
    if degree == 2:
        edge_id = {}
        mids = []
        conn = np.empty((tets.shape[0], 10), dtype=np.int64)
        conn[:, :4] = tets
        for e, t in enumerate(tets):
            for q, (a, b) in enumerate(TET_EDGES):
                key = (min(t[a], t[b]), max(t[a], t[b]))
                if key not in edge_id:
                    edge_id[key] = verts.shape[0] + len(mids)
                    mids.append(0.5 * (verts[t[a]] + verts[t[b]]))
                conn[e, 4 + q] = edge_id[key]
        nodes = np.concatenate([verts, np.array(mids)])
        tets = conn
    elif degree > 2:
        # a node is identified by its (vertex, count) pairs with nonzero count,
        # so edge and face nodes are shared between the tets that meet there;
        # new nodes are numbered in order of first appearance
        counts = tet_lagrange_counts(degree)
        key_id, extra = {}, []
        conn = np.empty((tets.shape[0], len(counts)), dtype=np.int64)
        for e, t in enumerate(tets):
            for m, cnt in enumerate(counts):
                if max(cnt) == degree:
                    conn[e, m] = t[cnt.index(degree)]
                    continue
                key = tuple(sorted((int(t[i]), c) for i, c in enumerate(cnt) if c))
                if key not in key_id:
                    key_id[key] = verts.shape[0] + len(extra)
                    extra.append(sum(c * verts[t[i]] for i, c in enumerate(cnt)) / degree)
                conn[e, m] = key_id[key]
        nodes = np.concatenate([verts, np.array(extra)])
        tets = conn
    n_nodes = nodes.shape[0]
    fixed = np.zeros((n_nodes, 3), dtype=bool)
    tol = 1e-9
    fixed[np.abs(nodes[:, 2]) < tol, :] = True
    fixed[(np.abs(nodes[:, 0]) < tol) | (np.abs(nodes[:, 0] - length) < tol), 0] = True
    fixed[(np.abs(nodes[:, 1]) < tol) | (np.abs(nodes[:, 1] - width) < tol), 1] = True
    freedofs = np.flatnonzero(~fixed.ravel()).astype(np.int64)
    # the reference's rule for the element degree (bit-compatible inputs), or
    # a collapsed Gauss-Jacobi rule with quad_n points per direction
    xi, wq = tet_quadrature_reference(degree) if quad_n is None else gauss_jacobi_tet(quad_n)
    _, d1, d2, d3 = tet_lagrange_tabulate(degree, xi)           # (n_p, nq)
    X = nodes[tets[:, :4]]                                     # (E, 4, 3)
    Jm = np.stack([X[:, 1] - X[:, 0], X[:, 2] - X[:, 0], X[:, 3] - X[:, 0]], axis=2)  # dx / dxi (E, 3, 3)
    det = np.linalg.det(Jm)
    Jinv = np.linalg.inv(Jm)                                   # dxi / dx
    R = np.stack([d1, d2, d3], axis=0)                         # (3, n_p, nq)
    G = np.einsum("eki,kpq->eiqp", Jinv, R)                     # (E, 3, nq, n_p): d phi_p / d x_i
    c_bar, phi_red = davis_b_reduction(c0, phi_deg, psi_deg, lam)
    lame = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))
    shear = E / (2.0 * (1.0 + nu))
    bulk = lame + 2.0 * shear / 3.0
    ne, nq = tets.shape[0], wq.size
    full = lambda v: np.full((ne, nq), float(v))  # noqa: E731
    phi_vals = tet_lagrange_tabulate(degree, xi)[0]            # (n_p, nq)
    load = np.zeros(3 * n_nodes)
    np.add.at(load, 3 * tets + 2, -gamma * np.einsum("e,q,pq->ep", np.abs(det), wq, phi_vals))
    elems = (3 * tets[:, :, None] + np.arange(3)).reshape(ne, -1)
    return {
        "nodes": nodes, "elems_scalar": tets, "elems": elems, "freedofs": freedofs, "u_0": np.zeros(3 * n_nodes),
        "dphix": G[:, 0], "dphiy": G[:, 1], "dphiz": G[:, 2], "quad_weight": np.abs(det)[:, None] * wq[None, :],
        "c_bar": full(2.0 * c_bar * math.cos(math.radians(phi_red))), "sin_phi": full(math.sin(math.radians(phi_red))),
        "shear": full(shear), "bulk": full(bulk), "lame": full(lame), "force": load,
    }


# The 3-D family's element rules for P1 / P2 tetrahedra, in the digits and
# point order of src/problems/slope_stability_3d/support/mesh.py:935-1010 so
# element inputs are bit-compatible: the centroid rule and Keast's 11-point
# rule (one negative weight), weights already scaled to the volume 1/6.
KEAST11_A, KEAST11_B = 0.0714285714285714, 0.785714285714286
KEAST11_C, KEAST11_D = 0.399403576166799, 0.100596423833201
KEAST11_W = (-0.013155555555555, 0.007622222222222, 0.024888888888888)


# P4 tetrahedra: Keast's 24-point rule (exact to degree 6), the reference's
# digits (src/problems/slope_stability_3d/support/mesh.py:1003-1101): three
# 4-point orbits (a, a, a, 1 - 3a) and one 12-point orbit of (p, p, q, r);
# its weights are listed for the unit simplex and divided by 6 there.
KEAST24_ORBITS4 = ((0.2146028712591517, 0.3561913862225449, 0.0399227502581679),
                   (0.0406739585346113, 0.8779781243961660, 0.0100772110553207),
                   (0.3223378901422757, 0.0329863295731731, 0.0553571815436544))
KEAST24_PQR = (0.0636610018750175, 0.2696723314583159, 0.6030056647916491)
KEAST24_W12 = 0.0482142857142857


def tet_quadrature_reference(degree):
    """(xi (3, nq), w (nq,)) of the reference's tetrahedral rule for element degree 1, 2 or 4."""
    if degree == 1:
        return np.full((3, 1), 0.25), np.array([1.0 / 6.0])
    if degree == 4:
        pts, w = [], []
        for a, b, wt in KEAST24_ORBITS4:                 # point order (b,a,a) (a,a,a) (a,a,b) (a,b,a)
            pts += [(b, a, a), (a, a, a), (a, a, b), (a, b, a)]
            w += [wt] * 4
        p_, q_, r_ = KEAST24_PQR
        pts += [(q_, p_, p_), (p_, q_, p_), (p_, p_, q_), (r_, p_, p_), (p_, r_, p_), (p_, p_, r_),
                (p_, q_, r_), (q_, r_, p_), (r_, p_, q_), (p_, r_, q_), (q_, p_, r_), (r_, q_, p_)]
        w += [KEAST24_W12] * 12
        return np.array(pts, dtype=np.float64).T, np.array(w, dtype=np.float64) / 6.0
    if degree != 2:
        raise ValueError("the reference's tetrahedral rules here: degree 1, 2 or 4")
    a, b, c, d = KEAST11_A, KEAST11_B, KEAST11_C, KEAST11_D
    pts = [(0.25, 0.25, 0.25)]
    pts += [(a, a, a), (b, a, a), (a, b, a), (a, a, b)]                  # orbit (a, a, a, b)
    pts += [(c, d, d), (d, c, d), (d, d, c), (c, c, d), (c, d, c), (d, c, c)]  # orbit (c, c, d, d)
    w = [KEAST11_W[0]] + [KEAST11_W[1]] * 4 + [KEAST11_W[2]] * 6
    return np.array(pts, dtype=np.float64).T, np.array(w, dtype=np.float64)
