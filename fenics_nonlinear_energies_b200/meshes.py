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
