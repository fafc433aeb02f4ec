"""Device layout build (``fne_layout_build_device``) against the host build.

Every array (perm, iperm, total_to_free_reord, COO and owned COO rows /
columns, element owners) and the owned range must be identical to
``fne_layout_build``, which the CPU suite pins to the oracle and the
reference's goldens: all four families, both reorder modes, 1-3 ranks, a
given adjacency (in a non-canonical storage order), a permutation override,
coordinate ties across signed zeros and negative values, empty meshes, the
error paths, and the full-size P4 slope.
"""

import numpy as np
import pytest
from scipy import sparse

from oracle import layout as L
from fenics_nonlinear_energies_b200 import _lib, meshes

pytestmark = pytest.mark.gpu

KEYS = ("perm", "iperm", "total_to_free_reord", "coo_rows", "coo_cols", "owned_rows", "owned_cols", "elem_owner")


def _both(**kw):
    import torch

    torch.cuda.init()
    host = _lib.build_layout(**kw)
    dev = _lib.build_layout(device=True, **kw)
    for k in KEYS:
        np.testing.assert_array_equal(dev[k], host[k], err_msg=k)
    assert (dev["lo"], dev["hi"], dev["n_free"]) == (host["lo"], host["hi"], host["n_free"])
    return host


def _args(params, bs, coord_key, dir_key):
    return dict(freedofs=np.asarray(params["freedofs"]), elems=np.asarray(params["elems"]),
                n_total=len(params[dir_key]), block_size=bs, coords=params[coord_key])


@pytest.mark.parametrize("size", [1, 2, 3])
@pytest.mark.parametrize("reorder", ["none", "block_xyz"])
@pytest.mark.parametrize("family", ["plaplace", "gl", "he", "mc_p2", "mc_p4"])
def test_device_layout_matches_host(family, reorder, size):
    if family == "plaplace":
        params, _ = meshes.plaplace_problem(n=23, numbering="x_fast")
        a = _args(params, 1, "nodes", "u_0")
    elif family == "gl":
        params, _ = meshes.gl_problem(n=31)
        a = _args(params, 1, "nodes", "u_0")
    elif family == "he":
        params, _ = meshes.he_beam_problem(nx=9, ny=3, nz=2)
        a = _args(params, 3, "nodes2coord", "u_0_ref")
    else:
        params = meshes.slope_problem(level=1, degree=int(family[-1]), lam=1.0)
        a = _args(params, 2, "nodes", "u_0")
    for rank in range(size):
        _both(reorder=reorder, rank=rank, size=size, **a)


def test_device_layout_given_adjacency_and_override():
    params, _ = meshes.gl_problem(n=17, numbering="x_fast")
    free = params["freedofs"]
    adj = L.element_adjacency(params["elems"], free, len(params["u_0"])).tocsr()
    # non-canonical storage order: reverse the columns inside every row
    ind = adj.indices.copy()
    for r in range(adj.shape[0]):
        ind[adj.indptr[r]:adj.indptr[r + 1]] = ind[adj.indptr[r]:adj.indptr[r + 1]][::-1]
    adj_rev = sparse.csr_matrix((adj.data, ind, adj.indptr), shape=adj.shape)
    perm = np.random.default_rng(0).permutation(free.size)
    a = _args(params, 1, "nodes", "u_0")
    for kw in ({"adjacency": adj}, {"adjacency": adj_rev}, {"perm_override": perm},
               {"adjacency": adj_rev, "perm_override": perm}):
        for rank, size in ((0, 1), (1, 2)):
            _both(reorder="block_xyz", rank=rank, size=size, **kw, **a)


def test_device_layout_coordinate_ties():
    # ties on x and y across -0.0 / +0.0 and negative values: the stable
    # lexicographic order must match std::stable_sort with operator<
    rng = np.random.default_rng(5)
    n = 400
    vals = np.array([-1.5, -0.0, 0.0, 0.25, -2.0, 3.0])
    coords = vals[rng.integers(0, vals.size, size=(n, 3))]
    elems = np.stack([rng.permutation(n)[:4] for _ in range(300)])
    free = np.sort(rng.choice(n, size=350, replace=False))
    for bs_elems, bs in ((elems, 1),):
        _both(freedofs=free, elems=bs_elems, n_total=n, block_size=bs, coords=coords, reorder="block_xyz")
    # block size 2 on a 2-D variant
    c2 = coords[:, :2]
    e2 = np.concatenate([2 * elems[:, :, None] + np.arange(2)], axis=2).reshape(elems.shape[0], -1)
    f2 = np.sort(np.concatenate([2 * free, 2 * free + 1]))
    _both(freedofs=f2, elems=e2, n_total=2 * n, block_size=2, coords=c2, reorder="block_xyz", rank=1, size=3)


def test_device_layout_empty_and_errors():
    lay = _lib.build_layout(freedofs=np.zeros(0, np.int64), elems=np.zeros((0, 3), np.int64), n_total=0,
                            block_size=1, reorder="none", device=True)
    assert lay["owned_rows"].size == 0 and lay["hi"] == 0
    # elements whose DOFs are all Dirichlet
    lay = _both(freedofs=np.array([3, 4]), elems=np.array([[0, 1, 2], [2, 3, 4]]), n_total=5, block_size=1,
                reorder="none")
    assert lay["elem_owner"].tolist() == [-1, 0]
    with pytest.raises(_lib.FneError):
        _lib.build_layout(freedofs=np.array([2, 1]), elems=np.array([[0, 1, 2]]), n_total=3, block_size=1,
                          reorder="none", device=True)
    with pytest.raises(_lib.FneError):
        _lib.build_layout(freedofs=np.arange(3), elems=np.array([[0, 1, 2]]), n_total=3, block_size=1,
                          reorder="none", perm_override=np.array([0, 0, 1]), device=True)
    bad = sparse.csr_matrix((np.ones(2), np.array([0, 7]), np.array([0, 1, 2, 2])), shape=(3, 8))
    with pytest.raises(_lib.FneError) as ei:
        _lib.build_layout(freedofs=np.arange(3), elems=np.array([[0, 1, 2]]), n_total=3, block_size=1,
                          reorder="none", adjacency=bad, device=True)
    assert ei.value.code == _lib.FNE_EBOUNDS


def test_device_layout_full_size_slope_p4():
    params = meshes.slope_problem(h=0.08, degree=4, lam=1.0)
    lay = _both(**_args(params, 2, "nodes", "u_0"), reorder="block_xyz")
    assert lay["owned_rows"].size == 152_345_168
