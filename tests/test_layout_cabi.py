"""The C++ layout builder (libfne_asm.so) reproduces the reference layout bit for bit.

Runs on CPU: ``fne_layout_build`` is host code.  The checker is the NumPy
restatement in ``oracle/layout.py`` (itself pinned by the reference's goldens).
"""

import re
from pathlib import Path

import numpy as np
import pytest

from oracle import layout as L
from fenics_nonlinear_energies_b200 import _lib, meshes

ROOT = Path(__file__).resolve().parents[1]


def _compare(params, *, bs, coord_key, dir_key, reorder, rank=0, size=1, adjacency=None, perm_override=None):
    free = np.asarray(params["freedofs"])
    elems = np.asarray(params["elems"])
    n_total = len(params[dir_key])
    lay = _lib.build_layout(freedofs=free, elems=elems, n_total=n_total, block_size=bs, reorder=reorder,
                            coords=params[coord_key], rank=rank, size=size, adjacency=adjacency,
                            perm_override=perm_override)
    adj = adjacency if adjacency is not None else L.element_adjacency(elems, free, n_total)
    if perm_override is not None:
        perm = np.asarray(perm_override)
    else:
        perm = L.select_permutation(reorder, adjacency=adj, coords_all=params[coord_key], freedofs=free,
                                    block_size=bs)
    ref = L.build_global_layout(free, elems, n_total, adj, perm, rank=rank, size=size, block_size=bs)
    for k in ("perm", "iperm", "total_to_free_reord", "coo_rows", "coo_cols", "owned_rows", "owned_cols",
              "elem_owner"):
        np.testing.assert_array_equal(lay[k], getattr(ref, k), err_msg=k)
    assert (lay["lo"], lay["hi"]) == (ref.lo, ref.hi)


@pytest.mark.parametrize("numbering", ["x_slow", "x_fast"])
@pytest.mark.parametrize("reorder", ["none", "block_xyz"])
def test_tri_layout(numbering, reorder):
    params, _ = meshes.gl_problem(n=7, numbering=numbering)
    _compare(params, bs=1, coord_key="nodes", dir_key="u_0", reorder=reorder)


@pytest.mark.parametrize("size", [2, 3])
def test_tri_layout_ranks(size):
    params, _ = meshes.plaplace_problem(n=6, numbering="x_fast")
    for rank in range(size):
        _compare(params, bs=1, coord_key="nodes", dir_key="u_0", reorder="block_xyz", rank=rank, size=size)


@pytest.mark.parametrize("reorder", ["none", "block_xyz"])
def test_tet_layout(reorder):
    params, _ = meshes.he_beam_problem(nx=4, ny=2, nz=2)
    _compare(params, bs=3, coord_key="nodes2coord", dir_key="u_0_ref", reorder=reorder)
    _compare(params, bs=3, coord_key="nodes2coord", dir_key="u_0_ref", reorder=reorder, rank=1, size=2)


def test_given_adjacency_and_override():
    params, _ = meshes.gl_problem(n=5, numbering="x_fast")
    free = params["freedofs"]
    adj = L.element_adjacency(params["elems"], free, len(params["u_0"]))
    perm = np.random.default_rng(0).permutation(free.size)
    _compare(params, bs=1, coord_key="nodes", dir_key="u_0", reorder="none", adjacency=adj, perm_override=perm)


def test_reference_goldens_through_cabi():
    # tests/test_reordered_element_base.py:12-52 goldens, through the C++ builder
    coords = np.array([[1.0, 0.0], [0.0, 1.0], [0.0, 0.0], [1.0, 1.0]])
    lay = _lib.build_layout(freedofs=np.arange(4), elems=np.array([[0, 1, 2], [1, 2, 3]]), n_total=4,
                            block_size=1, coords=coords)
    assert lay["perm"].tolist() == [2, 1, 0, 3]
    coords3 = np.array([[1.0, 0.0, 0.0], [0.0, 0.0, 0.0]])
    lay = _lib.build_layout(freedofs=np.arange(6), elems=np.array([[0, 1, 2, 3, 4, 5]]), n_total=6,
                            block_size=3, coords=coords3)
    assert lay["perm"].tolist() == [3, 4, 5, 0, 1, 2]


def test_layout_errors():
    with pytest.raises(_lib.FneError):
        _lib.build_layout(freedofs=np.array([2, 1]), elems=np.array([[0, 1, 2]]), n_total=3, block_size=1,
                          reorder="none")
    with pytest.raises(_lib.FneError):
        _lib.build_layout(freedofs=np.arange(3), elems=np.array([[0, 1, 2]]), n_total=3, block_size=1,
                          reorder="none", perm_override=np.array([0, 0, 1]))


def test_empty_mesh_layout():
    lay = _lib.build_layout(freedofs=np.zeros(0, np.int64), elems=np.zeros((0, 3), np.int64), n_total=0,
                            block_size=1, reorder="none")
    assert lay["owned_rows"].size == 0 and lay["hi"] == 0


def test_library_exports_every_declared_symbol():
    header = (ROOT / "include" / "fne_asm.h").read_text()
    names = set(re.findall(r"^\s*(?:int|void|const char\*)\s+(fne_\w+)\s*\(", header, re.M))
    assert len(names) >= 12
    for n in sorted(names):
        assert hasattr(_lib.lib, n), n


@pytest.mark.parametrize("reorder", ["none", "block_xyz"])
@pytest.mark.parametrize("size", [1, 2, 3])
def test_slope3d_p2_layout(reorder, size):
    """The 3-D family's layout (P2 tetrahedra, 3 DOFs per node, 30 DOFs per
    element) through the same C++ builder, bit for bit against the oracle."""
    p = meshes.slope3d_problem(nx=3, ny=2, nz=2, degree=2)
    for rank in range(size):
        _compare(p, bs=3, coord_key="nodes", dir_key="u_0", reorder=reorder, rank=rank, size=size)


def test_device_cg_argument_checks_on_host():
    """DeviceCG reaches fne_cg_create with the documented argument checks, which
    run on the host before any device call: an entry outside the n x n block
    is FNE_EBOUNDS, mismatched row / column arrays are rejected in Python."""
    from fenics_nonlinear_energies_b200.newton import DeviceCG

    with pytest.raises(_lib.FneError) as ei:
        DeviceCG(3, np.array([0, 1, 3]), np.array([0, 1, 2]), device="cpu")
    assert ei.value.code == _lib.FNE_EBOUNDS
    with pytest.raises(_lib.FneError) as ei:
        DeviceCG(3, np.array([0, 1, 2]), np.array([0, -1, 2]), device="cpu")
    assert ei.value.code == _lib.FNE_EBOUNDS
    with pytest.raises(ValueError):
        DeviceCG(3, np.array([0, 1]), np.array([0, 1, 2]), device="cpu")
    with pytest.raises(_lib.FneError) as ei:
        DeviceCG(3, np.array([0, 1, 2]), np.array([0, 1, 2]), device="cpu", chunk=0)
    assert ei.value.code == _lib.FNE_EINVAL


def test_mc3d_descriptor_checks_on_host():
    """fne_create for the 3-D Mohr-Coulomb family checks its descriptor on the
    host before any device call: nodes per element (4, 10 or 35), block size
    3, 1 to 16 quadrature points (P1, P2) or 1 to 32 (P4) and the presence of
    the per-point arrays."""
    import ctypes as C

    p = meshes.slope3d_problem(nx=2, ny=2, nz=1, degree=1)
    el, pel = _lib.i64(p["elems"])
    t2f, pt2f = _lib.i64(np.full(p["u_0"].size, -1, dtype=np.int64))
    dirv, pdir = _lib.f64(p["u_0"])
    keep = [el, t2f, dirv]

    def desc(**kw):
        d = _lib.Desc()
        d.family, d.precision, d.n_elem, d.npe, d.block_size = _lib.FNE_MOHR_COULOMB_3D, 0, el.shape[0], 4, 3
        d.elems, d.n_total, d.total_to_free_reord, d.dirichlet, d.nq = pel, p["u_0"].size, pt2f, pdir, 1
        for k, v in kw.items():
            setattr(d, k, v)
        return d

    h = C.c_void_p()
    for kw, what in (({"npe": 6}, "tetrahedra"), ({"block_size": 2}, "block_size"), ({"nq": 17}, "quadrature"),
                     ({"npe": 35, "nq": 33}, "quadrature"), ({}, "missing")):
        rc = _lib.lib.fne_create(C.byref(desc(**kw)), C.byref(h))
        assert rc == _lib.FNE_EINVAL, (kw, rc)
        assert what in _lib.lib.fne_last_error().decode(), _lib.lib.fne_last_error()
    del keep
