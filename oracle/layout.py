"""NumPy restatement of the reference's DOF layout and scatter map (oracle).

Test infrastructure only (see ``oracle/__init__.py``).  Every function cites
the reference function it restates; ``comm`` objects are replaced by plain
``rank`` / ``size`` integers.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy import sparse
from scipy.sparse.csgraph import reverse_cuthill_mckee


def petsc_ownership_range(n, rank, size, block_size=1):
    """``src/core/petsc/dof_partition.py:27-55``."""
    if block_size < 1:
        raise ValueError("block_size must be >= 1")
    if block_size > 1:
        if n % block_size != 0:
            raise ValueError("n not divisible by block_size")
        lo_b, hi_b = petsc_ownership_range(n // block_size, rank, size, 1)
        return lo_b * block_size, hi_b * block_size
    q, r = divmod(int(n), int(size))
    if rank < r:
        lo = rank * (q + 1)
        return lo, lo + q + 1
    lo = rank * q + r
    return lo, lo + q


def rank_of_dof_vec(dof_indices, n_total, size, block_size=1):
    """``src/core/petsc/dof_partition.py:502-521``."""
    dof_indices = np.asarray(dof_indices, dtype=np.int64)
    if block_size > 1:
        return rank_of_dof_vec(dof_indices // block_size, n_total // block_size, size, 1)
    q, r = divmod(int(n_total), int(size))
    boundary = r * (q + 1)
    out = np.empty(len(dof_indices), dtype=np.int64)
    below = dof_indices < boundary
    out[below] = dof_indices[below] // (q + 1)
    if q > 0:
        out[~below] = r + (dof_indices[~below] - boundary) // q
    return out


def expand_block_perm(block_perm, block_size):
    """``src/core/petsc/reordered_element_base.py:134-141``."""
    block_perm = np.asarray(block_perm, dtype=np.int64)
    if block_size <= 1:
        return block_perm
    perm = np.empty(block_perm.size * block_size, dtype=np.int64)
    for comp in range(block_size):
        perm[comp::block_size] = block_perm * block_size + comp
    return perm


def perm_block_xyz(coords_all, freedofs, block_size):
    """``src/core/petsc/reordered_element_base.py:159-170``: lexsort by (x, y, z)."""
    freedofs = np.asarray(freedofs, dtype=np.int64)
    node_ids = freedofs[::block_size] // block_size
    coords = np.asarray(coords_all[node_ids], dtype=np.float64)
    keys = tuple(coords[:, d] for d in reversed(range(coords.shape[1])))
    return expand_block_perm(np.lexsort(keys).astype(np.int64), block_size)


def _block_graph(adjacency, block_size):
    """``src/core/petsc/reordered_element_base.py:120-131``."""
    rows, cols = adjacency.nonzero()
    nb = adjacency.shape[0] // block_size
    g = sparse.coo_matrix(
        (np.ones(rows.size, dtype=np.int8), (rows // block_size, cols // block_size)),
        shape=(nb, nb),
    ).tocsr()
    g.data[:] = 1
    g.eliminate_zeros()
    return g


def perm_block_rcm(adjacency, block_size):
    """``src/core/petsc/reordered_element_base.py:148-156``."""
    graph = adjacency.tocsr() if block_size <= 1 else _block_graph(adjacency, block_size)
    bp = np.asarray(reverse_cuthill_mckee(graph, symmetric_mode=True), dtype=np.int64)
    return expand_block_perm(bp, block_size)


def select_permutation(mode, *, adjacency, coords_all, freedofs, block_size):
    """``src/core/petsc/reordered_element_base.py:183-200`` (METIS omitted: not installed)."""
    if mode == "none":
        return np.arange(len(freedofs), dtype=np.int64)
    if mode == "block_rcm":
        return perm_block_rcm(adjacency, block_size)
    if mode == "block_xyz":
        return perm_block_xyz(coords_all, freedofs, block_size)
    raise ValueError(f"Unsupported element reorder mode: {mode!r}")


def inverse_permutation(perm):
    """``src/core/petsc/reordered_element_base.py:203-206``."""
    perm = np.asarray(perm, dtype=np.int64)
    iperm = np.empty_like(perm)
    iperm[perm] = np.arange(perm.size, dtype=np.int64)
    return iperm


def local_vec_from_full(full_reordered, total_to_free_reord, local_total_nodes, dirichlet_full):
    """``src/core/petsc/reordered_element_base.py:225-235``."""
    local_reord = total_to_free_reord[local_total_nodes]
    v_local = np.asarray(dirichlet_full[local_total_nodes], dtype=np.float64).copy()
    free = local_reord >= 0
    if np.any(free):
        v_local[free] = full_reordered[local_reord[free]]
    return v_local


def element_adjacency(elems, freedofs, n_total):
    """Free-DOF element-pair adjacency, as built by the reference's mesh helpers
    (``src/problems/plaplace_u3/support/mesh.py:74-93``,
    ``src/problems/slope_stability/support/mesh.py:638-667``)."""
    freedofs = np.asarray(freedofs, dtype=np.int64)
    elems = np.asarray(elems, dtype=np.int64)
    n_free = freedofs.size
    full_to_free = np.full(int(n_total), -1, dtype=np.int64)
    full_to_free[freedofs] = np.arange(n_free, dtype=np.int64)
    local = full_to_free[elems]
    k = local.shape[1]
    rr = np.repeat(local, k, axis=1).reshape(-1)
    cc = np.tile(local, (1, k)).reshape(-1)
    mask = (rr >= 0) & (cc >= 0)
    adj = sparse.coo_matrix(
        (np.ones(int(mask.sum()), dtype=np.float64), (rr[mask], cc[mask])),
        shape=(n_free, n_free),
    )
    adj.sum_duplicates()
    adj.data[:] = 1.0
    return adj


@dataclass
class GlobalLayout:
    perm: np.ndarray
    iperm: np.ndarray
    lo: int
    hi: int
    n_free: int
    total_to_free_reord: np.ndarray
    coo_rows: np.ndarray
    coo_cols: np.ndarray
    owned_rows: np.ndarray
    owned_cols: np.ndarray
    owned_keys_sorted: np.ndarray
    owned_pos_sorted: np.ndarray
    elem_owner: np.ndarray


def build_global_layout(freedofs, elems, n_total, adjacency, perm, *, rank=0, size=1, block_size=1):
    """``src/core/petsc/reordered_element_base.py:380-506`` (global-adjacency branch)."""
    freedofs = np.asarray(freedofs, dtype=np.int64)
    elems = np.asarray(elems, dtype=np.int64)
    n_free = int(freedofs.size)
    iperm = inverse_permutation(perm)
    lo, hi = petsc_ownership_range(n_free, rank, size, block_size=block_size)
    t2f_orig = np.full(int(n_total), -1, dtype=np.int64)
    t2f_orig[freedofs] = np.arange(n_free, dtype=np.int64)
    t2f = np.full(int(n_total), -1, dtype=np.int64)
    m = t2f_orig >= 0
    t2f[m] = iperm[t2f_orig[m]]
    key_base = np.int64(n_free)
    row_adj, col_adj = adjacency.tocsr().nonzero()
    coo_rows = iperm[np.asarray(row_adj, dtype=np.int64)]
    coo_cols = iperm[np.asarray(col_adj, dtype=np.int64)]
    owned = (coo_rows >= lo) & (coo_rows < hi)
    owned_rows = coo_rows[owned]
    owned_cols = coo_cols[owned]
    keys = owned_rows * key_base + owned_cols
    order = np.argsort(keys, kind="mergesort")
    er = t2f[elems]
    masked = np.where(er >= 0, er, np.int64(n_free))
    emin = np.min(masked, axis=1)
    valid = emin < n_free
    owner = np.full(len(elems), -1, dtype=np.int64)
    if np.any(valid):
        owner[valid] = rank_of_dof_vec(emin[valid], n_free, size, block_size)
    return GlobalLayout(
        perm=np.asarray(perm, dtype=np.int64), iperm=iperm, lo=lo, hi=hi, n_free=n_free,
        total_to_free_reord=t2f, coo_rows=coo_rows, coo_cols=coo_cols,
        owned_rows=owned_rows, owned_cols=owned_cols,
        owned_keys_sorted=keys[order], owned_pos_sorted=order.astype(np.int64),
        elem_owner=owner,
    )


@dataclass
class LocalOverlapData:
    local_elem_idx: np.ndarray
    local_total_nodes: np.ndarray
    elems_local_np: np.ndarray
    elems_reordered: np.ndarray
    energy_weights: np.ndarray


def build_local_overlap_data(elems, layout, *, rank=0):
    """``src/core/petsc/reordered_element_base.py:509-597`` (non-distributed branch)."""
    elems = np.asarray(elems, dtype=np.int64)
    er = layout.total_to_free_reord[elems]
    local = np.any((er >= layout.lo) & (er < layout.hi), axis=1)
    idx = np.where(local)[0].astype(np.int64)
    weights = (layout.elem_owner[idx] == rank).astype(np.float64)
    local_elems_total = elems[idx]
    ltn, inv = np.unique(local_elems_total.ravel(), return_inverse=True)
    return LocalOverlapData(
        local_elem_idx=idx,
        local_total_nodes=ltn.astype(np.int64),
        elems_local_np=inv.reshape(local_elems_total.shape).astype(np.int32),
        elems_reordered=layout.total_to_free_reord[local_elems_total],
        energy_weights=weights,
    )


@dataclass
class ScatterData:
    owned_local_pos: np.ndarray
    hess_e: np.ndarray
    hess_i: np.ndarray
    hess_j: np.ndarray
    hess_positions: np.ndarray


def build_scatter_data(layout, local):
    """``src/core/petsc/reordered_element_base.py:1464-1534`` (``coo`` backend)."""
    er = local.elems_reordered
    lr = layout.total_to_free_reord[local.local_total_nodes]
    own = (lr >= layout.lo) & (lr < layout.hi)
    olp = np.full(layout.hi - layout.lo, -1, dtype=np.int64)
    olp[lr[own] - layout.lo] = np.where(own)[0]
    if np.any(olp < 0):
        raise RuntimeError("Failed to map all owned reordered DOFs to overlap-local indices")
    rows = er[:, :, None]
    cols = er[:, None, :]
    valid = (rows >= layout.lo) & (rows < layout.hi) & (cols >= 0)
    vi = np.where(valid)
    keys = er[vi[0], vi[1]] * np.int64(layout.n_free) + er[vi[0], vi[2]]
    kp = np.searchsorted(layout.owned_keys_sorted, keys)
    if np.any(kp >= layout.owned_keys_sorted.size):
        raise RuntimeError("Scatter lookup exceeded owned COO pattern size")
    if not np.array_equal(layout.owned_keys_sorted[kp], keys):
        raise RuntimeError("Scatter lookup found mismatched owned COO entries")
    return ScatterData(
        owned_local_pos=olp,
        hess_e=vi[0].astype(np.int64), hess_i=vi[1].astype(np.int64), hess_j=vi[2].astype(np.int64),
        hess_positions=layout.owned_pos_sorted[kp],
    )
