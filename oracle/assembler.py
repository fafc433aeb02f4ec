"""CPU restatement of ``ReorderedElementAssemblerBase``'s three callbacks (oracle).

Test infrastructure only.  ``OracleAssembler`` follows
``src/core/petsc/reordered_element_base.py``: construction mirrors
``__init__`` (:652-901) minus PETSc/KSP, and the callbacks mirror
``energy_fn`` (:1579-1611), ``gradient_fn`` (:1613-1633) and
``assemble_hessian_element`` (:1733-1775), including the ``np.add.at``
scatter into the owned COO values.
"""

from __future__ import annotations

import numpy as np

from oracle import energies, layout as L

FAMILY_KEYS = {
    "plaplace": ("dvx", "dvy", "vol"),
    "gl": ("dvx", "dvy", "vol"),
    "he": ("dphix", "dphiy", "dphiz", "vol"),
    "mc": ("elem_B", "quad_weight", "eps_p_old"),
}


class OracleAssembler:
    """One-rank (or one-rank-of-``size``) restatement of the reference assembler."""

    def __init__(self, family, params, adjacency=None, *, block_size=1, coordinate_key="nodes",
                 dirichlet_key="u_0", reorder_mode="block_xyz", rank=0, size=1, perm_override=None,
                 layout=None):
        """``layout``: optional precomputed global layout (an object with
        ``perm, iperm, lo, hi, n_free, total_to_free_reord, owned_rows,
        owned_cols, elem_owner``, e.g. a CUDA assembler's ``layout``, whose
        builders are checked bit-for-bit against the reference's); the sorted
        owned keys are rebuilt from it.  Saves the restated layout build on
        large meshes."""
        self.family = family
        self.params = params
        self.block_size = int(block_size)
        freedofs = np.asarray(params["freedofs"], dtype=np.int64)
        elems = np.asarray(params["elems"], dtype=np.int64)
        n_total = len(np.asarray(params[dirichlet_key]))
        if layout is not None:
            self.adjacency = None
            self.layout = self._adopt_layout(layout)
        else:
            if adjacency is None:
                adjacency = L.element_adjacency(elems, freedofs, n_total)
            self.adjacency = adjacency
            if perm_override is None:
                perm = L.select_permutation(
                    reorder_mode, adjacency=adjacency,
                    coords_all=np.asarray(params[coordinate_key], dtype=np.float64),
                    freedofs=freedofs, block_size=self.block_size,
                )
            else:
                perm = np.asarray(perm_override, dtype=np.int64)
            self.layout = L.build_global_layout(freedofs, elems, n_total, adjacency, perm,
                                                rank=rank, size=size, block_size=self.block_size)
        self.local = L.build_local_overlap_data(elems, self.layout, rank=rank)
        self.scatter = L.build_scatter_data(self.layout, self.local)
        self.dirichlet_full = np.asarray(params[dirichlet_key], dtype=np.float64)
        self.elem_data = {k: np.asarray(params[k], dtype=np.float64)[self.local.local_elem_idx]
                          for k in FAMILY_KEYS[family]}
        self.f_owned = self._rhs_owned()
        # rank 0 only (ginzburg_landau/jax_petsc/reordered_element_assembler.py:34-36)
        self.dirichlet_only_energy = self._dirichlet_only_energy() if (family == "gl" and rank == 0) else 0.0

    @staticmethod
    def _adopt_layout(lay):
        g = lambda k: np.asarray(getattr(lay, k) if not isinstance(lay, dict) else lay[k])  # noqa: E731
        lo, hi, n_free = (int(getattr(lay, k) if not isinstance(lay, dict) else lay[k]) for k in ("lo", "hi", "n_free"))
        rows, cols = g("owned_rows").astype(np.int64), g("owned_cols").astype(np.int64)
        keys = rows * np.int64(n_free) + cols
        order = np.argsort(keys, kind="mergesort")
        return L.GlobalLayout(
            perm=g("perm").astype(np.int64), iperm=g("iperm").astype(np.int64), lo=lo, hi=hi, n_free=n_free,
            total_to_free_reord=g("total_to_free_reord").astype(np.int64), coo_rows=rows, coo_cols=cols,
            owned_rows=rows, owned_cols=cols, owned_keys_sorted=keys[order],
            owned_pos_sorted=order.astype(np.int64), elem_owner=g("elem_owner").astype(np.int64))

    def restricted_rows(self, u_full_reordered, rows):
        """Owned gradient entries and owned COO values of the reordered rows
        ``rows`` only (see ``restricted_rows`` below)."""
        return restricted_rows(self.family, self.params, self.layout, u_full_reordered, rows,
                               dirichlet_full=self.dirichlet_full, f_owned=self.f_owned)

    # -- reference helpers -------------------------------------------------
    def _rhs_owned(self):
        """``plaplace/jax_petsc/reordered_element_assembler.py:67-72``; others: zeros."""
        lay = self.layout
        if self.family == "plaplace":
            rhs = np.asarray(self.params["f"], dtype=np.float64)
            free = np.asarray(self.params["freedofs"], dtype=np.int64)
            return rhs[free][lay.perm][lay.lo:lay.hi].copy()
        if self.family == "mc" and "force" in self.params:
            rhs = np.asarray(self.params["force"], dtype=np.float64)
            free = np.asarray(self.params["freedofs"], dtype=np.int64)
            return rhs[free][lay.perm][lay.lo:lay.hi].copy()
        return np.zeros(lay.hi - lay.lo)

    def _dirichlet_only_energy(self):
        """``ginzburg_landau/jax_petsc/reordered_element_assembler.py:34-52``."""
        elems = np.asarray(self.params["elems"], dtype=np.int64)
        mask = np.all(self.layout.total_to_free_reord[elems] < 0, axis=1)
        if not np.any(mask):
            return 0.0
        v_e = np.asarray(self.params["u_0"], dtype=np.float64)[elems[mask]]
        data = {k: np.asarray(self.params[k], dtype=np.float64)[mask] for k in ("dvx", "dvy", "vol")}
        e, _, _ = energies.element_derivatives("gl", v_e, data, self.params, want_hessian=False)
        return float(np.sum(e))

    def v_local(self, u_full_reordered):
        return L.local_vec_from_full(np.asarray(u_full_reordered, dtype=np.float64),
                                     self.layout.total_to_free_reord,
                                     self.local.local_total_nodes, self.dirichlet_full)

    def update_dirichlet(self, u0_new):
        """``reordered_element_base.py:1560-1566``."""
        self.dirichlet_full = np.asarray(u0_new, dtype=np.float64)

    def _derivs(self, u, want_hessian):
        v = self.v_local(u)
        v_e = v[self.local.elems_local_np]
        return v, energies.element_derivatives(self.family, v_e, self.elem_data, self.params,
                                               want_hessian=want_hessian)

    # -- the three callbacks ------------------------------------------------
    def energy_fn(self, u_full_reordered):
        _, (e, _, _) = self._derivs(u_full_reordered, False)
        val = float(np.sum(e * self.local.energy_weights))
        u_owned = np.asarray(u_full_reordered)[self.layout.lo:self.layout.hi]
        if self.f_owned.size:
            val -= float(np.dot(self.f_owned, u_owned))
        return val + self.dirichlet_only_energy

    def element_energy_sum(self, u_full_reordered):
        """Weighted element energy only (no load term, no Dirichlet-only constant)."""
        _, (e, _, _) = self._derivs(u_full_reordered, False)
        return float(np.sum(e * self.local.energy_weights))

    def gradient_fn(self, u_full_reordered):
        v, (_, g_e, _) = self._derivs(u_full_reordered, False)
        g_local = np.zeros(v.size)
        np.add.at(g_local, self.local.elems_local_np, g_e)
        g = g_local[self.scatter.owned_local_pos]
        if self.f_owned.size:
            g = g - self.f_owned
        return g

    def assemble_hessian_element(self, u_full_reordered):
        _, (_, _, h_e) = self._derivs(u_full_reordered, True)
        sc = self.scatter
        contrib = h_e[sc.hess_e, sc.hess_i, sc.hess_j]
        vals = np.zeros(self.layout.owned_rows.size)
        np.add.at(vals, sc.hess_positions, contrib)
        return vals

    def all_in_one(self, u_full_reordered):
        """(energy, gradient, owned Hessian values) from one derivative pass."""
        v, (e, g_e, h_e) = self._derivs(u_full_reordered, True)
        val = float(np.sum(e * self.local.energy_weights))
        u_owned = np.asarray(u_full_reordered)[self.layout.lo:self.layout.hi]
        if self.f_owned.size:
            val -= float(np.dot(self.f_owned, u_owned))
        val += self.dirichlet_only_energy
        g_local = np.zeros(v.size)
        np.add.at(g_local, self.local.elems_local_np, g_e)
        g = g_local[self.scatter.owned_local_pos]
        if self.f_owned.size:
            g = g - self.f_owned
        sc = self.scatter
        vals = np.zeros(self.layout.owned_rows.size)
        np.add.at(vals, sc.hess_positions, h_e[sc.hess_e, sc.hess_i, sc.hess_j])
        return val, g, vals


def restricted_rows(family, params, layout, u_full_reordered, rows, *, dirichlet_full, f_owned=None,
                    with_scale=False):
    """Gradient entries and owned COO Hessian values of the owned reordered
    rows ``rows`` only, from the elements that touch them: the same sums as
    ``gradient_fn`` / ``assemble_hessian_element`` restricted to those rows
    (``reordered_element_base.py:1613-1633, 1733-1762``), without building the
    full overlap / scatter data -- for meshes where the full oracle pass is
    too slow.  ``layout`` needs ``lo, n_free, total_to_free_reord,
    owned_rows, owned_cols``.  Returns ``(grad[sorted rows], positions,
    values)`` with positions into the owned COO order; with ``with_scale`` also
    the per-row sum of |element contributions| (+ |load|), the scale of the
    rounding of a low-precision gradient sum."""
    get = (lambda k: layout[k]) if isinstance(layout, dict) else (lambda k: getattr(layout, k))  # noqa: E731
    lo, n_free = int(get("lo")), int(get("n_free"))
    t2f = np.asarray(get("total_to_free_reord"), dtype=np.int64)
    orow, ocol = np.asarray(get("owned_rows"), dtype=np.int64), np.asarray(get("owned_cols"), dtype=np.int64)
    rows = np.unique(np.asarray(rows, dtype=np.int64))
    elems = np.asarray(params["elems"], dtype=np.int64)
    er_all = t2f[elems]
    sel_all = np.isin(er_all, rows)
    idx = np.flatnonzero(sel_all.any(axis=1))
    er, sel = er_all[idx], sel_all[idx]
    u = np.asarray(u_full_reordered, dtype=np.float64)
    v_e = np.where(er >= 0, u[np.maximum(er, 0)], np.asarray(dirichlet_full, dtype=np.float64)[elems[idx]])
    data = {k: np.asarray(params[k][idx], dtype=np.float64) for k in FAMILY_KEYS[family]}
    _, g_e, h_e = energies.element_derivatives(family, v_e, data, params, want_hessian=True)
    grad = np.zeros(rows.size)
    ei, li = np.nonzero(sel)
    np.add.at(grad, np.searchsorted(rows, er[ei, li]), g_e[ei, li])
    scale = np.zeros(rows.size)
    np.add.at(scale, np.searchsorted(rows, er[ei, li]), np.abs(g_e[ei, li]))
    if f_owned is not None and np.size(f_owned):
        grad -= np.asarray(f_owned)[rows - lo]
        scale += np.abs(np.asarray(f_owned)[rows - lo])
    pos_all = np.flatnonzero(np.isin(orow, rows))
    keys_sub = orow[pos_all] * np.int64(n_free) + ocol[pos_all]
    order = np.argsort(keys_sub, kind="mergesort")
    ei, li, lj = np.nonzero(sel[:, :, None] & (er[:, None, :] >= 0))
    keys = er[ei, li] * np.int64(n_free) + er[ei, lj]
    kp = np.searchsorted(keys_sub[order], keys)
    if np.any(kp >= keys_sub.size) or not np.array_equal(keys_sub[order][kp], keys):
        raise RuntimeError("element pair outside the owned COO pattern")
    pos = pos_all[order][kp]
    uniq, inv = np.unique(pos, return_inverse=True)
    vals = np.zeros(uniq.size)
    np.add.at(vals, inv, h_e[ei, li, lj])
    if with_scale:
        return grad, uniq, vals, scale
    return grad, uniq, vals
