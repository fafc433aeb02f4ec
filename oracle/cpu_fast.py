"""Multi-core CPU assembly of the P1-triangle families (numba, all host threads).

Test and measurement infrastructure only: the stronger CPU line beside the
autodiff restatement (``oracle/assembler.py``) in the benchmark's CPU
baseline; nothing in the package imports it.  Same outputs as the
reference's ``energy_fn`` / ``gradient_fn`` / ``assemble_hessian_element``
(``src/core/petsc/reordered_element_base.py:1579-1633, 1733-1762``) for
p-Laplace (``plaplace/jax_petsc/reordered_element_assembler.py:16-19``) and
Ginzburg-Landau (``ginzburg_landau/jax_petsc/reordered_element_assembler.py:18-24``),
computed with the closed-form element derivatives instead of autodiff, and
two parallel, deterministic phases instead of ``np.add.at``:

1. ``prange`` over elements: energy, 3 gradient and 9 Hessian entries;
2. ``prange`` over owned COO positions (and owned gradient rows): sum the
   contributions listed for that position, in element order.

The contribution lists come from the oracle's scatter data (built once).
"""

from __future__ import annotations

import numpy as np

try:
    import numba
    from numba import njit, prange
except ImportError:  # pragma: no cover - numba is in the image
    numba = None


def _csr_from_targets(targets, n):
    """Sources grouped by target (stable: source order within a target)."""
    order = np.argsort(targets, kind="stable")
    counts = np.bincount(targets, minlength=n)
    ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=ptr[1:])
    return ptr, order.astype(np.int64)


if numba is not None:

    @njit(parallel=True, fastmath=False, cache=False)
    def _elements(fam, v, dvx, dvy, vol, p, eps, ip, w, e_out, g_out, h_out):
        ne = v.shape[0]
        for e in prange(ne):
            fx = v[e, 0] * dvx[e, 0] + v[e, 1] * dvx[e, 1] + v[e, 2] * dvx[e, 2]
            fy = v[e, 0] * dvy[e, 0] + v[e, 1] * dvy[e, 1] + v[e, 2] * dvy[e, 2]
            ve = vol[e]
            if fam == 1:  # p-Laplace: (1/p) s^(p/2), s = |grad u|^2
                s = fx * fx + fy * fy
                if s > 0.0:
                    sp = s ** (0.5 * p)
                    a1 = sp / s              # s^(p/2 - 1)
                    a2 = (p - 2.0) * a1 / s  # (p - 2) s^(p/2 - 2)
                else:                        # limit at s = 0 (p > 2): zero derivatives
                    sp = 0.0
                    a1 = 0.0
                    a2 = 0.0
                e_out[e] = ve * sp / p
                for a in range(3):
                    da = fx * dvx[e, a] + fy * dvy[e, a]
                    g_out[e, a] = ve * a1 * da
                    for b in range(3):
                        db = fx * dvx[e, b] + fy * dvy[e, b]
                        h_out[e, 3 * a + b] = ve * (a1 * (dvx[e, a] * dvx[e, b] + dvy[e, a] * dvy[e, b])
                                                    + a2 * da * db)
            else:  # Ginzburg-Landau: eps/2 |grad u|^2 + 1/4 sum_q w_q ((v ip)_q^2 - 1)^2
                pot = 0.0
                nq0 = v[e, 0] * ip[0, 0] + v[e, 1] * ip[1, 0] + v[e, 2] * ip[2, 0]
                nq1 = v[e, 0] * ip[0, 1] + v[e, 1] * ip[1, 1] + v[e, 2] * ip[2, 1]
                nq2 = v[e, 0] * ip[0, 2] + v[e, 1] * ip[1, 2] + v[e, 2] * ip[2, 2]
                nq = (nq0, nq1, nq2)
                for q in range(3):
                    t = nq[q] * nq[q] - 1.0
                    pot += w[q] * t * t
                e_out[e] = ve * (0.5 * eps * (fx * fx + fy * fy) + 0.25 * pot)
                for a in range(3):
                    ga = eps * (fx * dvx[e, a] + fy * dvy[e, a])
                    for q in range(3):
                        ga += w[q] * (nq[q] * nq[q] - 1.0) * nq[q] * ip[a, q]
                    g_out[e, a] = ve * ga
                    for b in range(3):
                        hab = eps * (dvx[e, a] * dvx[e, b] + dvy[e, a] * dvy[e, b])
                        for q in range(3):
                            hab += w[q] * (3.0 * nq[q] * nq[q] - 1.0) * ip[a, q] * ip[b, q]
                        h_out[e, 3 * a + b] = ve * hab

    @njit(parallel=True, cache=False)
    def _gather(ptr, src_idx, src, out):
        for p in prange(out.shape[0]):
            acc = 0.0
            for j in range(ptr[p], ptr[p + 1]):
                acc += src[src_idx[j]]
            out[p] = acc

    @njit(parallel=True, cache=False)
    def _weighted_sum(e, wts):
        acc = 0.0
        for i in prange(e.shape[0]):
            acc += e[i] * wts[i]
        return acc


class FastTriangleAssembler:
    """Numba-parallel E + grad + Hess of a P1-triangle family, in the owned COO
    order of an ``OracleAssembler`` (``orc``), whose layout and scatter data
    it reuses."""

    def __init__(self, orc):
        if numba is None:
            raise RuntimeError("numba is not installed")
        if orc.family not in ("plaplace", "gl"):
            raise ValueError("P1 triangle families only")
        self.orc = orc
        self.fam = 1 if orc.family == "plaplace" else 2
        d = orc.elem_data
        self.dvx = np.ascontiguousarray(d["dvx"], dtype=np.float64)
        self.dvy = np.ascontiguousarray(d["dvy"], dtype=np.float64)
        self.vol = np.ascontiguousarray(d["vol"], dtype=np.float64)
        prm = orc.params
        self.p = float(prm.get("p", 2.0))
        self.eps = float(prm.get("eps", 0.0))
        self.ip = np.ascontiguousarray(prm.get("ip", np.zeros((3, 3))), dtype=np.float64).reshape(3, 3)
        self.w = np.ascontiguousarray(prm.get("w", np.zeros(3)), dtype=np.float64).reshape(3)
        sc = orc.scatter
        ne = self.vol.size
        # Hessian: contribution (e, i, j) -> flat source e * 9 + 3 i + j, grouped by COO position
        src = sc.hess_e.astype(np.int64) * 9 + sc.hess_i.astype(np.int64) * 3 + sc.hess_j.astype(np.int64)
        nnz = orc.layout.owned_rows.size
        self.h_ptr, order = _csr_from_targets(np.asarray(sc.hess_positions, dtype=np.int64), nnz)
        self.h_src = src[order]
        # gradient: local DOF of element node -> owned row
        local_rows = np.full(orc.local.local_total_nodes.size, -1, dtype=np.int64)
        own = sc.owned_local_pos
        local_rows[own] = np.arange(own.size, dtype=np.int64)
        er = local_rows[orc.local.elems_local_np]                # (E, 3) owned row or -1
        e_idx, k_idx = np.nonzero(er >= 0)
        self.g_ptr, order = _csr_from_targets(er[e_idx, k_idx], own.size)
        self.g_src = (e_idx * 3 + k_idx)[order].astype(np.int64)
        self.e = np.empty(ne)
        self.g = np.empty((ne, 3))
        self.h = np.empty((ne, 9))
        self.vals = np.empty(nnz)
        self.grad = np.empty(own.size)
        self.weights = np.ascontiguousarray(orc.local.energy_weights, dtype=np.float64)

    def all_in_one(self, u_full_reordered):
        """(energy, owned gradient, owned COO values) like ``OracleAssembler.all_in_one``."""
        orc = self.orc
        v = orc.v_local(u_full_reordered)[orc.local.elems_local_np]
        _elements(self.fam, np.ascontiguousarray(v), self.dvx, self.dvy, self.vol, self.p, self.eps, self.ip,
                  self.w, self.e, self.g, self.h)
        _gather(self.h_ptr, self.h_src, self.h.reshape(-1), self.vals)
        _gather(self.g_ptr, self.g_src, self.g.reshape(-1), self.grad)
        val = float(_weighted_sum(self.e, self.weights))
        u_owned = np.asarray(u_full_reordered)[orc.layout.lo: orc.layout.hi]
        grad = self.grad
        if orc.f_owned.size:
            val -= float(np.dot(orc.f_owned, u_owned))
            grad = grad - orc.f_owned
        return val + orc.dirichlet_only_energy, grad, self.vals

    @staticmethod
    def threads():
        return int(numba.get_num_threads()) if numba is not None else 1
