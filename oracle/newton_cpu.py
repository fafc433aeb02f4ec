"""CPU Newton over the oracle assembler (the timed CPU baseline of the Newton workloads).

Test infrastructure only.  The same loop as the device driver
(``fenics_nonlinear_energies_b200/newton.py``, itself the golden-section
branch of ``src/core/petsc/minimizers.py:181-1038``): gradient, stop on
``||g|| < max(tolg, tolg_rel ||g_0||)``, assembled Hessian, Jacobi CG
(``oracle/krylov.py``, SciPy CSR products), interval repair and
golden-section line search (the package's host functions, which are plain
Python), accept a step only if it lowers the energy.  Everything runs in
NumPy float64 on the host.
"""

from __future__ import annotations

import math
import time

import numpy as np
from scipy import sparse

from oracle import krylov


def newton_cpu(asm, x0, *, tolg=0.0, tolg_rel=1e-6, maxit=100, linesearch_interval=(-0.5, 2.0),
               linesearch_tol=1e-3, ksp_rtol=1e-3, ksp_max_it=500):
    from fenics_nonlinear_energies_b200.newton import golden_section_search, repair_linesearch_interval

    lay = asm.layout
    rows = np.asarray(lay.owned_rows, dtype=np.int64) - lay.lo
    cols = np.asarray(lay.owned_cols, dtype=np.int64)
    n = rows.max() + 1 if rows.size else 0
    x = np.array(x0, dtype=np.float64)
    t0 = time.perf_counter()

    def energy(v):
        e = float(asm.energy_fn(v))
        return e if math.isfinite(e) else math.inf

    fx = energy(x)
    g0 = None
    nit, ksp_total = 0, 0
    message = "Maximum number of iterations reached"
    for _ in range(maxit):
        g = np.asarray(asm.gradient_fn(x))
        normg = float(np.linalg.norm(g))
        if g0 is None:
            g0 = normg
        if normg < max(tolg, tolg_rel * g0):
            message = "Gradient norm converged"
            break
        nit += 1
        vals = np.asarray(asm.assemble_hessian_element(x), dtype=np.float64)
        A = sparse.csr_matrix((vals, (rows, cols)), shape=(n, n))
        p, its, _ = krylov.pcg(A, krylov.jacobi_scaling(A.diagonal()), -g, ksp_rtol, ksp_max_it)
        ksp_total += its

        def f_alpha(alpha):
            return energy(x + alpha * p)

        a, b, _, _ = repair_linesearch_interval(f_alpha, *linesearch_interval, center=0.0, center_value=fx,
                                                tol=linesearch_tol)
        alpha, _ = golden_section_search(f_alpha, a, b, linesearch_tol)
        f_new = f_alpha(alpha)
        if not (math.isfinite(f_new) and f_new < fx):
            message = "Line search made no progress"
            break
        x = x + alpha * p
        fx = f_new
    g = np.asarray(asm.gradient_fn(x))
    normg = float(np.linalg.norm(g))
    return x, {"iterations": nit, "ksp_its": ksp_total, "energy": fx, "grad_norm": normg, "grad_norm0": g0,
               "converged": g0 is not None and normg < max(tolg, tolg_rel * g0) * (1.0 + 1e-12),
               "message": message, "time_s": time.perf_counter() - t0}
