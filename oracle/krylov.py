"""Scalar Jacobi-preconditioned CG (oracle for the device CG, ``fne_cg_*``).

Test infrastructure only.  The Newton driver's linear solve stands in for the
KSP solve the reference runs on the assembled Hessian
(``src/core/petsc/scalar_problem_driver.py:154-226``: ``ksp.setTolerances(rtol,
max_it)``, ``ksp.solve``, ``ksp.getIterationNumber``) with PETSc's CG
conventions: unpreconditioned-residual test ``||r|| <= rtol ||b||`` from a zero
start, Jacobi scaling ``1 / |a_ii|``, and a stop at non-positive curvature
``p.Ap <= 0`` that keeps the last iterate (the right-hand side itself when it
happens at the first iteration, so that a Newton direction stays a descent
direction).  The device solver must take the same number of iterations and
return the same iterate to rounding.
"""

from __future__ import annotations

import numpy as np

CONVERGED, NEGATIVE_CURVATURE, ITERATION_LIMIT, ZERO_RHS = range(4)


def jacobi_scaling(diag):
    """``1 / |d|``, with 1 where the diagonal is zero, missing (NaN) or not finite in magnitude."""
    d = np.abs(np.asarray(diag, dtype=np.float64))
    d = np.where(d > 0, d, 1.0)
    return 1.0 / d


def pcg(A, dinv, b, rtol, maxit):
    """Returns ``(x, iterations, reason)`` for ``A x = b`` (``A`` anything with ``@``)."""
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b)
    bnorm = np.linalg.norm(b)
    if bnorm == 0.0:
        return x, 0, ZERO_RHS
    r = b.copy()
    z = dinv * r
    p = z.copy()
    rz = r @ z
    for it in range(1, maxit + 1):
        Ap = A @ p
        pAp = p @ Ap
        if not pAp > 0.0:
            return (x if it > 1 else b.copy()), it, NEGATIVE_CURVATURE
        alpha = rz / pAp
        x = x + alpha * p
        r = r - alpha * Ap
        if np.linalg.norm(r) <= rtol * bnorm:
            return x, it, CONVERGED
        z = dinv * r
        rz_new = r @ z
        p = z + (rz_new / rz) * p
        rz = rz_new
    return x, maxit, ITERATION_LIMIT
