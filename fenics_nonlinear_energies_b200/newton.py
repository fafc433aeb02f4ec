"""Device-resident Newton driver used for end-to-end runs on one GPU.

The reference's driver (``src/core/petsc/minimizers.py``) stays the production
caller of the assembler; this module restates the parts of it the GPU runs
need so that Newton iterations can be counted without PETSc:

* ``golden_section_search`` -- ``minimizers.py:14-61`` (same bracket updates,
  best-point tracking and final midpoint evaluation);
* ``repair_linesearch_interval`` -- ``minimizers.py:74-127`` (bisect
  non-finite interval ends back toward the finite centre);
* ``newton`` -- the golden-section branch of ``minimizers.py:181-1038``:
  gradient, stop on ``||g|| < max(tolg, tolg_rel * ||g_0||)``, linear solve
  of ``H p = -g``, line search on ``[a, b]``, accept a step only if it lowers
  the energy, optional stop on the energy change.

The linear solve is Jacobi-preconditioned conjugate gradients on the
assembled owned COO values (``DeviceCG``: the library's own CG kernels,
``fne_cg_*``, every iteration on the device); CG stops at a
negative-curvature direction and returns the last iterate (or the steepest
descent direction), which keeps the Newton direction a descent direction for
the non-convex Ginzburg-Landau energy.
"""

from __future__ import annotations

import ctypes
import math
import time

import numpy as np
import torch

from fenics_nonlinear_energies_b200 import _lib


def golden_section_search(f, a, b, tol):
    """Minimise ``f`` on ``[a, b]``; returns ``(alpha, n_evals)``.

    Golden-section bracketing in the reference's evaluation order
    (``core/petsc/minimizers.py:14-61``): both ends and both interior points
    are evaluated first; each step keeps the sub-bracket around the smaller
    interior value and evaluates one new interior point; the smallest value
    seen anywhere is tracked; the bracket's midpoint is evaluated last.
    """
    ratio = 0.5 + math.sqrt(5.0) / 2.0
    lo, hi = float(a), float(b)
    f_lo, f_hi = f(lo), f(hi)
    right = (hi - lo) / ratio + lo
    left = lo + hi - right
    f_left, f_right = f(left), f(right)
    n_evals = 4
    arg_min, f_min = lo, f_lo
    for t, ft in ((hi, f_hi), (left, f_left), (right, f_right)):
        if ft < f_min:
            arg_min, f_min = t, ft
    while hi - lo > tol:
        if f_left < f_right:  # minimum in [lo, right]: old left becomes the right point
            hi = right
            right, left = left, lo + hi - left
            f_right, f_left = f_left, f(left)
            fresh = ((right, f_right), (left, f_left))
        else:  # minimum in [left, hi]: old right becomes the left point
            lo = left
            left, right = right, lo + hi - right
            f_left, f_right = f_right, f(right)
            fresh = ((left, f_left), (right, f_right))
        for t, ft in fresh:
            if ft < f_min:
                arg_min, f_min = t, ft
        n_evals += 1
    mid = 0.5 * (lo + hi)
    f_mid = f(mid)
    n_evals += 1
    if f_mid < f_min:
        arg_min = mid
    return float(arg_min), n_evals


def repair_linesearch_interval(f, a, b, center=0.0, center_value=None, tol=1e-6, max_bisect=60):
    """Shrink non-finite interval ends toward the finite centre; ``(a, b, n_evals, repaired)``."""
    n_evals = 0
    repaired = False
    if center_value is None:
        center_value = f(center)
        n_evals += 1
    if not math.isfinite(center_value):
        return a, b, n_evals, repaired
    tol = max(float(tol), 1e-12)

    def side(bound, sign):
        nonlocal n_evals, repaired
        if (sign < 0 and not bound < center) or (sign > 0 and not bound > center):
            return bound
        fb = f(bound)
        n_evals += 1
        if math.isfinite(fb):
            return bound
        repaired = True
        good, bad = center, bound
        for _ in range(max_bisect):
            mid = 0.5 * (good + bad)
            fm = f(mid)
            n_evals += 1
            if math.isfinite(fm):
                good = mid
            else:
                bad = mid
            if abs(bad - good) <= tol:
                break
        return good

    return side(float(a), -1.0), side(float(b), 1.0), n_evals, repaired


class DeviceCG:
    """Jacobi-preconditioned CG on an assembler's owned COO Hessian (``fne_cg_*``).

    The pattern is the one-rank owned COO pattern (``owned_rows - lo``,
    ``owned_cols``); values are taken in COO order from
    ``assembler.owned_values`` (FP32 or FP64 storage, FP64 arithmetic).  Every
    CG iteration runs on the device; the host reads the solver state once per
    CUDA graph of ``chunk`` iterations.
    """

    REASONS = ("converged", "non-positive curvature", "iteration limit", "zero right-hand side")

    def __init__(self, n, rows, cols, *, fp32=False, device="cuda", chunk=16):
        self._h = None
        self.n = int(n)
        self.device = torch.device(device)
        self.fp32 = bool(fp32)
        rows_np, rp = _lib.i64(rows)  # the arrays stay referenced until the call returns
        cols_np, cp = _lib.i64(cols)
        if rows_np.size != cols_np.size:
            raise ValueError("rows and cols differ in length")
        h = ctypes.c_void_p()
        _lib.check(_lib.lib.fne_cg_create(self.n, int(rows_np.size), rp, cp, int(self.fp32), int(chunk),
                                          ctypes.byref(h)))
        self._h = h
        self.chunk = int(chunk)
        self.reason = None
        self.launches = 0  # kernels launched by update() and solve() so far

    @classmethod
    def for_assembler(cls, assembler, chunk=16):
        lay = assembler.layout
        rows = np.asarray(lay.owned_rows, dtype=np.int64) - lay.lo
        return cls(assembler.n_owned, rows, lay.owned_cols, fp32=assembler.owned_values.dtype == torch.float32,
                   device=assembler.device, chunk=chunk)

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def update(self, values):
        want = torch.float32 if self.fp32 else torch.float64
        if values.dtype != want or not values.is_contiguous():
            raise TypeError(f"COO values must be a contiguous {want} tensor")
        self._values = values
        _lib.check(_lib.lib.fne_cg_set_matrix(self._h, values.data_ptr(), self._stream()))
        self.launches += 1

    def solve(self, b, rtol=1e-3, maxit=500, out=None):
        """``x`` with ``A x = b`` to ``rtol`` (stopping rules of ``fne_cg_solve``); returns ``(x, iterations)``."""
        b = b.contiguous()
        x = torch.empty_like(b) if out is None else out
        its, why = ctypes.c_int32(), ctypes.c_int32()
        _lib.check(_lib.lib.fne_cg_solve(self._h, b.data_ptr(), x.data_ptr(), float(rtol), int(maxit),
                                         ctypes.byref(its), ctypes.byref(why), self._stream()))
        self.reason = self.REASONS[why.value]
        # one initialisation kernel, then graphs of `chunk` iterations of two
        # kernels until the iteration that stopped the solve
        self.launches += 1 + 2 * self.chunk * (-(-int(its.value) // self.chunk))
        return x, int(its.value)

    def close(self):
        if self._h:
            _lib.lib.fne_cg_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def newton(assembler, x0, *, tolg=0.0, tolg_rel=1e-6, tolf=0.0, maxit=100, linesearch_interval=(-0.5, 2.0),
           linesearch_tol=1e-3, ksp_rtol=1e-3, ksp_max_it=500, verbose=False, cg=None):
    """Minimise the assembler's energy from ``x0`` (device tensor of the owned reordered DOFs).

    Returns ``(x, info)`` with ``info["iterations"]`` the number of Newton
    steps taken, ``info["converged"]``, the final energy and gradient norm.
    ``cg``: a ``DeviceCG`` for this assembler's pattern to reuse across calls
    (one is created and released per call otherwise).
    """
    dev = assembler.device
    x = torch.as_tensor(x0, dtype=torch.float64, device=dev).clone()
    own_cg = cg is None
    if own_cg:
        cg = DeviceCG.for_assembler(assembler)
    flags_eg = _lib.FNE_ENERGY | _lib.FNE_GRAD
    e_buf = torch.empty(1, dtype=torch.float64, device=dev)
    g = torch.empty(assembler.n_owned, dtype=torch.float64, device=dev)
    x_trial = torch.empty_like(x)

    def energy_at(xv):
        val = float(assembler.eval(xv, _lib.FNE_ENERGY, energy=e_buf)[0].item())
        return val if math.isfinite(val) else math.inf

    t0 = time.perf_counter()
    assembler.eval(x, flags_eg, energy=e_buf, grad=g)
    fx = float(e_buf.item())
    g0 = None
    history = []
    message = "Maximum number of iterations reached"
    nit = 0
    for _ in range(maxit):
        if not math.isfinite(fx):
            message = "Non-finite energy"
            break
        assembler.eval(x, _lib.FNE_GRAD, grad=g)
        normg = float(torch.linalg.vector_norm(g))
        if not math.isfinite(normg):
            message = "Non-finite gradient norm"
            break
        if g0 is None:
            g0 = normg
        target = max(tolg, tolg_rel * g0)
        if normg < target:
            message = "Gradient norm converged"
            break
        nit += 1
        assembler.eval(x, _lib.FNE_HESS)
        cg.update(assembler.owned_values)
        p, ksp_its = cg.solve(-g, rtol=ksp_rtol, maxit=ksp_max_it)

        def f_alpha(alpha):
            torch.add(x, p, alpha=alpha, out=x_trial)
            return energy_at(x_trial)

        a, b, n_rep, _ = repair_linesearch_interval(f_alpha, *linesearch_interval, center=0.0, center_value=fx,
                                                    tol=linesearch_tol)
        alpha, n_ls = golden_section_search(f_alpha, a, b, linesearch_tol)
        f_new = f_alpha(alpha)
        accepted = math.isfinite(f_new) and f_new < fx
        dE = fx - f_new if accepted else 0.0
        if accepted:
            x.copy_(x_trial)
            fx = f_new
        history.append({"it": nit, "energy": fx, "grad_norm": normg, "alpha": alpha, "ksp_its": ksp_its,
                        "ls_evals": n_rep + n_ls + 1, "accepted": accepted})
        if verbose:
            print(f"it={nit} J={fx:.10g} |g|={normg:.3e} alpha={alpha:.4f} ksp={ksp_its}", flush=True)
        if not accepted:
            message = "Line search made no progress"
            break
        if tolf > 0.0 and abs(dE) < tolf:
            message = "Energy change converged"
            break
    assembler.eval(x, _lib.FNE_GRAD, grad=g)
    normg = float(torch.linalg.vector_norm(g))
    info = {"iterations": nit, "message": message, "energy": fx, "grad_norm": normg, "grad_norm0": g0,
            "converged": g0 is not None and normg < max(tolg, tolg_rel * g0) * (1.0 + 1e-12),
            "time_s": time.perf_counter() - t0, "history": history}
    if own_cg:
        cg.close()
    return x, info
