"""Device CG (``fne_cg_*``) against the scalar CG oracle (``oracle/krylov.py``).

Same iteration count and stop reason, the same iterate to 1e-9 relative
(FP64 arithmetic, different summation order), on shuffled COO patterns with
FP64 and FP32 value storage; the stopping rules at the edges (first-iteration
negative curvature, later negative curvature, iteration limits that are not
a multiple of the graph length, zero right-hand side, missing and zero
diagonals); bitwise reproducibility and independence of the graph length;
and the Hessians the assemblers produce.
"""

import numpy as np
import pytest
import torch

from oracle import krylov
from oracle.assembler import OracleAssembler
from fenics_nonlinear_energies_b200 import meshes

pytestmark = pytest.mark.gpu


def _laplacian_coo(m, shift, seed, drop_diag=()):
    """Symmetric 5-point pattern on an m x m grid, random symmetric values, shuffled COO order."""
    rng = np.random.default_rng(seed)
    idx = np.arange(m * m).reshape(m, m)
    rows, cols = [idx.ravel()], [idx.ravel()]
    for a, b in ((idx[:, :-1], idx[:, 1:]), (idx[:-1, :], idx[1:, :])):
        rows += [a.ravel(), b.ravel()]
        cols += [b.ravel(), a.ravel()]
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    off = rows != cols
    w = np.zeros(rows.size)
    key = np.minimum(rows, cols) * (m * m) + np.maximum(rows, cols)
    _, inv = np.unique(key, return_inverse=True)
    w_sym = -(0.5 + rng.random(inv.max() + 1))
    w[off] = w_sym[inv[off]]
    diag = np.zeros(m * m)
    np.add.at(diag, rows[off], -w[off])
    w[~off] = diag[rows[~off]] + shift[rows[~off]] if np.ndim(shift) else diag[rows[~off]] + shift
    keep = ~np.isin(np.where(~off, rows, -1), np.asarray(drop_diag, dtype=np.int64))
    rows, cols, w = rows[keep], cols[keep], w[keep]
    order = rng.permutation(rows.size)
    return m * m, rows[order], cols[order], w[order]


def _dense(n, rows, cols, vals):
    A = np.zeros((n, n))
    np.add.at(A, (rows, cols), vals)
    return A


def _solve_both(n, rows, cols, vals, b, rtol, maxit, fp32=False, chunk=16):
    from fenics_nonlinear_energies_b200.newton import DeviceCG

    v = vals.astype(np.float32).astype(np.float64) if fp32 else vals
    A = _dense(n, rows, cols, v)
    diag = np.full(n, np.nan)
    on = rows == cols
    diag[rows[on]] = v[on]
    x_ref, it_ref, why_ref = krylov.pcg(A, krylov.jacobi_scaling(diag), b, rtol, maxit)
    cg = DeviceCG(n, rows, cols, fp32=fp32, chunk=chunk)
    cg.update(torch.as_tensor(vals, dtype=torch.float32 if fp32 else torch.float64, device="cuda"))
    x, it = cg.solve(torch.as_tensor(b, device="cuda"), rtol=rtol, maxit=maxit)
    why = cg.REASONS.index(cg.reason)
    cg.close()
    return x.cpu().numpy(), it, why, x_ref, it_ref, why_ref


@pytest.mark.parametrize("fp32", [False, True])
@pytest.mark.parametrize("m", [3, 40, 130])
def test_cg_spd_matches_oracle(m, fp32):
    n, rows, cols, vals = _laplacian_coo(m, 0.05, seed=m)
    b = np.random.default_rng(m + 1).standard_normal(n)
    x, it, why, x_ref, it_ref, why_ref = _solve_both(n, rows, cols, vals, b, 1e-8, 2000, fp32=fp32)
    assert (it, why) == (it_ref, why_ref) == (it_ref, krylov.CONVERGED)
    np.testing.assert_allclose(x, x_ref, rtol=0, atol=1e-9 * np.abs(x_ref).max())


def test_cg_negative_curvature_first_and_later():
    n, rows, cols, vals = _laplacian_coo(30, -1e6, seed=3)   # negative definite
    b = np.random.default_rng(4).standard_normal(n)
    x, it, why, x_ref, it_ref, why_ref = _solve_both(n, rows, cols, vals, b, 1e-10, 500)
    assert (it, why) == (it_ref, why_ref) == (1, krylov.NEGATIVE_CURVATURE)
    assert np.array_equal(x, b)
    shift = np.full(n, 0.02)
    shift[:5] = -3.0                                          # a few negative modes
    n, rows, cols, vals = _laplacian_coo(30, shift, seed=5)
    x, it, why, x_ref, it_ref, why_ref = _solve_both(n, rows, cols, vals, b, 1e-12, 500)
    assert (it, why) == (it_ref, why_ref) and why == krylov.NEGATIVE_CURVATURE and it > 1
    np.testing.assert_allclose(x, x_ref, rtol=0, atol=1e-9 * np.abs(x_ref).max())


@pytest.mark.parametrize("maxit,chunk", [(0, 16), (1, 16), (7, 16), (37, 16), (37, 3), (16, 16), (17, 1)])
def test_cg_iteration_limit(maxit, chunk):
    n, rows, cols, vals = _laplacian_coo(50, 1e-3, seed=6)
    b = np.random.default_rng(7).standard_normal(n)
    x, it, why, x_ref, it_ref, why_ref = _solve_both(n, rows, cols, vals, b, 1e-14, maxit, chunk=chunk)
    assert (it, why) == (it_ref, why_ref) == (maxit, krylov.ITERATION_LIMIT)
    np.testing.assert_allclose(x, x_ref, rtol=0, atol=1e-9 * max(1.0, np.abs(x_ref).max()))


def test_cg_zero_rhs_and_diagonal_edge_cases():
    n, rows, cols, vals = _laplacian_coo(20, 0.1, seed=8)
    x, it, why, *_ = _solve_both(n, rows, cols, vals, np.zeros(n), 1e-8, 100)
    assert (it, why) == (0, krylov.ZERO_RHS) and not x.any()
    # a missing diagonal entry and a zero one: Jacobi scale 1 there
    n, rows, cols, vals = _laplacian_coo(20, 0.1, seed=9, drop_diag=[3])
    vals = vals.copy()
    vals[(rows == 7) & (cols == 7)] = 0.0
    b = np.random.default_rng(10).standard_normal(n)
    x, it, why, x_ref, it_ref, why_ref = _solve_both(n, rows, cols, vals, b, 1e-8, 1000)
    assert (it, why) == (it_ref, why_ref)
    np.testing.assert_allclose(x, x_ref, rtol=0, atol=1e-8 * np.abs(x_ref).max())


def test_cg_reproducible_and_chunk_independent():
    from fenics_nonlinear_energies_b200.newton import DeviceCG

    n, rows, cols, vals = _laplacian_coo(90, 0.01, seed=11)
    b = torch.as_tensor(np.random.default_rng(12).standard_normal(n), device="cuda")
    v = torch.as_tensor(vals, device="cuda")
    outs = []
    for chunk in (16, 16, 5, 1):
        cg = DeviceCG(n, rows, cols, chunk=chunk)
        cg.update(v)
        outs.append(cg.solve(b, rtol=1e-9, maxit=3000))
        # the same handle again, with another right-hand side in between
        cg.solve(2.0 * b, rtol=1e-3, maxit=3000)
        outs.append(cg.solve(b, rtol=1e-9, maxit=3000))
        cg.close()
    for x, it in outs[1:]:
        assert it == outs[0][1] and torch.equal(x, outs[0][0])


@pytest.mark.parametrize("family", ["gl", "he"])
def test_cg_on_assembled_hessian(family):
    from fenics_nonlinear_energies_b200 import _lib
    from fenics_nonlinear_energies_b200.assembler import GLCudaAssembler, HECudaAssembler
    from fenics_nonlinear_energies_b200.newton import DeviceCG

    if family == "gl":
        params, u = meshes.gl_problem(n=48, seed=1)
        asm, ref = GLCudaAssembler(params), OracleAssembler("gl", params)
    else:
        params, u = meshes.he_beam_problem(nx=12, ny=3, nz=3)
        u = u + 1e-3 * np.random.default_rng(2).standard_normal(u.size)
        asm = HECudaAssembler(params)
        ref = OracleAssembler("he", params, block_size=3, coordinate_key="nodes2coord", dirichlet_key="u_0_ref")
    ud = torch.as_tensor(u, device="cuda")
    _, g, _ = asm.eval(ud, _lib.FNE_GRAD | _lib.FNE_HESS)
    lay = asm.layout
    rows = np.asarray(lay.owned_rows) - lay.lo
    cols = np.asarray(lay.owned_cols)
    hv = asm.owned_values.double().cpu().numpy()
    A = _dense(asm.n_owned, rows, cols, hv)
    x_ref, it_ref, why_ref = krylov.pcg(A, krylov.jacobi_scaling(np.diag(A)), -g.cpu().numpy(), 1e-6, 1000)
    cg = DeviceCG.for_assembler(asm)
    cg.update(asm.owned_values)
    x, it = cg.solve(-g, rtol=1e-6, maxit=1000)
    assert it == it_ref and cg.REASONS.index(cg.reason) == why_ref
    np.testing.assert_allclose(x.cpu().numpy(), x_ref, rtol=0, atol=1e-8 * np.abs(x_ref).max())
    cg.close()
    asm.cleanup()
    del ref
