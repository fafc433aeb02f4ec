"""Plane-strain Mohr-Coulomb kernels (P2 / P4 slope) vs the CPU oracle, through the C ABI.

FP64 mode within 1e-12 relative (energies vs the sum of |element energy|,
gradient / Hessian vs the largest entry); FP32 mode within 2e-5.
"""

import numpy as np
import pytest
import torch

from oracle.assembler import OracleAssembler
from fenics_nonlinear_energies_b200 import _lib, meshes

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 2e-5


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).max(initial=0.0) / max(np.abs(b).max(initial=0.0), 1e-300)


def _pair(params, **kw):
    from fenics_nonlinear_energies_b200.assembler import SlopeStabilityCudaAssembler

    gpu = SlopeStabilityCudaAssembler(params, **kw)
    okw = {}
    params = dict(params)
    if kw.get("constitutive_mode") == "elastic":
        params["elastic"] = True
    ref = OracleAssembler("mc", params, block_size=2)
    return gpu, ref


def _abs_scale(ref, u):
    from oracle import energies

    v = ref.v_local(u)[ref.local.elems_local_np]
    e, _, _ = energies.element_derivatives("mc", v, ref.elem_data, ref.params, want_hessian=False)
    return float(np.abs(e).sum() + abs(ref.f_owned @ np.asarray(u)[: ref.f_owned.size]))


@pytest.mark.parametrize("variant", ["auto", "cuda_cores"])
@pytest.mark.parametrize("degree,level", [(2, 1), (4, 1), (2, 2)])
@pytest.mark.parametrize("scale", [0.0, 0.05])
def test_mc_fp64_matches_oracle(degree, level, scale, variant):
    """FP64 P2 / P4: the DMMA tensor-core kernel (automatic) and the CUDA-core
    kernel, both at the FP64 bar."""
    params = meshes.slope_problem(level=level, degree=degree, lam=1.2, with_elem_B=True)
    gpu, ref = _pair(params, kernel_variant=variant)
    u = scale * np.random.default_rng(degree + level).standard_normal(gpu.layout.n_free)
    e_ref, g_ref, h_ref = ref.all_in_one(u)
    e, g, h = gpu.eval(torch.as_tensor(u, device="cuda"), 7)
    assert abs(float(e.item()) - e_ref) <= 1e-12 * max(_abs_scale(ref, u), 1.0)
    assert _rel(g.cpu().numpy(), g_ref) <= 1e-12
    assert _rel(h.cpu().numpy(), h_ref) <= 1e-12
    assert gpu.info["kernel_variant"] == (9 if variant == "auto" else 5)


@pytest.mark.parametrize("degree", [2, 4])
def test_mc_fp64_dmma_path(degree):
    """The FP64 DMMA kernel against the FP64 CUDA-core kernel (same
    arithmetic up to summation order), bit-repeatable, with every flag
    combination (energy / gradient passes of the automatic path agree)."""
    params = meshes.slope_problem(level=2, degree=degree, lam=1.2, with_elem_B=True)
    gpu, ref = _pair(params)
    cc, _ = _pair(params, kernel_variant="cuda_cores")
    assert gpu.info["kernel_variant"] == 9 and cc.info["kernel_variant"] == 5
    u = 0.05 * np.random.default_rng(13).standard_normal(gpu.layout.n_free)
    ut = torch.as_tensor(u, device="cuda")
    e, g, h = [t.clone() for t in gpu.eval(ut, 7)]
    ec, gc, hc = [t.clone() for t in cc.eval(ut, 7)]
    assert _rel(h.cpu().numpy(), hc.cpu().numpy()) <= 1e-13
    assert _rel(g.cpu().numpy(), gc.cpu().numpy()) <= 1e-13
    assert abs(float(e.item()) - float(ec.item())) <= 1e-13 * _abs_scale(ref, u)
    e2, g2, h2 = gpu.eval(ut, 7)
    assert torch.equal(h, h2) and torch.equal(g, g2) and torch.equal(e, e2)
    # other flag sets are other template instances (the compiler may contract
    # multiply-adds differently): agreement to rounding
    for flags in (_lib.FNE_HESS, _lib.FNE_HESS | _lib.FNE_ENERGY, _lib.FNE_HESS | _lib.FNE_GRAD):
        ef, gf, hf = gpu.eval(ut, flags)
        assert _rel(hf.cpu().numpy(), h.cpu().numpy()) <= 1e-14
        if flags & _lib.FNE_GRAD:
            assert _rel(gf.cpu().numpy(), g.cpu().numpy()) <= 1e-14
        if flags & _lib.FNE_ENERGY:
            assert abs(float(ef.item()) - float(e.item())) <= 1e-14 * _abs_scale(ref, u)
    assert abs(float(gpu.eval(ut, _lib.FNE_ENERGY)[0].item()) - float(e.item())) <= 1e-13 * _abs_scale(ref, u)
    assert _rel(gpu.eval(ut, _lib.FNE_GRAD)[1].cpu().numpy(), g.cpu().numpy()) <= 1e-13


def test_mc_plastic_points_present():
    """The displacement scale used above drives part of the quadrature points plastic."""
    from oracle import energies

    params = meshes.slope_problem(level=1, degree=4, lam=1.2, with_elem_B=True)
    ref = OracleAssembler("mc", params, block_size=2)
    u = 0.05 * np.random.default_rng(5).standard_normal(ref.layout.n_free)
    v = ref.v_local(u)[ref.local.elems_local_np]
    strain = np.einsum("eqij,ej->eqi", ref.elem_data["elem_B"], v)
    el = energies.element_derivatives("mc", v, ref.elem_data, dict(params, elastic=True), want_hessian=False)[0]
    pl = energies.element_derivatives("mc", v, ref.elem_data, params, want_hessian=False)[0]
    assert np.mean(np.abs(el - pl) > 1e-12 * np.abs(el)) > 0.1
    assert strain.shape[1] == 19


def test_mc_fp32():
    params = meshes.slope_problem(level=1, degree=4, lam=1.2, with_elem_B=True)
    gpu, ref = _pair(params, precision="fp32", hess_dtype=torch.float32)
    u = 0.05 * np.random.default_rng(9).standard_normal(gpu.layout.n_free)
    e_ref, g_ref, h_ref = ref.all_in_one(u)
    e, g, h = gpu.eval(torch.as_tensor(u, device="cuda"), 7)
    assert h.dtype == torch.float32
    assert abs(float(e.item()) - e_ref) <= 1e-5 * _abs_scale(ref, u)
    assert _rel(g.cpu().numpy(), g_ref) <= 1e-4
    assert _rel(h.double().cpu().numpy(), h_ref) <= 2e-5


def test_elastic_tangent_equals_mc_tangent_at_zero():
    """tests/test_slope_stability_petsc.py:559-585 of the reference: at u = 0 the
    elastic and the Mohr-Coulomb tangents coincide."""
    params = meshes.slope_problem(level=2, degree=2, lam=1.0)
    from fenics_nonlinear_energies_b200.assembler import SlopeStabilityCudaAssembler

    mc = SlopeStabilityCudaAssembler(params)
    el = SlopeStabilityCudaAssembler(params, constitutive_mode="elastic")
    u = torch.zeros(mc.layout.n_free, dtype=torch.float64, device="cuda")
    h_mc = mc.eval(u, _lib.FNE_HESS)[2].clone()
    h_el = el.eval(u, _lib.FNE_HESS)[2].clone()
    np.testing.assert_array_equal(mc.layout.owned_rows, el.layout.owned_rows)
    assert torch.allclose(h_mc, h_el, rtol=1e-10, atol=0)


def test_mc_energy_only_and_repeatability():
    params = meshes.slope_problem(level=2, degree=4, lam=1.1)
    from fenics_nonlinear_energies_b200.assembler import SlopeStabilityCudaAssembler

    gpu = SlopeStabilityCudaAssembler(params)
    u = torch.as_tensor(0.03 * np.random.default_rng(1).standard_normal(gpu.layout.n_free), device="cuda")
    e1, g1, h1 = [t.clone() for t in gpu.eval(u, 7)]
    e2, g2, h2 = [t.clone() for t in gpu.eval(u, 7)]
    assert torch.equal(h1, h2) and torch.equal(g1, g2) and torch.equal(e1, e2)
    # the energy-only pass is the tiled energy / gradient kernel: same value
    # to rounding (other summation order)
    e_only = gpu.eval(u, _lib.FNE_ENERGY)[0].clone()
    assert abs(float(e_only.item()) - float(e1.item())) <= 1e-14 * max(1.0, abs(float(e1.item())))
    assert torch.equal(e_only, gpu.eval(u, _lib.FNE_ENERGY)[0])


@pytest.mark.parametrize("degree", [2, 4])
def test_mc_tensor_core_path(degree):
    """FP32 P2 / P4 runs the tcgen05 kernel (3xTF32 Bt.D.B): same FP32
    tolerances against the FP64 oracle, agreement with the CUDA-core FP32
    kernel, bit-repeatable, and the device status word stays clear."""
    params = meshes.slope_problem(level=2, degree=degree, lam=1.2, with_elem_B=True)
    gpu, ref = _pair(params, precision="fp32", hess_dtype=torch.float32)
    assert gpu.info["kernel_variant"] == 6
    cc, _ = _pair(params, precision="fp32", hess_dtype=torch.float32, kernel_variant="cuda_cores")
    assert cc.info["kernel_variant"] == 5
    np.testing.assert_array_equal(gpu.layout.owned_cols, cc.layout.owned_cols)
    u = 0.05 * np.random.default_rng(11).standard_normal(gpu.layout.n_free)
    e_ref, g_ref, h_ref = ref.all_in_one(u)
    ut = torch.as_tensor(u, device="cuda")
    e, g, h = [t.clone() for t in gpu.eval(ut, 7)]
    gpu.check_device_status()
    assert abs(float(e.item()) - e_ref) <= 1e-5 * _abs_scale(ref, u)
    assert _rel(g.cpu().numpy(), g_ref) <= 1e-4
    assert _rel(h.double().cpu().numpy(), h_ref) <= 2e-5
    e2, g2, h2 = gpu.eval(ut, 7)
    assert torch.equal(h, h2) and torch.equal(g, g2) and torch.equal(e, e2)
    ec, gc, hc = cc.eval(ut, 7)
    assert _rel(h.double().cpu().numpy(), hc.double().cpu().numpy()) <= 2e-5
    # energy-only and gradient-only passes use the CUDA-core kernel and agree
    assert abs(float(gpu.eval(ut, _lib.FNE_ENERGY)[0].item()) - float(e.item())) <= 1e-6 * _abs_scale(ref, u)
    gg = gpu.eval(ut, _lib.FNE_GRAD)[1]
    assert _rel(gg.cpu().numpy(), g.cpu().numpy()) <= 1e-5


def test_mc_tensor_core_hessian_only_and_plastic_mix():
    """Hessian-only pass through the tensor-core kernel at a state with
    elastic, line-return and apex points; ragged last tile (element count not
    a multiple of the tile)."""
    params = meshes.slope_problem(level=1, degree=4, lam=1.3, with_elem_B=True)
    gpu, ref = _pair(params, precision="fp32", hess_dtype=torch.float32)
    assert gpu.info["n_elem"] % 24 != 0
    u = 0.2 * np.random.default_rng(12).standard_normal(gpu.layout.n_free)
    _, _, h_ref = ref.all_in_one(u)
    h = gpu.eval(torch.as_tensor(u, device="cuda"), _lib.FNE_HESS)[2]
    gpu.check_device_status()
    assert _rel(h.double().cpu().numpy(), h_ref) <= 2e-5


@pytest.mark.parametrize("degree", [2, 4])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_matrix_free_products(degree, precision):
    """Matrix-free H(u) x and diag H(u) against the assembled owned COO values
    (FP64: 1e-12; FP32: 2e-5 relative to the largest entry), at a state with
    plastic points, and against central differences of the oracle gradient."""
    from scipy import sparse

    params = meshes.slope_problem(level=2, degree=degree, lam=1.2, with_elem_B=True)
    hd = torch.float32 if precision == "fp32" else torch.float64
    gpu, ref = _pair(params, precision=precision, hess_dtype=hd)
    u = 0.05 * np.random.default_rng(21).standard_normal(gpu.layout.n_free)
    ut = torch.as_tensor(u, device="cuda")
    h = gpu.eval(ut, _lib.FNE_HESS)[2].double().cpu().numpy()
    A = sparse.coo_matrix((h, (gpu.layout.owned_rows, gpu.layout.owned_cols)),
                          shape=(gpu.layout.n_free,) * 2).tocsr()
    gpu.prepare_matrix_free_operator(ut, mode="matfree_element")
    tol = 1e-12 if precision == "fp64" else 2e-5
    for seed in (0, 1):
        x = np.random.default_rng(seed).standard_normal(gpu.layout.n_free)
        y = gpu.matrix_free_mult("matfree_element", torch.as_tensor(x, device="cuda")).cpu().numpy()
        y_ref = A @ x
        assert np.abs(y - y_ref).max() <= tol * np.abs(y_ref).max()
    d = gpu.matrix_free_get_diagonal("matfree_element").cpu().numpy()
    assert np.abs(d - A.diagonal()).max() <= tol * np.abs(A.diagonal()).max()
    # repeat calls are bit-identical (fixed summation order)
    y2 = gpu.matrix_free_mult("matfree_element", torch.as_tensor(x, device="cuda")).cpu().numpy()
    assert np.array_equal(y, y2)
    if precision == "fp64":
        hstep = 1e-6
        fd = (ref.gradient_fn(u + hstep * x) - ref.gradient_fn(u - hstep * x)) / (2 * hstep)
        assert np.abs(y - fd).max() <= 1e-4 * np.abs(fd).max()


def test_matrix_free_requires_prepare():
    from fenics_nonlinear_energies_b200._lib import FneError

    params = meshes.slope_problem(level=1, degree=2, lam=1.0)
    from fenics_nonlinear_energies_b200.assembler import SlopeStabilityCudaAssembler

    gpu = SlopeStabilityCudaAssembler(params)
    x = torch.zeros(gpu.layout.n_free, dtype=torch.float64, device="cuda")
    with pytest.raises(RuntimeError):
        gpu.matrix_free_mult("matfree_element", x)
    out = torch.empty(max(1, gpu.n_owned), dtype=torch.float64, device="cuda")
    with pytest.raises(FneError):
        _lib.check(_lib.lib.fne_hvp(gpu._handle, x.data_ptr(), out.data_ptr(), None))


@pytest.mark.parametrize("degree", [2, 4])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_mc_nonzero_previous_plastic_strain(degree, precision):
    """A non-zero eps_p_old (strain = B u - eps_p_old at every quadrature
    point) through the CUDA-core FP64 kernel, the tensor-core FP32 kernel and
    the matrix-free product, against the oracle."""
    from scipy import sparse

    params = meshes.slope_problem(level=1, degree=degree, lam=1.2, with_elem_B=True)
    rng = np.random.default_rng(41)
    params["eps_p_old"] = 2e-4 * rng.standard_normal(params["eps_p_old"].shape)
    hd = torch.float32 if precision == "fp32" else torch.float64
    gpu, ref = _pair(params, precision=precision, hess_dtype=hd)
    assert gpu.info["kernel_variant"] == (6 if precision == "fp32" else 9)
    u = 0.03 * rng.standard_normal(gpu.layout.n_free)
    e_ref, g_ref, h_ref = ref.all_in_one(u)
    ut = torch.as_tensor(u, device="cuda")
    e, g, h = gpu.eval(ut, 7)
    tol = FP64_TOL if precision == "fp64" else FP32_TOL
    etol = 1e-12 if precision == "fp64" else 1e-5
    assert abs(float(e.item()) - e_ref) <= etol * _abs_scale(ref, u)
    assert _rel(g.cpu().numpy(), g_ref) <= (tol if precision == "fp64" else 1e-4)
    assert _rel(h.double().cpu().numpy(), h_ref) <= tol
    gpu.prepare_matrix_free_operator(ut)
    x = rng.standard_normal(gpu.layout.n_free)
    A = sparse.coo_matrix((h_ref, (gpu.layout.owned_rows, gpu.layout.owned_cols)),
                          shape=(gpu.layout.n_free,) * 2).tocsr()
    y = gpu.matrix_free_mult("matfree_element", torch.as_tensor(x, device="cuda")).cpu().numpy()
    assert np.abs(y - A @ x).max() <= tol * np.abs(A @ x).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("degree", [1, 2, 4])
def test_mc_energy_gradient_kernel(degree, precision):
    """Energy-only, gradient-only and energy + gradient calls (the tiled
    energy / gradient kernel) against the oracle, against the CUDA-core
    kernel, with a non-zero previous plastic strain, bit-repeatable."""
    params = meshes.slope_problem(level=1, degree=degree, lam=1.2, with_elem_B=True)
    rng = np.random.default_rng(17 + degree)
    params["eps_p_old"] = 1e-4 * rng.standard_normal(params["eps_p_old"].shape)
    hd = torch.float32 if precision == "fp32" else torch.float64
    gpu, ref = _pair(params, precision=precision, hess_dtype=hd)
    cc, _ = _pair(params, precision=precision, hess_dtype=hd, kernel_variant="cuda_cores")
    u = 0.04 * rng.standard_normal(gpu.layout.n_free)
    ut = torch.as_tensor(u, device="cuda")
    e_ref, g_ref, _ = ref.all_in_one(u)
    scale = _abs_scale(ref, u)
    etol, gtol = (1e-12, 1e-12) if precision == "fp64" else (1e-5, 1e-4)
    e1 = float(gpu.eval(ut, _lib.FNE_ENERGY)[0].item())
    g2 = gpu.eval(ut, _lib.FNE_GRAD)[1].clone()
    e3, g3, _ = gpu.eval(ut, _lib.FNE_ENERGY | _lib.FNE_GRAD)
    assert abs(e1 - e_ref) <= etol * scale and abs(float(e3.item()) - e_ref) <= etol * scale
    assert _rel(g2.cpu().numpy(), g_ref) <= gtol and _rel(g3.cpu().numpy(), g_ref) <= gtol
    ec = float(cc.eval(ut, _lib.FNE_ENERGY)[0].item())
    gc = cc.eval(ut, _lib.FNE_GRAD)[1]
    ctol = 1e-13 if precision == "fp64" else 1e-5
    assert abs(e1 - ec) <= ctol * scale
    assert _rel(g2.cpu().numpy(), gc.cpu().numpy()) <= ctol
    assert torch.equal(gpu.eval(ut, _lib.FNE_GRAD)[1], g2)
    assert float(gpu.eval(ut, _lib.FNE_ENERGY)[0].item()) == e1


def test_tensor_core_wait_timeout_is_reported():
    """The tcgen05 kernel's MMA-completion wait, set to give up at once
    (fne_set_wait_limit 0): the pass returns, the status word reports
    FNE_ETIMEOUT (polled without a sync by the callbacks, or read
    synchronously), and with the default bound restored the same handle
    gives correct values again (the context stayed usable)."""
    params = meshes.slope_problem(level=1, degree=2, lam=1.2, with_elem_B=True)
    gpu, ref = _pair(params, precision="fp32", hess_dtype=torch.float32)
    assert gpu.info["kernel_variant"] == 6
    u = 0.05 * np.random.default_rng(3).standard_normal(gpu.layout.n_free)
    ut = torch.as_tensor(u, device="cuda")
    _lib.check(_lib.lib.fne_set_wait_limit(gpu._handle, 0))
    gpu.eval(ut, 7)
    torch.cuda.synchronize()
    assert _lib.lib.fne_check_device_status(gpu._handle) == _lib.FNE_ETIMEOUT
    assert _lib.lib.fne_check_device_status(gpu._handle) == _lib.FNE_OK  # cleared
    with pytest.raises(_lib.FneError) as err:
        gpu.assemble_hessian(u)
    assert err.value.code == _lib.FNE_ETIMEOUT
    _lib.check(_lib.lib.fne_set_wait_limit(gpu._handle, -1))
    _, _, h_ref = ref.all_in_one(u)
    gpu.assemble_hessian(u)  # no error now
    assert _rel(gpu.owned_values.double().cpu().numpy(), h_ref) <= FP32_TOL
    gpu.check_device_status()
