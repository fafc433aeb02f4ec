"""CUDA kernels vs the CPU oracle, through the C ABI (libfne_asm.so).

Tolerances: FP64 mode within 1e-12 relative (energies: relative to the sum
of absolute element energies; gradient / Hessian: relative to the largest
entry); FP32 mode within 2e-5 relative for gradient / Hessian and 1e-7 for the
FP64-reduced energy.
"""

import numpy as np
import pytest
import torch

from oracle.assembler import OracleAssembler
from fenics_nonlinear_energies_b200 import _lib, meshes

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32_TOL = 2e-5


def _asm_classes():
    from fenics_nonlinear_energies_b200.assembler import GLCudaAssembler, HECudaAssembler, PLaplaceCudaAssembler

    return {"plaplace": PLaplaceCudaAssembler, "gl": GLCudaAssembler, "he": HECudaAssembler}


def _make(family, params, **kw):
    cls = _asm_classes()[family]
    bs = 3 if family == "he" else 1
    okw = dict(block_size=bs)
    if family == "he":
        okw.update(coordinate_key="nodes2coord", dirichlet_key="u_0_ref")
    return cls(params, **kw), OracleAssembler(family, params, **okw)


def _rel(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(initial=0.0), 1e-300)
    return np.abs(a - b).max(initial=0.0) / scale


def _check(gpu, ref, u, tol, *, energy_scale=None):
    e_ref, g_ref, h_ref = ref.all_in_one(u)
    ut = torch.as_tensor(u, device="cuda")
    e, g, h = gpu.eval(ut, _lib.FNE_ENERGY | _lib.FNE_GRAD | _lib.FNE_HESS)
    torch.cuda.synchronize()
    scale = energy_scale if energy_scale is not None else max(abs(e_ref), 1.0)
    assert abs(float(e.item()) - e_ref) <= tol * scale, (float(e.item()), e_ref)
    assert _rel(g.cpu().numpy()[: gpu.n_owned], g_ref) <= tol
    assert _rel(h.double().cpu().numpy(), h_ref) <= tol
    # the separate callbacks agree with the fused pass
    assert abs(gpu.energy_fn(u) - e_ref) <= tol * scale
    gg = np.zeros(gpu.n_owned)
    gpu.gradient_fn(u, gg)
    assert _rel(gg, g_ref) <= tol
    gpu.assemble_hessian(u)
    assert _rel(gpu.owned_values.double().cpu().numpy(), h_ref) <= tol


def _abs_energy_scale(ref, u):
    """sum_e |e_e|: the natural scale of a sum of element energies."""
    from oracle import energies

    v = ref.v_local(u)[ref.local.elems_local_np]
    e, _, _ = energies.element_derivatives(ref.family, v, ref.elem_data, ref.params, want_hessian=False)
    return float(np.abs(e).sum() + np.abs(ref.f_owned @ np.asarray(u)[: ref.f_owned.size]) + 1e-300)


@pytest.mark.parametrize("variant", ["auto", "cluster", "row_gather", "incidence", "push"])
@pytest.mark.parametrize("numbering", ["x_slow", "x_fast"])
def test_plaplace_fp64(numbering, variant):
    params, _ = meshes.plaplace_problem(n=40, numbering=numbering)
    gpu, ref = _make("plaplace", params, kernel_variant=variant)
    u = np.random.default_rng(0).random(gpu.layout.n_free)
    _check(gpu, ref, u, FP64_TOL, energy_scale=_abs_energy_scale(ref, u))


def test_plaplace_zero_initial_guess():
    params, _ = meshes.plaplace_problem(n=8)
    gpu, ref = _make("plaplace", params)
    u = np.zeros(gpu.layout.n_free)
    _check(gpu, ref, u, FP64_TOL)
    assert torch.all(gpu.owned_values == 0)


@pytest.mark.parametrize("variant", ["auto", "cluster", "row_gather", "incidence", "push"])
@pytest.mark.parametrize("numbering", ["x_slow", "x_fast"])
def test_gl_fp64(numbering, variant):
    params, u0 = meshes.gl_problem(n=16, seed=3, numbering=numbering)
    gpu, ref = _make("gl", params, kernel_variant=variant)
    _check(gpu, ref, u0, FP64_TOL, energy_scale=_abs_energy_scale(ref, u0))


@pytest.mark.parametrize("variant", ["auto", "cluster", "row_gather", "incidence", "push"])
def test_gl_fp32(variant):
    params, u0 = meshes.gl_problem(n=40, seed=4)
    gpu, ref = _make("gl", params, precision="fp32", hess_dtype=torch.float32, kernel_variant=variant)
    e_ref, g_ref, h_ref = ref.all_in_one(u0)
    e, g, h = gpu.eval(torch.as_tensor(u0, device="cuda"), 7)
    assert h.dtype == torch.float32
    assert abs(float(e.item()) - e_ref) <= 1e-7 * _abs_energy_scale(ref, u0)
    assert _rel(g.cpu().numpy(), g_ref) <= FP32_TOL
    assert _rel(h.double().cpu().numpy(), h_ref) <= FP32_TOL


def test_he_fp64():
    params, y0 = meshes.he_beam_problem(nx=8, ny=2, nz=2)
    gpu, ref = _make("he", params)
    rng = np.random.default_rng(5)
    u = y0 + 2e-3 * rng.standard_normal(y0.size)
    _check(gpu, ref, u, FP64_TOL, energy_scale=_abs_energy_scale(ref, u))


def test_he_rotated_boundary_fp64_and_fp32():
    params, y0 = meshes.he_beam_problem(nx=8, ny=2, nz=2)
    gpu, ref = _make("he", params)
    gpu32 = _asm_classes()["he"](params, precision="fp32")
    u0 = meshes.rotate_right_face_from_reference(params["u_0_ref"], params["nodes2coord"], 0.3,
                                                 params["right_nodes"])
    for a in (gpu, ref, gpu32):
        a.update_dirichlet(u0)
    u = y0 + 1e-3 * np.random.default_rng(6).standard_normal(y0.size)
    _check(gpu, ref, u, FP64_TOL, energy_scale=_abs_energy_scale(ref, u))
    e_ref, g_ref, h_ref = ref.all_in_one(u)
    e, g, h = gpu32.eval(torch.as_tensor(u, device="cuda"), 7)
    assert _rel(g.cpu().numpy(), g_ref) <= 1e-4
    assert _rel(h.cpu().numpy(), h_ref) <= FP32_TOL


def test_he_inverted_element_gives_nonfinite_energy():
    params, y0 = meshes.he_beam_problem(nx=4, ny=1, nz=1)
    gpu, ref = _make("he", params)
    u = y0.copy()
    u[0::3] *= -1.0  # mirror x of free nodes -> negative det F somewhere
    e = gpu.energy_fn(u)
    assert not np.isfinite(e) or np.isfinite(ref.energy_fn(u))
    assert np.isnan(e) == np.isnan(ref.energy_fn(u))


def test_gl_dirichlet_only_energy_constant():
    params, u0 = meshes.gl_problem(n=8)
    gpu, ref = _make("gl", params)
    assert ref.dirichlet_only_energy > 0
    assert abs(gpu.energy_fn(u0) - ref.energy_fn(u0)) < 1e-12 * _abs_energy_scale(ref, u0)


def test_deterministic_and_energy_paths_agree():
    params, u0 = meshes.gl_problem(n=64, seed=9)
    gpu, _ = _make("gl", params, precision="fp32", hess_dtype=torch.float32)
    ut = torch.as_tensor(u0, device="cuda")
    e1, g1, h1 = [t.clone() for t in gpu.eval(ut, 7)]
    e2, g2, h2 = [t.clone() for t in gpu.eval(ut, 7)]
    assert torch.equal(h1, h2) and torch.equal(g1, g2) and torch.equal(e1, e2)
    e_only = gpu.eval(ut, _lib.FNE_ENERGY)[0].clone()
    # the fused pass sums FP32 element energies in FP64; the energy-only pass is FP64 throughout
    assert abs(float(e_only.item()) - float(e1.item())) < 1e-6 * abs(float(e1.item()))


def test_autograd_energy_function():
    from fenics_nonlinear_energies_b200.assembler import energy

    params, u0 = meshes.gl_problem(n=16, seed=2)
    gpu, ref = _make("gl", params)
    u = torch.as_tensor(u0, device="cuda").requires_grad_(True)
    J = energy(u, gpu)
    J.backward()
    np.testing.assert_allclose(u.grad.cpu().numpy(), ref.gradient_fn(u0), rtol=0, atol=1e-12 * np.abs(ref.gradient_fn(u0)).max())


def test_autograd_energy_function_rank_split():
    """Two ranks' EnergyFunction gradients are shaped like u and sum to dJ/du."""
    from types import SimpleNamespace

    from fenics_nonlinear_energies_b200.assembler import GLCudaAssembler, energy

    params, u0 = meshes.gl_problem(n=24, seed=3)
    ref = OracleAssembler("gl", params)
    total = np.zeros_like(u0)
    for r in range(2):
        gpu = GLCudaAssembler(params, SimpleNamespace(rank=r, size=2))
        u = torch.as_tensor(u0, device="cuda").requires_grad_(True)
        energy(u, gpu).backward()
        assert u.grad.shape == u.shape
        total += u.grad.cpu().numpy()
    g_ref = ref.gradient_fn(u0)
    np.testing.assert_allclose(total, g_ref, rtol=0, atol=1e-12 * np.abs(g_ref).max())


def test_empty_and_tiny_meshes():
    # 1x1 grid: no free DOF at all; 2x2 grid: a single free node
    for n in (1, 2):
        params, u0 = meshes.gl_problem(n=n)
        gpu, ref = _make("gl", params)
        e, g, h = gpu.eval(torch.as_tensor(u0, device="cuda"), 7) if gpu.layout.n_free else (None, None, None)
        assert abs(gpu.energy_fn(u0) - ref.energy_fn(u0)) < 1e-14
        if gpu.layout.n_free:
            assert _rel(h.cpu().numpy(), ref.assemble_hessian_element(u0)) <= FP64_TOL


def test_full_size_gl_properties():
    """1024 x 1024 GL, FP32 Hessian: FP64 energy vs the oracle's closed form,
    directional-derivative consistency and Hessian symmetry."""
    from scipy import sparse

    params, u0 = meshes.gl_problem(n=1024, seed=0)
    gpu = _asm_classes()["gl"](params, precision="fp32", hess_dtype=torch.float32)
    ut = torch.as_tensor(u0, device="cuda")
    e, g, h = [t.clone() for t in gpu.eval(ut, 7)]
    # energy: vectorised FP64 closed form of the restated density
    v = np.zeros(len(params["u_0"]))
    v[params["freedofs"]] = u0
    ve = v[params["elems"]]
    fx = np.sum(ve * params["dvx"], 1)
    fy = np.sum(ve * params["dvy"], 1)
    n = ve @ params["ip"]
    dens = 0.5 * params["eps"] * (fx**2 + fy**2) + (0.25 * (n**2 - 1.0) ** 2) @ params["w"]
    e_ref = float(np.sum(dens * params["vol"]))
    assert abs(float(e.item()) - e_ref) <= 1e-7 * float(np.sum(np.abs(dens * params["vol"])))
    # directional derivative of the FP64 energy vs the FP32 gradient
    d = torch.as_tensor(np.random.default_rng(1).standard_normal(u0.size), device="cuda")
    hstep = 1e-4
    ep = float(gpu.eval(ut + hstep * d, 1)[0].item())
    em = float(gpu.eval(ut - hstep * d, 1)[0].item())
    assert abs((ep - em) / (2 * hstep) - float(g @ d)) <= 1e-4 * abs(float(g @ d))
    # Hessian symmetry
    rows, cols = gpu.layout.owned_rows, gpu.layout.owned_cols
    A = sparse.coo_matrix((h.double().cpu().numpy(), (rows, cols)), shape=(gpu.layout.n_free,) * 2).tocsr()
    assert abs(A - A.T).max() <= 1e-6 * abs(A).max()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_he_element_pass_matches_row_gather(precision):
    """The element-parallel tet pass (opt-in) and the row-gather kernel
    (default) give the same values (FP64: 1e-12; FP32: 2e-5), bit-repeatably."""
    params, y0 = meshes.he_beam_problem(nx=6, ny=3, nz=2)
    cls = _asm_classes()["he"]
    hd = torch.float32 if precision == "fp32" else torch.float64
    a = cls(params, precision=precision, hess_dtype=hd, kernel_variant="element")
    b = cls(params, precision=precision, hess_dtype=hd)
    assert a.info["kernel_variant"] == 7 and b.info["kernel_variant"] == 2
    u = torch.as_tensor(y0 + 1e-3 * np.random.default_rng(8).standard_normal(y0.size), device="cuda")
    ea, ga, ha = [t.clone() for t in a.eval(u, 7)]
    eb, gb, hb = [t.clone() for t in b.eval(u, 7)]
    tol = FP64_TOL if precision == "fp64" else FP32_TOL
    assert abs(float(ea.item()) - float(eb.item())) <= 1e-12 * abs(float(eb.item()))
    assert _rel(ga.cpu().numpy(), gb.cpu().numpy()) <= tol
    assert _rel(ha.double().cpu().numpy(), hb.double().cpu().numpy()) <= tol
    ea2, ga2, ha2 = a.eval(u, 7)
    assert torch.equal(ha, ha2) and torch.equal(ga, ga2) and torch.equal(ea, ea2)
    # gradient-only and Hessian-only passes agree with the fused one
    assert torch.equal(a.eval(u, _lib.FNE_GRAD)[1], ga)
    assert torch.equal(a.eval(u, _lib.FNE_HESS)[2], ha)


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("variant", ["row_gather", "row_lanes_2", "row_lanes_4", "row_lanes_8"])
def test_he_row_lanes(variant, precision):
    """The tet row kernel with 1, 2, 4 or 8 lanes per output row (each lane
    its own shared-memory slice, summed in lane order) against the oracle,
    bit-repeatable; the automatic choice gives a small beam several lanes."""
    params, y0 = meshes.he_beam_problem(nx=10, ny=3, nz=3)
    hd = torch.float32 if precision == "fp32" else torch.float64
    gpu, ref = _make("he", params, precision=precision, hess_dtype=hd, kernel_variant=variant)
    lanes = {"row_gather": 1, "row_lanes_2": 2, "row_lanes_4": 4, "row_lanes_8": 8}[variant]
    assert gpu.info["kernel_variant"] == 2 and gpu.info["row_lanes"] == lanes
    u = y0 + 1e-3 * np.random.default_rng(12).standard_normal(y0.size)
    ut = torch.as_tensor(u, device="cuda")
    if precision == "fp64":
        _check(gpu, ref, u, FP64_TOL, energy_scale=_abs_energy_scale(ref, u))
    else:
        e_ref, g_ref, h_ref = ref.all_in_one(u)
        e, g, h = gpu.eval(ut, 7)
        assert abs(float(e.item()) - e_ref) <= 1e-6 * _abs_energy_scale(ref, u)
        assert _rel(g.cpu().numpy(), g_ref) <= 1e-4
        assert _rel(h.double().cpu().numpy(), h_ref) <= FP32_TOL
    e1, g1, h1 = [t.clone() for t in gpu.eval(ut, 7)]
    e2, g2, h2 = gpu.eval(ut, 7)
    assert torch.equal(h1, h2) and torch.equal(g1, g2) and torch.equal(e1, e2)
    auto, _ = _make("he", params, precision=precision, hess_dtype=hd)
    assert auto.info["row_lanes"] == 8  # 1,000-odd rows: far below 1024 row lanes per SM


@pytest.mark.parametrize("family", ["plaplace", "gl", "he", "mc"])
@pytest.mark.parametrize("size", [2, 3])
def test_rank_split_matches_oracle(family, size):
    """Each rank of a size-way split (owned rows [lo, hi), overlap elements,
    0/1 energy weights, rank-0-only constants) against the oracle of the same
    rank: FP64 within 1e-12; the rank energies sum to the one-rank energy."""
    from types import SimpleNamespace

    from fenics_nonlinear_energies_b200.assembler import SlopeStabilityCudaAssembler

    if family == "mc":
        params = meshes.slope_problem(level=2, degree=2, lam=1.2, with_elem_B=True)
        u = 0.05 * np.random.default_rng(31).standard_normal(int(np.asarray(params["freedofs"]).size))
        make_gpu = lambda comm: SlopeStabilityCudaAssembler(params, comm)  # noqa: E731
        okw = dict(block_size=2)
    else:
        if family == "plaplace":
            params, _ = meshes.plaplace_problem(n=20)
        elif family == "gl":
            params, _ = meshes.gl_problem(n=20, seed=5)
        else:
            params, _ = meshes.he_beam_problem(nx=8, ny=2, nz=2)
        cls = _asm_classes()[family]
        make_gpu = lambda comm: cls(params, comm)  # noqa: E731
        okw = dict(block_size=3, coordinate_key="nodes2coord", dirichlet_key="u_0_ref") if family == "he" else {}
        n_free = int(np.asarray(params["freedofs"]).size)
        rng = np.random.default_rng(32)
        if family == "he":
            y0 = np.asarray(params["u_0_ref"])[params["freedofs"]]
            u = y0 + 1e-3 * rng.standard_normal(n_free)
        else:
            u = rng.uniform(-0.5, 0.5, n_free)
    fam = "mc" if family == "mc" else family
    total = 0.0
    for r in range(size):
        gpu = make_gpu(SimpleNamespace(rank=r, size=size))
        ref = OracleAssembler(fam, params, rank=r, size=size, **okw)
        ur = u[np.asarray(gpu.layout.perm)] if family != "he" else u
        np.testing.assert_array_equal(gpu.layout.owned_rows, ref.layout.owned_rows)
        e_ref, g_ref, h_ref = ref.all_in_one(ur)
        e, g, h = gpu.eval(torch.as_tensor(ur, device="cuda"), 7)
        scale = max(1.0, abs(e_ref))
        assert abs(float(e.item()) - e_ref) <= 1e-12 * scale * 10
        if g_ref.size:
            assert _rel(g.cpu().numpy()[: gpu.n_owned], g_ref) <= FP64_TOL
        if h_ref.size:
            assert _rel(h.cpu().numpy(), h_ref) <= FP64_TOL
        total += float(e.item())
    one = OracleAssembler(fam, params, **okw)
    u1 = u[np.asarray(one.layout.perm)] if family != "he" else u
    e1 = one.all_in_one(u1)[0]
    assert abs(total - e1) <= 1e-11 * max(1.0, abs(e1))


def test_cluster_kernel_copy_wait_timeout_is_reported():
    """The row-cluster kernel's (kernel_variant "cluster") waits for its TMA
    bulk copies, set to give up at once (fne_set_wait_limit 0): the pass returns with a NaN energy, the
    status word reports FNE_ETIMEOUT (polled by the callbacks, or read
    synchronously), and with the default bound restored the same handle gives
    the oracle's values again (the context stayed usable)."""
    params, _ = meshes.gl_problem(n=24, seed=0)
    gpu, ref = _make("gl", params, kernel_variant="cluster")
    assert gpu.info["kernel_variant"] == 10
    u = np.random.default_rng(4).uniform(-0.5, 0.5, gpu.layout.n_free)
    ut = torch.as_tensor(u, device="cuda")
    _lib.check(_lib.lib.fne_set_wait_limit(gpu._handle, 0))
    e, _, _ = gpu.eval(ut, 7)
    torch.cuda.synchronize()
    assert np.isnan(float(e.item()))
    assert _lib.lib.fne_check_device_status(gpu._handle) == _lib.FNE_ETIMEOUT
    assert _lib.lib.fne_check_device_status(gpu._handle) == _lib.FNE_OK  # cleared
    with pytest.raises(_lib.FneError) as err:
        gpu.assemble_hessian(u)
    assert err.value.code == _lib.FNE_ETIMEOUT
    _lib.check(_lib.lib.fne_set_wait_limit(gpu._handle, -1))
    _check(gpu, ref, u, FP64_TOL)
    gpu.check_device_status()


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_cluster_kernel_is_bit_reproducible(precision):
    """Two passes of the row-cluster kernel give identical bits."""
    params, u0 = meshes.gl_problem(n=96, seed=1)
    hd = torch.float32 if precision == "fp32" else torch.float64
    gpu, _ = _make("gl", params, precision=precision, hess_dtype=hd, kernel_variant="cluster")
    assert gpu.info["kernel_variant"] == 10
    ut = torch.as_tensor(np.random.default_rng(5).uniform(-0.5, 0.5, gpu.layout.n_free), device="cuda")
    a = [t.clone() for t in gpu.eval(ut, 7)]
    b = gpu.eval(ut, 7)
    for x, y in zip(a, b):
        assert torch.equal(x, y)
