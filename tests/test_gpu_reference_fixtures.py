"""CUDA assemblers against outputs of the reference itself, through the C ABI.

``tests/golden/reference_*.npz`` hold what the reference's own assembler
classes returned (``tests/golden/make_fixtures.py``): per rank of 1-, 2- and
3-rank splits the layout, the energy, the owned gradient and the owned COO
Hessian values handed to ``Mat.setValuesCOO``.  The CUDA assemblers get the
same inputs and must give the same layout bit-for-bit and the same values:
FP64 mode within 1e-12 relative (energy vs max(1, |E|), gradient / Hessian
vs their largest entry); FP32-Hessian mode within 2e-5 (Hessian), 1e-4
(gradient) and 1e-6 (energy, reduced in FP64).
"""

from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from fenics_nonlinear_energies_b200 import _lib, meshes

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
FP64_TOL = 1e-12
FP32_H_TOL, FP32_G_TOL, FP32_E_TOL = 2e-5, 1e-4, 1e-6
LAYOUT_KEYS = ("perm", "iperm", "total_to_free_reord", "owned_rows", "owned_cols", "elem_owner")


def load(name):
    return dict(np.load(GOLDEN / f"reference_{name}.npz"))


def fixture_params(fx):
    params = {k[3:]: v for k, v in fx.items() if k.startswith("in_")}
    for k, v in fx.items():
        if k.startswith("sc_"):
            params[k[3:]] = float(v)
    return params


def splits(fx):
    return [(r, s) for s in (1, 2, 3) for r in range(s) if f"r{s}_{r}_energy" in fx]


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.abs(a - b).max(initial=0.0) / max(np.abs(b).max(initial=0.0), 1e-300)


def _assembler(name, params, comm, precision):
    from fenics_nonlinear_energies_b200.assembler import (
        GLCudaAssembler, HECudaAssembler, PLaplaceCudaAssembler, SlopeStabilityCudaAssembler)

    kw = dict(precision=precision, hess_dtype=torch.float32 if precision == "fp32" else torch.float64)
    if name == "plaplace":
        return PLaplaceCudaAssembler(params, comm, **kw)
    if name == "gl":
        return GLCudaAssembler(params, comm, **kw)
    if name == "he":
        return HECudaAssembler(params, comm, **kw)
    return SlopeStabilityCudaAssembler(params, comm, **kw)


def _check(name, params, fx, precision, dirichlet=None):
    for r, size in splits(fx):
        key = f"r{size}_{r}_"
        asm = _assembler(name, params, SimpleNamespace(rank=r, size=size), precision)
        for k in LAYOUT_KEYS:
            np.testing.assert_array_equal(getattr(asm.layout, k), fx[key + k], err_msg=f"{name} {r}/{size} {k}")
        if dirichlet is not None:
            asm.update_dirichlet(dirichlet)
        u = torch.as_tensor(fx["in_u"], device="cuda")
        e, g, h = asm.eval(u, _lib.FNE_ENERGY | _lib.FNE_GRAD | _lib.FNE_HESS)
        torch.cuda.synchronize()
        e, g, h = float(e.item()), g[: asm.n_owned].cpu().numpy(), h.double().cpu().numpy()
        e_ref = float(fx[key + "energy"])
        if precision == "fp64":
            tols = (FP64_TOL, FP64_TOL, FP64_TOL)
        else:  # Mohr-Coulomb FP32 energies sum many FP32 return-map densities: 1e-5
            tols = (1e-5 if name == "mc" else FP32_E_TOL, FP32_G_TOL, FP32_H_TOL)
        assert abs(e - e_ref) <= tols[0] * max(1.0, abs(e_ref)), (name, r, size, e, e_ref)
        assert rel(g, fx[key + "grad"]) <= tols[1], (name, r, size, rel(g, fx[key + "grad"]))
        assert rel(h, fx[key + "hess"]) <= tols[2], (name, r, size, rel(h, fx[key + "hess"]))
        if precision == "fp64":  # the per-assembly timing record carries the reference's keys
            t = asm.assemble_hessian(u)
            missing = set(fx[key + "timing_keys"].tolist()) - set(t)
            assert not missing, missing


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("name", ["plaplace", "gl", "he"])
def test_p1_families_match_reference(name, precision):
    fx = load(name)
    _check(name, fixture_params(fx), fx, precision, dirichlet=fx.get("in_dirichlet"))


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("degree", [2, 4])
def test_mc_matches_reference(degree, precision):
    """Slope P2 (the reference's own generator: isoparametric map, curved
    slope-side elements) and P4 (same-mesh, affine), level 1, partly plastic
    state: the mesh generator's arrays equal the fixture's inputs (CPU test),
    so the assembler runs on them; default kernels (DMMA FP64, tcgen05 FP32)."""
    fx = load(f"mc_p{degree}")
    params = meshes.slope_problem(level=int(fx["sc_level"]), degree=degree, E=float(fx["sc_E"]),
                                  nu=float(fx["sc_nu"]))
    np.testing.assert_array_equal(params["elems"], fx["in_elems"])
    _check("mc", params, fx, precision)


@pytest.mark.parametrize("variant", ["auto", "cuda_cores"])
def test_mc_accepts_reference_problem_data(variant):
    """The reference's own P2 problem data (``elem_B`` / ``quad_weight``, no
    element map): the assembler recovers the per-point map and matches the
    reference's outputs, on the tensor-core and CUDA-core kernels."""
    from fenics_nonlinear_energies_b200.assembler import SlopeStabilityCudaAssembler

    fx = load("mc_p2")
    params = fixture_params(fx)
    gen = meshes.slope_problem(level=int(fx["sc_level"]), degree=2)
    params.update({k: gen[k] for k in ("dhat1", "dhat2", "quad_w")})
    asm = SlopeStabilityCudaAssembler(params, kernel_variant=variant)
    e, g, h = asm.eval(torch.as_tensor(fx["in_u"], device="cuda"), 7)
    torch.cuda.synchronize()
    assert abs(float(e.item()) - float(fx["r1_0_energy"])) <= FP64_TOL * max(1.0, abs(float(fx["r1_0_energy"])))
    assert rel(g.cpu().numpy(), fx["r1_0_grad"]) <= FP64_TOL
    assert rel(h.cpu().numpy(), fx["r1_0_hess"]) <= FP64_TOL


def test_plaplace_zero_state_matches_reference():
    """The p-Laplace configuration's assembly start: energy and gradient at u = 0."""
    from fenics_nonlinear_energies_b200.assembler import PLaplaceCudaAssembler

    fx, z = load("plaplace"), load("plaplace_zero")
    asm = PLaplaceCudaAssembler(fixture_params(fx))
    u = torch.zeros(asm.layout.n_free, dtype=torch.float64, device="cuda")
    e, g, _ = asm.eval(u, _lib.FNE_ENERGY | _lib.FNE_GRAD)
    torch.cuda.synchronize()
    assert abs(float(e.item()) - float(z["energy"])) <= FP64_TOL
    assert rel(g[: asm.n_owned].cpu().numpy(), z["grad"]) <= FP64_TOL
