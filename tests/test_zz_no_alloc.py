"""fne_energy_p1tri_noalloc: the energy entry point that allocates no device memory.

It serves callers that cannot let the library call cudaMalloc -- a framework
whose caching allocator already owns the GPU's memory, or a solver that
forbids allocation after set-up.  Its scratch is a fixed array inside the
library.  The test calls it through the C ABI, twice in a row (the second
call must not see the first call's leftovers), and compares it with the
regular handle-based entry point (fne_eval with FNE_ENERGY) within the FP64
tolerance the parity tests use.  This file is collected last so that a run
stopping at the first failure has run every other test; it also passes on
its own in a fresh process.
"""

import ctypes as C

import numpy as np
import pytest
import torch

from fenics_nonlinear_energies_b200 import _lib, meshes

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _soa_inputs(asm, params):
    """Device float64 element arrays and int32 gather codes, from the assembler's layout."""
    elems = np.asarray(params["elems"], dtype=np.int64)
    t2f = asm.layout.total_to_free_reord
    r = t2f[elems]
    codes = np.where(r >= 0, r, -1 - elems).astype(np.int32)
    dev = asm.device
    weights = (asm.layout.elem_owner == 0).astype(np.float64)
    return {
        "codes": torch.as_tensor(codes.ravel(), device=dev),
        "dvx": torch.as_tensor(np.ascontiguousarray(params["dvx"]).ravel(), device=dev),
        "dvy": torch.as_tensor(np.ascontiguousarray(params["dvy"]).ravel(), device=dev),
        "vol": torch.as_tensor(np.ascontiguousarray(params["vol"]), device=dev),
        "weights": torch.as_tensor(weights, device=dev),
        "dir": torch.as_tensor(np.asarray(params["u_0"], dtype=np.float64), device=dev),
    }


def _noalloc_energy(family, n_elem, d, u, scalars, rhs=None, n_owned=0, out=None):
    if out is None:
        out = torch.full((1,), float("nan"), dtype=torch.float64, device=u.device)
    sc = (C.c_double * 16)(*scalars)
    stream = torch.cuda.current_stream(u.device).cuda_stream
    _lib.check(_lib.lib.fne_energy_p1tri_noalloc(
        family, n_elem, d["codes"].data_ptr(), d["dvx"].data_ptr(), d["dvy"].data_ptr(), d["vol"].data_ptr(),
        d["weights"].data_ptr(), u.data_ptr(), d["dir"].data_ptr(), sc,
        rhs.data_ptr() if rhs is not None else None, n_owned, 0, out.data_ptr(), stream))
    return out


@pytest.mark.parametrize("family", ["gl", "plaplace"])
def test_noalloc_energy_matches_fne_eval_twice(family):
    from fenics_nonlinear_energies_b200.assembler import GLCudaAssembler, PLaplaceCudaAssembler

    if family == "gl":
        params, u0 = meshes.gl_problem(n=96, seed=5)
        asm = GLCudaAssembler(params)
        fam = _lib.FNE_GINZBURG_LANDAU
    else:
        params, _ = meshes.plaplace_problem(n=80)
        u0 = np.random.default_rng(6).random(params["freedofs"].size)
        asm = PLaplaceCudaAssembler(params)
        fam = _lib.FNE_PLAPLACE
    d = _soa_inputs(asm, params)
    u = torch.as_tensor(u0, device=asm.device)
    scalars = list(asm._scalars()) + [0.0] * (16 - len(asm._scalars()))
    rhs = torch.as_tensor(asm._f_owned, device=asm.device) if asm._f_owned is not None else None
    n_owned = asm.n_owned if rhs is not None else 0
    ref = float(asm.eval(u, _lib.FNE_ENERGY)[0].item())
    if family == "gl":  # fne_eval adds the Dirichlet-only element energy; the SoA call covers all elements
        all_w = torch.ones_like(d["weights"])
        d = dict(d, weights=all_w)
    n_elem = len(params["elems"])
    # Warm-up call: the first call on a device may load the library's device code.
    _noalloc_energy(fam, n_elem, d, u, scalars, rhs, n_owned)
    first = torch.full((1,), float("nan"), dtype=torch.float64, device=u.device)
    second = torch.full((1,), float("nan"), dtype=torch.float64, device=u.device)
    torch.cuda.synchronize()
    free_before, _ = torch.cuda.mem_get_info(u.device)
    stats_before = torch.cuda.memory_stats(u.device)
    _noalloc_energy(fam, n_elem, d, u, scalars, rhs, n_owned, out=first)
    _noalloc_energy(fam, n_elem, d, u, scalars, rhs, n_owned, out=second)
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info(u.device)
    stats_after = torch.cuda.memory_stats(u.device)
    # The defining property: the two calls allocated no device memory, neither
    # through the driver (free memory unchanged) nor through torch's allocator.
    assert free_after == free_before, (free_before, free_after)
    for key in ("allocation.all.allocated", "segment.all.allocated"):
        assert stats_after.get(key, 0) == stats_before.get(key, 0), key
    scale = max(1.0, abs(ref))
    assert abs(float(first.item()) - ref) <= FP64_TOL * scale, (float(first.item()), ref)
    assert abs(float(second.item()) - ref) <= FP64_TOL * scale, (float(second.item()), ref)


def test_noalloc_rejects_oversized_input():
    u = torch.zeros(1, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    sc = (C.c_double * 16)(3.0)
    code = _lib.lib.fne_energy_p1tri_noalloc(_lib.FNE_PLAPLACE, 2**31, u.data_ptr(), u.data_ptr(), u.data_ptr(),
                                             u.data_ptr(), None, u.data_ptr(), u.data_ptr(), sc, None, 0, 0,
                                             out.data_ptr(), None)
    assert code == _lib.FNE_EBOUNDS
    assert b"2^31-1" in _lib.lib.fne_last_error()
