"""Write the reference-generated golden fixtures ``tests/golden/reference_*.npz``.

Run in a container that holds the reference sources (read-only)::

    python tests/golden/make_fixtures.py [--reference /path/to/fenics_nonlinear_energies]

The reference's own classes and functions produce every output stored here;
``refshim`` supplies the modules that are not installed (torch stands in for
JAX -- so derivatives are torch autodiff of the reference's own energy code --
plus one-process fakes for mpi4py / petsc4py).  Inputs come from this
repository's synthetic mesh generators (small sizes) and are stored beside
the outputs, so a test can rebuild the same problem from the fixture alone.

What is run (reference file:line):
* ``ReorderedElementAssemblerBase.__init__`` / ``energy_fn`` /
  ``gradient_fn`` / ``assemble_hessian_element``
  (``src/core/petsc/reordered_element_base.py:652-901, 1579-1633, 1733-1775``)
  through the family subclasses ``PLaplaceReorderedElementAssembler``,
  ``GLReorderedElementAssembler``, ``HEReorderedElementAssembler`` and
  ``SlopeStabilityReorderedElementAssembler``; the COO values are those
  handed to ``Mat.setValuesCOO``.  One rank, and every rank of 2- and
  3-rank splits (layout arrays, per-rank energy, owned gradient, owned COO).
* ``_triangle_operators`` (``plaplace_u3/support/mesh.py:51-71``) on the
  structured grids: P1 ``dvx, dvy, vol``.
* ``rotate_right_face_from_reference`` (``hyperelasticity/support/rotate_boundary.py:4-22``)
  and ``update_dirichlet`` (``reordered_element_base.py:1560-1566``).
* ``build_case_data`` (``slope_stability/support/mesh.py:816-878``: the P2
  slope generator, 13-digit 7-point rule, ``elem_B``, gravity load, free
  DOFs) and ``_build_same_mesh_lagrange_case_data_impl`` (:995-1091) for P4.
  basix is absent, so for P4 its element points, tabulation and quadrature
  come from this repository's restatement (``meshes.lagrange_points``,
  ``lagrange_tabulate``, ``slope_quadrature``); the P4 fixture therefore pins
  the reference's connectivity, operator, gravity and free-DOF code given
  that basis, not basix itself.
* ``davis_b_reduction`` (``slope_stability/support/reduction.py:8-29``).
* 3-D Mohr-Coulomb element functions (``slope_stability_3d/jax/jax_energy_3d.py``):
  ``element_energy_3d`` (:214-236), its ``jax.grad`` (``element_residual_3d``,
  :279) and ``constitutive_element_hessian_3d`` (:324-357, the assembler's
  ``autodiff_tangent_mode="constitutive"``); the elastic mode's
  ``elastic_element_energy_3d`` / ``constitutive_elastic_element_hessian_3d``.
  Inputs: this repository's synthetic 3-D slope (``meshes.slope3d_problem``,
  P1 / P2 / P4 tets) at a seeded state (``--only mc3d`` writes this fixture
  alone).
"""

from __future__ import annotations

import argparse
import math
import sys
import time
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

from tests.golden import refshim  # noqa: E402


def _basix_standin():
    """basix names used by slope_stability/support/mesh.py, backed by meshes.py."""
    from fenics_nonlinear_energies_b200 import meshes

    bx = sys.modules["basix"]
    bx.ElementFamily = types.SimpleNamespace(P="P")
    bx.CellType = types.SimpleNamespace(triangle="triangle")
    bx.LagrangeVariant = types.SimpleNamespace(equispaced="equispaced")
    bx.finite_element = types.SimpleNamespace(FiniteElement=object)

    class _Element:
        def __init__(self, degree):
            self.degree = int(degree)
            self.points = meshes.lagrange_points(self.degree)

        def tabulate(self, n, pts):
            pts = np.asarray(pts, dtype=np.float64)
            val, dx, dy = meshes.lagrange_tabulate(self.degree, pts.T)  # (n_p, nq)
            return np.stack([val.T, dx.T, dy.T])[..., None]

    bx.create_element = lambda family, cell, degree, variant=None: _Element(degree)

    def make_quadrature(cell, degree):
        # the reference asks for degree 2p+1: map back to the Lagrange degree
        xi, w = meshes.slope_quadrature((int(degree) - 1) // 2)
        return xi.T.copy(), w.copy()

    bx.make_quadrature = make_quadrature


def _savez(name, **arrays):
    path = HERE / f"reference_{name}.npz"
    np.savez_compressed(path, **{k: np.asarray(v) for k, v in arrays.items()})
    print(f"wrote {path.name}: {path.stat().st_size / 1024:.0f} KB")


def _run_assembler(cls, params, adjacency, u_full, *, rank=0, size=1, dirichlet=None, **kw):
    """One rank of the reference assembler: layout, energy, gradient, COO values."""
    comm = refshim.FakeComm(rank, size)
    comm.full = np.asarray(u_full, dtype=np.float64)
    asm = cls(params, comm, adjacency, **kw)
    if dirichlet is not None:
        asm.update_dirichlet(dirichlet)
    lay = asm.layout
    vec = asm.create_vec(u_full)
    energy = asm.energy_fn(vec)
    g = asm.create_vec()
    asm.gradient_fn(vec, g)
    timings = asm.assemble_hessian(np.asarray(u_full[lay.lo: lay.hi]))
    out = {
        "perm": lay.perm, "iperm": lay.iperm, "lo": lay.lo, "hi": lay.hi, "n_free": lay.n_free,
        "total_to_free_reord": lay.total_to_free_reord, "owned_rows": lay.owned_rows,
        "owned_cols": lay.owned_cols, "elem_owner": lay.elem_owner,
        "energy": energy, "grad": g.array.copy(), "hess": asm.A.values.copy(),
        "coo_rows": asm.A.coo_rows, "coo_cols": asm.A.coo_cols,
        "energy_weights": asm.local_data.energy_weights, "local_elem_idx": asm.local_data.local_elem_idx,
        "timing_keys": np.array(sorted(timings.keys())),
    }
    return out


def _family_case(name, cls, params, adjacency, u_full, keys, *, scalars, dirichlet=None, ranks=(1, 2, 3), **kw):
    store = {f"in_{k}": np.asarray(params[k]) for k in keys}
    for k, v in scalars.items():
        store[f"sc_{k}"] = np.asarray(v)
    store["in_u"] = np.asarray(u_full)
    if dirichlet is not None:
        store["in_dirichlet"] = np.asarray(dirichlet)
    for size in ranks:
        for r in range(size):
            t0 = time.perf_counter()
            res = _run_assembler(cls, params, adjacency, u_full, rank=r, size=size, dirichlet=dirichlet, **kw)
            for k, v in res.items():
                store[f"r{size}_{r}_{k}"] = np.asarray(v)
            print(f"  {name} rank {r}/{size}: {time.perf_counter() - t0:.1f} s")
    _savez(name, **store)


def main(reference):
    refshim.install()
    _basix_standin()
    sys.path.insert(0, str(reference))
    from src.problems.ginzburg_landau.jax_petsc.reordered_element_assembler import GLReorderedElementAssembler
    from src.problems.hyperelasticity.jax_petsc.reordered_element_assembler import HEReorderedElementAssembler
    from src.problems.hyperelasticity.support.rotate_boundary import rotate_right_face_from_reference
    from src.problems.plaplace.jax_petsc.reordered_element_assembler import PLaplaceReorderedElementAssembler
    from src.problems.plaplace_u3.support.mesh import _build_scalar_adjacency, _triangle_operators
    from src.problems.slope_stability.jax_petsc.reordered_element_assembler import (
        SlopeStabilityReorderedElementAssembler,
    )
    from src.problems.slope_stability.support import mesh as slope_mesh
    from src.problems.slope_stability.support.reduction import davis_b_reduction

    from fenics_nonlinear_energies_b200 import meshes

    # -- P1 geometry ------------------------------------------------------
    geo = {}
    for n in (4, 16):
        nodes, elems, _ = meshes.square_p1(n, -1.0, 1.0)
        dvx, dvy, vol = _triangle_operators(nodes, elems)
        geo.update({f"n{n}_nodes": nodes, f"n{n}_elems": elems, f"n{n}_dvx": dvx, f"n{n}_dvy": dvy,
                    f"n{n}_vol": vol})
    # -- Davis-B ----------------------------------------------------------
    lams = np.array([0.1, 0.5, 0.9, 1.0, 1.21, 1.5, 2.0])
    db = np.array([davis_b_reduction(6.0, 45.0, 0.0, float(lam)) for lam in lams])
    _savez("support", lams=lams, davis_b=db, **geo)

    # -- p-Laplace: random state and the zero state (energy / gradient only) --
    params, _ = meshes.plaplace_problem(n=16)
    adj = _build_scalar_adjacency(params["elems"], params["freedofs"])
    n_free = params["freedofs"].size
    u = 0.3 * np.random.default_rng(7).standard_normal(n_free)
    print("plaplace")
    _family_case("plaplace", PLaplaceReorderedElementAssembler, params, adj, u,
                 ("nodes", "u_0", "freedofs", "elems", "dvx", "dvy", "vol", "f"), scalars={"p": params["p"]})
    comm = refshim.FakeComm()
    asm = PLaplaceReorderedElementAssembler(params, comm, adj)
    z = np.zeros(n_free)
    vec = asm.create_vec(z)
    g = asm.create_vec()
    asm.gradient_fn(vec, g)
    _savez("plaplace_zero", energy=asm.energy_fn(vec), grad=g.array.copy())

    # -- Ginzburg-Landau --------------------------------------------------
    params, u = meshes.gl_problem(n=16, seed=3)
    adj = _build_scalar_adjacency(params["elems"], params["freedofs"])
    print("gl")
    _family_case("gl", GLReorderedElementAssembler, params, adj, u,
                 ("nodes", "u_0", "freedofs", "elems", "dvx", "dvy", "vol", "ip", "w"), scalars={"eps": params["eps"]})

    # -- Neo-Hookean beam, right face twisted ----------------------------
    params, y0 = meshes.he_beam_problem(nx=6, ny=2, nz=2)
    adj = slope_mesh._build_dof_adjacency(params["elems"], params["freedofs"])
    angle = 3 * 4.0 * math.pi / 24.0
    rotated = rotate_right_face_from_reference(params["u_0_ref"], params["nodes2coord"], angle,
                                               params["right_nodes"])
    # free DOFs follow the twist linearly along the beam, plus a seeded perturbation
    x = params["nodes2coord"][:, 0] / params["nodes2coord"][:, 0].max()
    a = angle * x
    twisted = params["nodes2coord"].copy()
    twisted[:, 1] = np.cos(a) * params["nodes2coord"][:, 1] + np.sin(a) * params["nodes2coord"][:, 2]
    twisted[:, 2] = -np.sin(a) * params["nodes2coord"][:, 1] + np.cos(a) * params["nodes2coord"][:, 2]
    y_full = twisted.reshape(-1) + 2e-4 * np.random.default_rng(8).standard_normal(twisted.size)
    comm = refshim.FakeComm()
    probe = HEReorderedElementAssembler(params, comm, adj, use_near_nullspace=False)
    y = np.zeros(probe.layout.n_free)
    y[probe.layout.total_to_free_reord[params["freedofs"]]] = y_full[params["freedofs"]]
    print("he")
    _family_case("he", HEReorderedElementAssembler, params, adj, y,
                 ("u_0", "u_0_ref", "freedofs", "elems", "elems_scalar", "dphix", "dphiy", "dphiz", "vol",
                  "nodes2coord", "right_nodes"),
                 scalars={"C1": params["C1"], "D1": params["D1"], "angle": angle}, dirichlet=rotated,
                 use_near_nullspace=False)

    # -- Mohr-Coulomb slope, P2 (reference generator) and P4 ------------------
    for degree, level in ((2, 1), (4, 1)):
        case = (slope_mesh.build_case_data(slope_mesh.case_name_for_level(level)) if degree == 2 else
                slope_mesh._build_same_mesh_lagrange_case_data_impl(slope_mesh.case_name_for_level(level),
                                                                    degree=degree))
        coh, phi = davis_b_reduction(6.0, 45.0, 0.0, 1.0)
        params = {
            "nodes": case.nodes, "elems_scalar": case.elems_scalar, "elems": case.elems,
            "freedofs": case.freedofs, "q_mask": case.q_mask, "u_0": case.u_0, "force": case.force,
            "elem_B": case.elem_B, "quad_weight": case.quad_weight, "eps_p_old": case.eps_p_old,
            "E": 2.0e4, "nu": 0.49, "phi_deg": phi, "cohesion": coh, "reg": 1.0e-12,
        }
        adj = case.adjacency
        probe = SlopeStabilityReorderedElementAssembler(params, refshim.FakeComm(), adj, use_near_nullspace=False)
        nodes = case.nodes
        # a smooth field that drives part of the slope into the plastic branches
        ux = 2e-3 * np.sin(0.11 * nodes[:, 0]) * (nodes[:, 1] / 20.0)
        uy = -4e-3 * (nodes[:, 1] / 20.0) ** 2 + 1e-3 * np.cos(0.07 * nodes[:, 0] + 0.2 * nodes[:, 1])
        u_nodal = np.stack([ux, uy], axis=1).reshape(-1)
        u = np.zeros(probe.layout.n_free)
        u[probe.layout.total_to_free_reord[case.freedofs]] = u_nodal[case.freedofs]
        print(f"mc_p{degree}")
        _family_case(f"mc_p{degree}", SlopeStabilityReorderedElementAssembler, params, adj, u,
                     ("nodes", "elems_scalar", "elems", "freedofs", "q_mask", "u_0", "force", "elem_B",
                      "quad_weight", "eps_p_old"),
                     scalars={"E": 2.0e4, "nu": 0.49, "phi_deg": phi, "cohesion": coh, "reg": 1.0e-12,
                              "gamma": case.gamma, "level": level, "h": case.h},
                     ranks=(1, 2) if degree == 2 else (1,), use_near_nullspace=False)


def mc3d_case(reference):
    """Element energy, residual and Hessians of the reference's 3-D density."""
    refshim.install()
    sys.path.insert(0, str(reference))
    import torch

    from src.problems.slope_stability_3d.jax import jax_energy_3d as R3

    from fenics_nonlinear_energies_b200 import meshes

    def t(a):
        return torch.as_tensor(np.asarray(a, dtype=np.float64))

    store = {}
    for degree, n, n_el in ((1, (2, 1, 1), 12), (2, (2, 1, 1), 12), (4, (1, 1, 1), 2)):
        p = meshes.slope3d_problem(nx=n[0], ny=n[1], nz=n[2], degree=degree, lam=1.5)
        rng = np.random.default_rng(20 + degree)
        u = p["u_0"].copy()
        u[p["freedofs"]] = 4e-2 * rng.standard_normal(p["freedofs"].size)
        keys = ("dphix", "dphiy", "dphiz", "quad_weight", "c_bar", "sin_phi", "shear", "bulk", "lame")
        out = {k: [] for k in ("energy", "grad", "hess", "el_energy", "el_hess")}
        ins = {k: np.asarray(p[k][:n_el]) for k in keys}
        ue = np.stack([u[p["elems"][e]] for e in range(n_el)])
        t0 = time.perf_counter()
        for e in range(n_el):
            args = [t(ins[k][e]) for k in keys]
            x = t(ue[e])
            out["energy"].append(float(R3.element_energy_3d(x, *args)))
            out["grad"].append(R3.element_residual_3d(x, *args).numpy())
            out["hess"].append(R3.constitutive_element_hessian_3d(x, *args).numpy())
            el_args = [args[i] for i in (0, 1, 2, 3, 6, 7, 8)]
            out["el_energy"].append(float(R3.elastic_element_energy_3d(x, *el_args)))
            out["el_hess"].append(R3.constitutive_elastic_element_hessian_3d(x, *el_args).numpy())
        print(f"  mc3d P{degree}: {n_el} elements, {time.perf_counter() - t0:.1f} s")
        store[f"p{degree}_u_elem"] = ue
        for k, v in ins.items():
            store[f"p{degree}_{k}"] = v
        for k, v in out.items():
            if v:
                store[f"p{degree}_{k}"] = np.asarray(v)
    _savez("mc3d", **store)


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--only", choices=["all", "mc3d"], default="all",
                    help="mc3d: write only the 3-D Mohr-Coulomb element fixture")
    args = ap.parse_args()
    if args.only == "all":
        main(Path(args.reference))
    mc3d_case(Path(args.reference))
