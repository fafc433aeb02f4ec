"""CPU oracle for the element energy / gradient / Hessian assembly path.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package imports this
directory; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` use it, and only as the checker.

What it restates (reference paths are relative to the
Beremi/fenics_nonlinear_energies project root):

* ``oracle.layout`` -- DOF permutation, PETSc ownership split, owned COO
  pattern, overlap data and the element->COO scatter map
  (``src/core/petsc/reordered_element_base.py``,
  ``src/core/petsc/dof_partition.py``).
* ``oracle.energies`` -- the per-element energy densities of the four
  families (p-Laplace, Ginzburg-Landau, Neo-Hookean, Mohr-Coulomb), written
  line by line after the JAX functions.  Derivatives come from
  ``torch.func`` autodiff in float64 (an autodiff independent of the
  hand-written CUDA adjoints, standing in for JAX, which is not installed).
* ``oracle.assembler`` -- ``energy_fn`` / ``gradient_fn`` /
  ``assemble_hessian_element`` with the reference's ``np.add.at`` scatter.
* ``oracle.slope`` -- the plane-strain P2/P4 geometry builders.

Pinning.  The layout functions are pinned by the reference's own unit
goldens (``tests/test_reordered_element_base.py:12-73``), the Davis-B
reduction by ``tests/test_slope_stability_jax.py:20-24`` and the slope mesh
counts by ``tests/test_slope_stability_support.py``.  Element VALUES have no
numeric golden in the reference's tests (only finiteness / shape / central
finite-difference consistency), so element-value parity is pinned by the
reference's own method: central finite differences of the restated energy
plus an independent autodiff (torch.func).  JAX itself cannot run here.
"""
