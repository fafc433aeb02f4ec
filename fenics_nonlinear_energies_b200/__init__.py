"""B200-native element energy / gradient / Hessian assembly.

A drop-in for the element-assembly callables of Beremi/fenics_nonlinear_energies
(``ReorderedElementAssemblerBase`` and its p-Laplace, Ginzburg-Landau,
Neo-Hookean and Mohr-Coulomb subclasses), computed by hand-written sm_100a
CUDA kernels in ``libfne_asm.so`` (C ABI: ``include/fne_asm.h``).

Import the assemblers from ``fenics_nonlinear_energies_b200.assembler``; the
mesh builders in ``fenics_nonlinear_energies_b200.meshes`` need no GPU.
"""

__version__ = "0.1.0"
