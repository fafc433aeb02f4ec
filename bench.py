"""Benchmark: fused energy + gradient + Hessian assembly, elements/s.

Default workload (``--workload gl1024_fp64``, one "step"): Ginzburg-Landau,
eps = 0.01 on [-1, 1]^2, structured 1024 x 1024 grid of P1 triangles
(2,097,152 elements, 1,046,529 free DOFs, 7,317,521 owned COO entries),
u ~ U[-0.5, 0.5] from a fixed seed, FP64 throughout (the reference's
arithmetic).  One step = one fused E+grad+Hess pass over every element into
the device gradient and the owned COO values (the reference's energy_fn +
gradient_fn + assemble_hessian_element).  ``gl1024_fp32h`` is the same
configuration with FP32 element gradients / Hessians.

``error_vs_fp64_oracle`` (outside the timed region): the largest relative
error of the energy, gradient and COO values of one pass against the FP64
oracle on the same configuration (every entry; the P4 slope on 400 sampled
owned rows).

Other workloads (same JSON line, same timing rules; ``--workload NAME``):
p-Laplace 128x128 P1 (FP64, zero state), Ginzburg-Landau 1024^2 in FP64,
the Neo-Hookean beam 160x8x8 hexes x 6 tets (FP64 and FP32 Hessian) and its
320x16x16 refinement, and the plane-strain Mohr-Coulomb slope with P4 / P2
triangles at h = 0.08 (203,000 elements); the matrix-free Mohr-Coulomb
Hessian-vector product; and whole Newton solves (``*_newton_*``: metric
"Newton s to 1e-6 rel-grad", lower is better; the roofline line is one
device CG iteration on the Hessian at the solution, timed on its own).

``--pass energy`` times the energy-only pass instead (the line-search
callback, ``energy_fn``): algorithmic bytes are the connectivity, geometry
and state reads only.

``value``: device-resident inputs, CUDA events around each pass, L2 flushed
(1 GiB write) between passes outside the timed events; its length also keeps
the GPU busy while the host enqueues the timed pass, so no launch gap
falls inside the events.
``e2e``: the same pass through the public assembler API with host buffers:
H2D of u from pinned memory, the pass, D2H of energy, gradient and COO values.

Multi-GPU: every rank runs its own replica of the workload (weak scaling).
``--impl reference``: the CPU restatement of the reference path (the JAX
element kernels + np.add.at scatter, restated in oracle/) on the host cores,
on the same configuration where one pass takes seconds (P1 triangles,
tetrahedra), else on a bounded sample of the same workload family.
``cpu_baseline`` (``--impl b200``): for the P1-triangle families a
numba-parallel CPU assembly of the full configuration on all host threads
(closed-form element derivatives, parallel deterministic gathers) -- the
stronger CPU line -- with the autodiff restatement on its sample and the
reference's archived single-thread figure beside it; for the other families
the autodiff restatement on a bounded sample.
"""


from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))



def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# L2 flush between timed passes: 8x the 126 MB L2; the write (~170 us) also
# covers the host's enqueue of the next pass.
FLUSH_BYTES = 1 << 30

# DRAM bytes (read + write) per launch of the dominant kernel, from one ncu
# capture of the same workload (dram__bytes_read.sum + dram__bytes_write.sum),
# with the profile summary that records it.  Keyed by (workload, kernel).
NCU_TRAFFIC = {
    ("gl1024_fp32h", "k_sweep_tri"): (213.2e6, "profiles/k_sweep_tri_gl1024_fp32.md"),
    ("gl1024_fp64", "k_sweep_tri"): (330.6e6, "profiles/k_sweep_tri_gl1024_fp64.md"),
    # one CG iteration: k_cg_spmv 117.4 MB + k_cg_update 41.9 MB
    ("gl1024_newton_fp64", "k_cg_spmv+k_cg_update"): (159.3e6, "profiles/k_cg_gl1024_newton_fp64.md"),
}

# CG iterations timed on their own for the Newton workloads' roofline line.
CG_TIMED_ITERATIONS = 800


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        # raw samples in the temporary directory (the JSON line carries the summary)
        self.path = Path(tempfile.gettempdir()) / f"fne_clocks_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist_setup():
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and not dist.is_initialized():
        import datetime

        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def _barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist

    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
# workloads
# ---------------------------------------------------------------------------
class Workload:
    """One benchmark configuration.

    ``build(rank)`` returns ``(assembler, u_owned_reordered)``;
    ``conn_nodes`` / ``geom_values`` are the node-level connectivity entries
    and the per-element geometry values one pass reads (algorithmic bytes);
    ``sample()`` returns ``(family, oracle_kwargs, params, u, n_el, label)`` for
    the bounded CPU restatement run; ``full()`` (where set) the same for the
    whole configuration.
    """

    def __init__(self, name, family, precision, hess_fp32, conn_nodes, geom_values, geom_bytes, has_rhs, desc,
                 build, sample, op="egh", newton_kw=None, full=None):
        self.op = op  # "egh": fused E+grad+Hess pass; "hvp": matrix-free H(u) x; "newton": one Newton solve
        self.newton_kw = dict(newton_kw or {})  # Newton settings of the "newton" workloads
        self.name, self.family, self.precision, self.hess_fp32 = name, family, precision, hess_fp32
        self.conn_nodes, self.geom_values, self.geom_bytes, self.has_rhs = conn_nodes, geom_values, geom_bytes, has_rhs
        self.desc, self.build, self.sample = desc, build, sample
        # full(): the whole configuration for the CPU restatement (same tuple as sample()),
        # or None where one CPU pass would take minutes
        self.full = full if full is not None else (getattr(build, "full", None) if op == "egh" else None)

    @property
    def dtype(self):
        if self.precision == "fp32":
            return "f32 (element grad/Hessian), f64 (energy)"
        return "f64"


# kernel choice passed to the assembler ("auto" unless --kernel-variant is given)
KERNEL_VARIANT = {"value": "auto"}


def _reordered(asm, u_free):
    import numpy as np

    return np.ascontiguousarray(np.asarray(u_free, dtype=np.float64)[np.asarray(asm.layout.perm)])


def twisted_beam_positions(params, theta):
    """Deformed positions of the beam twisted about its axis by ``theta * x / L``
    (the right face carries the full rotation of the load step)."""
    import numpy as np

    X = params["nodes2coord"]
    a = theta * X[:, 0] / float(X[:, 0].max())
    c, s = np.cos(a), np.sin(a)
    return np.stack([X[:, 0], c * X[:, 1] + s * X[:, 2], -s * X[:, 1] + c * X[:, 2]], axis=1).ravel()


def slope_state(params, amplitude=0.02):
    """Smooth synthetic slope displacement (u_x, u_y) interleaved per node."""
    import numpy as np

    x, y = params["nodes"][:, 0], params["nodes"][:, 1]
    ux = amplitude * 4.0 * (y / 20.0) * (x / 40.0) * (1.0 - x / 40.0)
    uy = -amplitude * (y / 20.0) ** 2
    return np.stack([ux, uy], axis=1).ravel()


def _tri(kind, n, precision, seed_from_rank=True, start_seed=None, sample_n=None):
    """``start_seed``: p-Laplace start U[0, 1) from this seed (zero state when
    None); ``sample_n``: grid of the bounded CPU sample (default min(n, 512))."""

    def build(rank):
        import torch

        from fenics_nonlinear_energies_b200 import meshes
        from fenics_nonlinear_energies_b200.assembler import GLCudaAssembler, PLaplaceCudaAssembler

        hd = torch.float32 if precision == "fp32" else torch.float64
        if kind == "gl":
            params, u0 = meshes.gl_problem(n=n, seed=rank)
            asm = GLCudaAssembler(params, precision=precision, hess_dtype=hd, kernel_variant=KERNEL_VARIANT["value"])
        else:
            params, u0 = meshes.plaplace_problem(n=n, seed=start_seed)
            asm = PLaplaceCudaAssembler(params, precision=precision, hess_dtype=hd, kernel_variant=KERNEL_VARIANT["value"])
        return asm, _reordered(asm, u0)

    def sample():
        from fenics_nonlinear_energies_b200 import meshes

        m = sample_n or min(n, 512)
        if kind == "gl":
            params, u0 = meshes.gl_problem(n=m, seed=0)
        else:
            params, u0 = meshes.plaplace_problem(n=m, seed=start_seed)
        return kind, {}, params, u0, 2 * m * m, f"{m}x{m} P1 grid"

    def full():
        from fenics_nonlinear_energies_b200 import meshes

        if kind == "gl":
            params, u0 = meshes.gl_problem(n=n, seed=0)
        else:
            params, u0 = meshes.plaplace_problem(n=n, seed=start_seed)
        return kind, {}, params, u0, 2 * n * n, f"{n}x{n} P1 grid"

    build.full = full
    return build, sample


def _he(nx, ny, nz, precision, theta=4.0 * 3.141592653589793 / 24.0):
    def build(rank):
        import torch

        from fenics_nonlinear_energies_b200 import meshes
        from fenics_nonlinear_energies_b200.assembler import HECudaAssembler

        params, _ = meshes.he_beam_problem(nx=nx, ny=ny, nz=nz)
        hd = torch.float32 if precision == "fp32" else torch.float64
        asm = HECudaAssembler(params, precision=precision, hess_dtype=hd, kernel_variant=KERNEL_VARIANT["value"])
        pos = twisted_beam_positions(params, theta)
        asm.update_dirichlet(pos)
        return asm, _reordered(asm, pos[params["freedofs"]])

    def sample():
        from fenics_nonlinear_energies_b200 import meshes

        sx = max(1, nx // 8)
        params, _ = meshes.he_beam_problem(nx=sx, ny=ny, nz=nz)
        pos = twisted_beam_positions(params, theta)
        params = dict(params, u_0_ref=pos)
        return "he", {"block_size": 3, "coordinate_key": "nodes2coord", "dirichlet_key": "u_0_ref"}, params, \
            pos[params["freedofs"]], 6 * sx * ny * nz, f"{sx}x{ny}x{nz}-hex beam"

    def full():
        from fenics_nonlinear_energies_b200 import meshes

        params, _ = meshes.he_beam_problem(nx=nx, ny=ny, nz=nz)
        pos = twisted_beam_positions(params, theta)
        params = dict(params, u_0_ref=pos)
        return "he", {"block_size": 3, "coordinate_key": "nodes2coord", "dirichlet_key": "u_0_ref"}, params, \
            pos[params["freedofs"]], 6 * nx * ny * nz, f"{nx}x{ny}x{nz}-hex beam"

    build.full = full
    return build, sample


def _he_newton(nx, ny, nz, precision, theta=4.0 * 3.141592653589793 / 24.0):
    """First load step of the twisted beam: Dirichlet right face rotated by
    ``theta``, Newton from the reference configuration."""

    def rotated(params):
        from fenics_nonlinear_energies_b200 import meshes

        return meshes.rotate_right_face_from_reference(params["u_0_ref"], params["nodes2coord"], theta,
                                                       params["right_nodes"])

    def build(rank):
        import torch

        from fenics_nonlinear_energies_b200 import meshes
        from fenics_nonlinear_energies_b200.assembler import HECudaAssembler

        params, _ = meshes.he_beam_problem(nx=nx, ny=ny, nz=nz)
        hd = torch.float32 if precision == "fp32" else torch.float64
        asm = HECudaAssembler(params, precision=precision, hess_dtype=hd, kernel_variant=KERNEL_VARIANT["value"])
        rot = rotated(params)
        asm.update_dirichlet(rot)
        return asm, _reordered(asm, rot[params["freedofs"]])

    def sample():
        from fenics_nonlinear_energies_b200 import meshes

        sx = max(1, nx // 8)
        params, _ = meshes.he_beam_problem(nx=sx, ny=ny, nz=nz)
        rot = rotated(params)
        params = dict(params, u_0_ref=rot)
        return "he", {"block_size": 3, "coordinate_key": "nodes2coord", "dirichlet_key": "u_0_ref"}, params, \
            rot[params["freedofs"]], 6 * sx * ny * nz, f"{sx}x{ny}x{nz}-hex beam"

    return build, sample


def _mc(degree, h, precision):
    def build(rank):
        import torch

        from fenics_nonlinear_energies_b200 import meshes
        from fenics_nonlinear_energies_b200.assembler import SlopeStabilityCudaAssembler

        params = meshes.slope_problem(h=h, degree=degree, lam=1.0)
        hd = torch.float32 if precision == "fp32" else torch.float64
        asm = SlopeStabilityCudaAssembler(params, precision=precision, hess_dtype=hd,
                                          kernel_variant=KERNEL_VARIANT["value"])
        return asm, _reordered(asm, slope_state(params)[params["freedofs"]])

    def sample():
        from fenics_nonlinear_energies_b200 import meshes

        params = meshes.slope_problem(level=3, degree=degree, lam=1.0, with_elem_B=True)
        u = slope_state(params)[params["freedofs"]]
        return "mc", {"block_size": 2}, params, u, int(params["elems_scalar"].shape[0]), \
            f"slope h=1 P{degree}"

    return build, sample


def slope3d_state(params, amplitude=0.05):
    """A smooth closed-form displacement of the 3-D slope (zero on the fixed
    faces by the factor z x (L - x) y (W - y) in the constrained components),
    large enough to reach the plastic branches."""
    import numpy as np

    X = np.asarray(params["nodes"], dtype=np.float64)
    L, W, H = X[:, 0].max(), X[:, 1].max(), X[:, 2].max()
    x, y, z = X[:, 0] / L, X[:, 1] / W, X[:, 2] / H
    u = np.zeros((X.shape[0], 3))
    u[:, 0] = amplitude * z * x * (1 - x) * np.sin(3.0 * y + 1.0)
    u[:, 1] = amplitude * z * y * (1 - y) * np.cos(2.0 * x)
    u[:, 2] = -amplitude * z * (1.0 + 0.5 * np.sin(4.0 * x) * np.cos(3.0 * y))
    return u.ravel()


def _mc3d(nx, ny, nz, precision, degree=2):
    def build(rank):
        import torch

        from fenics_nonlinear_energies_b200 import meshes
        from fenics_nonlinear_energies_b200.assembler import SlopeStability3DCudaAssembler

        params = meshes.slope3d_problem(nx=nx, ny=ny, nz=nz, degree=degree, lam=1.0)
        hd = torch.float32 if precision == "fp32" else torch.float64
        asm = SlopeStability3DCudaAssembler(params, precision=precision, hess_dtype=hd)
        return asm, _reordered(asm, slope3d_state(params)[params["freedofs"]])

    def sample():
        from fenics_nonlinear_energies_b200 import meshes

        n = (2, 2, 1) if degree == 2 else (1, 1, 1)
        params = meshes.slope3d_problem(nx=n[0], ny=n[1], nz=n[2], degree=degree, lam=1.0)
        return "mc3d", {}, params, slope3d_state(params)[params["freedofs"]], int(params["elems"].shape[0]), \
            f"3-D slope {n[0]}x{n[1]}x{n[2]} hexes, P{degree} tets"

    return build, sample


WORKLOADS = {
    "gl1024_fp32h": Workload(
        "gl1024_fp32h", "gl", "fp32", True, 3, 7, 4, False,
        "Ginzburg-Landau eps=0.01 on [-1,1]^2, 1024x1024 P1 triangles (2,097,152 elements), "
        "u ~ U[-0.5,0.5] seeded; FP32 element grad/Hessian, FP64 energy", *_tri("gl", 1024, "fp32")),
    "gl1024_fp64": Workload(
        "gl1024_fp64", "gl", "fp64", False, 3, 7, 8, False,
        "Ginzburg-Landau eps=0.01 on [-1,1]^2, 1024x1024 P1 triangles (2,097,152 elements), FP64",
        *_tri("gl", 1024, "fp64")),
    "plaplace128_fp64": Workload(
        "plaplace128_fp64", "plaplace", "fp64", False, 3, 7, 8, True,
        "p-Laplace p=3, f=-10, unit square 128x128 P1 triangles (32,768 elements), zero state, FP64",
        *_tri("plaplace", 128, "fp64")),
    "he160x8x8_fp64": Workload(
        "he160x8x8_fp64", "he", "fp64", False, 4, 13, 8, False,
        "Neo-Hookean beam [0,0.4]x[-0.01,0.01]^2, 160x8x8 hexes x 6 tets (61,440), E=10, nu=0.3, "
        "state twisted by 4pi/24 (first load step), FP64", *_he(160, 8, 8, "fp64")),
    "he160x8x8_fp32h": Workload(
        "he160x8x8_fp32h", "he", "fp32", True, 4, 13, 4, False,
        "Neo-Hookean beam 160x8x8 hexes x 6 tets (61,440), first load step, FP32 element grad/Hessian",
        *_he(160, 8, 8, "fp32")),
    "he320x16x16_fp64": Workload(
        "he320x16x16_fp64", "he", "fp64", False, 4, 13, 8, False,
        "Neo-Hookean beam 320x16x16 hexes x 6 tets (491,520), first load step, FP64", *_he(320, 16, 16, "fp64")),
    "mc_p4_h0.08_fp64": Workload(
        "mc_p4_h0.08_fp64", "mc", "fp64", False, 15, 5, 8, True,
        "Mohr-Coulomb plane-strain slope 40x20 (height 10, 1:1), P4 triangles h=0.08 (203,000 elements), "
        "c=6, phi=45 deg, E=2e4, nu=0.49, lambda=1 (Davis-B), 19-point degree-9 rule, smooth synthetic state, FP64",
        *_mc(4, 0.08, "fp64")),
    "mc_p4_h0.08_fp32": Workload(
        "mc_p4_h0.08_fp32", "mc", "fp32", True, 15, 5, 8, True,
        "Mohr-Coulomb slope P4 h=0.08 (203,000 elements), FP32 element grad/Hessian", *_mc(4, 0.08, "fp32")),
    "mc_p4_h0.16_fp64": Workload(
        "mc_p4_h0.16_fp64", "mc", "fp64", False, 15, 5, 8, True,
        "Mohr-Coulomb slope P4 h=0.16 (about 51,000 elements), FP64 (profiling size)", *_mc(4, 0.16, "fp64")),
    "mc_p4_h0.16_fp32": Workload(
        "mc_p4_h0.16_fp32", "mc", "fp32", True, 15, 5, 8, True,
        "Mohr-Coulomb slope P4 h=0.16 (about 51,000 elements), FP32 element grad/Hessian (profiling size)",
        *_mc(4, 0.16, "fp32")),
    "mc_p4_h0.08_hvp_fp64": Workload(
        "mc_p4_h0.08_hvp_fp64", "mc", "fp64", False, 15, 5, 8, False,
        "Mohr-Coulomb slope P4 h=0.08 (203,000 elements): one matrix-free Hessian-vector product H(u) x "
        "at a linearized state (the PMG smoother's operator), FP64", *_mc(4, 0.08, "fp64"), op="hvp"),
    "mc_p4_h0.08_hvp_fp32": Workload(
        "mc_p4_h0.08_hvp_fp32", "mc", "fp32", False, 15, 5, 8, False,
        "Mohr-Coulomb slope P4 h=0.08: one matrix-free Hessian-vector product, FP32 element arithmetic",
        *_mc(4, 0.08, "fp32"), op="hvp"),
    "mc_p2_h0.08_fp64": Workload(
        "mc_p2_h0.08_fp64", "mc", "fp64", False, 6, 5, 8, True,
        "Mohr-Coulomb slope P2 h=0.08 (203,000 elements), 7-point rule, FP64", *_mc(2, 0.08, "fp64")),
    "mc3d_p2_fp64": Workload(
        "mc3d_p2_fp64", "mc3d", "fp64", False, 10, 396, 8, True,
        "Mohr-Coulomb 3-D slope (length 40, width 10, heights 20 / 10), 40x16x16 hexes x 6 P2 tetrahedra "
        "(61,440 elements), reference 11-point rule, c=6, phi=45 deg, E=2e4, nu=0.3, lambda=1 (Davis-B), smooth "
        "synthetic state, FP64", *_mc3d(40, 16, 16, "fp64")),
    "mc3d_p4_fp64": Workload(
        "mc3d_p4_fp64", "mc3d", "fp64", False, 35, 2664, 8, True,
        "Mohr-Coulomb 3-D slope (length 40, width 10, heights 20 / 10), 23x8x8 hexes x 6 P4 tetrahedra "
        "(8,832 elements, 35 nodes each), reference 24-point rule, c=6, phi=45 deg, E=2e4, nu=0.3, lambda=1 "
        "(Davis-B), smooth synthetic state, FP64", *_mc3d(23, 8, 8, "fp64", degree=4)),
    "plaplace128_newton_fp64": Workload(
        "plaplace128_newton_fp64", "plaplace", "fp64", False, 3, 7, 8, True,
        "Newton to ||g|| <= 1e-6 ||g_0||: p-Laplace p=3, f=-10, unit square 128x128 P1 triangles (32,768 "
        "elements), start U[0,1) seed 0; Jacobi CG rtol 1e-3, golden-section line search on [-0.5, 2], FP64",
        *_tri("plaplace", 128, "fp64", start_seed=0, sample_n=128), op="newton"),
    "gl1024_newton_fp64": Workload(
        "gl1024_newton_fp64", "gl", "fp64", False, 3, 7, 8, False,
        "Newton to ||g|| <= 1e-6 ||g_0||: Ginzburg-Landau eps=0.01, 1024x1024 P1 triangles (2,097,152 "
        "elements), u ~ U[-0.5,0.5] seeded; Jacobi CG rtol 1e-3, golden-section line search on [-0.5, 2], FP64",
        *_tri("gl", 1024, "fp64", sample_n=96), op="newton"),
    "he160x8x8_newton_fp64": Workload(
        "he160x8x8_newton_fp64", "he", "fp64", False, 4, 13, 8, False,
        "Newton to ||g|| <= 1e-6 ||g_0||: Neo-Hookean beam 160x8x8 hexes x 6 tets (61,440), E=10, nu=0.3, "
        "first load step (right face rotated by 4pi/24) from the reference configuration; Jacobi CG rtol 1e-2, "
        "golden-section line search on [-0.5, 2], FP64", *_he_newton(160, 8, 8, "fp64"), op="newton",
        newton_kw={"ksp_rtol": 1e-2, "ksp_max_it": 2000, "maxit": 200}),
    "gl1024_newton_fp32h": Workload(
        "gl1024_newton_fp32h", "gl", "fp32", True, 3, 7, 4, False,
        "Newton to ||g|| <= 1e-6 ||g_0||: Ginzburg-Landau 1024x1024 as gl1024_newton_fp64 with FP32 element "
        "gradients / Hessians (FP32 COO values in the CG), FP64 energy, state and CG arithmetic",
        *_tri("gl", 1024, "fp32", sample_n=96), op="newton"),
}
DEFAULT_WORKLOAD = "gl1024_fp64"

# The reference's own archived per-assembly timings at the 1024^2 GL grid
# (GL level 9, one MPI rank, one thread, JAX on the CPU; hardware not
# recorded): element Hessians 42.76 ms + np.add.at scatter 152.3 ms + COO
# insert 27.17 ms (total 229.9 ms) + gradient 37.4 ms, median per assembly,
# archive/results/raw_results_historical/experiment_results_cache/
# gl_final_suite/jax_petsc_element_l9_np1.json.
REFERENCE_ARCHIVED = {
    "gl": {"value": 2097152 / (0.2299 + 0.0374), "unit": "elements/s", "cores": 1,
           "what": "E+grad+Hess assembled into COO values (229.9 ms Hessian assembly + 37.4 ms gradient per pass), "
                   "reference JAX-CPU, one thread, archived run (gl_final_suite/jax_petsc_element_l9_np1.json), "
                   "hardware not recorded"},
}

KERNEL_NAMES = {1: "k_rows_tri", 2: "k_rows_tet", 3: "k_inc_tri", 4: "k_sweep_tri",
                5: "k_mc_elem+k_node_gather+k_rowgrad", 6: "k_mc_tc+k_fixup2+k_rowgrad", 7: "k_he_elem+k_node_gather",
                8: "k_push_tri", 9: "k_mc_dmma+k_fixup2+k_rowgrad", 10: "k_cluster_tri",
                11: "k_mc3d_elem+k_node_gather"}


def algorithmic_bytes(w, asm, n_el, energy_only=False):
    """Bytes one pass must move: node-level connectivity (int32), per-element
    geometry, the free state u (FP64), the load vector where the family has one,
    and -- unless energy only -- the owned gradient write (FP64) and the owned
    COO value write."""
    n_free = asm.layout.n_free
    nnz = int(asm.owned_values.numel())
    hb = 4 if w.hess_fp32 else 8
    b = n_el * (4 * w.conn_nodes + w.geom_bytes * w.geom_values) + n_free * 8
    if not energy_only:
        b += asm.n_owned * 8 + nnz * hb
    if w.has_rhs:
        b += asm.n_owned * 8
    return b


ENERGY_KERNELS = {"plaplace": "k_energy_tri", "gl": "k_energy_tri", "he": "k_energy_tet", "mc": "k_mc_eg",
                  "mc3d": "k_mc3d_elem (energy)"}


# ---------------------------------------------------------------------------
# CPU restatement (the oracle) on a bounded sample
# ---------------------------------------------------------------------------
def _oracle_sample(w, min_seconds=8.0, max_passes=5):
    import torch

    from oracle.assembler import OracleAssembler

    family, okw, params, u, n_el, label = w.sample()
    asm = OracleAssembler(family, params, **okw)
    u = u[asm.layout.perm]
    return asm, u, n_el, label, min_seconds, max_passes, int(torch.get_num_threads())


def cpu_mc3d_baseline(w, energy_only=False):
    """3-D Mohr-Coulomb: the oracle's element derivatives (the reference's
    density restated, stress and tangent by torch float64 autodiff through
    eigvalsh) over every element of a small slope, plus the np.add.at
    scatter of the element blocks."""
    import numpy as np
    import torch

    from oracle import energies3d as E3

    _, _, p, u_free, n_el, label = w.sample()
    u = p["u_0"].copy()
    u[p["freedofs"]] = u_free
    n = u.size

    def step():
        g, e_tot = np.zeros(n), 0.0
        vals = []
        for e in range(p["elems"].shape[0]):
            args = (p["dphix"][e], p["dphiy"][e], p["dphiz"][e], p["quad_weight"][e],
                    *[p[k][e] for k in ("c_bar", "sin_phi", "shear", "bulk", "lame")])
            if energy_only:
                eps = E3.strain6(u[p["elems"][e]], *args[:3])
                e_tot += float(np.sum(args[3] * E3.mc_density(eps, *args[4:])[0]))
                continue
            ee, ge, He, _ = E3.element_derivatives(u[p["elems"][e]], *args)
            e_tot += ee
            np.add.at(g, p["elems"][e], ge)
            vals.append(He)
        return e_tot

    t = time.perf_counter()
    step()
    dt = time.perf_counter() - t
    what = "energy passes" if energy_only else "fused E+grad+Hess passes (element derivatives + np.add.at)"
    return {"value": n_el / dt, "unit": "elements/s", "cores": int(torch.get_num_threads()), "kind": "port",
            "sample": f"{label} ({n_el} elements), 1 of the {what} of the CPU restatement",
            "seconds_per_pass": dt}


def cpu_port_baseline(w, energy_only=False):
    """The oracle (CPU restatement of the reference path) on a bounded sample."""
    if w.family == "mc3d":
        return cpu_mc3d_baseline(w, energy_only)
    asm, u, n_el, label, min_s, max_p, cores = _oracle_sample(w)
    step = (lambda: asm.energy_fn(u)) if energy_only else (lambda: asm.all_in_one(u))  # noqa: E731
    step()  # warm-up
    times = []
    while len(times) < (20 if energy_only else max_p) and sum(times) < min_s:
        t = time.perf_counter()
        step()
        times.append(time.perf_counter() - t)
    dt = sum(times) / len(times)
    what = ("energy passes of the CPU restatement (the reference element energy, NumPy float64)" if energy_only
            else "fused E+grad+Hess passes of the CPU restatement (torch.func float64 autodiff of the reference "
                 "element energy + np.add.at scatter)")
    return {"value": n_el / dt, "unit": "elements/s", "cores": cores, "kind": "port",
            "sample": f"{label} ({n_el} elements), {len(times)} {what}", "seconds_per_pass": dt}


def run_reference(args):
    world, rank, _ = _dist_setup()
    if rank != 0:
        return 0
    import torch

    torch.set_num_threads(os.cpu_count() or 1)
    w = WORKLOADS[args.workload]
    if w.family == "mc3d":  # the 3-D restatement: element loop of the oracle on a small slope
        times = [cpu_mc3d_baseline(w, args.pass_ == "energy") for _ in range(max(1, min(args.steps, 3)))]
        dt = sum(t["seconds_per_pass"] for t in times) / len(times)
        base = times[0]
        value = base["value"] * base["seconds_per_pass"] / dt
        print(json.dumps({
            "impl": "reference", "metric": "elements/s (energy)" if args.pass_ == "energy" else "elements/s (E+grad+Hess)",
            "value": value, "unit": "elements/s", "n_gpus": world, "steps": len(times), "warmup": 0,
            "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (closed-form state on the generated mesh)",
            "config": {"workload": w.name, "description": w.desc, "sample": base["sample"]},
            "cpu_baseline": dict(base, value=value),
            "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}),
            flush=True)
        return 0
    full = w.full is not None and w.op == "egh"
    if full:  # the whole configuration: one pass takes seconds on the host
        from oracle.assembler import OracleAssembler

        family, okw, params, u, _, label = w.full()
        asm = OracleAssembler(family, params, **okw)
        u = u[asm.layout.perm]
        n_el = int(asm.local.local_elem_idx.size)
    else:
        asm, u, n_el, label, _, _, _ = _oracle_sample(w)
    if w.op == "hvp":
        # the reference's "matfree_element" product: element Hessians of the
        # linearization point (computed once), then sum_e H_e x_e by np.add.at
        import numpy as np

        from oracle import energies

        v = asm.v_local(u)[asm.local.elems_local_np]
        _, _, H = energies.element_derivatives(asm.family, v, asm.elem_data, asm.params)
        x = np.random.default_rng(0).standard_normal(asm.layout.n_free)
        xf = np.asarray(asm.layout.total_to_free_reord)[asm.local.local_total_nodes]
        xl = np.zeros(xf.size)

        def step():  # tangent with zero Dirichlet part, element products, scatter
            xl[:] = 0.0
            xl[xf >= 0] = x[xf[xf >= 0]]
            ye = np.einsum("eij,ej->ei", H, xl[asm.local.elems_local_np])
            out = np.zeros(xl.size)
            np.add.at(out, asm.local.elems_local_np.ravel(), ye.ravel())
            return out
    elif w.op == "newton":
        from oracle.newton_cpu import newton_cpu

        def step():
            return newton_cpu(asm, u, tolg_rel=1e-6, **w.newton_kw)
    elif args.pass_ == "energy":
        def step():
            return asm.energy_fn(u)
    else:
        def step():
            return asm.all_in_one(u)
    for _ in range(min(args.warmup, 1) if w.op == "newton" else args.warmup):
        step()
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        step()
        times.append(time.perf_counter() - t)
    dt = sum(times) / len(times)
    newton_op = w.op == "newton"
    value, unit = (dt, "s") if newton_op else (n_el / dt, "elements/s")
    energy_op = w.op == "egh" and args.pass_ == "energy"
    metric = {"hvp": "elements/s (matrix-free H(u) x)", "newton": "Newton s to 1e-6 rel-grad"}.get(
        w.op, "elements/s (energy)" if energy_op else "elements/s (E+grad+Hess)")
    what = ("one Newton solve to 1e-6 relative gradient (oracle assembler, NumPy/SciPy Jacobi CG, the same "
            "golden-section line search)" if newton_op else
            "energy pass of the CPU restatement of the reference element energy" if energy_op else
            "CPU restatement of the reference JAX element kernels (torch.func float64 autodiff) + np.add.at scatter")
    if full:
        config = workload_config(w, n_el, asm.layout.n_free, asm.layout.owned_rows.size, world)
    else:
        config = {"workload": w.name, "description": w.desc, "sample": label, "elements_per_step": n_el}
    line = {
        "impl": "reference", "metric": metric, "value": value, "unit": unit,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": not newton_op, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded / closed-form state on the generated mesh)",
        "config": config,
        "cpu_baseline": {"value": value, "unit": unit, "cores": int(torch.get_num_threads()),
                         "kind": "port", "sample": f"{'full configuration' if full else 'sample'}: {label} "
                                                   f"({n_el} elements) per step; {what}"},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(w, n_el, n_free, nnz, world):
    """The workload's ``config`` object, identical in both arms."""
    return {"workload": w.name, "description": w.desc, "elements": int(n_el), "free_dofs": int(n_free),
            "coo_nnz": int(nnz), "l2": "flushed by a 1 GiB write between passes (outside the timed events)",
            "parallelism": f"{world} independent replica(s), one per GPU"}


# Mohr-Coulomb P4 meshes above this size are checked on sampled rows only.
ORACLE_FULL_LIMIT = {"mc4": 60_000}


def oracle_error(w, asm, u_host, e_dev, g_dev, h_dev):
    """Largest relative errors of one pass against the FP64 oracle on the
    same configuration: energy vs max(1, sum |e_e| + |load|), gradient and
    COO values vs their largest entry.  Returns (dict, oracle assembler or None)."""
    import numpy as np

    from oracle import energies
    from oracle.assembler import OracleAssembler, restricted_rows

    fam = w.family
    if fam == "mc3d":  # the autodiff oracle takes ~0.4 s per P2 element: checked by the parity tests instead
        return None, None
    okw = {"block_size": asm.block_size, "coordinate_key": asm.coordinate_key, "dirichlet_key": asm.dirichlet_key}
    params = dict(asm.params)
    g = g_dev[: asm.n_owned].double().cpu().numpy()
    h = h_dev.double().cpu().numpy()
    e = float(e_dev.item())
    lay = asm.layout
    t0 = time.perf_counter()

    def rel(a, b):
        return float(np.abs(a - b).max(initial=0.0) / max(np.abs(b).max(initial=0.0), 1e-300))

    if fam == "mc" and int(asm.npe) == 15 and asm.info["n_elem"] > ORACLE_FULL_LIMIT["mc4"]:
        from fenics_nonlinear_energies_b200 import meshes

        class _ElemB:
            def __getitem__(self, idx):
                return meshes.slope_elem_B({"dhat1": params["dhat1"], "dhat2": params["dhat2"],
                                            "inv_jac": params["inv_jac"][idx]})

        params["elem_B"] = _ElemB()
        rows = np.sort(np.random.default_rng(11).choice(np.arange(lay.lo, lay.hi), 400, replace=False))
        force = np.asarray(params["force"])[params["freedofs"]][lay.perm][lay.lo: lay.hi]
        g_ref, pos, h_ref = restricted_rows("mc", params, lay, u_host, rows, dirichlet_full=asm.dirichlet_full,
                                            f_owned=force)
        return {"energy": None, "grad": rel(g[rows - lay.lo], g_ref), "hess": rel(h[pos], h_ref),
                "scope": "400 sampled owned rows (all their gradient entries and COO values)",
                "oracle_s": time.perf_counter() - t0}, None
    if fam == "mc":
        from fenics_nonlinear_energies_b200 import meshes

        params["elem_B"] = meshes.slope_elem_B(params)
    orc = OracleAssembler(fam, params, layout=lay, **okw)
    if fam == "he":
        orc.update_dirichlet(asm.dirichlet_full)
    e_ref, g_ref, h_ref = orc.all_in_one(u_host)
    v = orc.v_local(u_host)[orc.local.elems_local_np]
    e_el, _, _ = energies.element_derivatives(fam, v, orc.elem_data, orc.params, want_hessian=False)
    load = abs(float(orc.f_owned @ u_host[lay.lo: lay.hi])) if orc.f_owned.size else 0.0
    scale = max(1.0, float(np.abs(e_el).sum()) + load + abs(orc.dirichlet_only_energy))
    return {"energy": abs(e - e_ref) / scale, "grad": rel(g, g_ref), "hess": rel(h, h_ref),
            "scope": "every owned gradient entry and COO value", "energy_scale": "sum |e_e| + |load|",
            "oracle_s": time.perf_counter() - t0}, orc


def cpu_fast_baseline(orc, u_host, n_el, label):
    """The numba-parallel CPU assembly on the full configuration."""
    from oracle.cpu_fast import FastTriangleAssembler

    fast = FastTriangleAssembler(orc)
    fast.all_in_one(u_host)  # compile + warm-up
    times = []
    while len(times) < 20 and sum(times) < 8.0:
        t = time.perf_counter()
        fast.all_in_one(u_host)
        times.append(time.perf_counter() - t)
    dt = statistics.median(times)
    return {"value": n_el / dt, "unit": "elements/s", "cores": fast.threads(), "kind": "port",
            "sample": f"full configuration ({label}, {n_el} elements), median of {len(times)} fused "
                      f"E+grad+Hess passes into the owned COO values: numba-parallel closed-form element "
                      f"derivatives + parallel fixed-order gathers on all host threads",
            "seconds_per_pass": dt}


# ---------------------------------------------------------------------------
# the CUDA path
# ---------------------------------------------------------------------------
def run_hvp(args, w, world, rank, local):
    """One step = one matrix-free H(u) x over every element (linearized once
    at the workload state outside the timed region)."""
    import numpy as np
    import torch

    from fenics_nonlinear_energies_b200 import _lib

    t_setup = time.perf_counter()
    asm, u0 = w.build(rank)
    t_setup = time.perf_counter() - t_setup
    n_el = int(asm.info["n_elem"])
    dev = torch.device("cuda", local)
    asm.prepare_matrix_free_operator(torch.as_tensor(u0, device=dev), mode="matfree_element")
    x = torch.as_tensor(np.random.default_rng(rank).standard_normal(asm.layout.n_free), device=dev)
    y = torch.empty(max(1, asm.n_owned), dtype=torch.float64, device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    h = asm._handle

    def step(xv):
        _lib.check(_lib.lib.fne_hvp(h, xv.data_ptr(), y.data_ptr(), stream.cuda_stream))

    for _ in range(args.warmup):
        step(x)
        flush.fill_(1.0)
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        _barrier(world)
        torch.cuda.synchronize()
        for i in range(args.steps):
            flush.fill_(float(i))
            evs[i][0].record(stream)
            step(x)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        _barrier(world)
    ms = [a.elapsed_time(b) for a, b in evs]
    total_s = _max_over_ranks(sum(ms) * 1e-3, world)
    value = world * n_el * args.steps / total_s
    # e2e: tangent H2D from pinned memory, product, D2H of the owned result
    pin_x = x.cpu().pin_memory()
    host_y = torch.empty(asm.n_owned, dtype=torch.float64).pin_memory()
    dx = torch.empty_like(x)
    e2e = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        flush.fill_(float(i))
        e2e[i][0].record(stream)
        dx.copy_(pin_x, non_blocking=True)
        step(dx)
        host_y.copy_(y[: asm.n_owned], non_blocking=True)
        e2e[i][1].record(stream)
    torch.cuda.synchronize()
    e2e_s = _max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e) * 1e-3, world)
    rsz = 4 if w.precision == "fp32" else 8
    nq = int(asm.params["quad_w"].size)
    n_dof_e = 2 * int(asm.npe)
    alg = n_el * (nq * 6 * rsz + 4 * n_dof_e + 8 * w.geom_values) + asm.layout.n_free * 8 + asm.n_owned * 8
    peak, peak_kind = _peaks()
    achieved = alg / (sum(ms) / len(ms) * 1e-3) / 1e9
    if rank == 0:
        line = {
            "metric": "elements/s (matrix-free H(u) x)", "value": value, "unit": "elements/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_s * 1e3 / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": w.dtype,
            "data": "synthetic (closed-form state, seeded tangent)",
            "config": {"workload": w.name, "description": w.desc, "elements": n_el, "free_dofs": asm.layout.n_free,
                       "setup_s": t_setup, "l2": "flushed by a 1 GiB write between products",
                       "parallelism": f"{world} independent replica(s), one per GPU"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": f"{peak_kind} burst copy (hbm_gbs)", "traffic": None,
                         "algorithmic_bytes_per_launch": alg, "kernel": "k_mc_hvp+k_rowgrad",
                         "launches_per_pass": 2},
            "e2e": {"value": world * n_el * args.steps / e2e_s, "unit": "elements/s",
                    "h2d_bytes_per_step": int(x.numel() * 8), "d2h_bytes_per_step": int(asm.n_owned * 8)},
            "gpu_launches": 2 * args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": None,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


class _CountingAssembler:
    """Forwards to an assembler and counts the kernels its evaluations launch."""

    def __init__(self, asm):
        self._asm = asm
        self.launches = 0

    def eval(self, u, flags, **kw):
        self.launches += self._asm.launches_per_eval(flags)
        return self._asm.eval(u, flags, **kw)

    def __getattr__(self, name):
        return getattr(self._asm, name)


def cpu_newton_baseline(w):
    """The CPU Newton (oracle assembler + scalar CG oracle) on the workload's bounded sample."""
    import numpy as np
    import torch

    from oracle.assembler import OracleAssembler
    from oracle.newton_cpu import newton_cpu

    family, okw, params, u, n_el, label = w.sample()
    asm = OracleAssembler(family, params, **okw)
    u = np.asarray(u)[np.asarray(asm.layout.perm)]
    times = []
    while len(times) < 5 and sum(times) < 8.0:  # repeated solves of the same start: at least ~8 s of work
        x, info = newton_cpu(asm, u, tolg_rel=1e-6, **w.newton_kw)
        times.append(info["time_s"])
    return {"value": sum(times) / len(times), "unit": "s", "cores": int(torch.get_num_threads()), "kind": "port",
            "sample": f"{label} ({n_el} elements): Newton solve to 1e-6 relative gradient on the host "
                      f"(oracle assembler, NumPy/SciPy CG, same line search), mean of {len(times)}: "
                      f"{info['iterations']} Newton, {info['ksp_its']} CG iterations, converged={info['converged']}",
            "newton_iterations": info["iterations"], "ksp_iterations": info["ksp_its"]}


def run_newton(args, w, world, rank, local):
    """One step = one Newton solve from the workload's seeded start to
    ||g|| <= 1e-6 ||g_0|| on the device: assembly kernels, the device CG
    (fne_cg_*) and the golden-section line search, host logic in between."""
    import numpy as np
    import torch

    from fenics_nonlinear_energies_b200.newton import DeviceCG, newton

    t_setup = time.perf_counter()
    asm, u0 = w.build(rank)
    t_setup = time.perf_counter() - t_setup
    n_el = int(asm.info["n_elem"])
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    cg = DeviceCG.for_assembler(asm)
    casm = _CountingAssembler(asm)
    kw = dict(tolg_rel=1e-6, cg=cg, **w.newton_kw)
    u = torch.as_tensor(u0, device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        newton(casm, u, **kw)
        flush.fill_(1.0)
    torch.cuda.synchronize()
    casm.launches, cg.launches = 0, 0
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    e2e = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    pin_u = torch.from_numpy(np.ascontiguousarray(u0)).pin_memory()
    host_x = torch.empty(asm.n_owned, dtype=torch.float64).pin_memory()
    infos = []
    # The solve is host-driven (line-search decisions, one read per CG graph),
    # so both timed loops run under the same clock sampling load on the host.
    with ClockSampler(local) as clk:
        _barrier(world)
        torch.cuda.synchronize()
        for i in range(args.steps):
            flush.fill_(float(i))
            evs[i][0].record(stream)
            x, info = newton(casm, u, **kw)
            evs[i][1].record(stream)
            infos.append(info)
        torch.cuda.synchronize()
        _barrier(world)
        launches = casm.launches + cg.launches
        # e2e: start vector H2D from pinned memory, the solve, D2H of the solution
        for i in range(args.steps):
            flush.fill_(float(i))
            e2e[i][0].record(stream)
            du = pin_u.to(dev, non_blocking=True)
            x, _ = newton(casm, du, **kw)
            host_x.copy_(x, non_blocking=True)
            e2e[i][1].record(stream)
        torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in evs]
    total_s = _max_over_ranks(sum(ms) * 1e-3, world)
    s_per_solve = total_s / args.steps
    e2e_s = _max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e) * 1e-3, world) / args.steps

    # roofline of the dominant kernel pair (one CG iteration: k_cg_spmv +
    # k_cg_update) on the Hessian at the solution, timed on its own
    from fenics_nonlinear_energies_b200 import _lib

    asm.eval(x, _lib.FNE_HESS)
    cg.update(asm.owned_values)
    b = torch.as_tensor(np.random.default_rng(rank).standard_normal(asm.n_owned), device=dev)
    cg.solve(b, rtol=0.0, maxit=64)
    flush.fill_(2.0)
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    _, cg_its = cg.solve(b, rtol=0.0, maxit=CG_TIMED_ITERATIONS)
    c1.record(stream)
    torch.cuda.synchronize()
    us_it = c0.elapsed_time(c1) * 1e3 / max(1, cg_its)
    n, nnz = asm.n_owned, int(asm.owned_values.numel())
    vb = asm.owned_values.element_size()
    alg = nnz * (vb + 4) + (n + 1) * 4 + 12 * n * 8
    peak, peak_kind = _peaks()
    achieved = alg / (us_it * 1e-6) / 1e9
    traffic = NCU_TRAFFIC.get((w.name, "k_cg_spmv+k_cg_update"))
    its = [i["iterations"] for i in infos]
    ksp = [sum(h["ksp_its"] for h in i["history"]) for i in infos]
    if rank == 0:
        cpu = cpu_newton_baseline(w) if (world == 1 and not args.no_cpu_baseline) else None
        line = {
            "metric": "Newton s to 1e-6 rel-grad", "value": s_per_solve, "unit": "s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": s_per_solve * 1e3,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": w.dtype,
            "data": "synthetic (seeded start on the generated mesh)",
            "config": {"workload": w.name, "description": w.desc, "elements": n_el, "free_dofs": asm.layout.n_free,
                       "coo_nnz": nnz, "newton_iterations": its, "cg_iterations": ksp,
                       "converged": [bool(i["converged"]) for i in infos], "energy": infos[-1]["energy"],
                       "solves_per_s_all_gpus": world / s_per_solve, "setup_s": t_setup,
                       "l2": "flushed by a 1 GiB write between solves",
                       "parallelism": f"{world} independent replica(s), one per GPU"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": f"{peak_kind} burst copy (hbm_gbs)",
                         "traffic": traffic[0] if traffic else None,
                         "traffic_source": traffic[1] if traffic else None,
                         "algorithmic_bytes_per_launch": alg, "kernel": "k_cg_spmv+k_cg_update",
                         "unit_of_launch": "one CG iteration (two kernels)", "us_per_cg_iteration": us_it,
                         "cg_iterations_timed": cg_its},
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": int(u0.nbytes),
                    "d2h_bytes_per_step": int(host_x.numel() * 8)},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    cg.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def run(args):
    import numpy as np
    import torch

    world, rank, local = _dist_setup()
    torch.cuda.set_device(local)
    from fenics_nonlinear_energies_b200 import _lib

    w = WORKLOADS[args.workload]
    if w.op == "hvp":
        return run_hvp(args, w, world, rank, local)
    if w.op == "newton":
        return run_newton(args, w, world, rank, local)
    t_setup = time.perf_counter()
    asm, u0 = w.build(rank)
    t_setup = time.perf_counter() - t_setup
    n_el = int(asm.info["n_elem"])
    dev = torch.device("cuda", local)
    u = torch.as_tensor(u0, device=dev)
    energy_only = args.pass_ == "energy"
    flags = _lib.FNE_ENERGY if energy_only else _lib.FNE_ENERGY | _lib.FNE_GRAD | _lib.FNE_HESS
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    launches_per_pass = asm.launches_per_eval(flags)

    for _ in range(args.warmup):
        asm.eval(u, flags)
        flush.fill_(1.0)
    torch.cuda.synchronize()

    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local) as clk:
        _barrier(world)
        torch.cuda.synchronize()
        for i in range(args.steps):
            flush.fill_(float(i))
            evs[i][0].record(stream)
            asm.eval(u, flags)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        _barrier(world)
    kernel_ms = [a.elapsed_time(b) for a, b in evs]
    total_s = _max_over_ranks(sum(kernel_ms) * 1e-3, world)
    value = world * n_el * args.steps / total_s
    ms_step = total_s * 1e3 / args.steps
    energy = float(asm.eval(u, flags)[0].item())

    # end to end through the public API with host buffers
    pin_u = torch.from_numpy(np.ascontiguousarray(u0)).pin_memory()
    host_g = torch.empty(asm.n_owned, dtype=torch.float64).pin_memory()
    host_h = torch.empty(asm.owned_values.numel(), dtype=asm.owned_values.dtype).pin_memory()
    host_e = torch.empty(1, dtype=torch.float64).pin_memory()
    dev_u = torch.empty_like(u)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    def e2e_pass():
        dev_u.copy_(pin_u, non_blocking=True)
        e, g, h = asm.eval(dev_u, flags)
        host_e.copy_(e, non_blocking=True)
        if not energy_only:
            host_g.copy_(g, non_blocking=True)
            host_h.copy_(h, non_blocking=True)

    for _ in range(args.warmup):
        e2e_pass()
    torch.cuda.synchronize()
    _barrier(world)
    for i in range(args.steps):
        flush.fill_(float(i))
        e2e_ev[i][0].record(stream)
        e2e_pass()
        e2e_ev[i][1].record(stream)
    torch.cuda.synchronize()
    e2e_s = _max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_ev) * 1e-3, world)
    e2e_value = world * n_el * args.steps / e2e_s

    # roofline of the pass (one kernel launch per pass for the P1 families)
    alg_bytes = algorithmic_bytes(w, asm, n_el, energy_only)
    peak, peak_kind = _peaks()
    avg_launch_s = (sum(kernel_ms) / len(kernel_ms)) * 1e-3
    achieved = alg_bytes / avg_launch_s / 1e9
    kname = ENERGY_KERNELS[w.family] if energy_only else KERNEL_NAMES.get(asm.info["kernel_variant"], "?")
    traffic = NCU_TRAFFIC.get((w.name, kname))
    nnz = int(asm.owned_values.numel())

    cpu, err, extra = None, None, {}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        orc = None
        if not energy_only:  # accuracy of this pass against the FP64 oracle (outside the timed region)
            e_d, g_d, h_d = asm.eval(u, flags)
            torch.cuda.synchronize()
            err, orc = oracle_error(w, asm, np.asarray(u0, dtype=np.float64), e_d, g_d, h_d)
        if orc is not None and w.family in ("gl", "plaplace") and w.full is not None:
            cpu = cpu_fast_baseline(orc, np.asarray(u0, dtype=np.float64), n_el, w.full()[5])
            extra["cpu_baseline_autodiff"] = cpu_port_baseline(w)
            if w.family in REFERENCE_ARCHIVED and n_el >= 2_000_000:
                extra["reference_archived"] = REFERENCE_ARCHIVED[w.family]
        else:
            cpu = cpu_port_baseline(w, energy_only)
    if rank == 0:
        line = {
            "metric": "elements/s (energy)" if energy_only else "elements/s (E+grad+Hess)", "value": value,
            "unit": "elements/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": w.dtype,
            "data": "synthetic (seeded / closed-form state on the generated mesh)",
            "config": workload_config(w, n_el, asm.layout.n_free, nnz, world),
            "details": {"energy": energy, "setup_s": t_setup},
            "error_vs_fp64_oracle": err,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": f"{peak_kind} burst copy (hbm_gbs)",
                         "traffic": traffic[0] if traffic else None,
                         "traffic_source": traffic[1] if traffic else None,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "kernel": kname, "kernel_variant": args.kernel_variant,
                         "launches_per_pass": launches_per_pass},
            "e2e": {"value": e2e_value, "unit": "elements/s",
                    "h2d_bytes_per_step": int(u0.nbytes),
                    "d2h_bytes_per_step": 8 if energy_only else
                    int(8 + host_g.numel() * 8 + host_h.numel() * host_h.element_size())},
            "gpu_launches": args.steps * launches_per_pass,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
            **extra,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--pass", dest="pass_", default="egh", choices=["egh", "energy"],
                    help="egh: fused energy + gradient + Hessian pass (default); energy: the energy-only pass "
                         "(the line-search callback)")
    ap.add_argument("--kernel-variant", default="auto", choices=["auto", "sweep", "cluster", "row_gather", "incidence", "element", "cuda_cores",
                                                                  "push", "row_lanes_2", "row_lanes_4", "row_lanes_8"])
    args = ap.parse_args()
    KERNEL_VARIANT["value"] = args.kernel_variant
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run(args)


if __name__ == "__main__":
    sys.exit(main())
