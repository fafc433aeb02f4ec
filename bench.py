"""Benchmark: fused energy + gradient + Hessian assembly, elements/s.

Workload (one "step"): Ginzburg-Landau, eps = 0.01 on [-1, 1]^2, structured
1024 x 1024 grid of P1 triangles (2,097,152 elements, 1,046,529 free DOFs,
7,317,521 owned COO entries), u ~ U[-0.5, 0.5] from a fixed seed; FP32
element gradients / Hessians (float32 COO values), FP64 energy reduction.
One step = one fused E+grad+Hess pass over every element into the device
gradient and the owned COO values (the reference's energy_fn + gradient_fn +
assemble_hessian_element).

``value``: device-resident inputs, CUDA events around each pass, L2 flushed
(256 MiB write) between passes outside the timed events.
``e2e``: the same pass through the public assembler API with host buffers:
H2D of u from pinned memory, the pass, D2H of energy, gradient and COO values.

Multi-GPU: every rank runs its own replica of the workload (weak scaling).
``--impl reference``: the CPU restatement of the reference path (the JAX
element kernels + np.add.at scatter, restated in oracle/) on the host cores.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

GRID = 1024
WORKLOAD = "ginzburg_landau_p1_1024x1024_fp32hess"


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def _traffic_per_launch():
    p = ROOT / "profiles" / "k_rows_tri_gl_fp32_traffic.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["dram_bytes_per_launch"])
        except Exception:
            return None
    return None


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = ROOT / "gpurun_out" / f"clocks_bench_{os.getpid()}.csv"

    def __enter__(self):
        try:
            self.path.parent.mkdir(exist_ok=True)
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


def cpu_port_baseline(grid=512, passes=3):
    """The oracle (CPU restatement of the reference path) on a bounded sample."""
    import torch

    from oracle.assembler import OracleAssembler
    from fenics_nonlinear_energies_b200 import meshes

    params, u0 = meshes.gl_problem(n=grid, seed=0)
    asm = OracleAssembler("gl", params)
    asm.all_in_one(u0)  # warm-up
    t = time.perf_counter()
    for _ in range(passes):
        asm.all_in_one(u0)
    dt = (time.perf_counter() - t) / passes
    n_el = 2 * grid * grid
    return {"value": n_el / dt, "unit": "elements/s", "cores": int(torch.get_num_threads()), "kind": "port",
            "sample": f"GL {grid}x{grid} P1 grid ({n_el} elements), {passes} fused E+grad+Hess passes, "
                      "torch.func float64 autodiff + np.add.at scatter",
            "seconds_per_pass": dt}


def run_reference(args):
    world, rank, _ = _dist_setup()
    if rank != 0:
        return 0
    import torch

    torch.set_num_threads(os.cpu_count() or 1)
    grid = 512
    from oracle.assembler import OracleAssembler
    from fenics_nonlinear_energies_b200 import meshes

    params, u0 = meshes.gl_problem(n=grid, seed=0)
    asm = OracleAssembler("gl", params)
    for _ in range(args.warmup):
        asm.all_in_one(u0)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        asm.all_in_one(u0)
        times.append(time.perf_counter() - t)
    n_el = 2 * grid * grid
    dt = sum(times) / len(times)
    value = n_el / dt
    line = {
        "impl": "reference", "metric": "elements/s (E+grad+Hess)", "value": value, "unit": "elements/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "sample_grid": f"{grid}x{grid}", "elements_per_step": n_el},
        "cpu_baseline": {"value": value, "unit": "elements/s", "cores": int(torch.get_num_threads()),
                         "kind": "port",
                         "sample": f"GL {grid}x{grid} P1 grid ({n_el} elements) per step; CPU restatement of the "
                                   "reference JAX element kernels (torch.func float64 autodiff) + np.add.at scatter"},
        "e2e": {"value": value, "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run(args):
    import torch

    world, rank, local = _dist_setup()
    torch.cuda.set_device(local)
    from fenics_nonlinear_energies_b200 import _lib
    from fenics_nonlinear_energies_b200.assembler import GLCudaAssembler
    from fenics_nonlinear_energies_b200 import meshes

    params, u0 = meshes.gl_problem(n=GRID, seed=rank)
    asm = GLCudaAssembler(params, precision="fp32", hess_dtype=torch.float32)
    n_el = int(params["elems"].shape[0])
    dev = torch.device("cuda", local)
    u = torch.as_tensor(u0, device=dev)
    flags = _lib.FNE_ENERGY | _lib.FNE_GRAD | _lib.FNE_HESS
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)

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

    # end to end through the public API with host buffers
    pin_u = torch.from_numpy(u0).pin_memory()
    host_g = torch.empty(asm.n_owned, dtype=torch.float64).pin_memory()
    host_h = torch.empty(asm.owned_values.numel(), dtype=torch.float32).pin_memory()
    host_e = torch.empty(1, dtype=torch.float64).pin_memory()
    dev_u = torch.empty_like(u)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for _ in range(args.warmup):
        dev_u.copy_(pin_u, non_blocking=True)
        e, g, h = asm.eval(dev_u, flags)
        host_e.copy_(e, non_blocking=True), host_g.copy_(g, non_blocking=True), host_h.copy_(h, non_blocking=True)
    torch.cuda.synchronize()
    _barrier(world)
    for i in range(args.steps):
        flush.fill_(float(i))
        e2e_ev[i][0].record(stream)
        dev_u.copy_(pin_u, non_blocking=True)
        e, g, h = asm.eval(dev_u, flags)
        host_e.copy_(e, non_blocking=True)
        host_g.copy_(g, non_blocking=True)
        host_h.copy_(h, non_blocking=True)
        e2e_ev[i][1].record(stream)
    torch.cuda.synchronize()
    e2e_s = _max_over_ranks(sum(a.elapsed_time(b) for a, b in e2e_ev) * 1e-3, world)
    e2e_value = world * n_el * args.steps / e2e_s

    # roofline of the fused row-gather kernel (one launch per step)
    n_free = asm.layout.n_free
    nnz = int(asm.owned_values.numel())
    alg_bytes = n_el * (3 * 4 + 7 * 4) + n_free * 8 + asm.n_owned * 8 + nnz * 4
    peak, peak_kind = _peaks()
    avg_launch_s = (sum(kernel_ms) / len(kernel_ms)) * 1e-3
    achieved = alg_bytes / avg_launch_s / 1e9
    traffic = _traffic_per_launch()

    if rank == 0:
        cpu = cpu_port_baseline() if (world == 1 and not args.no_cpu_baseline) else None
        line = {
            "metric": "elements/s (E+grad+Hess)", "value": value, "unit": "elements/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (element grad/Hessian), f64 (energy)",
            "data": "synthetic (seeded U[-0.5,0.5] initial guess on the structured grid)",
            "config": {"workload": WORKLOAD, "elements": n_el, "free_dofs": n_free, "coo_nnz": nnz,
                       "l2": "flushed by a 256 MiB write between passes (outside the timed events)",
                       "parallelism": f"{world} independent replica(s), one per GPU"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": f"{peak_kind} burst copy",
                         "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
                         "kernel": {1: "k_rows_tri", 2: "k_rows_tet", 3: "k_inc_tri",
                                    4: "k_sweep_tri"}.get(asm.info["kernel_variant"], "?")
                                   + "<float, GL, E|G|H, float>"},
            "e2e": {"value": e2e_value, "unit": "elements/s",
                    "h2d_bytes_per_step": int(u0.nbytes),
                    "d2h_bytes_per_step": int(8 + host_g.numel() * 8 + host_h.numel() * 4)},
            "gpu_launches": args.steps,
            "clocks": clk.summary(),
            "cpu_baseline": cpu,
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
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run(args)


if __name__ == "__main__":
    sys.exit(main())
