"""bench.py bookkeeping on the CPU: algorithmic byte counts of the fused and
the energy-only passes, the workload table, and the reference arm's JSON
line for a small Newton workload sample."""

import json
import os
import subprocess
import sys
from types import SimpleNamespace

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _fake_asm(n_free, n_owned, nnz):
    return SimpleNamespace(layout=SimpleNamespace(n_free=n_free), n_owned=n_owned,
                           owned_values=SimpleNamespace(numel=lambda: nnz))


def test_algorithmic_bytes_fused_and_energy_only():
    import bench

    w = bench.WORKLOADS["gl1024_fp32h"]
    n_el, n_free, nnz = 2_097_152, 1_046_529, 7_317_521
    asm = _fake_asm(n_free, n_free, nnz)
    # connectivity (3 int32) + geometry (7 FP32) per element, u, grad write, FP32 COO values
    fused = n_el * (3 * 4 + 7 * 4) + n_free * 8 + n_free * 8 + nnz * 4
    assert bench.algorithmic_bytes(w, asm, n_el) == fused
    assert bench.algorithmic_bytes(w, asm, n_el, energy_only=True) == n_el * 40 + n_free * 8
    wp = bench.WORKLOADS["plaplace128_fp64"]  # has a load vector: read in both passes
    a2 = _fake_asm(16_129, 16_129, 111_889)
    assert bench.algorithmic_bytes(wp, a2, 32_768, energy_only=True) == 32_768 * (12 + 56) + 2 * 16_129 * 8


def test_workload_table():
    import bench

    for name, w in bench.WORKLOADS.items():
        assert w.name == name and w.op in ("egh", "hvp", "newton")
        assert callable(w.build) and callable(w.sample)
        if w.op == "newton":
            assert set(w.newton_kw) <= {"ksp_rtol", "ksp_max_it", "maxit", "linesearch_tol", "tolf"}
    assert bench.DEFAULT_WORKLOAD == "gl1024_fp64"
    assert bench.WORKLOADS[bench.DEFAULT_WORKLOAD].dtype == "f64"
    assert bench.KERNEL_NAMES[9] == "k_mc_dmma+k_fixup2+k_rowgrad"
    assert bench.ENERGY_KERNELS["mc"] == "k_mc_eg"
    for name in ("gl1024_fp64", "gl1024_fp32h", "plaplace128_fp64", "he160x8x8_fp64"):
        assert bench.WORKLOADS[name].full is not None, name
    assert set(bench.ENERGY_KERNELS) == {"plaplace", "gl", "he", "mc", "mc3d"}
    assert bench.KERNEL_NAMES[11] == "k_mc3d_elem+k_node_gather"


@pytest.mark.timeout(600)
def test_reference_arm_line_for_newton_sample(tmp_path):
    """--impl reference prints one JSON line with the contract's keys (CPU Newton over the oracle)."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "gl1024_newton_fp64", "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                         cwd=tmp_path, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference" and line["unit"] == "s" and line["higher_is_better"] is False
    assert line["metric"] == "Newton s to 1e-6 rel-grad" and line["value"] > 0
    for key in ("cpu_baseline", "e2e", "config", "n_gpus", "steps", "warmup", "ms_per_step"):
        assert key in line


@pytest.mark.timeout(600)
def test_reference_arm_runs_the_full_configuration(tmp_path):
    """For P1 workloads the reference arm times the whole configuration and
    prints the same ``config`` object the CUDA arm prints."""
    import bench
    from oracle.assembler import OracleAssembler

    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "plaplace128_fp64", "--steps", "2", "--warmup", "1"], capture_output=True, text=True,
                         cwd=tmp_path, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    w = bench.WORKLOADS["plaplace128_fp64"]
    family, okw, params, _, _, _ = w.full()
    orc = OracleAssembler(family, params, **okw)
    n_el = int(orc.local.local_elem_idx.size)
    assert line["config"] == bench.workload_config(w, n_el, orc.layout.n_free, orc.layout.owned_rows.size, 1)
    # elements with a free DOF (the two corner triangles have none), owned COO entries
    assert line["config"]["elements"] == 32_766 and line["config"]["coo_nnz"] == 111_889
    assert line["cpu_baseline"]["sample"].startswith("full configuration")


@pytest.mark.timeout(300)
@pytest.mark.parametrize("workload", ["mc3d_p2_fp64", "mc3d_p4_fp64"])
def test_reference_arm_line_for_mc3d(tmp_path, workload):
    """--impl reference on the 3-D Mohr-Coulomb workloads (P2, P4 tets): the
    oracle's element loop on a small slope."""
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          workload, "--steps", "1", "--warmup", "0"], capture_output=True, text=True,
                         cwd=tmp_path, timeout=300)
    assert out.returncode == 0, out.stderr[-2000:]
    line = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference" and line["unit"] == "elements/s" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and line["e2e"]["h2d_bytes_per_step"] == 0
    assert line["config"]["workload"] == workload
