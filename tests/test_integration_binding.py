"""The drop-in subclass of INTEGRATION.md section 1, run as written under the
reference's own assembler classes (CPU; needs the reference sources, so it
is skipped where they are absent).

``integration_binding_driver.py`` executes the documented code block, builds
every family's unmodified reference assembler and the mixin assembler on the
same reference-fixture problems (1 and 2 ranks), and reports both sides.
The library is a stand-in that computes ``fne_eval`` from the descriptor
the mixin fills, so this checks the binding -- construction through the
reference's ``__init__`` and ``_warmup``, the descriptor contents, the
callbacks, ``setValuesCOO`` and the timing records -- not the CUDA kernels
(the GPU tests cover those against the same fixtures).
"""

import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
REFERENCE = Path(os.environ.get("FNE_REFERENCE_ROOT", "/root/reference"))


@pytest.mark.skipif(not (REFERENCE / "src" / "core" / "petsc" / "reordered_element_base.py").exists(),
                    reason="reference sources not present")
@pytest.mark.timeout(600)
def test_integration_subclass_runs_under_the_reference_base_class():
    out = subprocess.run([sys.executable, str(ROOT / "tests" / "integration_binding_driver.py"), str(REFERENCE)],
                         capture_output=True, text=True, timeout=600, cwd=str(ROOT))
    assert out.returncode == 0, out.stderr[-3000:]
    rep = json.loads([l for l in out.stdout.splitlines() if l.startswith("{")][-1])
    res = rep["results"]
    assert {r["case"] for r in res} == {"gl", "plaplace", "he", "mc_p2"}
    assert any(r["size"] == 2 for r in res)
    for r in res:
        e_ref, e_cuda = r["energy"]
        assert abs(e_cuda - e_ref) <= 1e-12 * max(1.0, abs(e_ref)), r
        assert r["grad_rel"] <= 1e-12 and r["hess_rel"] <= 1e-12, r
        assert r["coo_inserts"] == [1, 1], r
        assert r["timing_keys_missing"] == [], r
        assert r["iter_timings"] == [1, 1] and r["iter_timings_last_is_returned"], r
        assert r["callback_calls"][0] == r["callback_calls"][1], r
        assert not any(r["callback_keys_missing"].values()), r
        assert r["jit_stub_raises"], r
    assert rep["finite"]
    calls = rep["calls"]
    assert calls["create"] == len(res) and calls["destroy"] == len(res)
    assert calls["set_dirichlet"] >= sum(1 for r in res if r["case"] == "he")
