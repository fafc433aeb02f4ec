"""Build ``libfne_asm.so`` in-tree with nvcc for sm_100a.

``python -m fenics_nonlinear_energies_b200.build [--verbose]``
"""

from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libfne_asm.so"
SOURCES = ["fne_asm.cu", "fne_mc.cu", "fne_mc3d.cu", "fne_mlp.cu", "fne_krylov.cu", "fne_layout_dev.cu", "fne_plan.cpp", "fne_layout.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def sources():
    return [CSRC / s for s in SOURCES if (CSRC / s).exists()]


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(sources()) + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "fne_asm.h"]
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def _run(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + " ".join(cmd) + "\n" + res.stdout + res.stderr)
    return res.stdout + res.stderr


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile every translation unit to an object (in parallel), then link
    the shared library.  Objects go to a temporary folder."""
    import tempfile
    from concurrent.futures import ThreadPoolExecutor

    if not force and not needs_build():
        return LIB
    flags = [_nvcc(), "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC,-O3", "-Xptxas=-warn-spills"]
    if verbose:
        flags.append("-Xptxas=-v")
    with tempfile.TemporaryDirectory(prefix="fne_build_") as tmp:
        objs = [Path(tmp) / (src.stem + ".o") for src in sources()]
        cmds = [flags + ["-c", str(src), "-o", str(obj)] for src, obj in zip(sources(), objs)]
        with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
            logs = list(ex.map(_run, cmds))
        logs.append(_run([_nvcc(), *ARCH, "-shared", "-o", str(LIB), *map(str, objs)]))
    if verbose:
        sys.stdout.write("".join(logs))
    return LIB


if __name__ == "__main__":
    build(verbose="--verbose" in sys.argv, force=True)
    print(LIB)
