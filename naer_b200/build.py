"""Builds the CUDA library of the package in-tree: naer_b200/libnaer_b200.so.

All device code is compiled for sm_100a only (B200).  Run as
`python -m naer_b200.build` or call `build()`.
"""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libnaer_b200.so"
# the same sources with every computed global index bounds-checked (NAER_CHECKED)
LIB_CHECKED = PKG / "libnaer_b200_checked.so"

SOURCES = ["sim_kernels.cu", "build_kernels.cu", "engine.cu", "forms.cu", "probe.cu", "capi.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "--fmad=false",            # fp32 arithmetic repeated bit-for-bit by the oracle
    "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden",
    "-shared",
]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    return cand if Path(cand).exists() else "nvcc"


def _stale(lib: Path = LIB) -> bool:
    if not lib.exists():
        return True
    t = lib.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h"))
    deps += list((PKG.parent / "include" / "naer").glob("*.h"))
    return any(p.stat().st_mtime > t for p in deps)


def build(force: bool = False, verbose: bool = False, checked: bool = False) -> Path:
    """Builds libnaer_b200.so, or with checked=True libnaer_b200_checked.so
    (NAER_CHECKED: every global access at a computed index is checked
    against its buffer; violations are recorded, not made)."""
    lib = LIB_CHECKED if checked else LIB
    if not force and not _stale(lib):
        return lib
    tmp = lib.with_suffix(".so.tmp")
    extra = os.environ.get("NAER_NVCC_FLAGS", "").split()  # tuning sweeps, e.g. -DNAER_RUN_MIN_BLOCKS=3
    if checked:
        extra.append("-DNAER_CHECKED")
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-o", str(tmp), *[str(CSRC / s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=str(PKG))
    os.replace(tmp, lib)
    return lib


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True, checked="--checked" in sys.argv))
