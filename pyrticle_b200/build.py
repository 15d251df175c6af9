"""Builds libprt.so (sm_100a) in-tree with nvcc, and the CPU oracle with make.

Usage: ``python -m pyrticle_b200.build [--oracle]``.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libprt.so"
SOURCES = ["core.cu", "deposit.cu", "deposit_tc.cu", "grid.cu", "adjoint.cu", "stage_mixed.cu", "diagnostics.cu", "average.cu"]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC", "-shared",
    "--expt-relaxed-constexpr",
    "-Xptxas", "-warn-spills",
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: cannot build libprt.so")
    return cand


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build_lib(force: bool = False, verbose: bool = False, extra=()) -> Path:
    deps = [CSRC / s for s in SOURCES] + list(CSRC.glob("*.cuh")) + [ROOT / "include" / "prt.h"]
    if not force and not _stale(LIB, deps):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-I", str(ROOT / "include"),
           "-o", str(tmp), *[str(CSRC / s) for s in SOURCES]]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True, cwd=str(CSRC))
    os.replace(tmp, LIB)
    return LIB


def build_oracle(force: bool = False) -> None:
    odir = ROOT / "oracle"
    if force:
        subprocess.run(["make", "-C", str(odir), "clean"], check=True)
    subprocess.run(["make", "-C", str(odir)], check=True, stdout=subprocess.DEVNULL)


if __name__ == "__main__":
    build_lib(force="--force" in sys.argv, verbose=True)
    if "--oracle" in sys.argv:
        build_oracle(force="--force" in sys.argv)
