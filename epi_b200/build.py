"""Builds libepi_mech.so in-tree for sm_100a with nvcc.

The library is the product: hand-written CUDA kernels plus the C ABI declared
in include/epi_mech.h. It links the CUDA runtime statically so the .so
carries no dependency beyond the driver.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "libepi_mech.so"

SOURCES = ["epi_kernels.cu", "epi_adjoint.cu", "epi_field.cu", "epi_capi.cu", "epi_noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def compile_command(out: Path = LIB, extra=()) -> list:
    return [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "--shared",
            "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"), "-I", str(CSRC),
            *extra, "-o", str(out), *[str(CSRC / s) for s in SOURCES]]


def _stale(out: Path) -> bool:
    if not out.exists():
        return True
    deps = list(CSRC.glob("*")) + [ROOT / "include" / "epi_mech.h", Path(__file__)]
    return out.stat().st_mtime < max(p.stat().st_mtime for p in deps)


def build_library(force: bool = False, verbose: bool = False) -> Path:
    if not force and not _stale(LIB):
        return LIB
    cmd = compile_command(LIB, ("-Xptxas", "-v") if verbose else ())
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stderr[-6000:])
    if verbose:
        print(r.stderr)
    return LIB


if __name__ == "__main__":
    build_library(force=True, verbose=True)
