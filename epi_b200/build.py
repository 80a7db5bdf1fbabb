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
# the bounds-checked build (-DEPI_CHECK): every index derived from stored data
# is checked before use (EPI_ERR_CHECK); for tests, not for timing
LIB_CHECK = PKG / "libepi_mech_check.so"

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


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("nvcc failed:\n" + r.stderr[-6000:])
    return r.stderr


def build_library(force: bool = False, verbose: bool = False, check: bool = False) -> Path:
    """Compiles the translation units in parallel (one nvcc each), then links
    them into the shared library."""
    from concurrent.futures import ThreadPoolExecutor
    out = LIB_CHECK if check else LIB
    if not force and not _stale(out):
        return out
    extra = (("-Xptxas", "-v") if verbose else ()) + (("-DEPI_CHECK",) if check else ())
    objdir = PKG / "_build" / ("check" if check else "release")
    objdir.mkdir(parents=True, exist_ok=True)
    common = [nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
              "-I", str(ROOT / "include"), "-I", str(CSRC), *extra]
    jobs = [(common + ["-c", str(CSRC / src), "-o", str(objdir / (src + ".o"))])
            for src in SOURCES]
    with ThreadPoolExecutor(max_workers=len(jobs)) as ex:
        logs = list(ex.map(_run, jobs))
    _run([nvcc(), *ARCH, "--shared", "-o", str(out),
          *[str(objdir / (src + ".o")) for src in SOURCES]])
    if verbose:
        print("".join(logs))
    return out


if __name__ == "__main__":
    build_library(force=True, verbose=True)
