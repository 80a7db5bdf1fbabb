"""Build recipe for the compiled reference oracle (test infrastructure only).

Compiles the UNMODIFIED epi5_MT mechanics sources, where they lie under the
reference checkout, together with oracle/ref_harness.cpp and the project's TBB
stand-in (oracle/tbb_shim). Nothing from the reference is copied into the
repository; every output goes to oracle/_ref/ (git-ignored, shipped to the GPU
host with the other built files).

epi5_MT fixes its geometry at compile time (epi5_MT/define.h:66-99: TRI_MEMB,
NMX, NMY, LX, LY, LZ, MAX_CELL_NUM). For each geometry this script writes a
constant overlay of define.h into oracle/_ref/<geometry>/define.h -- the same
header with only those constants changed and TRI_MEMB undefined (square
membrane) -- and force-includes it. Because it defines the DEFINE_H guard, the
reference's own define.h then contributes nothing. No other source is altered.

Two variants per geometry:
  serial : TBB loops run in index order; -O2 -ffp-contract=off. This is the
           deterministic FP64 oracle.
  omp    : TBB loops become OpenMP loops; -O3 -march=x86-64-v3. This is the
           timed CPU baseline (AVX2/FMA level so the binary runs on any
           current x86 host).

A third variant, built on request (it needs epi_b200/libepi_mech.so):
  dropin : the same harness with the reference's cell_connection.cpp and
           cell_interaction.cpp replaced by the drop-in GPU mechanics
           (epi_b200/shim/epi5_gpu_mechanics.cpp) and linked to the library;
           every other translation unit is the reference's own. This is how
           epi5_MT itself would be built against the library.

Usage: python oracle/build_ref.py [--dropin] [geometry ...]   (default: all known)
"""
from __future__ import annotations

import math
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
# The reference checkout: EPI_REFERENCE_DIR, else a "reference" directory
# beside this repository.
REF_DIR = Path(os.environ.get("EPI_REFERENCE_DIR", str(ROOT.parent / "reference"))) / "epi5_MT"
OUT = HERE / "_ref"

# The mechanics path's translation units plus cell_state_renew (the harness's
# dyn mode runs the complete cell_dynamics); chemistry and I/O drivers are not
# needed.
SOURCES = [
    "cellmanager.cpp", "cell.cpp", "cell_connection.cpp", "cell_interaction.cpp",
    "cell_init.cpp", "cell_state_renew.cpp", "utils.cpp", "vec3.cpp", "DualValue.cpp",
    "map.cpp", "ext_stim.cpp",
]
# Random_gen.cpp is replaced by the harness's fixed-seed genrand_real (the
# reference seeds from std::random_device; see oracle/ref_harness.cpp).

# name -> (NMX, NMY or rows, LX, LY, LZ, MAX_CELL_NUM[, triangular[, define.h NMY]])
GEOMETRIES = {
    "sq16_L16": (16, 16, 16.0, 16.0, 32.0, 20000),
    "sq24_L24": (24, 24, 24.0, 24.0, 32.0, 40000),
    "sq32_L32": (32, 32, 32.0, 32.0, 32.0, 60000),
    "sq48_L48": (48, 48, 48.0, 48.0, 32.0, 80000),
    "sq64_L64": (64, 64, 64.0, 64.0, 32.0, 80000),
    "sq256_L256": (256, 256, 256.0, 256.0, 32.0, 1300000),
    # membrane at the reference's natural spacing (0.5) for the mixed-state case
    "sq32_L16": (32, 32, 16.0, 16.0, 32.0, 20000),
    # triangular membrane (the reference's default build): NMX x rows sites at
    # unit spacing, rows sqrt(3)/2 apart; the wiring uses only NMX and the
    # number of membrane particles (cellmanager.cpp:70-111)
    "tri16x18": (16, 18, 16.0, 18 * math.sqrt(3.0) / 2.0, 32.0, 20000, True),
    "tri32x36": (32, 36, 32.0, 36 * math.sqrt(3.0) / 2.0, 32.0, 60000, True),
    # the all-laws tissue on the triangular lattice at the natural 0.5 spacing
    "tri32x36_L16": (32, 36, 16.0, 36 * 0.5 * math.sqrt(3.0) / 2.0, 32.0, 20000, True),
    # the reference's own default geometry (define.h as shipped: TRI_MEMB,
    # NMX = NMY = 100, 50 x 50 x 100 box), for its shipped input files; the
    # triangular wiring has 114 rows there (NMY / (sqrt(3)/2), even)
    "default": (100, 114, 50.0, 50.0, 100.0, 100 * 100 + 50000 * 10, True, 100),
}


# Field grid (define.h NX, NY, NZ) per geometry, for the harness's field
# mode; the mechanics never read it. Geometries not listed keep the shipped
# 100 x 100 x 200. These give the reference's default resolution, 0.5.
GRIDS = {
    "sq16_L16": (32, 32, 64),
    "sq32_L16": (32, 32, 64),
    "tri16x18": (32, 32, 64),
    "sq64_L64": (128, 128, 64),
}


def is_tri(name: str) -> bool:
    return len(GEOMETRIES[name]) > 6 and GEOMETRIES[name][6]

COMMON_FLAGS = [
    "-std=c++14", "-w",
    "-include", "cstddef", "-include", "cstring", "-include", "cassert",
    # RESTRICT expands to __restrict__ (epi5_MT/define.h:21-25); g++ 13 rejects
    # binding restrict-qualified pointers to `const Cell* const&` keys
    # (cell_connection.cpp:142). Dropping the qualifier is an aliasing hint
    # only and changes no arithmetic.
    "-D__restrict__=",
    # The loader asserts that the first non-membrane cell is DER
    # (cellmanager.cpp:266-269), which rejects the DER-free configurations.
    # define.h:3 carries the reference's own (commented) NDEBUG switch; it
    # removes assert() only. The harness re-checks the capacity asserts it
    # loses (connection lists < 400 per cell, cell_connection.cpp:122).
    "-DNDEBUG",
]


def geometry_for(nmx: int, nmy: int, lx: float, ly: float, lz: float, lattice: int = 0) -> str:
    for name, g in GEOMETRIES.items():
        if g[:5] == (nmx, nmy, float(lx), float(ly), float(lz)) and is_tri(name) == bool(lattice):
            return name
    raise KeyError(f"no oracle geometry for NMX={nmx} NMY={nmy} L=({lx},{ly},{lz})")


def _fmt(v: float) -> str:
    return repr(float(v))


def write_overlay(name: str) -> Path:
    nmx, nmy, lx, ly, lz, maxc = GEOMETRIES[name][:6]
    tri = is_tri(name)
    # NMY as written into define.h (a triangular entry may differ from its rows)
    if len(GEOMETRIES[name]) > 7:
        nmy = GEOMETRIES[name][7]
    text = (REF_DIR / "define.h").read_text(encoding="latin-1")
    subs = [] if tri else [
        (r"#define\s+TRI_MEMB\s+1", "/* TRI_MEMB undefined: square membrane */")]
    subs += [
        (r"(unsigned int NMX\s*=\s*)\d+", rf"\g<1>{nmx}"),
        (r"(unsigned int NMY\s*=\s*)\d+", rf"\g<1>{nmy}"),
        (r"(cdefs MAX_CELL_NUM\s*=\s*)[^;]+", rf"\g<1>{maxc}"),
        (r"(cdefd LX\s*=\s*)[^;]+", rf"\g<1>{_fmt(lx)}"),
        (r"(cdefd LY\s*=\s*)[^;]+", rf"\g<1>{_fmt(ly)}"),
        (r"(cdefd LZ\s*=\s*)[^;]+", rf"\g<1>{_fmt(lz)}"),
    ]
    if name in GRIDS:
        gx, gy, gz = GRIDS[name]
        subs += [(r"(cdefs NX\s*=\s*)\d+", rf"\g<1>{gx}"),
                 (r"(cdefs NY\s*=\s*)\d+", rf"\g<1>{gy}"),
                 (r"(cdefs NZ\s*=\s*)\d+", rf"\g<1>{gz}")]
    for pat, rep in subs:
        text, k = re.subn(pat, rep, text, count=1)
        if k != 1:
            raise RuntimeError(f"define.h overlay: pattern {pat!r} not found")
    # The square build of epi5_MT does not compile as shipped: tri_memb_bend
    # (cell_interaction.cpp:488-499) sits outside any #ifdef and reads
    # Cell::Memb_data::memb[6], which cell.h:57-59 declares only under
    # TRI_MEMB. Pre-include cell.h once with TRI_MEMB defined, so the struct
    # carries that (never used) member, then undefine TRI_MEMB before any
    # translation unit's own code is compiled. Every code path that branches
    # on TRI_MEMB (define.h:148, cellmanager.cpp:70,318,
    # cell_interaction.cpp:502) therefore takes its square branch.
    text = text.rstrip()
    assert text.endswith("#endif // DEFINE_H"), "unexpected define.h tail"
    if not tri:
        text = text[: -len("#endif // DEFINE_H")] + (
            "#endif // DEFINE_H\n"
            "#ifdef __cplusplus\n"
            "#define TRI_MEMB 1\n"
            "#include \"cell.h\"\n"
            "#undef TRI_MEMB\n"
            "#endif\n"
        )
    else:
        text += "\n"
    d = OUT / name
    d.mkdir(parents=True, exist_ok=True)
    p = d / "define.h"
    if not p.exists() or p.read_text(encoding="latin-1") != text:
        p.write_text(text, encoding="latin-1")
    return p


def _compile(args):
    cmd, obj = args
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"compile failed: {' '.join(cmd)}\n{r.stderr[-4000:]}")
    return obj


def binary_path(name: str, variant: str) -> Path:
    return OUT / name / f"ref_harness_{variant}"


DROPIN_SHIM = ROOT / "epi_b200" / "shim" / "epi5_gpu_mechanics.cpp"
DROPIN_LIB = ROOT / "epi_b200" / "libepi_mech.so"
# the two translation units the drop-in replaces
DROPIN_REPLACED = ("cell_connection.cpp", "cell_interaction.cpp")


def build(name: str, variant: str, jobs: int = 8) -> Path:
    overlay = write_overlay(name)
    odir = OUT / name / variant
    odir.mkdir(parents=True, exist_ok=True)
    inc = ["-I", str(HERE / "tbb_shim"), "-I", str(REF_DIR), "-include", str(overlay)]
    srcs = [REF_DIR / s for s in SOURCES] + [HERE / "ref_harness.cpp"]
    libs = []
    deps = []
    if variant == "serial":
        flags = ["-O2", "-ffp-contract=off"]
    elif variant == "omp":
        flags = ["-O3", "-march=x86-64-v3", "-fopenmp", "-DEPI_TBB_SHIM_OPENMP"]
    elif variant in ("dropin", "dropin_omp"):
        # dropin_omp: the timed build (the reference's own loops and the
        # drop-in's host loops on all threads, as the omp build)
        flags = (["-O2", "-ffp-contract=off"] if variant == "dropin" else
                 ["-O3", "-march=x86-64-v3", "-fopenmp", "-DEPI_TBB_SHIM_OPENMP"])
        inc += ["-I", str(ROOT / "include")]
        srcs = [s for s in srcs if s.name not in DROPIN_REPLACED] + [DROPIN_SHIM]
        # relative rpath: the binary sits three levels below the repository root
        libs = [f"-L{DROPIN_LIB.parent}", "-lepi_mech", "-Wl,-rpath,$ORIGIN/../../../epi_b200"]
        deps = [DROPIN_LIB, ROOT / "include" / "epi_mech.h"]
    else:
        raise ValueError(variant)
    out = binary_path(name, variant)
    newest_src = max(p.stat().st_mtime for p in srcs + deps + [overlay, Path(__file__)])
    if out.exists() and out.stat().st_mtime > newest_src:
        return out
    work = []
    for s in srcs:
        obj = odir / (s.stem + ".o")
        work.append((["g++", *COMMON_FLAGS, *flags, *inc, "-c", str(s), "-o", str(obj)], obj))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(_compile, work))
    link = ["g++", *flags, *[str(o) for o in objs], *libs, "-o", str(out)]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed: {r.stderr[-4000:]}")
    return out


def available() -> bool:
    return (REF_DIR / "cell_interaction.cpp").exists()


def main(argv):
    variants = ["serial", "omp"]
    if "--dropin" in argv:
        argv = [a for a in argv if a != "--dropin"]
        variants += ["dropin", "dropin_omp"]
    names = argv or list(GEOMETRIES)
    if not available():
        print(f"reference sources not found under {REF_DIR}; nothing built")
        return 0
    for name in names:
        for variant in variants:
            p = build(name, variant)
            print(p)
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
