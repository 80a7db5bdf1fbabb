"""Python access to the oracle (TEST INFRASTRUCTURE ONLY).

Two checkers live here, both used only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg:

* OracleTissue -- ctypes binding of the C restatement (oracle/epi_oracle.c),
  built into oracle/liboracle.so by build_oracle().
* run_reference -- runs the compiled reference harness (oracle/_ref, built by
  oracle/build_ref.py from the reference sources) on a tissue and returns its
  frames.
* tangent_gradient -- the FP64 forward-mode gradient of a final-state loss
  with respect to the spring / LJ-epsilon / bending multipliers
  (oracle/epi_oracle_tangent.cpp, same library), the reference gradient of
  the adjoint tests.

Nothing in the product package imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from pathlib import Path
from typing import Optional

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_OUT = HERE / "_ref"
# the reference checkout (present where the oracle is built, not on GPU
# hosts): EPI_REFERENCE_DIR, else a "reference" directory beside this repository
REF_DIR = Path(os.environ.get("EPI_REFERENCE_DIR", str(HERE.parent.parent / "reference")))

_lib = None


def build_oracle(force: bool = False) -> Path:
    c_src = HERE / "epi_oracle.c"
    cpp_src = HERE / "epi_oracle_tangent.cpp"
    hdr = HERE / "epi_oracle.h"
    deps = [c_src, cpp_src, hdr, Path(__file__)]
    if (not force and LIB_PATH.exists()
            and LIB_PATH.stat().st_mtime > max(p.stat().st_mtime for p in deps)):
        return LIB_PATH
    # -ffp-contract=off: the restatement evaluates the reference's arithmetic
    # operation by operation (no fused multiply-adds)
    flags = ["-O2", "-ffp-contract=off", "-fPIC"]
    with tempfile.TemporaryDirectory() as d:
        c_obj, cpp_obj = os.path.join(d, "oracle.o"), os.path.join(d, "tangent.o")
        subprocess.run(["gcc", *flags, "-std=c11", "-c", str(c_src), "-o", c_obj], check=True)
        subprocess.run(["g++", *flags, "-std=c++17", "-c", str(cpp_src), "-o", cpp_obj],
                       check=True)
        tmp = str(LIB_PATH) + ".tmp"
        subprocess.run(["g++", "-shared", "-o", tmp, c_obj, cpp_obj, "-lm"], check=True)
        os.replace(tmp, LIB_PATH)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            build_oracle()
        L = ctypes.CDLL(str(LIB_PATH))
        P = ctypes.c_void_p
        d = ctypes.POINTER(ctypes.c_double)
        i32 = ctypes.POINTER(ctypes.c_int32)
        u8 = ctypes.POINTER(ctypes.c_uint8)
        L.ora_new.restype = P
        L.ora_new.argtypes = [ctypes.c_int32] * 5 + [ctypes.c_double] * 3 + [d] * 7 + [u8, i32, i32]
        L.ora_new_lattice.restype = P
        L.ora_new_lattice.argtypes = L.ora_new.argtypes + [ctypes.c_int32]
        L.ora_free.argtypes = [P]
        for f in ("ora_connect", "ora_interact"):
            getattr(L, f).argtypes = [P]
            getattr(L, f).restype = ctypes.c_int
        L.ora_step.argtypes = [P, ctypes.c_int32]
        L.ora_step.restype = ctypes.c_int
        L.ora_pos_copy.argtypes = [P]
        L.ora_periodic_fix.argtypes = [P]
        L.ora_get_positions.argtypes = [P, d, d, d]
        L.ora_set_positions.argtypes = [P, d, d, d]
        for f in ("ora_get_connections", "ora_get_connections_raw"):
            getattr(L, f).argtypes = [P, i32, i32, ctypes.c_int64]
            getattr(L, f).restype = ctypes.c_int64
        L.ora_get_dermis.argtypes = [P, i32]
        L.ora_error_info.argtypes = [P, i32, i32, d]
        L.ora_error_info.restype = ctypes.c_int
        L.ora_field_new.restype = P
        L.ora_field_new.argtypes = [P, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
        L.ora_field_free.argtypes = [P]
        L.ora_field_step.argtypes = [P, P, d]
        L.ora_field_step.restype = ctypes.c_int
        L.ora_field_get.argtypes = [P, i32, u8, d]
        L.ora_tangent_gradient.argtypes = (
            [ctypes.c_int32] * 5 + [ctypes.c_double] * 3 + [d] * 7 + [u8, i32, i32] +
            [ctypes.c_int32, ctypes.c_int32, d, d, d, ctypes.c_int32, ctypes.c_int32, d, d, d, d, d])
        L.ora_tangent_gradient.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


class OracleTissue:
    """FP64 serial restatement of the epi5_MT step for one tissue."""

    def __init__(self, t, params=None):
        L = lib()
        p = np.array((params or t.params).as_tuple(), dtype=np.float64)
        self._keep = [np.ascontiguousarray(a) for a in (
            t.x, t.y, t.z, t.radius, t.agek, t.spr_nat_len)]
        st = np.ascontiguousarray(t.state, dtype=np.uint8)
        pr = np.ascontiguousarray(t.pair, dtype=np.int32)
        rd = np.ascontiguousarray(t.rest_div_times, dtype=np.int32)
        self.n = t.n
        self._h = L.ora_new_lattice(t.n, t.nmemb, t.nder, t.nmx, t.nmy, t.lx, t.ly, t.lz,
                                    _p(p, ctypes.c_double),
                                    *[_p(a, ctypes.c_double) for a in self._keep],
                                    _p(st, ctypes.c_uint8), _p(pr, ctypes.c_int32),
                                    _p(rd, ctypes.c_int32), int(getattr(t, "lattice", 0)))
        if not self._h:
            raise ValueError("oracle rejected the tissue")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ora_free(self._h)
            self._h = None

    def step(self, n: int = 1) -> int:
        return lib().ora_step(self._h, n)

    def connect(self) -> int:
        return lib().ora_connect(self._h)

    def positions(self):
        x, y, z = (np.empty(self.n) for _ in range(3))
        lib().ora_get_positions(self._h, _p(x, ctypes.c_double), _p(y, ctypes.c_double),
                                _p(z, ctypes.c_double))
        return x, y, z

    def set_positions(self, x, y, z):
        x, y, z = (np.ascontiguousarray(a, dtype=np.float64) for a in (x, y, z))
        lib().ora_set_positions(self._h, _p(x, ctypes.c_double), _p(y, ctypes.c_double),
                                _p(z, ctypes.c_double))

    def connections(self, raw: bool = False):
        off = np.zeros(self.n + 1, np.int32)
        f = lib().ora_get_connections_raw if raw else lib().ora_get_connections
        tot = f(self._h, _p(off, ctypes.c_int32), None, 0)
        idx = np.zeros(max(int(tot), 1), np.int32)
        f(self._h, _p(off, ctypes.c_int32), _p(idx, ctypes.c_int32), tot)
        return off, idx[: int(tot)]

    def dermis(self):
        d = np.empty(self.n, np.int32)
        lib().ora_get_dermis(self._h, _p(d, ctypes.c_int32))
        return d

    def error(self):
        a = ctypes.c_int32()
        b = ctypes.c_int32()
        v = ctypes.c_double()
        code = lib().ora_error_info(self._h, ctypes.byref(a), ctypes.byref(b), ctypes.byref(v))
        return code, a.value, b.value, v.value


def reference_binary(t, variant: str = "serial") -> Optional[Path]:
    """Path of the compiled reference harness for this tissue's geometry, if built."""
    import importlib.util
    spec = importlib.util.spec_from_file_location("epi_build_ref", HERE / "build_ref.py")
    br = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(br)
    try:
        name = br.geometry_for(t.nmx, t.nmy, t.lx, t.ly, t.lz, getattr(t, "lattice", 0))
    except KeyError:
        return None
    p = br.binary_path(name, variant)
    return p if p.exists() else None


def run_reference(t, nsteps: int, every: int, variant: str = "serial",
                  env: Optional[dict] = None, mode: str = "run"):
    """Run the compiled reference on `t` (default parameters only: the reference
    fixes its constants at compile time). Returns the parsed frames. `env`
    adds environment variables (the dropin variant reads EPI_MECH_*, the
    harness EPI_HARNESS_RNG / EPI_HARNESS_SEED); mode "dyn" runs the complete
    cell_dynamics including state renewal."""
    from epi_b200.tissue import read_reference_frames
    exe = reference_binary(t, variant)
    if exe is None:
        raise FileNotFoundError("compiled reference harness not built for this geometry")
    full_env = dict(os.environ)
    full_env.update(env or {})
    with tempfile.TemporaryDirectory() as d:
        cells = os.path.join(d, "cells.dat")
        out = os.path.join(d, "frames.bin")
        t.write_reference_file(cells)
        r = subprocess.run([str(exe), mode, cells, str(nsteps), out, str(every)],
                           capture_output=True, text=True, env=full_env)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness failed ({r.returncode}): {r.stderr[-2000:]}")
        return read_reference_frames(out)


def read_gj_frames(path: str):
    """Parse the gap-junction dumps of the harness (EPI_HARNESS_GJ): per frame
    {step, dead (keys of removed cells per cell), off (CSR row offsets), idx,
    checked, value}."""
    data = open(path, "rb").read()
    off = 0
    frames = []
    entry = np.dtype([("idx", "<i4"), ("checked", "<i4"), ("value", "<f8")])
    while off < len(data):
        tag, step, n = np.frombuffer(data, np.int32, 3, off)
        assert tag == 0x504D4A47, "bad gap-junction frame tag"
        off += 12
        rows, dead, lens = [], np.zeros(n, np.int32), np.zeros(n, np.int64)
        for i in range(n):
            m, d = np.frombuffer(data, np.int32, 2, off)
            off += 8
            rows.append(np.frombuffer(data, entry, m, off))
            off += 16 * int(m)
            dead[i], lens[i] = d, m
        allr = np.concatenate(rows) if rows else np.zeros(0, entry)
        frames.append(dict(step=int(step), dead=dead,
                           off=np.concatenate([[0], np.cumsum(lens)]),
                           idx=allr["idx"].copy(), checked=allr["checked"].copy(),
                           value=allr["value"].copy()))
    return frames


def run_reference_gj(t, nsteps: int, every: int, variant: str = "serial",
                     env: Optional[dict] = None, mode: str = "run"):
    """run_reference with the gap-junction maps dumped beside each frame:
    returns (frames, gap-junction frames)."""
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "gj.bin")
        e = dict(env or {})
        e["EPI_HARNESS_GJ"] = path
        frames = run_reference(t, nsteps, every, variant=variant, env=e, mode=mode)
        return frames, read_gj_frames(path)


def time_reference(t, warmup: int, steps: int, threads: Optional[int] = None,
                   variant: str = "omp", env: Optional[dict] = None):
    """Time the OpenMP build of the reference on `t` (or another build: the
    drop-in's is "dropin_omp"); returns its JSON summary."""
    import json
    exe = reference_binary(t, variant)
    if exe is None:
        raise FileNotFoundError(f"compiled reference harness ({variant}) not built for this "
                                f"geometry")
    env = dict(os.environ, **(env or {}))
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory() as d:
        cells = os.path.join(d, "cells.dat")
        t.write_reference_file(cells)
        r = subprocess.run([str(exe), "time", cells, str(warmup), str(steps)],
                           capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness failed ({r.returncode}): {r.stderr[-2000:]}")
        return json.loads(r.stdout.strip().splitlines()[-1])


def tangent_gradient(t, nsteps: int, target=None, cells_only: bool = True, dual: bool = True,
                     params=None):
    """Forward-mode FP64 gradient (oracle/epi_oracle_tangent.cpp).

    Runs `nsteps` steps of tissue `t` and returns (loss, grad, positions):
    loss = mean over the loss set (non-membrane particles when `cells_only`)
    of the squared minimum-image distance to `target` (x, y, z arrays), and
    grad = d loss / d (s_spring, s_eps, s_bend), the multipliers of every
    spring constant, of eps_m and of kbend, at 1. With dual=False the
    plain-double instantiation runs (no gradient: grad is None).
    """
    L = lib()
    p = np.array((params or t.params).as_tuple(), dtype=np.float64)
    keep = [np.ascontiguousarray(a, dtype=np.float64) for a in (
        t.x, t.y, t.z, t.radius, t.agek, t.spr_nat_len)]
    st = np.ascontiguousarray(t.state, dtype=np.uint8)
    pr = np.ascontiguousarray(t.pair, dtype=np.int32)
    rd = np.ascontiguousarray(t.rest_div_times, dtype=np.int32)
    tgt = [np.ascontiguousarray(a, dtype=np.float64) for a in target] if target is not None \
        else [None] * 3
    loss = ctypes.c_double(0.0)
    grad = np.zeros(3)
    out = [np.empty(t.n) for _ in range(3)]
    rc = L.ora_tangent_gradient(
        t.n, t.nmemb, t.nder, t.nmx, t.nmy, t.lx, t.ly, t.lz, _p(p, ctypes.c_double),
        *[_p(a, ctypes.c_double) for a in keep], _p(st, ctypes.c_uint8),
        _p(pr, ctypes.c_int32), _p(rd, ctypes.c_int32), int(getattr(t, "lattice", 0)), nsteps,
        *[(_p(a, ctypes.c_double) if a is not None else None) for a in tgt],
        1 if cells_only else 0, 1 if dual else 0, ctypes.byref(loss),
        _p(grad, ctypes.c_double), *[_p(a, ctypes.c_double) for a in out])
    if rc != 0:
        raise RuntimeError(f"oracle tangent failed with code {rc}")
    return loss.value, (grad if dual else None), tuple(out)


class OracleField:
    """Cell maps and external stimulus of an OracleTissue (ora_field_*)."""

    def __init__(self, ora: "OracleTissue", nx: int, ny: int, nz: int):
        self.ora = ora
        self.dims = (nx + 1, ny + 1, nz + 1)
        self._h = lib().ora_field_new(ora._h, nx, ny, nz)
        if not self._h:
            raise ValueError("oracle rejected the field")

    def __del__(self):
        if getattr(self, "_h", None):
            lib().ora_field_free(self._h)
            self._h = None

    def step(self):
        z = ctypes.c_double()
        rc = lib().ora_field_step(self.ora._h, self._h, ctypes.byref(z))
        return rc, z.value

    def get(self):
        nv = int(np.prod(self.dims))
        m1 = np.empty(nv, np.int32)
        m2 = np.empty(nv, np.uint8)
        ex = np.empty(nv, np.float64)
        lib().ora_field_get(self._h, _p(m1, ctypes.c_int32), _p(m2, ctypes.c_uint8),
                            _p(ex, ctypes.c_double))
        return m1.reshape(self.dims), m2.reshape(self.dims), ex.reshape(self.dims)


def read_field_frames(path: str):
    """Field frames written by the reference harness's field mode."""
    data = open(path, "rb").read()
    off = 0
    frames = []
    while off < len(data):
        tag, step, n, X, Y, Z = np.frombuffer(data, np.int32, 6, off)
        assert tag == 0x46444C46, "bad field frame tag"
        off += 24
        zzmax = float(np.frombuffer(data, np.float64, 1, off)[0])
        off += 8
        pos = np.frombuffer(data, np.float64, 3 * n, off).reshape(3, n)
        off += 24 * n
        nv = int(X) * int(Y) * int(Z)
        m1 = np.frombuffer(data, np.int32, nv, off).reshape(X, Y, Z)
        off += 4 * nv
        m2 = np.frombuffer(data, np.uint8, nv, off).reshape(X, Y, Z)
        off += nv
        ex = np.frombuffer(data, np.float64, nv, off).reshape(X, Y, Z)
        off += 8 * nv
        frames.append(dict(step=int(step), zzmax=zzmax, x=pos[0].copy(), y=pos[1].copy(),
                           z=pos[2].copy(), cmap1=m1.copy(), cmap2=m2.copy(), ext=ex.copy()))
    return frames


def run_reference_field(t, nsteps: int, every: int):
    """The compiled reference's field mode (mechanics step, zzmax, cell maps,
    external-stimulus diffusion per step) on `t`."""
    exe = reference_binary(t, "serial")
    if exe is None:
        raise FileNotFoundError("compiled reference harness not built for this geometry")
    with tempfile.TemporaryDirectory() as d:
        cells = os.path.join(d, "cells.dat")
        out = os.path.join(d, "field.bin")
        t.write_reference_file(cells)
        r = subprocess.run([str(exe), "field", cells, str(nsteps), out, str(every)],
                           capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness failed ({r.returncode}): {r.stderr[-2000:]}")
        return read_field_frames(out)


def time_reference_field(t, warmup: int, steps: int, threads: Optional[int] = None):
    """Time the OpenMP build's field part of the step (zzmax, cell maps,
    external-stimulus update) on `t`; returns its JSON summary."""
    import json
    exe = reference_binary(t, "omp")
    if exe is None:
        raise FileNotFoundError("compiled reference harness (omp) not built for this geometry")
    env = dict(os.environ)
    if threads:
        env["OMP_NUM_THREADS"] = str(threads)
    with tempfile.TemporaryDirectory() as d:
        cells = os.path.join(d, "cells.dat")
        t.write_reference_file(cells)
        r = subprocess.run([str(exe), "time_field", cells, str(warmup), str(steps)],
                           capture_output=True, text=True, env=env)
        if r.returncode != 0:
            raise RuntimeError(f"reference harness failed ({r.returncode}): {r.stderr[-2000:]}")
        return json.loads(r.stdout.strip().splitlines()[-1])
