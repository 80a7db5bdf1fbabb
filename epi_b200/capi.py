"""ctypes binding of libepi_mech.so (include/epi_mech.h).

Python is glue here: tests and the benchmark drive the library through exactly
the C ABI a C or C++ caller uses. The library must be built in-tree
(epi_b200/build.py); loading fails loudly if it is missing.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path
from typing import List, Optional, Sequence

import numpy as np

from .tissue import Params, Tissue

# EPI_MECH_LIB selects another build of the same library, e.g. the
# bounds-checked libepi_mech_check.so the tests run.
LIB_PATH = Path(os.environ.get("EPI_MECH_LIB",
                               Path(__file__).resolve().parent / "libepi_mech.so"))

EPI_OK = 0
EPI_ERR_INVALID_ARG = 1
EPI_ERR_NO_DEVICE = 2
EPI_ERR_CUDA = 3
EPI_ERR_OOM = 4
EPI_ERR_BIN_RANGE = 5
EPI_ERR_BIN_OVERFLOW = 6
EPI_ERR_LIST_OVERFLOW = 7
EPI_ERR_COEF_RANGE = 8
EPI_ERR_MEMB_COEF_RANGE = 9
EPI_ERR_NONFINITE = 10
EPI_ERR_TIMEOUT = 11
EPI_ERR_STATE = 12
EPI_ERR_UNSUPPORTED = 13
EPI_ERR_CHECK = 14

EPI_PREC_FP64 = 0
EPI_PREC_MIXED = 1

# Every function the header declares (checked by tests/test_capi_host.py).
EXPORTED = [
    "epi_params_default", "epi_config_default", "epi_strerror", "epi_create", "epi_destroy",
    "epi_upload", "epi_connect", "epi_interact_commit", "epi_step", "epi_step_graph",
    "epi_step_per_tissue", "epi_sync", "epi_num_particles", "epi_download_positions",
    "epi_upload_positions", "epi_step_host", "epi_step_host_async", "epi_get_connections", "epi_get_dermis", "epi_error_info",
    "epi_stream", "epi_rebuild_count", "epi_launch_count", "epi_time_kernels", "epi_autotune",
    "epi_get_config", "epi_set_tuning", "epi_field_init",
    "epi_field_step", "epi_field_get", "epi_field_set_ext", "epi_adjoint", "epi_connect_noalloc",
]


class EpiError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        super().__init__(f"{where}: {strerror(code)} (status {code})")


class ParamsC(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "dt", "eps_m", "p_memb", "der_der_const", "k_total", "k_desmosome", "kspring",
        "kspring_d", "kbend", "delta_r", "para_ljp2", "kspring_division", "lj_thresh",
        "thresh_sp")]

    @classmethod
    def from_params(cls, p: Params) -> "ParamsC":
        return cls(*p.as_tuple())


_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)
_up = ctypes.POINTER(ctypes.c_uint8)


class TissueViewC(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int32), ("nmemb", ctypes.c_int32), ("nder", ctypes.c_int32),
                ("nmx", ctypes.c_int32), ("nmy", ctypes.c_int32),
                ("lx", ctypes.c_double), ("ly", ctypes.c_double), ("lz", ctypes.c_double),
                ("x", _dp), ("y", _dp), ("z", _dp), ("radius", _dp), ("agek", _dp),
                ("spr_nat_len", _dp), ("state", _up), ("pair", _ip),
                ("rest_div_times", _ip), ("lattice", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class LossC(ctypes.Structure):
    _fields_ = [("target_x", ctypes.POINTER(ctypes.c_double)),
                ("target_y", ctypes.POINTER(ctypes.c_double)),
                ("target_z", ctypes.POINTER(ctypes.c_double)),
                ("cells_only", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class ConfigC(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("max_conn", ctypes.c_int32), ("max_cand", ctypes.c_int32),
                ("skin", ctypes.c_double), ("variant", ctypes.c_int32),
                ("search_switch", ctypes.c_int32), ("rebuild_gate", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with epi_b200/build.py (no CPU fallback exists)")
        L = ctypes.CDLL(str(LIB_PATH))
        vp = ctypes.c_void_p
        L.epi_params_default.argtypes = [ctypes.POINTER(ParamsC)]
        L.epi_params_default.restype = None
        L.epi_config_default.argtypes = [ctypes.POINTER(ConfigC)]
        L.epi_config_default.restype = None
        L.epi_strerror.argtypes = [ctypes.c_int]
        L.epi_strerror.restype = ctypes.c_char_p
        L.epi_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(ConfigC)]
        L.epi_destroy.argtypes = [vp]
        L.epi_destroy.restype = None
        L.epi_upload.argtypes = [vp, ctypes.c_int32, ctypes.POINTER(TissueViewC),
                                 ctypes.POINTER(ParamsC)]
        for f in ("epi_connect", "epi_interact_commit", "epi_sync"):
            getattr(L, f).argtypes = [vp]
        for f in ("epi_step", "epi_step_graph", "epi_step_per_tissue"):
            getattr(L, f).argtypes = [vp, ctypes.c_int32]
        L.epi_num_particles.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.epi_download_positions.argtypes = [vp, _dp, _dp, _dp]
        L.epi_upload_positions.argtypes = [vp, _dp, _dp, _dp]
        L.epi_step_host.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.epi_step_host_async.argtypes = [vp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.epi_get_connections.argtypes = [vp, _ip, _ip, ctypes.c_int64,
                                          ctypes.POINTER(ctypes.c_int64)]
        L.epi_get_dermis.argtypes = [vp, _ip]
        L.epi_error_info.argtypes = [vp, _ip, _ip, _ip, _dp]
        L.epi_rebuild_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.epi_launch_count.argtypes = [vp, ctypes.POINTER(ctypes.c_int64)]
        L.epi_stream.argtypes = [vp]
        L.epi_stream.restype = vp
        L.epi_time_kernels.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, _dp, _ip,
                                       ctypes.POINTER(ctypes.c_char_p), _ip]
        L.epi_autotune.argtypes = [vp, ctypes.c_int32, _dp, _ip, _dp]
        L.epi_get_config.argtypes = [vp, ctypes.POINTER(ConfigC)]
        L.epi_set_tuning.argtypes = [vp, ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                                     ctypes.c_int32]
        L.epi_field_init.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]
        L.epi_field_step.argtypes = [vp, ctypes.c_int32]
        L.epi_field_get.argtypes = [vp, ctypes.c_int32, _ip, _up, _dp, _dp]
        L.epi_field_set_ext.argtypes = [vp, ctypes.c_int32, _dp]
        L.epi_adjoint.argtypes = [vp, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(LossC),
                                  _dp, _dp]
        for f in EXPORTED:
            if f not in ("epi_params_default", "epi_config_default", "epi_strerror",
                         "epi_destroy", "epi_stream"):
                getattr(L, f).restype = ctypes.c_int
        _lib = L
    return _lib


def strerror(code: int) -> str:
    try:
        return lib().epi_strerror(code).decode()
    except FileNotFoundError:
        return f"status {code}"


def _check(rc: int, where: str):
    if rc != EPI_OK:
        raise EpiError(rc, where)


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(ctypes.POINTER(ct))


def default_params() -> ParamsC:
    p = ParamsC()
    lib().epi_params_default(ctypes.byref(p))
    return p


class Context:
    """One epi_ctx: a batch of tissues resident on one GPU."""

    def __init__(self, precision: int = EPI_PREC_MIXED, max_conn: int = 64, device: int = 0,
                 max_cand: Optional[int] = None, skin: Optional[float] = None,
                 variant: Optional[int] = None, rebuild_gate: Optional[int] = None,
                 search_switch: Optional[int] = None):
        L = lib()
        cfg = ConfigC()
        L.epi_config_default(ctypes.byref(cfg))
        cfg.precision = precision
        cfg.max_conn = max_conn
        cfg.max_cand = max(max_cand if max_cand is not None else cfg.max_cand, max_conn)
        if skin is not None:
            cfg.skin = skin
        if variant is not None:
            cfg.variant = variant
        if rebuild_gate is not None:
            cfg.rebuild_gate = rebuild_gate
        if search_switch is not None:
            cfg.search_switch = search_switch
        cfg.device = device
        h = ctypes.c_void_p()
        _check(L.epi_create(ctypes.byref(h), ctypes.byref(cfg)), "epi_create")
        self._h = h
        self.precision = precision
        self.tissues: List[Tissue] = []
        self.offsets = np.zeros(1, np.int64)
        self._keep = []

    def close(self):
        if getattr(self, "_h", None) is not None and self._h.value:
            lib().epi_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- upload / state ---------------------------------------------------
    def upload(self, tissues: Sequence[Tissue], params: Optional[Sequence[Params]] = None):
        tissues = list(tissues)
        views = (TissueViewC * len(tissues))()
        pars = (ParamsC * len(tissues))()
        keep = []
        for k, t in enumerate(tissues):
            arrs = dict(
                x=np.ascontiguousarray(t.x, np.float64), y=np.ascontiguousarray(t.y, np.float64),
                z=np.ascontiguousarray(t.z, np.float64),
                radius=np.ascontiguousarray(t.radius, np.float64),
                agek=np.ascontiguousarray(t.agek, np.float64),
                spr=np.ascontiguousarray(t.spr_nat_len, np.float64),
                state=np.ascontiguousarray(t.state, np.uint8),
                pair=np.ascontiguousarray(t.pair, np.int32),
                rest=np.ascontiguousarray(t.rest_div_times, np.int32))
            keep.append(arrs)
            v = views[k]
            v.n, v.nmemb, v.nder, v.nmx, v.nmy = t.n, t.nmemb, t.nder, t.nmx, t.nmy
            v.lx, v.ly, v.lz = t.lx, t.ly, t.lz
            v.x, v.y, v.z = (_ptr(arrs[c], ctypes.c_double) for c in ("x", "y", "z"))
            v.radius = _ptr(arrs["radius"], ctypes.c_double)
            v.agek = _ptr(arrs["agek"], ctypes.c_double)
            v.spr_nat_len = _ptr(arrs["spr"], ctypes.c_double)
            v.state = _ptr(arrs["state"], ctypes.c_uint8)
            v.pair = _ptr(arrs["pair"], ctypes.c_int32)
            v.rest_div_times = _ptr(arrs["rest"], ctypes.c_int32)
            v.lattice = int(getattr(t, "lattice", 0))
            v.reserved = 0
            p = (params[k] if params is not None else t.params)
            pars[k] = ParamsC.from_params(p)
        rc = lib().epi_upload(self._h, len(tissues), views, pars)
        self.tissues = tissues
        self.offsets = np.concatenate([[0], np.cumsum([t.n for t in tissues])]).astype(np.int64)
        _check(rc, "epi_upload")

    @property
    def ntissues(self) -> int:
        return len(self.tissues)

    @property
    def n(self) -> int:
        v = ctypes.c_int64()
        _check(lib().epi_num_particles(self._h, ctypes.byref(v)), "epi_num_particles")
        return int(v.value)

    # --- the reference's step functions ------------------------------------
    def connect(self):
        _check(lib().epi_connect(self._h), "epi_connect")

    def interact_commit(self):
        _check(lib().epi_interact_commit(self._h), "epi_interact_commit")

    def step(self, nsteps: int = 1, mode: str = "eager"):
        fn = {"eager": lib().epi_step, "graph": lib().epi_step_graph,
              "per_tissue": lib().epi_step_per_tissue}[mode]
        _check(fn(self._h, nsteps), f"epi_step[{mode}]")

    def sync(self):
        _check(lib().epi_sync(self._h), "epi_sync")

    # --- results -------------------------------------------------------------
    def positions(self, out=None):
        n = self.n
        if out is None:
            out = (np.empty(n), np.empty(n), np.empty(n))
        x, y, z = out
        _check(lib().epi_download_positions(self._h, _ptr(x, ctypes.c_double),
                                            _ptr(y, ctypes.c_double), _ptr(z, ctypes.c_double)),
               "epi_download_positions")
        return x, y, z

    def set_positions(self, x, y, z):
        x, y, z = (np.ascontiguousarray(a, np.float64) for a in (x, y, z))
        _check(lib().epi_upload_positions(self._h, _ptr(x, ctypes.c_double),
                                          _ptr(y, ctypes.c_double), _ptr(z, ctypes.c_double)),
               "epi_upload_positions")

    def step_host(self, pos_in, pos_out=None, wait: bool = True):
        """epi_step_host: one step of a batch whose positions are in host
        memory (x, y, z arrays in, new positions out; the same arrays may be
        given for both). Pinned host arrays let the copies overlap. With
        wait=False (epi_step_host_async) the call returns once the step is
        queued; the arrays are valid after sync()."""
        x, y, z = pos_in
        for a in (x, y, z):
            if a.dtype != np.float64 or not a.flags.c_contiguous or a.shape != (self.n,):
                raise ValueError("positions must be contiguous float64 arrays of n entries")
        if pos_out is None:
            pos_out = (np.empty(self.n), np.empty(self.n), np.empty(self.n))
        ox, oy, oz = pos_out
        fn = lib().epi_step_host if wait else lib().epi_step_host_async
        _check(fn(self._h, *(_ptr(a, ctypes.c_double) for a in (x, y, z, ox, oy, oz))),
               "epi_step_host" if wait else "epi_step_host_async")
        return pos_out

    def connections(self):
        n = self.n
        off = np.zeros(n + 1, np.int32)
        tot = ctypes.c_int64()
        _check(lib().epi_get_connections(self._h, _ptr(off, ctypes.c_int32), None, 0,
                                         ctypes.byref(tot)), "epi_get_connections")
        idx = np.zeros(max(int(tot.value), 1), np.int32)
        _check(lib().epi_get_connections(self._h, _ptr(off, ctypes.c_int32),
                                         _ptr(idx, ctypes.c_int32), int(tot.value),
                                         ctypes.byref(tot)), "epi_get_connections")
        return off, idx[: int(tot.value)]

    def dermis(self):
        d = np.empty(self.n, np.int32)
        _check(lib().epi_get_dermis(self._h, _ptr(d, ctypes.c_int32)), "epi_get_dermis")
        return d

    def error_info(self):
        t, a, b = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        v = ctypes.c_double()
        code = lib().epi_error_info(self._h, ctypes.byref(t), ctypes.byref(a), ctypes.byref(b),
                                    ctypes.byref(v))
        return dict(code=code, tissue=t.value, particle=a.value, other=b.value, value=v.value)

    def rebuild_count(self) -> int:
        v = ctypes.c_int64()
        _check(lib().epi_rebuild_count(self._h, ctypes.byref(v)), "epi_rebuild_count")
        return int(v.value)

    def launch_count(self) -> int:
        v = ctypes.c_int64()
        _check(lib().epi_launch_count(self._h, ctypes.byref(v)), "epi_launch_count")
        return int(v.value)

    def stream_handle(self) -> int:
        return int(lib().epi_stream(self._h) or 0)

    def time_kernels(self, nsteps: int):
        K = 16
        ms = np.zeros(K)
        launches = np.zeros(K, np.int32)
        names = (ctypes.c_char_p * K)()
        ncls = ctypes.c_int32()
        _check(lib().epi_time_kernels(self._h, nsteps, K, _ptr(ms, ctypes.c_double),
                                      _ptr(launches, ctypes.c_int32), names,
                                      ctypes.byref(ncls)), "epi_time_kernels")
        return {names[k].decode(): (float(ms[k]), int(launches[k])) for k in range(ncls.value)}

    def adjoint(self, nsteps: int, target, checkpoint_every: int = 20, cells_only: bool = True):
        """epi_adjoint: runs nsteps steps and returns (loss per tissue, gradient
        per tissue as an array (ntissues, 3): d loss / d (s_spring, s_eps,
        s_bend)). `target` is (x, y, z) over all particles."""
        tx, ty, tz = (np.ascontiguousarray(a, np.float64) for a in target)
        assert len(tx) == len(ty) == len(tz) == self.n
        spec = LossC(_ptr(tx, ctypes.c_double), _ptr(ty, ctypes.c_double),
                     _ptr(tz, ctypes.c_double), 1 if cells_only else 0, 0)
        nt = self.ntissues
        loss = np.zeros(nt)
        grad = np.zeros(3 * nt)
        _check(lib().epi_adjoint(self._h, nsteps, checkpoint_every, ctypes.byref(spec),
                                 _ptr(loss, ctypes.c_double), _ptr(grad, ctypes.c_double)),
               "epi_adjoint")
        return loss, grad.reshape(nt, 3)

    def config(self) -> dict:
        """epi_get_config: the context's configuration (after autotune: its choice)."""
        cfg = ConfigC()
        _check(lib().epi_get_config(self._h, ctypes.byref(cfg)), "epi_get_config")
        return {k: getattr(cfg, k) for k, _ in ConfigC._fields_}

    def set_tuning(self, skin: float, variant: int, search_switch: int = 0,
                   rebuild_gate: int = 0):
        """epi_set_tuning: apply a tuning chosen earlier (e.g. cached)."""
        _check(lib().epi_set_tuning(self._h, float(skin), int(variant), int(search_switch),
                                    int(rebuild_gate)), "epi_set_tuning")

    def autotune(self, trial_steps: int = 64):
        """epi_autotune: returns (skin, variant, ms per step of the best trial)
        and keeps that pair in the context."""
        skin = ctypes.c_double()
        variant = ctypes.c_int32()
        ms = ctypes.c_double()
        _check(lib().epi_autotune(self._h, trial_steps, ctypes.byref(skin), ctypes.byref(variant),
                                  ctypes.byref(ms)), "epi_autotune")
        return float(skin.value), int(variant.value), float(ms.value)

    # --- cell maps and external stimulus ------------------------------------
    def field_init(self, nx: int, ny: int, nz: int):
        _check(lib().epi_field_init(self._h, nx, ny, nz), "epi_field_init")
        self.field_dims = (nx + 1, ny + 1, nz + 1)

    def field_step(self, nsteps: int = 1):
        _check(lib().epi_field_step(self._h, nsteps), "epi_field_step")

    def field(self, tissue: int = 0):
        """(cmap1, cmap2, ext, zzmax) of one tissue, grids shaped (nx+1, ny+1, nz+1)."""
        nv = int(np.prod(self.field_dims))
        m1 = np.empty(nv, np.int32)
        m2 = np.empty(nv, np.uint8)
        ex = np.empty(nv, np.float64)
        zz = ctypes.c_double()
        _check(lib().epi_field_get(self._h, tissue, _ptr(m1, ctypes.c_int32),
                                   _ptr(m2, ctypes.c_uint8), _ptr(ex, ctypes.c_double),
                                   ctypes.byref(zz)), "epi_field_get")
        d = self.field_dims
        return m1.reshape(d), m2.reshape(d), ex.reshape(d), float(zz.value)

    def field_set_ext(self, tissue: int, ext):
        e = np.ascontiguousarray(ext, np.float64).ravel()
        _check(lib().epi_field_set_ext(self._h, tissue, _ptr(e, ctypes.c_double)),
               "epi_field_set_ext")
