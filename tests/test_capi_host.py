"""The C-ABI library without a GPU: it loads, exports every declared entry
point, and reports errors instead of failing."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from epi_b200 import capi
from epi_b200.tissue import Params

HEADER = Path(__file__).resolve().parents[1] / "include" / "epi_mech.h"


def declared_functions():
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(epi_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_function(built):
    L = capi.lib()
    names = declared_functions()
    assert names, "no declarations parsed"
    for n in names:
        assert hasattr(L, n), f"{n} declared in include/epi_mech.h but not exported"
    assert sorted(capi.EXPORTED) == names


def test_strerror_covers_every_status(built):
    for code in range(0, 15):
        s = capi.strerror(code)
        assert s and "unknown" not in s
    assert "unknown" in capi.strerror(99)


def test_default_params_equal_reference_constants(built):
    p = capi.default_params()
    got = tuple(getattr(p, f) for f, _ in capi.ParamsC._fields_)
    assert got == Params().as_tuple()


def test_create_rejects_bad_arguments(built):
    L = capi.lib()
    assert L.epi_create(None, None) == capi.EPI_ERR_INVALID_ARG
    cfg = capi.ConfigC(0, 7, 64, 96, 0.3, 0, 0, 0, 0)  # unknown precision
    h = ctypes.c_void_p()
    assert L.epi_create(ctypes.byref(h), ctypes.byref(cfg)) in (
        capi.EPI_ERR_INVALID_ARG, capi.EPI_ERR_NO_DEVICE)
    cfg = capi.ConfigC(0, 1, 64, 32, 0.3, 0, 0, 0, 0)  # fewer candidates than connections
    assert L.epi_create(ctypes.byref(h), ctypes.byref(cfg)) in (
        capi.EPI_ERR_INVALID_ARG, capi.EPI_ERR_NO_DEVICE)
    cfg = capi.ConfigC(0, 1, 64, 96, -1.0, 0, 0, 0, 0)  # negative skin
    assert L.epi_create(ctypes.byref(h), ctypes.byref(cfg)) in (
        capi.EPI_ERR_INVALID_ARG, capi.EPI_ERR_NO_DEVICE)
    cfg = capi.ConfigC(0, 1, 64, 96, 0.1, 9, 0, 0, 0)  # unknown step-kernel variant
    assert L.epi_create(ctypes.byref(h), ctypes.byref(cfg)) in (
        capi.EPI_ERR_INVALID_ARG, capi.EPI_ERR_NO_DEVICE)
    # argument checks come before the device query: exact codes without a GPU
    cfg = capi.ConfigC(0, 1, 64, 96, 0.1, 0, -5, 0, 0)  # negative search switch
    assert L.epi_create(ctypes.byref(h), ctypes.byref(cfg)) == capi.EPI_ERR_INVALID_ARG
    cfg = capi.ConfigC(0, 1, 64, 96, 0.1, 0, 0, 3, 0)  # unknown rebuild node
    assert L.epi_create(ctypes.byref(h), ctypes.byref(cfg)) == capi.EPI_ERR_INVALID_ARG
    cfg = capi.ConfigC(0, 1, 64, 96, 0.1, 0, 0, 0, 7)  # reserved must be 0
    assert L.epi_create(ctypes.byref(h), ctypes.byref(cfg)) == capi.EPI_ERR_INVALID_ARG
    cfg = capi.ConfigC(0, 1, 500, 600, 0.1, 0, 0, 0, 0)  # beyond the reference's 400 connections
    assert L.epi_create(ctypes.byref(h), ctypes.byref(cfg)) == capi.EPI_ERR_INVALID_ARG
    assert L.epi_step(None, 1) == capi.EPI_ERR_INVALID_ARG
    assert L.epi_sync(None) == capi.EPI_ERR_INVALID_ARG
    assert L.epi_get_config(None, ctypes.byref(cfg)) == capi.EPI_ERR_INVALID_ARG
    assert L.epi_set_tuning(None, 0.1, 3, 0, 0) == capi.EPI_ERR_INVALID_ARG


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_has_gpu(), reason="a GPU is present")
def test_create_without_gpu_reports_no_device(built):
    with pytest.raises(capi.EpiError) as e:
        capi.Context()
    assert e.value.code == capi.EPI_ERR_NO_DEVICE
