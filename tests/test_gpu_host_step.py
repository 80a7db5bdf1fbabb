"""epi_step_host (one step of a batch held in host memory, its copies
overlapped with the kernels) against the three calls it stands for:
epi_upload_positions (connect), epi_interact_commit and
epi_download_positions.

Bar: bit-identical positions after every step, and identical connection
lists at the end, on a multi-group ensemble (rebuilds included), a single
tissue, the general (all force laws) path in FP64, and with the output
arrays aliasing the input arrays.
"""
import numpy as np
import pytest
import torch

from epi_b200 import capi
from epi_b200 import tissue as T

pytestmark = pytest.mark.gpu

FP64 = capi.EPI_PREC_FP64
MIXED = capi.EPI_PREC_MIXED


def pinned(a):
    t = torch.empty(a.shape[0], dtype=torch.float64, pin_memory=True)
    out = t.numpy()
    out[:] = a
    return out, t


def three_call_steps(tissues, steps, precision, **cfg):
    out = []
    with capi.Context(precision=precision, **cfg) as ctx:
        ctx.upload(tissues)
        x, y, z = ctx.positions()
        for _ in range(steps):
            ctx.set_positions(x, y, z)
            ctx.interact_commit()
            x, y, z = ctx.positions()
            out.append((x.copy(), y.copy(), z.copy()))
        off, idx = ctx.connections()
    return out, off, idx


def host_steps(tissues, steps, precision, alias=False, **cfg):
    out = []
    with capi.Context(precision=precision, **cfg) as ctx:
        ctx.upload(tissues)
        start = ctx.positions()
        keep = [pinned(a) for a in start]
        pos_in = tuple(k[0] for k in keep)
        keep_out = [pinned(np.zeros_like(a)) for a in start]
        pos_out = pos_in if alias else tuple(k[0] for k in keep_out)
        for _ in range(steps):
            ctx.step_host(pos_in, pos_out)
            out.append(tuple(a.copy() for a in pos_out))
            if not alias:
                for a, b in zip(pos_in, pos_out):
                    a[:] = b
        off, idx = ctx.connections()
    return out, off, idx


def assert_same(a, b):
    ra, offa, idxa = a
    rb, offb, idxb = b
    assert len(ra) == len(rb)
    for k, (pa, pb) in enumerate(zip(ra, rb)):
        for d in range(3):
            assert np.array_equal(pa[d], pb[d]), (k, d)
    assert np.array_equal(offa, offb) and np.array_equal(idxa, idxb)


def test_host_step_equals_three_calls_on_an_ensemble(built):
    tissues = T.config4(n_tissues=24)
    steps = 30
    assert_same(host_steps(tissues, steps, MIXED, max_conn=64),
                three_call_steps(tissues, steps, MIXED, max_conn=64))


def test_host_step_equals_three_calls_on_one_tissue_fp64(built):
    t = T.config1(2)
    assert_same(host_steps([t], 20, FP64), three_call_steps([t], 20, FP64))


def test_host_step_general_laws_and_aliased_arrays(built):
    tissues = [T.mixed_state_tissue(), T.mixed_state_tissue(seed=8)]
    cfg = dict(max_conn=96, max_cand=192)
    ref = three_call_steps(tissues, 25, FP64, **cfg)
    assert_same(host_steps(tissues, 25, FP64, **cfg), ref)
    assert_same(host_steps(tissues, 25, FP64, alias=True, **cfg), ref)


def test_host_step_triangular_membranes(built):
    tissues = [T.mixed_state_tissue(lattice=T.TRIANGULAR), T.tri_layered_tissue(16, 18, 2, 0)]
    cfg = dict(max_conn=96, max_cand=192)
    assert_same(host_steps(tissues, 20, MIXED, **cfg), three_call_steps(tissues, 20, MIXED, **cfg))


def test_async_host_steps_equal_sync_ones(built):
    """epi_step_host_async queued step after step on the same (aliased)
    pinned arrays, one sync at the end: the same positions as synchronous
    steps."""
    tissues = T.config4(n_tissues=24)
    steps = 12
    ref, _, _ = host_steps(tissues, steps, MIXED, alias=True, max_conn=64)
    with capi.Context(precision=MIXED, max_conn=64) as ctx:
        ctx.upload(tissues)
        keep = [pinned(a) for a in ctx.positions()]
        pos = tuple(k[0] for k in keep)
        for _ in range(steps):
            ctx.step_host(pos, pos, wait=False)
        ctx.sync()
        for d in range(3):
            assert np.array_equal(pos[d], ref[-1][d]), d


def test_host_step_rejects_bad_arrays(built):
    t = T.config1(1)
    with capi.Context(precision=MIXED) as ctx:
        ctx.upload([t])
        x, y, z = ctx.positions()
        with pytest.raises(ValueError):
            ctx.step_host((x[:-1], y, z))
        with pytest.raises(capi.EpiError) as e:
            capi._check(capi.lib().epi_step_host(ctx._h, None, None, None, None, None, None),
                        "epi_step_host")
        assert e.value.code == capi.EPI_ERR_INVALID_ARG
