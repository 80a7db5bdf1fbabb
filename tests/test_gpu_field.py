"""Cell maps and external-stimulus diffusion (epi_field_*) against the
oracle's restatement, which is pinned bit for bit to the reference's map.cpp
and ext_stim.cpp (tests/test_oracle.py).

The GPU runs the field step on exactly the oracle's positions (uploaded each
step), so every grid must agree bit for bit: the cell map (highest-index
cell wins where spheres overlap, as the reference's index-order loop
leaves it), the mask map and the stimulus (same operation order, no fused
multiply-adds).
"""
import numpy as np
import pytest

from epi_b200 import capi
from epi_b200 import tissue as T
from oracle import oracle as O

pytestmark = pytest.mark.gpu

GRID = (32, 32, 64)


def field_tissue_tri():
    return T.field_tissue(lattice=T.TRIANGULAR)


@pytest.mark.parametrize("factory", [T.field_tissue, field_tissue_tri, T.config1])
def test_field_bit_exact_vs_oracle_on_the_same_positions(built, factory):
    t = factory()
    ora = O.OracleTissue(t)
    fld = O.OracleField(ora, *GRID)
    with capi.Context(precision=capi.EPI_PREC_FP64, max_conn=96, max_cand=192) as ctx:
        ctx.upload([t])
        ctx.field_init(*GRID)
        for s in range(1, 31):
            assert ora.step(1) == 0
            ctx.set_positions(*ora.positions())
            rc, zz = fld.step()
            assert rc == 0
            ctx.field_step(1)
            if s % 10 == 0:
                m1, m2, ex, gzz = ctx.field(0)
                o1, o2, oex = fld.get()
                assert gzz == zz
                assert np.array_equal(m1, o1), (s, int((m1 != o1).sum()))
                assert np.array_equal(m2, o2), (s, int((m2 != o2).sum()))
                assert np.array_equal(ex, oex), (s, float(abs(ex - oex).max()))
    if factory is T.field_tissue:
        assert oex.max() > 0.1


def test_field_batch_and_device_trajectory(built):
    """Two tissues in one batch, the GPU stepping its own mechanics: each
    tissue's grids equal a single-tissue run's, and the maps equal the
    oracle's on the GPU's positions."""
    ta, tb = T.field_tissue(), T.config1(4)
    steps = 20
    res = {}
    for key, tissues in (("batch", [ta, tb]), ("a", [ta]), ("b", [tb])):
        with capi.Context(precision=capi.EPI_PREC_FP64, max_conn=96, max_cand=192) as ctx:
            ctx.upload(tissues)
            ctx.field_init(*GRID)
            for _ in range(steps):
                ctx.step(1)
                ctx.field_step(1)
            res[key] = [ctx.field(k) for k in range(len(tissues))]
            if key == "a":
                pos = ctx.positions()
    for k, key in ((0, "a"), (1, "b")):
        for u, v in zip(res["batch"][k][:3], res[key][0][:3]):
            assert np.array_equal(u, v)
    ora = O.OracleTissue(ta)
    ora.set_positions(*pos)
    fld = O.OracleField(ora, *GRID)
    assert fld.step()[0] == 0
    o1, o2, _ = fld.get()
    assert np.array_equal(res["a"][0][0], o1) and np.array_equal(res["a"][0][1], o2)


def test_field_survives_an_upload_that_keeps_the_tissue_count(built):
    t = T.field_tissue()
    with capi.Context(precision=capi.EPI_PREC_FP64, max_conn=96, max_cand=192) as ctx:
        ctx.upload([t])
        ctx.field_init(*GRID)
        ctx.field_step(5)
        ex0 = ctx.field(0)[2]
        ctx.upload([t])  # the drop-in re-uploads every step
        ex1 = ctx.field(0)[2]
        assert np.array_equal(ex0, ex1) and ex0.max() > 0
        ctx.field_step(1)
