"""Parity at the full workload sizes, through checks that stay cheap on the
CPU side.

* 1.1M-particle tissue (256x256 membrane + 1,048,576 cells), FP64: the
  initial connection lists bit-exact against the oracle; after a few steps
  positions within 1e-10 of the oracle's and the lists bit-exact against the
  oracle's lists at the GPU's positions; the mixed path within 1e-5. Over
  the workload's 200 steps, the same bars against the compiled reference.
* 512-tissue ensemble (6.56M particles), mixed precision, graph-replayed:
  every sampled tissue of the batch bit-identical to the same tissue run
  alone. The batch's rebuilds take the thread-per-particle candidate search
  and a single tissue's the warp-per-particle one, so this also pins their
  candidate order to each other at scale.
"""
import numpy as np
import pytest

from epi_b200 import capi
from epi_b200 import tissue as T
from oracle import oracle as O
from tests.helpers import lists_equal, list_diff_summary, rel_pos_err

pytestmark = pytest.mark.gpu

FP64 = capi.EPI_PREC_FP64
MIXED = capi.EPI_PREC_MIXED
TOL_FP64 = 1e-10
TOL_MIXED = 1e-5


def test_large_tissue_vs_oracle(built):
    t = T.config3()
    steps = 4
    ora = O.OracleTissue(t)  # runs the first connect
    ooff0, oidx0 = ora.connections()
    assert ora.step(steps) == 0
    opos = ora.positions()
    with capi.Context(precision=FP64, max_conn=64, max_cand=128) as ctx:
        ctx.upload([t])
        off0, idx0 = ctx.connections()
        ctx.step(steps, "graph")
        pos = ctx.positions()
        off, idx = ctx.connections()
    assert lists_equal(off0, idx0, ooff0, oidx0), list_diff_summary(off0, idx0, ooff0, oidx0)
    err = rel_pos_err(pos, opos, t.lx, t.ly)
    assert err <= TOL_FP64, err
    ora.set_positions(*pos)
    assert ora.connect() == 0
    ooff, oidx = ora.connections()
    assert lists_equal(off, idx, ooff, oidx), list_diff_summary(off, idx, ooff, oidx)
    with capi.Context(precision=MIXED, max_conn=64, max_cand=128) as ctx:
        ctx.upload([t])
        ctx.step(steps, "graph")
        mpos = ctx.positions()
    err = rel_pos_err(mpos, opos, t.lx, t.ly)
    assert err <= TOL_MIXED, err


def test_large_tissue_200_steps_vs_reference(built):
    """The 1.1M-particle tissue over its workload's 200 steps against the
    compiled reference (its OpenMP build on the host's threads; the serial
    oracle would take a quarter of an hour): FP64 positions within 1e-10 at
    steps 100 and 200, lists bit-exact there against the reference's and
    against the oracle's connect at the GPU's positions; the mixed path
    within 1e-5 at step 200."""
    t = T.config3()
    if O.reference_binary(t, "omp") is None:
        pytest.skip("compiled reference (omp) not built for the 256 x 256 geometry")
    frames = {f["step"]: f for f in O.run_reference(t, 200, 100, variant="omp")}
    assert sorted(frames) == [0, 100, 200]
    with capi.Context(precision=FP64, max_conn=64, max_cand=128) as ctx:
        ctx.upload([t])
        done = 0
        for s in (100, 200):
            ctx.step(s - done, "graph")
            done = s
            f = frames[s]
            pos = ctx.positions()
            err = rel_pos_err(pos, (f["x"], f["y"], f["z"]), t.lx, t.ly)
            assert err <= TOL_FP64, (s, err)
            off, idx = ctx.connections()
            assert lists_equal(off, idx, f["conn_off"], f["conn_idx"]), \
                (s, list_diff_summary(off, idx, f["conn_off"], f["conn_idx"]))
            ora = O.OracleTissue(t)
            ora.set_positions(*pos)
            assert ora.connect() == 0
            ooff, oidx = ora.connections()
            assert lists_equal(off, idx, ooff, oidx), s
    with capi.Context(precision=MIXED, max_conn=64, max_cand=128) as ctx:
        ctx.upload([t])
        ctx.step(200, "graph")
        f = frames[200]
        err = rel_pos_err(ctx.positions(), (f["x"], f["y"], f["z"]), t.lx, t.ly)
        assert err <= TOL_MIXED, err


def test_full_ensemble_batch_equals_single_tissue_runs(built):
    ts = T.config4()
    steps = 20
    with capi.Context(precision=MIXED, max_conn=64) as ctx:
        ctx.upload(ts)
        ctx.step(steps, "graph")
        pos = ctx.positions()
    offs = np.cumsum([0] + [t.n for t in ts])
    sizes = [t.n for t in ts]
    pick = sorted({int(np.argmax(sizes)), int(np.argmin(sizes)), 0, 255, len(ts) - 1})
    for k in pick:
        with capi.Context(precision=MIXED, max_conn=64) as ctx:
            ctx.upload([ts[k]])
            ctx.step(steps, "graph")
            alone = ctx.positions()
        for d in range(3):
            assert np.array_equal(pos[d][offs[k]:offs[k + 1]], alone[d]), (k, d)
