"""The reference's own initial state through the GPU path.

epi5_MT ships input_2layer_nfix16.dat: 11,400 membrane particles on its
default triangular lattice (TRI_MEMB, 100 columns x 114 rows at 0.5 spacing,
cellmanager.cpp:70-113), 2,312 dermis cells (DER, radius 1.4) and 16 stem
cells (FIX) in a 50 x 50 x 100 box. It exercises what the synthetic tissues
hold only a few of: DER-DER pairs (CI_der_to_der, cell_interaction.cpp:129-139),
FIX dermis springs (:174-183) and the dihedral bending (:451-499).

Checks, through the C ABI: lists and dermis bit-exact at every step for 20
steps against the oracle (pinned bit-exact to the reference's default build
on this input, tests/test_oracle.py) and at steps 0 and 20 against the
compiled reference's own frames (tests/golden/shipped.npz); FP64 positions
within 1e-10 of L_x, the mixed path within 1e-5. The drop-in compiled into
the default build reproduces the same frames.
"""
import numpy as np
import pytest

from epi_b200 import capi
from epi_b200 import tissue as T
from oracle import oracle as O
from tests.golden.make_golden import load, load_shipped_tissue
from tests.helpers import lists_equal, list_diff_summary, rel_pos_err

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
TOL_MIXED = 1e-5
STEPS = 20


def _frames():
    return {f["step"]: f for f in load("shipped")}


@pytest.mark.parametrize("precision", [capi.EPI_PREC_FP64, capi.EPI_PREC_MIXED])
def test_shipped_input_every_step_vs_oracle_and_reference(built, precision):
    t = load_shipped_tissue()
    assert (t.nmemb, t.nder, int((t.state == T.FIX).sum())) == (11400, 2312, 16)
    frames = _frames()
    fix = t.state == T.FIX
    tol = TOL_FP64 if precision == capi.EPI_PREC_FP64 else TOL_MIXED
    ora = O.OracleTissue(t)
    with capi.Context(precision=precision, max_conn=64, max_cand=128) as ctx:
        ctx.upload([t])
        off, idx = ctx.connections()
        g = frames[0]
        assert lists_equal(off, idx, g["conn_off"], g["conn_idx"]), \
            list_diff_summary(off, idx, g["conn_off"], g["conn_idx"])
        assert np.array_equal(ctx.dermis()[fix], g["dermis"][fix])
        for s in range(1, STEPS + 1):
            ctx.step(1)
            assert ora.step(1) == 0, ora.error()
            pos = ctx.positions()
            err = rel_pos_err(pos, ora.positions(), t.lx, t.ly)
            assert err <= tol, (s, err)
            off, idx = ctx.connections()
            # the lists of the GPU's positions, exactly as connect_cell makes them
            ora_at = O.OracleTissue(t)
            ora_at.set_positions(*pos)
            assert ora_at.connect() == 0
            ooff, oidx = ora_at.connections()
            assert lists_equal(off, idx, ooff, oidx), (s, list_diff_summary(off, idx, ooff, oidx))
            assert np.array_equal(ctx.dermis()[fix], ora_at.dermis()[fix]), s
        g = frames[STEPS]
        err = rel_pos_err(ctx.positions(), (g["x"], g["y"], g["z"]), t.lx, t.ly)
        assert err <= tol, err
        if precision == capi.EPI_PREC_FP64:
            off, idx = ctx.connections()
            assert lists_equal(off, idx, g["conn_off"], g["conn_idx"])
            assert np.array_equal(ctx.dermis()[fix], g["dermis"][fix])


def test_shipped_input_through_the_dropin_default_build(built):
    """epi5_MT's default build with connect_cell / cell_interaction replaced
    by the drop-in (epi_b200/shim over the C ABI), on its own input."""
    t = load_shipped_tissue()
    if O.reference_binary(t, "dropin") is None:
        pytest.skip("drop-in harness not built (python oracle/build_ref.py --dropin default)")
    frames = _frames()
    got = {f["step"]: f for f in O.run_reference(t, STEPS, STEPS, variant="dropin",
                                                  env={"EPI_MECH_PRECISION": "fp64"})}
    fix = t.state == T.FIX
    for s in (0, STEPS):
        f, g = got[s], frames[s]
        err = rel_pos_err((f["x"], f["y"], f["z"]), (g["x"], g["y"], g["z"]), t.lx, t.ly)
        assert err <= TOL_FP64, (s, err)
        assert lists_equal(f["conn_off"], f["conn_idx"], g["conn_off"], g["conn_idx"]), \
            list_diff_summary(f["conn_off"], f["conn_idx"], g["conn_off"], g["conn_idx"])
        assert np.array_equal(f["dermis"][fix], g["dermis"][fix]), s
