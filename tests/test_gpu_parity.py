"""GPU parity: the CUDA path through the C ABI against the oracle.

Bars (stated per test):
* connection lists and dermis: bit-exact (sorted per cell);
* FP64 path positions: max min-image |dr| / L_x <= 1e-10 after up to 1000
  steps (the only difference from the reference is the FP64 summation order);
* mixed path (FP32 forces, FP64 sums and positions): <= 1e-5 after 1000 steps;
* batched, graph-replayed and per-tissue launches: bit-identical to each other.
"""
import numpy as np
import pytest

from epi_b200 import capi
from epi_b200 import tissue as T
from oracle import oracle as O
from tests.golden.make_golden import load
from tests.helpers import lists_equal, list_diff_summary, rel_pos_err

pytestmark = pytest.mark.gpu

FP64 = capi.EPI_PREC_FP64
MIXED = capi.EPI_PREC_MIXED
TOL_FP64 = 1e-10
TOL_MIXED = 1e-5


def run_gpu(tissues, steps, precision=FP64, mode="eager", max_conn=64, skin=None, variant=None):
    with capi.Context(precision=precision, max_conn=max_conn, max_cand=2 * max_conn,
                      skin=skin, variant=variant) as ctx:
        ctx.upload(tissues)
        if steps:
            ctx.step(steps, mode)
        pos = ctx.positions()
        off, idx = ctx.connections()
        der = ctx.dermis()
    return pos, off, idx, der


def oracle_lists_at(t, pos):
    ora = O.OracleTissue(t)
    ora.set_positions(*pos)
    assert ora.connect() == 0
    return ora.connections(), ora.dermis()


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_initial_connect_bit_exact_vs_reference(built, precision):
    for name, factory in (("c1", T.config1), ("mixed", T.mixed_state_tissue)):
        f = load(name)[0]
        t = factory()
        _, off, idx, der = run_gpu([t], 0, precision, max_conn=96)
        assert lists_equal(off, idx, f["conn_off"], f["conn_idx"]), \
            list_diff_summary(off, idx, f["conn_off"], f["conn_idx"])
        fm = (t.state == T.FIX) | (t.state == T.MUSUME)
        assert np.array_equal(der[fm], f["dermis"][fm])


def test_fp64_c1_1000_steps_vs_reference_frames(built):
    frames = load("c1")
    t = T.config1()
    with capi.Context(precision=FP64) as ctx:
        ctx.upload([t])
        done = 0
        for f in frames[1:]:
            ctx.step(f["step"] - done)
            done = f["step"]
            pos = ctx.positions()
            err = rel_pos_err(pos, (f["x"], f["y"], f["z"]), t.lx, t.ly)
            assert err <= TOL_FP64, (f["step"], err)
            off, idx = ctx.connections()
            # lists equal the reference's own lists at the same step ...
            assert lists_equal(off, idx, f["conn_off"], f["conn_idx"])
            # ... and the oracle's connect applied to the GPU's positions
            (ooff, oidx), _ = oracle_lists_at(t, pos)
            assert lists_equal(off, idx, ooff, oidx)


def test_fp64_mixed_states_all_laws_vs_reference_frames(built):
    frames = load("mixed")
    t = T.mixed_state_tissue()
    fm = (t.state == T.FIX) | (t.state == T.MUSUME)
    with capi.Context(precision=FP64, max_conn=96, max_cand=192) as ctx:
        ctx.upload([t])
        done = 0
        for f in frames[1:]:
            ctx.step(f["step"] - done)
            done = f["step"]
            pos = ctx.positions()
            err = rel_pos_err(pos, (f["x"], f["y"], f["z"]), t.lx, t.ly)
            assert err <= TOL_FP64, (f["step"], err)
            off, idx = ctx.connections()
            (ooff, oidx), oder = oracle_lists_at(t, pos)
            assert lists_equal(off, idx, ooff, oidx)
            assert np.array_equal(ctx.dermis()[fm], oder[fm])


def test_mixed_precision_c1_1000_steps_within_1e5(built):
    f = load("c1")[-1]
    t = T.config1()
    pos, off, idx, _ = run_gpu([t], 1000, MIXED)
    err = rel_pos_err(pos, (f["x"], f["y"], f["z"]), t.lx, t.ly)
    assert err <= TOL_MIXED, err
    (ooff, oidx), _ = oracle_lists_at(t, pos)
    assert lists_equal(off, idx, ooff, oidx)


def test_mixed_precision_all_laws_300_steps_within_1e5(built):
    f = load("mixed")[-1]
    t = T.mixed_state_tissue()
    pos, off, idx, _ = run_gpu([t], 300, MIXED, max_conn=96)
    err = rel_pos_err(pos, (f["x"], f["y"], f["z"]), t.lx, t.ly)
    assert err <= TOL_MIXED, err


def test_fp64_c2_vs_oracle(built):
    t = T.config2()
    steps = 50
    ora = O.OracleTissue(t)
    assert ora.step(steps) == 0
    pos, off, idx, _ = run_gpu([t], steps, FP64)
    err = rel_pos_err(pos, ora.positions(), t.lx, t.ly)
    assert err <= TOL_FP64, err
    (ooff, oidx), _ = oracle_lists_at(t, pos)
    assert lists_equal(off, idx, ooff, oidx)


def test_ragged_batch_equals_single_tissue_runs(built):
    ts = [T.config1(3), T.mixed_state_tissue(), T.layered_tissue(24, 3, 9),
          T.layered_tissue(16, 5, 2, params=T.Params().scaled(1.7, 0.6, 1.3))]
    steps = 30
    pos_b, off_b, idx_b, der_b = run_gpu(ts, steps, FP64, max_conn=96)
    base = 0
    cbase = 0
    for t in ts:
        pos_s, off_s, idx_s, der_s = run_gpu([t], steps, FP64, max_conn=96)
        sl = slice(base, base + t.n)
        assert rel_pos_err(tuple(a[sl] for a in pos_b), pos_s, t.lx, t.ly) <= 1e-13
        rows = off_b[base: base + t.n + 1] - off_b[base]
        assert np.array_equal(rows, off_s)
        assert np.array_equal(idx_b[off_b[base]: off_b[base + t.n]], idx_s)
        assert np.array_equal(der_b[sl], der_s)
        base += t.n


def test_batch_with_scaled_params_vs_oracle(built):
    ts = [T.layered_tissue(16, 3, 21, params=T.Params().scaled(s, e, b))
          for s, e, b in ((0.5, 2.0, 1.0), (2.0, 0.5, 0.7), (1.0, 1.0, 2.0))]
    steps = 100
    pos, off, idx, _ = run_gpu(ts, steps, FP64)
    base = 0
    for t in ts:
        ora = O.OracleTissue(t)
        assert ora.step(steps) == 0
        sl = slice(base, base + t.n)
        err = rel_pos_err(tuple(a[sl] for a in pos), ora.positions(), t.lx, t.ly)
        assert err <= TOL_FP64, err
        base += t.n


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_graph_and_per_tissue_launches_are_bit_identical(built, precision):
    ts = [T.config1(1), T.layered_tissue(24, 2, 4)]
    ref = run_gpu(ts, 21, precision, "eager")
    for mode in ("graph", "per_tissue"):
        got = run_gpu(ts, 21, precision, mode)
        for a, b in zip(ref[0], got[0]):
            assert np.array_equal(a, b), mode
        assert np.array_equal(ref[1], got[1]) and np.array_equal(ref[2], got[2]), mode


@pytest.mark.parametrize("skin", [0.05, 0.3, 1.0])
def test_results_do_not_depend_on_skin(built, skin):
    """The candidate margin changes how often candidates are rebuilt, never
    which pairs connect: lists and FP64 positions match the oracle."""
    t = T.config1(2)
    steps = 200
    ora = O.OracleTissue(t)
    assert ora.step(steps) == 0
    pos, off, idx, _ = run_gpu([t], steps, FP64, skin=skin)
    assert rel_pos_err(pos, ora.positions(), t.lx, t.ly) <= TOL_FP64
    ooff, oidx = ora.connections()
    assert lists_equal(off, idx, ooff, oidx)


def test_simple_and_general_step_kernels_agree(built):
    """A batch holding one mixed-state tissue runs the general kernel for all
    its tissues; the ALIVE-only tissue in it must match its own (specialised)
    run to FP64 rounding and exactly in its lists."""
    t = T.config1(4)
    (pos_s, off_s, idx_s, _) = run_gpu([t], 100, FP64)
    (pos_b, off_b, idx_b, _) = run_gpu([t, T.mixed_state_tissue()], 100, FP64, max_conn=96)
    sl = slice(0, t.n)
    assert rel_pos_err(tuple(a[sl] for a in pos_b), pos_s, t.lx, t.ly) <= 1e-13
    assert np.array_equal(off_b[: t.n + 1], off_s)
    assert np.array_equal(idx_b[: off_s[-1]], idx_s)


@pytest.mark.parametrize("variant", [1, 2, 3, 4])
def test_step_kernel_variants_agree(built, variant):
    """Register-budget variants run the same formulas in the same order; only
    the compiler's multiply-add fusion may differ (FP64: rounding level)."""
    ts = [T.mixed_state_tissue(), T.config1(6)]
    ref = run_gpu(ts, 40, FP64, max_conn=96, variant=0)
    got = run_gpu(ts, 40, FP64, max_conn=96, variant=variant)
    base = 0
    for t in ts:
        sl = slice(base, base + t.n)
        assert rel_pos_err(tuple(a[sl] for a in got[0]), tuple(a[sl] for a in ref[0]),
                           t.lx, t.ly) <= 1e-13
        base += t.n
    assert np.array_equal(ref[1], got[1]) and np.array_equal(ref[2], got[2])


def test_repeat_runs_are_deterministic(built):
    t = T.config2()
    a = run_gpu([t], 20, MIXED)
    b = run_gpu([t], 20, MIXED)
    for u, v in zip(a[0], b[0]):
        assert np.array_equal(u, v)


# --- error behaviour: the reference's aborts become status codes ------------

def test_too_strong_interaction_reports_coef_range(built):
    t = T.config1()
    k = t.nmemb
    t.x[k + 1], t.y[k + 1], t.z[k + 1] = t.x[k] + 0.3, t.y[k], t.z[k]
    ora = O.OracleTissue(t)
    assert ora.step(1) == capi.EPI_ERR_COEF_RANGE
    with capi.Context(precision=FP64) as ctx:
        ctx.upload([t])
        with pytest.raises(capi.EpiError) as e:
            ctx.step(1)
        assert e.value.code == capi.EPI_ERR_COEF_RANGE
        info = ctx.error_info()
        assert {info["particle"], info["other"]} == {k, k + 1}
        assert abs(info["value"]) > 1000


def test_out_of_grid_reports_bin_range(built):
    t = T.config1()
    t.z[t.nmemb + 3] = 40.0
    with capi.Context(precision=FP64) as ctx:
        with pytest.raises(capi.EpiError) as e:
            ctx.upload([t])
        assert e.value.code == capi.EPI_ERR_BIN_RANGE


def test_nan_input_reports_nonfinite(built):
    t = T.config1()
    t.x[t.nmemb + 5] = np.nan
    with capi.Context(precision=FP64) as ctx:
        with pytest.raises(capi.EpiError) as e:
            ctx.upload([t])
        assert e.value.code == capi.EPI_ERR_NONFINITE


def test_list_capacity_overflow_reported(built):
    t = T.config1()
    with capi.Context(precision=FP64, max_conn=3, max_cand=64) as ctx:
        with pytest.raises(capi.EpiError) as e:
            ctx.upload([t])
        assert e.value.code == capi.EPI_ERR_LIST_OVERFLOW
    with capi.Context(precision=FP64, max_conn=3, max_cand=4) as ctx:
        with pytest.raises(capi.EpiError) as e:
            ctx.upload([t])
        assert e.value.code == capi.EPI_ERR_LIST_OVERFLOW


def test_context_usable_after_error(built):
    t = T.config1()
    bad = t.copy()
    bad.z[bad.nmemb] = 40.0
    with capi.Context(precision=FP64) as ctx:
        with pytest.raises(capi.EpiError):
            ctx.upload([bad])
        ctx.upload([t])
        ctx.step(5)
        ctx.sync()


def test_kernel_timing_reports_every_class(built):
    with capi.Context(precision=MIXED) as ctx:
        ctx.upload([T.config1()])
        tm = ctx.time_kernels(3)
    assert set(tm) == {"step", "prepass", "rebuild_bin", "rebuild_scan", "rebuild_sort",
                       "rebuild_search", "gate"}
    assert all(v[1] == 3 for v in tm.values())
    assert tm["step"][0] > 0
