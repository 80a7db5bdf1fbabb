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


@pytest.mark.parametrize("name,lattice", [("mixed", T.SQUARE), ("mixed_tri", T.TRIANGULAR)])
def test_fp64_mixed_states_all_laws_vs_reference_frames(built, name, lattice):
    frames = load(name)
    t = T.mixed_state_tissue(lattice=lattice)
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
            assert lists_equal(off, idx, f["conn_off"], f["conn_idx"])
            (ooff, oidx), oder = oracle_lists_at(t, pos)
            assert lists_equal(off, idx, ooff, oidx)
            assert np.array_equal(ctx.dermis()[fm], oder[fm])
            assert np.array_equal(ctx.dermis()[fm], f["dermis"][fm])


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


@pytest.mark.parametrize("variant", [None, 1, 2])
@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_graph_and_per_tissue_launches_are_bit_identical(built, precision, variant):
    """Also for the step-kernel forms whose gathers go through shared memory
    (variants 1 and 2)."""
    ts = [T.config1(1), T.layered_tissue(24, 2, 4), T.config1(7)]
    ref = run_gpu(ts, 21, precision, "eager")
    for mode in ("graph", "per_tissue"):
        got = run_gpu(ts, 21, precision, mode, variant=variant)
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


@pytest.mark.parametrize("precision", [FP64, MIXED])
def test_rebuild_nodes_and_search_paths_are_bit_identical(built, precision):
    """The step graph with the rebuild in a conditional node or always
    launched, and the candidate search by warps or by threads, give the same
    candidate rows in the same order: the steps agree bit for bit."""
    ts = [T.mixed_state_tissue(), T.config1(3), T.layered_tissue(24, 3, 5)]
    runs = []
    for gate, switch in ((1, 1 << 30), (2, 1 << 30), (1, 1), (2, 1)):
        with capi.Context(precision=precision, max_conn=96, max_cand=192, rebuild_gate=gate,
                          search_switch=switch) as ctx:
            ctx.upload(ts)
            ctx.step(30, "graph")
            runs.append((ctx.positions(), ctx.connections(), ctx.dermis()))
    for pos, (off, idx), der in runs[1:]:
        for a, b in zip(runs[0][0], pos):
            assert np.array_equal(a, b)
        assert np.array_equal(runs[0][1][0], off) and np.array_equal(runs[0][1][1], idx)
        assert np.array_equal(runs[0][2], der)


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


def test_upload_rejects_invalid_constants_and_views(built):
    t = T.config1()
    with capi.Context(precision=FP64) as ctx:
        for bad in (t.params.scaled(1, 1, 1), ):
            bad.lj_thresh = 1.0  # adhesion divides by (LJ_THRESH - 1)^2
            with pytest.raises(capi.EpiError) as e:
                ctx.upload([t], [bad])
            assert e.value.code == capi.EPI_ERR_INVALID_ARG
        bad = t.params.scaled(1, 1, 1)
        bad.dt = 0.0
        with pytest.raises(capi.EpiError) as e:
            ctx.upload([t], [bad])
        assert e.value.code == capi.EPI_ERR_INVALID_ARG
        r = t.copy()
        r.radius[r.nmemb + 2] = np.inf
        with pytest.raises(capi.EpiError) as e:
            ctx.upload([r])
        assert e.value.code == capi.EPI_ERR_INVALID_ARG
        ctx.upload([t])  # usable afterwards
        ctx.step(2)
        x, y, z = ctx.positions()
        x[3] = np.nan
        with pytest.raises(capi.EpiError) as e:
            ctx.set_positions(x, y, z)
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


def threshold_pair_tissue():
    """A dermis cell with one ALIVE cell at the largest FP64 separation the
    reference still connects and one at the smallest it does not (same axis,
    reference rounding), far from everything else. ljmain, which the DER
    applies to the ALIVE cell (cell_interaction.cpp:549-561), is not zero at
    the cut-off, so a misjudged pair moves the DER by ~4e-5."""
    side = 16
    nm = side * side
    jj, kk = np.meshgrid(np.arange(side), np.arange(side), indexing="xy")
    mx, my = (jj.ravel() + 0.5).astype(float), (kk.ravel() + 0.5).astype(float)
    xd, yd, zd = 8.0, 8.0, 6.0
    r_der, r_cell = T.R_DER, 0.5
    lt2 = 1.2 * 1.2
    rs = r_der + r_cell
    thr = lt2 * rs * rs

    def connected(xa):
        dx = xd - xa
        return dx * dx + 0.0 * 0.0 + 0.0 * 0.0 <= thr

    # largest xa > xd (ALIVE to the right) still connected: walk up from a guess
    xa = xd + 1.2 * rs
    while connected(np.nextafter(xa, np.inf)):
        xa = np.nextafter(xa, np.inf)
    while not connected(xa):
        xa = np.nextafter(xa, -np.inf)
    inside = xa
    # smallest xb < xd (to the left) not connected
    xb = xd - 1.2 * rs
    while connected(xb):
        xb = np.nextafter(xb, -np.inf)
    while not connected(np.nextafter(xb, np.inf)):
        xb = np.nextafter(xb, np.inf)
    outside = xb
    x = np.concatenate([mx, [xd, inside, outside]])
    y = np.concatenate([my, [yd, yd, yd]])
    z = np.concatenate([np.full(nm, 1.0), [zd, zd, zd]])
    n = nm + 3
    t = T.Tissue(nmx=side, nmy=side, lx=16.0, ly=16.0, lz=32.0, x=x, y=y, z=z,
                 radius=np.concatenate([np.full(nm, T.R_MEMB), [r_der, r_cell, r_cell]]),
                 state=np.concatenate([np.full(nm, T.MEMB, np.uint8),
                                       np.array([T.DER, T.ALIVE, T.ALIVE], np.uint8)]),
                 agek=np.zeros(n), spr_nat_len=np.zeros(n), pair=np.full(n, -1, np.int32),
                 rest_div_times=np.zeros(n, np.int32), nmemb=nm, nder=1, name="threshold")
    t.validate()
    return t


def test_mixed_path_decides_threshold_pairs_with_the_fp64_predicate(built):
    t = threshold_pair_tissue()
    d = t.nmemb
    _, off, idx, _ = run_gpu([t], 0, FP64)
    assert list(idx[off[d]:off[d + 1]]) == [d + 1]  # inside connected, outside not
    p64, _, _, _ = run_gpu([t], 1, FP64)
    pmx, _, _, _ = run_gpu([t], 1, MIXED)
    moved = abs(p64[0][d] - t.x[d])
    assert moved > 1e-5  # the inside pair pulls the DER
    # FP32 cannot separate these pairs; the mixed path must agree with FP64
    for k in range(3):
        assert abs(pmx[k][d] - p64[k][d]) < 1e-9, (k, pmx[k][d], p64[k][d])
        assert abs(pmx[k][d + 2] - p64[k][d + 2]) < 1e-9


def tri_c1():
    return T.tri_layered_tissue(16, 18, 2, 0)


def test_triangular_membrane_fp64_vs_reference_frames(built):
    """The reference's default build (TRI_MEMB): six lattice links and the
    dihedral bending of tri_memb_bend (cell_interaction.cpp:451-508)."""
    frames = load("tri")
    t = tri_c1()
    _, off, idx, _ = run_gpu([t], 0, FP64)
    assert lists_equal(off, idx, frames[0]["conn_off"], frames[0]["conn_idx"])
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
            assert lists_equal(off, idx, f["conn_off"], f["conn_idx"]), \
                list_diff_summary(off, idx, f["conn_off"], f["conn_idx"])


def test_triangular_membrane_mixed_precision(built):
    frames = load("tri")
    t = tri_c1()
    pos, _, _, _ = run_gpu([t], frames[-1]["step"], MIXED)
    f = frames[-1]
    assert rel_pos_err(pos, (f["x"], f["y"], f["z"]), t.lx, t.ly) <= TOL_MIXED


def test_square_and_triangular_tissues_in_one_batch(built):
    ts = [T.config1(3), tri_c1(), T.tri_layered_tissue(32, 36, 3, 5), T.mixed_state_tissue()]
    steps = 40
    pos_b, off_b, idx_b, _ = run_gpu(ts, steps, FP64, max_conn=96)
    o = 0
    for t in ts:
        pos_1, off_1, idx_1, _ = run_gpu([t], steps, FP64, max_conn=96)
        for k in range(3):
            assert np.array_equal(pos_b[k][o:o + t.n], pos_1[k])
        o += t.n


def test_mixed_precision_error_curve_c2_vs_fp64_oracle(built):
    """The 64x64-membrane, 32,768-cell tissue: the mixed path (FP32 forces,
    FP64 sums and positions) against the FP64 CPU oracle at every one of
    1000 steps, max over particles of |dr|_min-image / L_x. Bar 1e-5 at every
    step. The curve is printed (pytest -s) for the record."""
    t = T.config2()
    ora = O.OracleTissue(t)
    curve = []
    with capi.Context(precision=MIXED) as ctx:
        ctx.upload([t])
        for s in range(1, 1001):
            ctx.step(1)
            assert ora.step(1) == 0
            e = rel_pos_err(ctx.positions(), ora.positions(), t.lx, t.ly)
            curve.append(e)
            assert e <= TOL_MIXED, (s, e)
    picks = [1, 2, 5, 10, 20, 50, 100, 200, 500, 1000]
    print("mixed-vs-FP64-oracle error curve (step: max |dr|/L_x): " +
          ", ".join(f"{s}: {curve[s - 1]:.3e}" for s in picks))
    print(f"max over 1000 steps: {max(curve):.3e}")


def test_reupload_and_position_upload_regate_only_what_changed(built):
    """A same-shape re-upload (the drop-in's per-step connect) and a position
    upload keep the candidate lists of tissues nothing moved in; results stay
    those of a fresh context."""
    ts = T.config4(n_tissues=12)
    with capi.Context(precision=FP64) as ctx:
        ctx.upload(ts)
        ctx.step(20)
        pos = ctx.positions()
        r0 = ctx.rebuild_count()
        ctx.set_positions(*pos)  # unchanged positions: nothing to rebuild
        assert ctx.rebuild_count() == r0
        off_a, idx_a = ctx.connections()
        moved = [a.copy() for a in pos]
        moved[2][ts[0].n + 5] += 0.3  # one particle of tissue 1 jumps
        ctx.set_positions(*moved)
        assert ctx.rebuild_count() == r0 + 1
        off_b, idx_b = ctx.connections()
        # re-upload of the same tissues with new positions and one changed radius
        ts2 = [t.copy() for t in ts]
        o = 0
        for t in ts2:
            t.x[:], t.y[:], t.z[:] = moved[0][o:o + t.n], moved[1][o:o + t.n], moved[2][o:o + t.n]
            o += t.n
        ts2[3].radius[ts2[3].nmemb + 1] *= 1.01
        r1 = ctx.rebuild_count()
        ctx.upload(ts2)
        assert ctx.rebuild_count() == r1 + 1
        off_c, idx_c = ctx.connections()
        ctx.step(10)
        end = ctx.positions()
    for tissues, positions, (off, idx) in ((ts, pos, (off_a, idx_a)), (ts, moved, (off_b, idx_b))):
        fresh = [t.copy() for t in tissues]
        o = 0
        for t in fresh:
            t.x[:], t.y[:], t.z[:] = (positions[k][o:o + t.n] for k in range(3))
            o += t.n
        _, foff, fidx, _ = run_gpu(fresh, 0, FP64)
        assert lists_equal(off, idx, foff, fidx)
    fpos, foff, fidx, _ = run_gpu(ts2, 0, FP64)
    assert lists_equal(off_c, idx_c, foff, fidx)
    fpos, _, _, _ = run_gpu(ts2, 10, FP64)
    assert max(abs(a - b).max() for a, b in zip(end, fpos)) <= 1e-12


def test_launch_count_counts_the_step_sequence(built):
    """epi_launch_count: eager steps run 8 kernels each (6 rebuild kernels,
    the membrane sums, the step); a graph step runs the work-list kernel
    that sets the rebuild condition, the membrane sums and the step, one loop
    kernel per pass of two steps, and the 5 remaining rebuild kernels only in
    steps where some tissue was flagged."""
    with capi.Context(precision=MIXED) as ctx:
        ctx.upload([T.config1()])
        c0 = ctx.launch_count()
        ctx.step(10, "eager")
        assert ctx.launch_count() - c0 == 80
        c1 = ctx.launch_count()
        r1 = ctx.rebuild_count()
        ctx.step(10, "graph")
        n = ctx.launch_count() - c1
        rebuilt_steps = ctx.rebuild_count() - r1  # one tissue: one rebuild per rebuilding step
        assert n == 10 * 3 + 5 + 5 * rebuilt_steps
