"""The drop-in: epi5_MT's own step loop with connect_cell and cell_interaction
replaced by epi_b200/shim/epi5_gpu_mechanics.cpp over the C ABI.

The binary (oracle/_ref/<geometry>/ref_harness_dropin, built by
`python oracle/build_ref.py --dropin` where the reference sources are) is the
reference's harness compiled from the reference's own cellmanager, cell,
cell_init, utils ... translation units; only the two mechanics files differ.
Its frames must match the reference's golden frames to the library's FP64
bars: lists and dermis bit-exact, positions within 1e-10 of L_x after 1000
steps. In the default (mixed) precision the positions stay within 1e-5.
"""
import numpy as np
import pytest

from epi_b200 import tissue as T
from oracle import oracle as O
from tests.golden.make_golden import load
from tests.helpers import lists_equal, list_diff_summary, rel_pos_err

pytestmark = pytest.mark.gpu

TOL_FP64 = 1e-10
TOL_MIXED = 1e-5


def _dropin_frames(t, steps, every, precision):
    if O.reference_binary(t, "dropin") is None:
        pytest.skip("drop-in harness not built (python oracle/build_ref.py --dropin)")
    return O.run_reference(t, steps, every, variant="dropin",
                           env={"EPI_MECH_PRECISION": precision})


@pytest.mark.parametrize("name,factory,steps,every", [
    ("c1", T.config1, 1000, 100),
    ("mixed", T.mixed_state_tissue, 300, 50),
])
def test_dropin_fp64_matches_reference_frames(built, name, factory, steps, every):
    t = factory()
    golden = {f["step"]: f for f in load(name)}
    frames = {f["step"]: f for f in _dropin_frames(t, steps, every, "fp64")}
    fm = (t.state == T.FIX) | (t.state == T.MUSUME)
    for s, g in golden.items():
        f = frames[s]
        err = rel_pos_err((f["x"], f["y"], f["z"]), (g["x"], g["y"], g["z"]), t.lx, t.ly)
        assert err <= TOL_FP64, (name, s, err)
        assert lists_equal(f["conn_off"], f["conn_idx"], g["conn_off"], g["conn_idx"]), \
            list_diff_summary(f["conn_off"], f["conn_idx"], g["conn_off"], g["conn_idx"])
        assert np.array_equal(f["dermis"][fm], g["dermis"][fm]), (name, s)
        # positions come back wrapped into the box by the host's periodic fix
        assert (f["x"] >= 0).all() and (f["x"] <= t.lx).all()
        assert (f["y"] >= 0).all() and (f["y"] <= t.ly).all()


def test_dropin_mixed_precision_within_bar(built):
    t = T.config1()
    golden = {f["step"]: f for f in load("c1")}
    frames = {f["step"]: f for f in _dropin_frames(t, 1000, 100, "mixed")}
    for s, g in golden.items():
        f = frames[s]
        err = rel_pos_err((f["x"], f["y"], f["z"]), (g["x"], g["y"], g["z"]), t.lx, t.ly)
        assert err <= TOL_MIXED, (s, err)


def test_dropin_runs_the_reference_state_renewal_loop(built):
    """epi5_MT's complete cell_dynamics (cell_state_renew between pos_copy and
    the periodic fix, proc.cpp:22-32) with the drop-in: cells divide (the batch
    grows and is re-uploaded), are removed (the reference swaps the last cell
    into the gap) and cornify, and every frame still matches the serial
    reference's (division draw fixed at 0 in both)."""
    t = T.renewal_tissue()
    if O.reference_binary(t, "dropin") is None:
        pytest.skip("drop-in harness not built (python oracle/build_ref.py --dropin)")
    frames = {f["step"]: f for f in O.run_reference(
        t, 200, 1, variant="dropin", mode="dyn",
        env={"EPI_MECH_PRECISION": "fp64", "EPI_HARNESS_RNG": "zero"})}
    golden = load("renewal")
    assert len(golden[0]["x"]) != len(golden[-1]["x"])
    for g in golden:
        f = frames[g["step"]]
        assert len(f["x"]) == len(g["x"]), g["step"]
        err = rel_pos_err((f["x"], f["y"], f["z"]), (g["x"], g["y"], g["z"]), t.lx, t.ly)
        assert err <= TOL_FP64, (g["step"], err)
        assert lists_equal(f["conn_off"], f["conn_idx"], g["conn_off"], g["conn_idx"]), \
            list_diff_summary(f["conn_off"], f["conn_idx"], g["conn_off"], g["conn_idx"])
        assert np.array_equal(f["dermis"], g["dermis"]), g["step"]


def test_dropin_triangular_build_matches_reference_frames(built):
    """The drop-in compiled into the reference's default TRI_MEMB build."""
    t = T.tri_layered_tissue(16, 18, 2, 0)
    golden = {f["step"]: f for f in load("tri")}
    frames = {f["step"]: f for f in _dropin_frames(t, 300, 50, "fp64")}
    for s, g in golden.items():
        f = frames[s]
        err = rel_pos_err((f["x"], f["y"], f["z"]), (g["x"], g["y"], g["z"]), t.lx, t.ly)
        assert err <= TOL_FP64, (s, err)
        assert lists_equal(f["conn_off"], f["conn_idx"], g["conn_off"], g["conn_idx"])


@pytest.mark.parametrize("case", ["mixed", "renewal"])
def test_dropin_gap_junction_bookkeeping_matches_reference(built, case):
    """The gap-junction maps the drop-in's connect_cell leaves for the
    chemistry (gj_refresh, cell_connection.cpp:133-152; read by
    ca2p.cpp:204-207) equal the reference's: per cell the same partners,
    values and marks. With state renewal, cells are removed and the reference
    keeps their map keys (never dereferenced here); there the marked entries
    and each cell's key count are compared."""
    if case == "mixed":
        t, mode, env, steps, every = T.mixed_state_tissue(), "run", {}, 300, 50
    else:
        t, mode, env, steps, every = (T.renewal_tissue(), "dyn", {"EPI_HARNESS_RNG": "zero"},
                                      200, 20)
    if O.reference_binary(t, "dropin") is None or O.reference_binary(t, "serial") is None:
        pytest.skip("reference and drop-in harnesses not built (oracle/build_ref.py --dropin)")
    _, ref = O.run_reference_gj(t, steps, every, mode=mode, env=env)
    _, got = O.run_reference_gj(t, steps, every, variant="dropin", mode=mode,
                                env=dict(env, EPI_MECH_PRECISION="fp64"))
    assert [g["step"] for g in got] == [g["step"] for g in ref]
    for a, b in zip(ref, got):
        s = a["step"]
        if case == "mixed":
            for k in ("off", "idx", "checked", "value", "dead"):
                assert np.array_equal(a[k], b[k]), (s, k)
        else:
            keys_a = np.diff(a["off"]) + a["dead"]
            keys_b = np.diff(b["off"]) + b["dead"]
            assert np.array_equal(keys_a, keys_b), s
            row_a = np.repeat(np.arange(len(a["dead"])), np.diff(a["off"]))
            row_b = np.repeat(np.arange(len(b["dead"])), np.diff(b["off"]))
            ca, cb = a["checked"] == 1, b["checked"] == 1
            for arr_a, arr_b in ((row_a, row_b), (a["idx"], b["idx"]), (a["value"], b["value"])):
                assert np.array_equal(arr_a[ca], arr_b[cb]), s
