"""The oracle is pinned before it is trusted.

The C restatement (oracle/epi_oracle.c) must reproduce, bit for bit, the
frames the compiled reference (epi5_MT sources, serial TBB stand-in) wrote
into tests/golden/ -- positions, sorted connection lists and dermis -- and,
where the compiled reference is present, fresh runs of it.
"""
import numpy as np
import pytest

from epi_b200 import tissue as T
from oracle import oracle as O
from tests.golden.make_golden import load
from tests.helpers import lists_equal


def tri_c1():
    return T.tri_layered_tissue(16, 18, 2, 0)


@pytest.mark.parametrize("name,factory", [
    ("c1", T.config1), ("mixed", T.mixed_state_tissue), ("tri", tri_c1),
    ("mixed_tri", lambda: T.mixed_state_tissue(lattice=T.TRIANGULAR)),
])
def test_oracle_reproduces_reference_golden_frames(built, name, factory):
    frames = load(name)
    t = factory()
    ora = O.OracleTissue(t)
    done = 0
    fix_mu = (t.state == T.FIX) | (t.state == T.MUSUME)
    for f in frames:
        assert ora.step(f["step"] - done) == 0, ora.error()
        done = f["step"]
        x, y, z = ora.positions()
        assert np.array_equal(x, f["x"]) and np.array_equal(y, f["y"]) and np.array_equal(z, f["z"])
        off, idx = ora.connections()
        assert lists_equal(off, idx, f["conn_off"], f["conn_idx"])
        assert np.array_equal(ora.dermis()[fix_mu], f["dermis"][fix_mu])


def _ref_available(t):
    return O.reference_binary(t) is not None


@pytest.mark.parametrize("factory,steps", [
    (lambda: T.layered_tissue(24, 3, 11), 40),
    (lambda: T.layered_tissue(64, 8, 1), 3),
    (lambda: T.config1(5), 200),
    (lambda: T.tri_layered_tissue(32, 36, 4, 3), 50),
])
def test_oracle_matches_compiled_reference_live(built, factory, steps):
    t = factory()
    if not _ref_available(t):
        pytest.skip("compiled reference not built here (no reference checkout)")
    frames = O.run_reference(t, steps, steps)
    ora = O.OracleTissue(t)
    assert ora.step(steps) == 0
    x, y, z = ora.positions()
    f = frames[-1]
    assert np.array_equal(x, f["x"]) and np.array_equal(y, f["y"]) and np.array_equal(z, f["z"])
    off, idx = ora.connections()
    assert lists_equal(off, idx, f["conn_off"], f["conn_idx"])


def test_oracle_raw_lists_start_with_lattice_links(built):
    t = T.config1()
    ora = O.OracleTissue(t)
    off, idx = ora.connections(raw=True)
    # _memb_init pushes l, r, b, u first (cellmanager.cpp:160-163)
    row = idx[off[17]:off[18]]
    assert row[:4].tolist() == [16, 18, 1, 33]


def test_oracle_flags_too_strong_interaction(built):
    t = T.config1()
    k = t.nmemb
    t.x[k + 1], t.y[k + 1], t.z[k + 1] = t.x[k] + 0.3, t.y[k], t.z[k]
    ora = O.OracleTissue(t)
    code = ora.step(1)
    assert code == 8  # EPI_ERR_COEF_RANGE: the reference prints "Too strong interaction" and exits


def test_oracle_flags_out_of_grid(built):
    t = T.config1()
    t.z[t.nmemb + 3] = 40.0  # above LZ = 32: grid_init's range assert
    ora = O.OracleTissue(t)
    assert ora.error()[0] == 5


def test_renewal_fixture_reproduces_with_the_compiled_reference(built):
    """tests/golden/renewal.npz: the reference's complete cell_dynamics (state
    renewal included, division draw fixed at 0) is deterministic and the
    committed frames are what it writes."""
    t = T.renewal_tissue()
    if not _ref_available(t):
        pytest.skip("compiled reference not built here (no reference checkout)")
    golden = load("renewal")
    frames = {f["step"]: f for f in O.run_reference(t, 200, 1, mode="dyn",
                                                     env={"EPI_HARNESS_RNG": "zero"})}
    for g in golden:
        f = frames[g["step"]]
        for k in ("x", "y", "z", "conn_off", "conn_idx", "dermis"):
            assert np.array_equal(f[k], g[k]), (g["step"], k)
    # the run divides, cornifies and removes cells: the batch size changes
    assert len(golden[0]["x"]) != len(golden[-1]["x"])


SHIPPED_INPUT = O.REF_DIR / "epi5_MT" / "input_2layer_nfix16.dat"


def test_oracle_matches_reference_default_build_on_its_shipped_input(built):
    """The reference's own default build (define.h as shipped: TRI_MEMB,
    NMX = 100, 50 x 50 x 100 box) on its own initial state
    (epi5_MT/input_2layer_nfix16.dat: 11,400 membrane, 2,312 dermis and 16
    stem cells): the oracle reproduces it bit for bit. Runs where the
    reference checkout is present."""
    if not SHIPPED_INPUT.exists():
        pytest.skip("reference checkout not present")
    t = T.read_reference_file(str(SHIPPED_INPUT), 100, 50.0, 50.0, 100.0)
    assert (t.nmemb, t.nder, t.nmy) == (11400, 2312, 114)
    if not _ref_available(t):
        pytest.skip("compiled reference default build not present")
    f = O.run_reference(t, 20, 20)[-1]
    ora = O.OracleTissue(t)
    assert ora.step(20) == 0, ora.error()
    x, y, z = ora.positions()
    assert np.array_equal(x, f["x"]) and np.array_equal(y, f["y"]) and np.array_equal(z, f["z"])
    off, idx = ora.connections()
    assert lists_equal(off, idx, f["conn_off"], f["conn_idx"])
    fix = t.state == T.FIX
    assert np.array_equal(ora.dermis()[fix], f["dermis"][fix])


@pytest.mark.parametrize("factory", [T.field_tissue, T.config1])
def test_oracle_field_matches_compiled_reference(built, factory):
    """Cell maps and external stimulus (setup_map_lat, calc_ext_stim) after
    each mechanics step, bit for bit against the compiled reference's own
    map.cpp and ext_stim.cpp (32 x 32 x 64 grid)."""
    t = factory()
    if not _ref_available(t):
        pytest.skip("compiled reference not built here (no reference checkout)")
    frames = {f["step"]: f for f in O.run_reference_field(t, 20, 5)}
    ora = O.OracleTissue(t)
    fld = O.OracleField(ora, 32, 32, 64)
    for s in range(1, 21):
        assert ora.step(1) == 0
        rc, zz = fld.step()
        assert rc == 0
        if s in frames:
            f = frames[s]
            m1, m2, ex = fld.get()
            assert zz == f["zzmax"]
            assert np.array_equal(m1, f["cmap1"]) and np.array_equal(m2, f["cmap2"])
            assert np.array_equal(ex, f["ext"])
    if factory is T.field_tissue:
        assert f["ext"].max() > 0.1  # sources were on
