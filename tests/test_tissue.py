"""Synthetic tissue generator: determinism, shapes and the reference file format."""
import numpy as np

from epi_b200 import tissue as T


def test_splitmix64_known_values():
    # splitmix64 from seed 0: first outputs 0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4
    u = T.splitmix64_uniform(0, 2)
    assert u[0] == (0xE220A8397B1DCDAF >> 11) / 2.0**53
    assert u[1] == (0x6E789E6AA1B965F4 >> 11) / 2.0**53


def test_config_shapes():
    t1 = T.config1()
    assert (t1.nmemb, t1.n - t1.nmemb, t1.lx, t1.lz) == (256, 512, 16.0, 32.0)
    t2 = T.config2()
    assert (t2.nmemb, t2.n - t2.nmemb) == (4096, 32768)
    assert np.all((t1.x >= 0) & (t1.x < t1.lx)) and np.all((t1.y >= 0) & (t1.y < t1.ly))
    jit = t1.z[t1.nmemb:] - np.repeat([2.0, 3.0], 256)
    assert np.abs(jit).max() <= 0.1


def test_generator_is_deterministic():
    a, b = T.config1(0), T.config1(0)
    assert np.array_equal(a.x, b.x) and np.array_equal(a.z, b.z)
    c = T.config1(1)
    assert not np.array_equal(a.x, c.x)


def test_config4_ensemble_ranges():
    ts = T.config4(n_tissues=64)
    cells = np.array([t.n - t.nmemb for t in ts])
    assert np.all((cells >= 2048) & (cells <= 40000))
    assert {t.nmx for t in ts} <= set(T.C4_SIDES)
    ks = np.array([t.params.kbend / T.Params().kbend for t in ts])
    assert np.all((ks >= 0.5) & (ks <= 2.0))
    again = T.config4(n_tissues=64)
    assert all(np.array_equal(a.x, b.x) for a, b in zip(ts, again))


def test_reference_file_round_trip(tmp_path):
    t = T.mixed_state_tissue()
    p = tmp_path / "cells.dat"
    t.write_reference_file(str(p))
    rows = np.loadtxt(p)
    assert rows.shape == (t.n, 17)
    assert np.array_equal(rows[:, 1].astype(int), t.state)
    assert np.array_equal(rows[:, 6], t.x) and np.array_equal(rows[:, 8], t.z)
    assert np.array_equal(rows[:, 15].astype(int), t.pair)
    # pairs are mutual, as the reference loader builds them
    paired = np.nonzero(t.pair >= 0)[0]
    assert np.all(t.pair[t.pair[paired]] == paired)


def test_triangular_ensemble_fits_the_reference_grid():
    """config4_tri: the config-4 shapes with triangular membranes. Each box
    must be covered by the reference's grid ((int)(L / 2 + 0.5) bins of 2.0,
    cell_connection.cpp:22-26), rows even (the lattice wiring alternates
    row offsets), every position inside the box."""
    specs = T.config4_specs(n_tissues=16)
    ts = T.config4_tri(n_tissues=16)
    for (side, layers, _), t in zip(specs, ts):
        t.validate()
        rows = T.tri_rows(side)
        assert rows % 2 == 0 and rows >= side
        assert t.nmemb == side * rows
        for L in (t.lx, t.ly):
            assert int(L / 2.0 + 0.5) * 2.0 >= L
        x, y = np.asarray(t.x), np.asarray(t.y)
        assert x.min() >= 0 and x.max() < t.lx and y.min() >= 0 and y.max() < t.ly
