"""The reference gradient is pinned before it is trusted.

oracle/epi_oracle_tangent.cpp restates the step as a template: its plain
double instantiation must reproduce the C oracle (itself pinned to the
compiled reference) bit for bit, the dual-number instantiation must carry
the same values, and its gradient must match central finite differences of
the oracle's own step (h = 1e-4 relative).
"""
import numpy as np
import pytest

from epi_b200 import tissue as T
from oracle import oracle as O

STEPS = 200
H = 1e-4


def aged_tissue():
    """C1 with every other cell older than THRESH_SP and some DEAD / AIR cells,
    so that both adhesion constants (K_TOTAL for two old cells) take part."""
    t = T.config1(3).copy()
    cells = np.arange(t.nmemb, t.n)
    t.agek[cells[::2]] = 5.0
    t.agek[cells[::5]] = 4.0
    t.state[cells[3::7]] = T.DEAD
    t.state[cells[5::11]] = T.AIR
    t.validate()
    return t


def tri_tissue():
    """Two cell layers over a 16 x 18 triangular membrane (TRI_MEMB)."""
    return T.tri_layered_tissue(16, 18, 2, 0)


def min_image_loss(t, pos, target):
    d = [pos[k] - target[k] for k in range(3)]
    for k, L in ((0, t.lx), (1, t.ly)):
        d[k] = np.where(d[k] > 0.5 * L, d[k] - L, np.where(d[k] <= -0.5 * L, d[k] + L, d[k]))
    m = slice(t.nmemb, t.n)
    return float(np.mean(d[0][m] ** 2 + d[1][m] ** 2 + d[2][m] ** 2))


def oracle_positions(t, steps, params=None):
    ora = O.OracleTissue(t, params=params)
    assert ora.step(steps) == 0, ora.error()
    return ora.positions()


def mixed_tri():
    return T.mixed_state_tissue(lattice=T.TRIANGULAR)


@pytest.mark.parametrize("factory", [T.config1, aged_tissue, tri_tissue, T.mixed_state_tissue,
                                     mixed_tri])
def test_tangent_value_path_is_the_oracle_bit_for_bit(built, factory):
    t = factory()
    ref = oracle_positions(t, STEPS)
    _, _, plain = O.tangent_gradient(t, STEPS, dual=False)
    _, _, dual = O.tangent_gradient(t, STEPS, target=ref)
    for k in range(3):
        assert np.array_equal(plain[k], ref[k])
        assert np.array_equal(dual[k], ref[k])


@pytest.mark.parametrize("factory", [T.config1, aged_tissue, tri_tissue])
def test_tangent_gradient_matches_central_differences(built, factory):
    t = factory()
    target = oracle_positions(t, STEPS, t.params.scaled(1.1, 1.1, 1.1))
    loss, grad, pos = O.tangent_gradient(t, STEPS, target=target)
    assert loss == pytest.approx(min_image_loss(t, pos, target), rel=1e-12)
    for k in range(3):
        e = [1.0, 1.0, 1.0]
        e[k] = 1.0 + H
        lp = min_image_loss(t, oracle_positions(t, STEPS, t.params.scaled(*e)), target)
        e[k] = 1.0 - H
        lm = min_image_loss(t, oracle_positions(t, STEPS, t.params.scaled(*e)), target)
        fd = (lp - lm) / (2 * H)
        assert abs(fd - grad[k]) <= 1e-5 * abs(grad[k]), (k, fd, grad[k])


@pytest.mark.parametrize("factory", [T.mixed_state_tissue, mixed_tri])
def test_tangent_gradient_all_laws_matches_central_differences(built, factory):
    """Every cell state and law (DER, FIX, MUSUME with their dermis springs,
    pairs). Shorter run: DER pairs have laws that jump where their branches
    meet (CI_der_to_der at r = r_i + r_j, ljmain at the connection cut-off),
    which central differences must not straddle. The bending component is
    small here, so its bar adds 1e-6 of the largest component."""
    t = factory()
    steps = 10
    target = oracle_positions(t, steps, t.params.scaled(1.1, 1.1, 1.1))
    loss, grad, pos = O.tangent_gradient(t, steps, target=target)
    assert loss == pytest.approx(min_image_loss(t, pos, target), rel=1e-12)
    for k in range(3):
        e = [1.0, 1.0, 1.0]
        e[k] = 1.0 + H
        lp = min_image_loss(t, oracle_positions(t, steps, t.params.scaled(*e)), target)
        e[k] = 1.0 - H
        lm = min_image_loss(t, oracle_positions(t, steps, t.params.scaled(*e)), target)
        fd = (lp - lm) / (2 * H)
        assert abs(fd - grad[k]) <= 1e-5 * abs(grad[k]) + 1e-6 * np.max(np.abs(grad)), \
            (k, fd, grad[k])


def test_tangent_rejects_a_broken_layout(built):
    t = T.config1()
    t = t.copy()
    t.state[0] = T.ALIVE  # a membrane slot that is not a membrane particle
    with pytest.raises(RuntimeError):
        O.tangent_gradient(t, 1)
