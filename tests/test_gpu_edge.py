"""Edge cases and randomised tissues through the C ABI against the oracle.

* a membrane with no cells, a single cell, and tissues of very different sizes
  in one batch (ragged);
* seeded random variants of the all-laws tissue (jitter, ages, pairs, the
  membrane lattice, force constants): lists exact and FP64 positions within
  1e-10 of the oracle after 40 steps.
"""
import numpy as np
import pytest

from epi_b200 import capi
from epi_b200 import tissue as T
from oracle import oracle as O
from tests.helpers import lists_equal, list_diff_summary, rel_pos_err

pytestmark = pytest.mark.gpu

FP64 = capi.EPI_PREC_FP64


def gpu(tissues, steps, precision=FP64, params=None):
    with capi.Context(precision=precision, max_conn=96, max_cand=192) as ctx:
        ctx.upload(tissues, params)
        ctx.step(steps)
        return ctx.positions(), ctx.connections(), ctx.dermis()


def oracle(t, steps, params=None):
    ora = O.OracleTissue(t, params=params)
    assert ora.step(steps) == 0, ora.error()
    return ora.positions(), ora.connections(), ora.dermis()


def membrane_only():
    t = T.config1()
    keep = np.arange(t.nmemb)
    return T.Tissue(nmx=t.nmx, nmy=t.nmy, lx=t.lx, ly=t.ly, lz=t.lz, x=t.x[keep].copy(),
                    y=t.y[keep].copy(), z=t.z[keep].copy(), radius=t.radius[keep].copy(),
                    state=t.state[keep].copy(), agek=t.agek[keep].copy(),
                    spr_nat_len=t.spr_nat_len[keep].copy(), pair=t.pair[keep].copy(),
                    rest_div_times=t.rest_div_times[keep].copy(), nmemb=t.nmemb, nder=0,
                    name="membrane only")


def single_cell():
    t = membrane_only()
    n = t.n + 1
    return T.Tissue(nmx=t.nmx, nmy=t.nmy, lx=t.lx, ly=t.ly, lz=t.lz,
                    x=np.append(t.x, 8.05), y=np.append(t.y, 7.95), z=np.append(t.z, 2.0),
                    radius=np.append(t.radius, 0.5),
                    state=np.append(t.state, np.uint8(T.ALIVE)), agek=np.zeros(n),
                    spr_nat_len=np.zeros(n), pair=np.full(n, -1, np.int32),
                    rest_div_times=np.zeros(n, np.int32), nmemb=t.nmemb, nder=0,
                    name="single cell")


@pytest.mark.parametrize("factory", [membrane_only, single_cell])
def test_small_tissues_match_the_oracle(built, factory):
    t = factory()
    t.validate()
    steps = 50
    (p, (off, idx), _), (op, (ooff, oidx), _) = gpu([t], steps), oracle(t, steps)
    assert rel_pos_err(p, op, t.lx, t.ly) <= 1e-12
    assert lists_equal(off, idx, ooff, oidx)


def test_ragged_batch_matches_single_tissues(built):
    ts = [membrane_only(), T.config2(), single_cell(), T.mixed_state_tissue(),
          T.tri_layered_tissue(16, 18, 1, 3)]
    steps = 20
    p, (off, idx), der = gpu(ts, steps)
    o = 0
    for t in ts:
        op, (ooff, oidx), oder = oracle(t, steps)
        seg = [a[o:o + t.n] for a in p]
        assert rel_pos_err(seg, op, t.lx, t.ly) <= 1e-10, t.name
        rows = off[o:o + t.n + 1] - off[o]
        assert lists_equal(rows, idx[off[o]:off[o + t.n]], ooff, oidx), t.name
        fm = (t.state == T.FIX) | (t.state == T.MUSUME)
        assert np.array_equal(der[o:o + t.n][fm], oder[fm]), t.name
        o += t.n


def randomised(seed):
    rng = np.random.default_rng(seed)
    lattice = T.TRIANGULAR if seed % 2 else T.SQUARE
    t = T.mixed_state_tissue(seed=int(rng.integers(1, 1000)), lattice=lattice).copy()
    cells = np.arange(t.nmemb + t.nder, t.n)
    old = rng.random(len(cells)) < 0.4
    t.agek[cells[old]] = rng.uniform(3.1, 30.0, old.sum())
    t.params = t.params.scaled(*rng.uniform(0.6, 1.6, 3))
    return t


@pytest.mark.parametrize("seed", range(6))
def test_randomised_all_laws_tissues_match_the_oracle(built, seed):
    t = randomised(seed)
    steps = 40
    (p, (off, idx), der) = gpu([t], steps, params=[t.params])
    (op, (ooff, oidx), oder) = oracle(t, steps, params=t.params)
    assert rel_pos_err(p, op, t.lx, t.ly) <= 1e-10
    assert lists_equal(off, idx, ooff, oidx), list_diff_summary(off, idx, ooff, oidx)
    fm = (t.state == T.FIX) | (t.state == T.MUSUME)
    assert np.array_equal(der[fm], oder[fm])
