"""Reverse-mode adjoint (epi_adjoint) against the oracle's forward-mode
gradient and against central finite differences of the GPU's own step.

Loss: mean squared minimum-image distance of the final cell positions to a
target made by a run with every force constant +10% (spring, LJ epsilon,
bending), as the adjoint workload specifies. Gradient: d loss / d (s_spring,
s_eps, s_bend), the multipliers of those constants at 1.

Tissues: square membranes and a triangular one (TRI_MEMB, the reference's
default lattice), under ALIVE / DEAD / AIR cells, and tissues with every
cell state and law (DER, FIX, MUSUME, pairs) on both lattices.

Bars: FP64 adjoint vs the FP64 forward-mode reference gradient within 1e-6
relative per component; vs central differences (h = 1e-4 relative) within
1e-4 relative; independent of the checkpoint interval; per-tissue results
of a batch (one lattice or both) equal single-tissue runs.
"""
import numpy as np
import pytest

from epi_b200 import capi
from epi_b200 import tissue as T
from oracle import oracle as O
from tests.test_oracle_tangent import aged_tissue, min_image_loss, tri_tissue

pytestmark = pytest.mark.gpu

FP64 = capi.EPI_PREC_FP64
MIXED = capi.EPI_PREC_MIXED
H = 1e-4


def gpu_positions(t, steps, params=None, precision=FP64, **cfg):
    with capi.Context(precision=precision, **cfg) as ctx:
        ctx.upload([t], [params] if params is not None else None)
        ctx.step(steps)
        return ctx.positions()


def gpu_adjoint(tissues, steps, targets, K=20, precision=FP64, params=None, **cfg):
    with capi.Context(precision=precision, **cfg) as ctx:
        ctx.upload(tissues, params)
        tgt = [np.concatenate([tg[k] for tg in targets]) for k in range(3)]
        loss, grad = ctx.adjoint(steps, tgt, checkpoint_every=K)
        end = ctx.positions()
    return loss, grad, end


def target_of(t, steps, **cfg):
    return gpu_positions(t, steps, t.params.scaled(1.1, 1.1, 1.1), **cfg)


@pytest.mark.parametrize("factory,steps", [(T.config1, 200), (aged_tissue, 200),
                                           (T.config5, 200), (tri_tissue, 200)])
def test_adjoint_matches_forward_mode_reference_gradient(built, factory, steps):
    t = factory()
    target = target_of(t, steps)
    loss, grad, _ = gpu_adjoint([t], steps, [target])
    rloss, rgrad, _ = O.tangent_gradient(t, steps, target=target)
    assert loss[0] == pytest.approx(rloss, rel=1e-9)
    for k in range(3):
        assert abs(grad[0, k] - rgrad[k]) <= 1e-6 * abs(rgrad[k]), (k, grad[0], rgrad)


@pytest.mark.parametrize("factory", [T.config1, T.config5, tri_tissue])
def test_adjoint_matches_central_differences(built, factory):
    t = factory()
    steps = 200
    target = target_of(t, steps)
    _, grad, _ = gpu_adjoint([t], steps, [target])
    for k in range(3):
        e = [1.0, 1.0, 1.0]
        e[k] = 1.0 + H
        lp = min_image_loss(t, gpu_positions(t, steps, t.params.scaled(*e)), target)
        e[k] = 1.0 - H
        lm = min_image_loss(t, gpu_positions(t, steps, t.params.scaled(*e)), target)
        fd = (lp - lm) / (2 * H)
        assert abs(grad[0, k] - fd) <= 1e-4 * abs(fd), (k, grad[0, k], fd)


def test_adjoint_independent_of_checkpoint_interval_and_leaves_final_state(built):
    t = T.config1(2)
    steps = 60
    target = target_of(t, steps)
    ref_end = gpu_positions(t, steps)
    results = [gpu_adjoint([t], steps, [target], K=K) for K in (1, 7, 20, 60, 100)]
    l0, g0, _ = results[0]
    for loss, grad, end in results:
        assert loss[0] == pytest.approx(l0[0], rel=1e-13)
        assert np.allclose(grad, g0, rtol=1e-11, atol=0)
        for k in range(3):
            assert np.array_equal(end[k], ref_end[k])


def test_adjoint_batched_equals_single_tissue_runs(built):
    ta, tb = T.config1(1), aged_tissue()
    pa, pb = ta.params.scaled(0.7, 1.3, 1.8), tb.params.scaled(1.4, 0.6, 0.5)
    steps = 80
    tga = gpu_positions(ta, steps, pa.scaled(1.1, 1.1, 1.1))
    tgb = gpu_positions(tb, steps, pb.scaled(1.1, 1.1, 1.1))
    loss, grad, _ = gpu_adjoint([ta, tb], steps, [tga, tgb], params=[pa, pb])
    la, ga, _ = gpu_adjoint([ta], steps, [tga], params=[pa])
    lb, gb, _ = gpu_adjoint([tb], steps, [tgb], params=[pb])
    assert loss[0] == pytest.approx(la[0], rel=1e-12) and loss[1] == pytest.approx(lb[0], rel=1e-12)
    assert np.allclose(grad[0], ga[0], rtol=1e-10, atol=0)
    assert np.allclose(grad[1], gb[0], rtol=1e-10, atol=0)
    # a per-tissue parameter set is differentiated at its own constants
    rl, rg, _ = O.tangent_gradient(tb, steps, target=tgb, params=pb)
    assert np.allclose(grad[1], rg, rtol=1e-6, atol=0)


def test_adjoint_mixed_precision_close_to_fp64(built):
    t = T.config1()
    steps = 200
    target = target_of(t, steps)
    _, g64, _ = gpu_adjoint([t], steps, [target])
    _, gmx, _ = gpu_adjoint([t], steps, [target], precision=MIXED)
    assert np.allclose(gmx, g64, rtol=1e-2, atol=0), (gmx, g64)


MIXED_CFG = dict(max_conn=96, max_cand=192)


def mixed_tri():
    return T.mixed_state_tissue(lattice=T.TRIANGULAR)


@pytest.mark.parametrize("factory", [T.mixed_state_tissue, mixed_tri])
def test_adjoint_all_laws_matches_forward_mode_reference_gradient(built, factory):
    """Every cell state and law: DER (CI_der_to_der, wall), FIX and MUSUME
    with their dermis springs, pairs of dividing cells, old cells."""
    t = factory()
    steps = 60
    target = target_of(t, steps, **MIXED_CFG)
    loss, grad, _ = gpu_adjoint([t], steps, [target], **MIXED_CFG)
    rloss, rgrad, _ = O.tangent_gradient(t, steps, target=target)
    assert loss[0] == pytest.approx(rloss, rel=1e-9)
    for k in range(3):
        assert abs(grad[0, k] - rgrad[k]) <= 1e-6 * abs(rgrad[k]) + 1e-9 * np.max(np.abs(rgrad)), \
            (k, grad[0], rgrad)


@pytest.mark.parametrize("factory", [T.mixed_state_tissue, mixed_tri])
def test_adjoint_all_laws_matches_central_differences(built, factory):
    """Short run: DER laws jump where their branches meet, which central
    differences must not straddle; the small bending component's bar adds
    1e-6 of the largest component."""
    t = factory()
    steps = 10
    target = target_of(t, steps, **MIXED_CFG)
    _, grad, _ = gpu_adjoint([t], steps, [target], **MIXED_CFG)
    g = grad[0]
    for k in range(3):
        e = [1.0, 1.0, 1.0]
        e[k] = 1.0 + H
        lp = min_image_loss(t, gpu_positions(t, steps, t.params.scaled(*e), **MIXED_CFG), target)
        e[k] = 1.0 - H
        lm = min_image_loss(t, gpu_positions(t, steps, t.params.scaled(*e), **MIXED_CFG), target)
        fd = (lp - lm) / (2 * H)
        assert abs(g[k] - fd) <= 1e-4 * abs(fd) + 1e-6 * np.max(np.abs(g)), (k, g[k], fd)


def test_adjoint_rejects_invalid_arguments(built):
    t = T.config1()
    with capi.Context(precision=FP64) as ctx:
        ctx.upload([t])
        with pytest.raises(capi.EpiError) as e:
            ctx.adjoint(5, (t.x, t.y, t.z), checkpoint_every=0)
        assert e.value.code == capi.EPI_ERR_INVALID_ARG


def test_adjoint_square_and_triangular_tissues_in_one_batch(built):
    """A batch mixing both lattices: each tissue's gradient equals its own
    single-tissue run (the bending-product buffer and the gathers are per
    tissue and per lattice)."""
    ta, tb = T.config1(1), tri_tissue()
    steps = 60
    tga, tgb = target_of(ta, steps), target_of(tb, steps)
    loss, grad, _ = gpu_adjoint([ta, tb], steps, [tga, tgb])
    la, ga, _ = gpu_adjoint([ta], steps, [tga])
    lb, gb, _ = gpu_adjoint([tb], steps, [tgb])
    assert loss[0] == pytest.approx(la[0], rel=1e-12) and loss[1] == pytest.approx(lb[0], rel=1e-12)
    assert np.allclose(grad[0], ga[0], rtol=1e-10, atol=0)
    assert np.allclose(grad[1], gb[0], rtol=1e-10, atol=0)
