"""epi_autotune: picks a (skin, variant) pair from its grid by timing, leaves
the simulation state untouched, and the chosen configuration gives the same
results as the default one (connection sets are exact for every skin)."""
import numpy as np
import pytest

from epi_b200 import capi
from epi_b200 import tissue as T
from tests.helpers import lists_equal, rel_pos_err

pytestmark = pytest.mark.gpu


def test_autotune_keeps_state_and_results(built):
    tissues = T.config4(n_tissues=24)
    with capi.Context(precision=capi.EPI_PREC_FP64) as ctx:
        ctx.upload(tissues)
        ctx.step(10)
        before = ctx.positions()
        skin, variant, ms = ctx.autotune(8)
        assert skin in (0.05, 0.08, 0.1, 0.15, 0.2, 0.3)
        assert variant in (1, 2, 3, 4)
        assert ms > 0
        after = ctx.positions()
        for a, b in zip(before, after):
            assert np.array_equal(a, b)
        ctx.step(40, "graph")
        tuned = ctx.positions()
        off_t, idx_t = ctx.connections()
    with capi.Context(precision=capi.EPI_PREC_FP64) as ref:
        ref.upload(tissues)
        ref.step(50)
        base = ref.positions()
        off_b, idx_b = ref.connections()
    # the only freedom left to the variants is multiply-add contraction
    assert max(abs(a - b).max() for a, b in zip(tuned, base)) <= 1e-12
    assert lists_equal(off_t, idx_t, off_b, idx_b)
