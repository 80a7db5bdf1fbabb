"""The bounds-checked build (libepi_mech_check.so, -DEPI_CHECK): every index
a kernel derives from stored data -- candidate entries, bin slots, sorted
keys, lattice sites, pair and dermis partners -- is checked against its
range before use (EPI_ERR_CHECK on a failure). It stands in for a memory
checker. Run on the parity cases (square and triangular membranes, every
cell state, a ragged batch, both precisions, eager and graph steps), it
must report nothing and give the release build's results."""
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np
import pytest

from epi_b200 import build as B
from epi_b200 import capi
from epi_b200 import tissue as T

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]

CASES = {
    "c1": lambda: [T.config1()],
    "mixed": lambda: [T.mixed_state_tissue()],
    "mixed_tri": lambda: [T.mixed_state_tissue(lattice=T.TRIANGULAR)],
    "ragged": lambda: [T.config1(1), T.layered_tissue(24, 3, 2), T.tri_layered_tissue(16, 18, 2, 0)],
}

RUNNER = r"""
import json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from epi_b200 import capi
from tests.test_gpu_checked_build import CASES
out = {}
for name, make in CASES.items():
    for prec in (capi.EPI_PREC_FP64, capi.EPI_PREC_MIXED):
        for mode in ("eager", "graph"):
            with capi.Context(precision=prec, max_conn=96, max_cand=192) as ctx:
                ctx.upload(make())
                ctx.step(30, mode)
                x, y, z = ctx.positions()
                off, idx = ctx.connections()
            out[f"{name}/{prec}/{mode}"] = [x.tolist(), y.tolist(), z.tolist(),
                                            off.tolist(), idx.tolist()]
json.dump(out, open(sys.argv[2], "w"))
"""


def _run(lib: Path, path: str):
    env = dict(os.environ, EPI_MECH_LIB=str(lib))
    r = subprocess.run([sys.executable, "-c", RUNNER, str(ROOT), path], env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.load(open(path))


def test_checked_build_reports_nothing_and_matches_release(built):
    lib = B.build_library(check=True)
    with tempfile.TemporaryDirectory() as d:
        got = _run(lib, os.path.join(d, "checked.json"))
        ref = _run(B.LIB, os.path.join(d, "release.json"))
    assert got.keys() == ref.keys()
    for k in ref:
        gx, gy, gz, goff, gidx = got[k]
        rx, ry, rz, roff, ridx = ref[k]
        assert goff == roff and gidx == ridx, k
        # the two builds may contract multiply-adds differently: rounding
        # level in FP64, FP32 rounding level of the forces in the mixed path
        tol = 1e-12 if k.split("/")[1] == str(capi.EPI_PREC_FP64) else 1e-8
        for a, b in ((gx, rx), (gy, ry), (gz, rz)):
            assert np.max(np.abs(np.array(a) - np.array(b))) <= tol, k
