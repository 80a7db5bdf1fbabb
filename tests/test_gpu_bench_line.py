"""bench.py's own arm on the GPU: the JSON line the driver reads, on a small
slice of the ensemble (16 tissues).

The line must carry the contract's keys, a positive device-timed value, the
end-to-end block with the bytes it copies, the number of the library's
launches in the timed steps, the roofline of the step kernel and the
per-kernel split, whose replay of the warm-up and timed steps must land on
the timed run's positions bit for bit.
"""
import json
import os
import subprocess
import sys
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def test_bench_line_on_a_slice_of_the_ensemble(built, tmp_path):
    env = dict(os.environ, EPI_AUTOTUNE_CACHE=str(tmp_path / "autotune.json"))
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--tissues", "16", "--steps", "6",
                        "--warmup", "3", "--no-cpu-baseline", "--dropin-steps", "0",
                        "--adjoint-steps", "0", "--field-steps", "0", "--accuracy-steps", "0",
                        "--tune-steps", "16", "--retune"],
                       capture_output=True, text=True, timeout=900, cwd=ROOT, env=env)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "gpu_launches", "clocks", "e2e", "roofline", "kernel_ms_per_step",
                "kernel_split", "fp64_plain", "fp64_batched"):
        assert key in d, key
    assert d["value"] > 0 and d["steps"] == 6 and d["warmup"] == 3 and d["n_gpus"] == 1
    assert d["gpu_launches"] > 0
    n = d["config"]["particles"]
    e2e = d["e2e"]
    assert e2e["value"] > 0 and e2e["h2d_bytes_per_step"] == e2e["d2h_bytes_per_step"] == 24 * n
    roof = d["roofline"]
    assert roof["bound"] == "hbm" and roof["unit"] == "GB/s" and roof["launch_ms"] > 0
    assert abs(roof["frac"] - roof["achieved"] / roof["peak"]) < 1e-12
    assert d["kernel_split"]["replay_bit_identical"] is True
    assert d["kernel_ms_per_step"]["step"] == pytest.approx(roof["launch_ms"])
    assert d["config"]["autotune"]["cached"] is False
