"""bench.py's reference arm on the CPU: the JSON line the driver reads.

`bench.py --impl reference` times the compiled epi5_MT (the reference's own
CPU path) on a bounded sample of the workload, without a GPU. Its single
line must carry the metric, a positive value, and the cpu_baseline / e2e
keys of the contract; where the compiled reference is absent it prints an
`unavailable` line instead.
"""
import json
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_reference_arm_prints_one_contract_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference",
                        "--steps", "1", "--warmup", "1", "--ref-particles", "4000"],
                       capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [l for l in r.stdout.splitlines() if l.strip()]
    assert len(lines) == 1, r.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    if "unavailable" in d:
        return
    assert d["value"] > 0 and d["unit"] == "cell-updates/s" and d["higher_is_better"] is True
    for key in ("metric", "n_gpus", "steps", "warmup", "ms_per_step", "scaling", "dtype",
                "data", "config"):
        assert key in d, key
    cb = d["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}
