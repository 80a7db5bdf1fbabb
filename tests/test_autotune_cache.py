"""The autotuner's cache (epi_b200/autotune.py) on the host: a batch shape
tunes once, later runs of the same shape apply the stored choice, and any
change of shape, precision or GPU tunes again. A stand-in context records
the calls (no GPU needed)."""
import json

from epi_b200 import autotune as A
from epi_b200 import tissue as T


class FakeCtx:
    def __init__(self, precision=1):
        self.precision = precision
        self.tuned_with = None
        self.autotuned = 0

    def autotune(self, steps):
        self.autotuned += 1
        return 0.15, 4, 0.42

    def config(self):
        return {"search_switch": 16384, "rebuild_gate": 2}

    def set_tuning(self, skin, variant, switch, gate):
        self.tuned_with = (skin, variant, switch, gate)


def test_cache_tunes_once_per_shape(tmp_path, monkeypatch):
    monkeypatch.setattr(A, "gpu_name", lambda device=0: "B200 x148")
    cache = tmp_path / "c.json"
    ts = [T.config1(s) for s in range(3)]
    a = FakeCtx()
    first = A.tuned(a, ts, 16, cache=cache)
    assert a.autotuned == 1 and not first["cached"]
    assert (first["skin"], first["variant"], first["search_switch"]) == (0.15, 4, 16384)
    b = FakeCtx()
    again = A.tuned(b, [T.config1(s) for s in range(3)], 16, cache=cache)
    assert b.autotuned == 0 and again["cached"] and b.tuned_with == (0.15, 4, 16384, 2)
    # another shape, another precision, another GPU: tuned anew
    c = FakeCtx()
    A.tuned(c, ts[:2], 16, cache=cache)
    d = FakeCtx(precision=0)
    A.tuned(d, ts, 16, cache=cache)
    monkeypatch.setattr(A, "gpu_name", lambda device=0: "B200 x132")
    e = FakeCtx()
    A.tuned(e, ts, 16, cache=cache)
    assert c.autotuned == d.autotuned == e.autotuned == 1
    assert len(json.loads(cache.read_text())) == 4
    # retune ignores the stored choice
    f = FakeCtx()
    A.tuned(f, ts, 16, cache=cache, retune=True)
    assert f.autotuned == 1
