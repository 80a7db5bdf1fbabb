"""Regenerates the golden fixtures from the compiled reference (epi5_MT).

Runs the reference's own mechanics (oracle/_ref, built by oracle/build_ref.py
from the unmodified reference sources, serial TBB stand-in) on seeded
synthetic tissues and stores selected frames: positions, per-cell sorted
connection lists and the dermis of FIX / MUSUME cells. Needs the reference
checkout, so it runs in the build container only; the fixtures it writes are
committed and the tests read them anywhere.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from epi_b200 import tissue as T  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = Path(__file__).resolve().parent

# name -> (tissue factory, steps, frame steps kept)
CASES = {
    "c1": (T.config1, 1000, (0, 100, 1000)),
    "mixed": (T.mixed_state_tissue, 300, (0, 50, 300)),
}


def make(name: str) -> Path:
    factory, steps, keep = CASES[name]
    t = factory()
    every = int(np.gcd.reduce([k for k in keep if k > 0] + [steps]))
    frames = [f for f in O.run_reference(t, steps, every) if f["step"] in keep]
    assert [f["step"] for f in frames] == list(keep)
    out = OUT / f"{name}.npz"
    np.savez_compressed(
        out,
        steps=np.array(keep, np.int32),
        x=np.stack([f["x"] for f in frames]),
        y=np.stack([f["y"] for f in frames]),
        z=np.stack([f["z"] for f in frames]),
        conn_off=np.stack([f["conn_off"] for f in frames]),
        conn_idx=np.concatenate([f["conn_idx"] for f in frames]),
        conn_len=np.array([len(f["conn_idx"]) for f in frames], np.int64),
        dermis=np.stack([f["dermis"] for f in frames]),
    )
    return out


def load(name: str):
    d = np.load(OUT / f"{name}.npz")
    frames = []
    cut = np.concatenate([[0], np.cumsum(d["conn_len"])])
    for k, s in enumerate(d["steps"]):
        frames.append(dict(step=int(s), x=d["x"][k], y=d["y"][k], z=d["z"][k],
                           conn_off=d["conn_off"][k], conn_idx=d["conn_idx"][cut[k]:cut[k + 1]],
                           dermis=d["dermis"][k]))
    return frames


if __name__ == "__main__":
    for n in CASES:
        print(make(n))
