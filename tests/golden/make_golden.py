"""Regenerates the golden fixtures from the compiled reference (epi5_MT).

Runs the reference's own mechanics (oracle/_ref, built by oracle/build_ref.py
from the unmodified reference sources, serial TBB stand-in) on seeded
synthetic tissues and stores selected frames: positions, per-cell sorted
connection lists and the dermis of FIX / MUSUME cells. Needs the reference
checkout, so it runs in the build container only; the fixtures it writes are
committed and the tests read them anywhere.

    python tests/golden/make_golden.py [case ...]

Cases "c1", "mixed" and "tri" (triangular membrane, the reference's default
TRI_MEMB build) run the mechanics step (interaction, commit, wrap, connect).
Case "renewal" runs the complete cell_dynamics including the reference's
state renewal, with the harness's division draw fixed at 0 (every division
test that is reached passes), so cells divide, cornify and are removed and
the frames differ in size. Case "shipped" is the reference's own initial
state (epi5_MT/input_2layer_nfix16.dat: 11,400 triangular-lattice membrane
particles, 2,312 dermis cells, 16 stem cells) run by its default build
(define.h as shipped); the fixture also stores that initial state, so the
tests need no reference checkout to load it.
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

# name -> (tissue factory, steps, frame steps kept, harness mode, harness environment)
CASES = {
    "c1": (T.config1, 1000, (0, 100, 1000), "run", {}),
    "mixed": (T.mixed_state_tissue, 300, (0, 50, 300), "run", {}),
    "renewal": (T.renewal_tissue, 200, (0, 1, 20, 100, 200), "dyn", {"EPI_HARNESS_RNG": "zero"}),
    # triangular membrane: the reference's default TRI_MEMB build
    "tri": (lambda: T.tri_layered_tissue(16, 18, 2, 0), 300, (0, 50, 300), "run", {}),
    "mixed_tri": (lambda: T.mixed_state_tissue(lattice=T.TRIANGULAR), 300, (0, 50, 300), "run",
                  {}),
    # the reference's shipped initial state under its default build
    "shipped": (lambda: shipped_input(), 20, (0, 20), "run", {}),
}

# per-particle arrays of the initial state stored with the "shipped" case
STATE_KEYS = ("x", "y", "z", "radius", "state", "agek", "ageb", "spr_nat_len", "pair",
              "rest_div_times")
# define.h as shipped: NMX = 100 membrane columns, LX = LY = 50, LZ = 100
SHIPPED_GEOMETRY = dict(nmx=100, lx=50.0, ly=50.0, lz=100.0)


def shipped_input():
    """The reference's input_2layer_nfix16.dat (reference checkout needed)."""
    path = O.REF_DIR / "epi5_MT" / "input_2layer_nfix16.dat"
    g = SHIPPED_GEOMETRY
    return T.read_reference_file(str(path), g["nmx"], g["lx"], g["ly"], g["lz"])


def load_shipped_tissue():
    """The shipped initial state from the committed fixture."""
    d = np.load(OUT / "shipped.npz")
    st = d["init_state"]
    nmemb = int((st == T.MEMB).sum())
    g = SHIPPED_GEOMETRY
    return T.Tissue(nmx=g["nmx"], nmy=nmemb // g["nmx"], lx=g["lx"], ly=g["ly"], lz=g["lz"],
                    x=d["init_x"], y=d["init_y"], z=d["init_z"], radius=d["init_radius"],
                    state=st, agek=d["init_agek"], ageb=d["init_ageb"],
                    spr_nat_len=d["init_spr_nat_len"], pair=d["init_pair"],
                    rest_div_times=d["init_rest_div_times"], nmemb=nmemb,
                    nder=int((st == T.DER).sum()), name="input_2layer_nfix16.dat",
                    lattice=T.TRIANGULAR)


def make(name: str) -> Path:
    factory, steps, keep, mode, env = CASES[name]
    t = factory()
    every = int(np.gcd.reduce([k for k in keep if k > 0] + [steps]))
    frames = [f for f in O.run_reference(t, steps, every, mode=mode, env=env)
              if f["step"] in keep]
    assert [f["step"] for f in frames] == list(keep)
    out = OUT / f"{name}.npz"
    cat = lambda key: np.concatenate([f[key] for f in frames])
    init = ({f"init_{k}": getattr(t, k) for k in STATE_KEYS} if name == "shipped" else {})
    np.savez_compressed(
        out,
        **init,
        steps=np.array(keep, np.int32),
        n=np.array([len(f["x"]) for f in frames], np.int64),
        x=cat("x"), y=cat("y"), z=cat("z"),
        conn_off=cat("conn_off"),
        # int16 where the indices fit (halves the largest array); load() widens
        conn_idx=cat("conn_idx").astype(np.int16 if len(frames[0]["x"]) < 32768 else np.int32),
        conn_len=np.array([len(f["conn_idx"]) for f in frames], np.int64),
        dermis=cat("dermis"),
    )
    return out


def load(name: str):
    d = np.load(OUT / f"{name}.npz")
    frames = []
    n = d["n"]
    pcut = np.concatenate([[0], np.cumsum(n)])
    ocut = np.concatenate([[0], np.cumsum(n + 1)])
    ccut = np.concatenate([[0], np.cumsum(d["conn_len"])])
    for k, s in enumerate(d["steps"]):
        a, b = pcut[k], pcut[k + 1]
        frames.append(dict(step=int(s), x=d["x"][a:b], y=d["y"][a:b], z=d["z"][a:b],
                           conn_off=d["conn_off"][ocut[k]:ocut[k + 1]],
                           conn_idx=d["conn_idx"][ccut[k]:ccut[k + 1]].astype(np.int32),
                           dermis=d["dermis"][a:b]))
    return frames


if __name__ == "__main__":
    for n in (sys.argv[1:] or CASES):
        print(make(n))
