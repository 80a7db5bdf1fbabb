"""Cached autotuning: epi_autotune's choice stored per batch shape.

epi_autotune times trials of the uploaded batch (skin x step-kernel variant,
then the candidate-search switch); its choice depends only on the batch's
shape, its precision and the GPU, not on the positions. tuned() looks the
shape up in a JSON cache first and applies a stored choice with
epi_set_tuning, so repeated runs of one workload tune once.

Key: precision, GPU name and SM count, tissue count, and a digest of every
tissue's (particles, membrane particles, lattice, box).
"""
from __future__ import annotations

import hashlib
import json
import os
from pathlib import Path
from typing import Optional, Sequence

DEFAULT_CACHE = Path(__file__).resolve().parent / "autotune_cache.json"


def shape_key(tissues: Sequence, precision: int, gpu: str) -> str:
    h = hashlib.sha1()
    for t in tissues:
        h.update(f"{t.n},{t.nmemb},{getattr(t, 'lattice', 0)},{t.lx:.6g},{t.ly:.6g},"
                 f"{t.lz:.6g};".encode())
    return f"p{precision}|{gpu}|{len(tissues)}|{h.hexdigest()[:16]}"


def gpu_name(device: int = 0) -> str:
    try:
        import torch
        p = torch.cuda.get_device_properties(device)
        return f"{p.name} x{p.multi_processor_count}"
    except Exception:
        return "unknown"


def _load(path: Path) -> dict:
    try:
        return json.loads(path.read_text())
    except (OSError, ValueError):
        return {}


def tuned(ctx, tissues: Sequence, trial_steps: int = 128, cache: Optional[Path] = None,
          device: int = 0, retune: bool = False) -> dict:
    """Applies the cached choice for this batch shape to ctx, or runs
    epi_autotune and stores its choice. Returns {skin, variant,
    search_switch, rebuild_gate, trial_ms_per_step, cached}."""
    path = Path(cache or os.environ.get("EPI_AUTOTUNE_CACHE", DEFAULT_CACHE))
    key = shape_key(tissues, ctx.precision, gpu_name(device))
    db = _load(path)
    hit = db.get(key)
    if hit and not retune:
        ctx.set_tuning(hit["skin"], hit["variant"], hit["search_switch"],
                       hit.get("rebuild_gate", 0))
        return dict(hit, cached=True)
    skin, variant, ms = ctx.autotune(trial_steps)
    cfg = ctx.config()
    rec = {"skin": skin, "variant": variant, "search_switch": int(cfg["search_switch"]),
           "rebuild_gate": int(cfg["rebuild_gate"]),
           "trial_ms_per_step": ms, "trial_steps": trial_steps}
    db[key] = rec
    try:
        path.write_text(json.dumps(db, indent=1, sort_keys=True) + "\n")
    except OSError:
        pass  # a read-only checkout still tunes, it only does not remember
    return dict(rec, cached=False)
