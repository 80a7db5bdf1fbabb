"""Comparison helpers shared by the tests."""
from __future__ import annotations

import numpy as np


def min_image_err(a, b, lx, ly):
    """Per-particle |r_a - r_b| with minimum-image x/y differences."""
    ax, ay, az = a
    bx, by, bz = b
    dx = ax - bx
    dy = ay - by
    dx = dx - lx * np.round(dx / lx)
    dy = dy - ly * np.round(dy / ly)
    return np.sqrt(dx * dx + dy * dy + (az - bz) ** 2)


def rel_pos_err(a, b, lx, ly):
    """max_i |dr_i| / L_x, the position-error measure used throughout."""
    return float(min_image_err(a, b, lx, ly).max() / lx)


def lists_equal(off_a, idx_a, off_b, idx_b) -> bool:
    return np.array_equal(np.asarray(off_a), np.asarray(off_b)) and np.array_equal(
        np.asarray(idx_a), np.asarray(idx_b))


def list_diff_summary(off_a, idx_a, off_b, idx_b, limit=5):
    out = []
    n = len(off_a) - 1
    for i in range(n):
        ra = set(idx_a[off_a[i]:off_a[i + 1]].tolist())
        rb = set(idx_b[off_b[i]:off_b[i + 1]].tolist())
        if ra != rb:
            out.append((i, sorted(ra - rb), sorted(rb - ra)))
            if len(out) >= limit:
                break
    return out
