"""Shared helpers of the parity tests: seeded sequences and comparisons."""
from __future__ import annotations

import functools

import numpy as np

from fastfusion_b200 import scene

SCALING = 1.0 / 5000.0
MAXCAM = 4.0


@functools.lru_cache(maxsize=8)
def circle_frames(seed: int, n_frames: int, width: int, height: int, total: int = 100):
    """Frames 0..n_frames-1 of the room-circle sequence (cached)."""
    seq = scene.room_circle_sequence(seed, total, width, height)
    return seq.K, [seq.frame(k) for k in range(n_frames)]


def queue_set(q) -> set:
    return set(int(x) for x in q)
