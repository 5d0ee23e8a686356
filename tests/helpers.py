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


BRANCHINIT = 0xFFFFFFFE


def tree_shape(tree) -> list:
    """The octree with its branch numbering taken out: per branch, in a
    depth-first walk from the root in octant order, its eight leaf entries
    and which of its eight children exist.  Branch indices are handed out in
    the order threads reach them on the GPU and in traversal order on the
    CPU, so two octrees of the same map compare equal in this form."""
    tree = np.asarray(tree, np.uint32)
    out = []
    stack = [0] if len(tree) >= 16 else []
    while stack:
        b = stack.pop()
        row = tree[b:b + 16]
        out.append((tuple(int(x) for x in row[:8]), tuple(bool(x != BRANCHINIT) for x in row[8:])))
        for co in range(7, -1, -1):
            c = int(row[8 + co])
            if c != BRANCHINIT:
                stack.append(c)
    return out
