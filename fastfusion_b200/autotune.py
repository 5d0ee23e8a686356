"""Autotuner of the batched fusion's launch shapes (ff_tuning).

Sweeps the de-duplication tile height, the voxel update's block shape
(bricks per block, register budget) and grid, the insert's block size and
CUDA-graph replay on the batched workload -- independent rooms of uneven
size, one frame of every map per ff_add_maps_u16_device call -- and keeps
the fastest.  Launch shapes never change results (the batched tests check
every shape against one-by-one fusion), so all candidates run on one set of
maps: after a warm-up, candidates take turns on consecutive frame sets
(each timed with CUDA events) and each keeps the median of its turns.  One
parameter is settled at a time, in the order below.

    python -m fastfusion_b200.autotune [--maps 16] [--rounds 5]

writes tuning.json next to this file, keyed by GPU name; load_tuning()
returns the entry of the current GPU (empty: defaults).
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from fastfusion_b200 import fusion as ff

TUNING_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json")
DEFAULT = dict(dedupe_rows=0, fuse_shape=0, fuse_blocks_per_sm=0, insert_block=0, graph=False)
SCALING, MAXCAM = 1.0 / 5000.0, 4.0


def gpu_name() -> str:
    import torch
    return torch.cuda.get_device_name(torch.cuda.current_device())


def load_tuning(path: str = TUNING_PATH) -> dict:
    """The tuned launch shapes of this GPU (ff_tuning fields), or {}."""
    try:
        with open(path) as f:
            table = json.load(f)
        entry = table.get(gpu_name(), {})
    except (OSError, ValueError, RuntimeError, AssertionError):
        return {}
    return dict(entry.get("tuning", {}))


class BatchWorkload:
    """The batched workload on the GPU: frames rendered once, maps on the
    current torch stream."""

    def __init__(self, n_maps: int = 16, n_frames: int = 40, storage: str = "fp32", seed0: int = 100):
        import torch
        from fastfusion_b200.scene import batch_sequences, render_torch
        self.torch = torch
        dev = torch.device("cuda", torch.cuda.current_device())
        self.seqs = batch_sequences(n_maps, n_frames=n_frames, seed0=seed0)
        self.frames = []
        for seq, _ in self.seqs:
            d = torch.empty((n_frames, seq.height, seq.width), dtype=torch.int16, device=dev)
            c = torch.empty((n_frames, seq.height, seq.width, 3), dtype=torch.uint8, device=dev)
            for k in range(n_frames):
                dk, ck = render_torch(seq.scene, *seq.poses[k], seq.width, seq.height, seq.K, seq.seed, k,
                                      device=dev)
                d[k].copy_(dk)
                c[k].copy_(ck)
            self.frames.append((d, c))
        self.n_frames = n_frames
        self.cams = [[ff.CameraInfo(seq.K, *seq.poses[k]) for k in range(n_frames)] for seq, _ in self.seqs]
        self.widths = [seq.width for seq, _ in self.seqs]
        self.heights = [seq.height for seq, _ in self.seqs]
        self.stream = torch.cuda.current_stream()
        self.maps = []
        for seq, voxel in self.seqs:
            m = ff.FusionMipMapCPU(0, 0, 0, voxel, 2 * voxel, 0, True, leaves_max=400000, branches_max=8000000,
                                   storage=storage)
            m.set_stream(self.stream.cuda_stream)
            self.maps.append(m)
        self.k = 0

    def frame_sets(self, count: int):
        """Fuse the next `count` frame sets (frames wrap around)."""
        for _ in range(count):
            k = self.k % self.n_frames
            ff.add_maps_device(self.maps, [f[0][k].data_ptr() for f in self.frames],
                               [f[1][k].data_ptr() for f in self.frames], self.widths, self.heights,
                               [c[k] for c in self.cams], SCALING, MAXCAM)
            self.k += 1

    def time_sets(self, tuning: dict, count: int) -> float:
        """ms per frame set of `count` frame sets under the given shapes."""
        torch = self.torch
        self.maps[0].set_tuning(**{**DEFAULT, **tuning})
        self.frame_sets(1)  # (records the graph when replay is on)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(self.stream)
        self.frame_sets(count)
        e1.record(self.stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / count

    def close(self):
        for m in self.maps:
            m.close()


SPACE = [
    ("fuse_shape", [0, 1, 2, 3]),
    ("fuse_blocks_per_sm", [0, 1, 2, 4, 16]),
    ("dedupe_rows", [0, 8, 16, 32]),
    ("insert_block", [0, 128, 512]),
    ("graph", [False, True]),
]


def tune(work: BatchWorkload, rounds: int = 5, sets: int = 6, log=print) -> tuple[dict, dict]:
    """Coordinate search over the ff_tuning fields; returns (best, record)."""
    best = dict(DEFAULT)
    record = {}
    for name, values in SPACE:
        times = {v: [] for v in values}
        for _ in range(rounds):
            for v in values:
                times[v].append(work.time_sets({**best, name: v}, sets))
        med = {v: float(np.median(t)) for v, t in times.items()}
        choice = min(med, key=med.get)
        best[name] = choice
        record[name] = {str(v): round(t, 4) for v, t in med.items()}
        log(f"{name}: " + ", ".join(f"{v}={t:.3f} ms" for v, t in med.items()) + f" -> {choice}", flush=True)
    return best, record


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m fastfusion_b200.autotune")
    ap.add_argument("--maps", type=int, default=16)
    ap.add_argument("--frames", type=int, default=40)
    ap.add_argument("--rounds", type=int, default=5)
    ap.add_argument("--sets", type=int, default=6, help="frame sets per timed turn")
    ap.add_argument("--warmup", type=int, default=20, help="frame sets before the search")
    ap.add_argument("--out", default=TUNING_PATH)
    a = ap.parse_args(argv)
    t0 = time.time()
    work = BatchWorkload(a.maps, a.frames)
    work.frame_sets(a.warmup)
    best, record = tune(work, a.rounds, a.sets)
    base = float(np.median([work.time_sets(DEFAULT, a.sets) for _ in range(a.rounds)]))
    tuned = float(np.median([work.time_sets(best, a.sets) for _ in range(a.rounds)]))
    work.close()
    try:
        with open(a.out) as f:
            table = json.load(f)
    except (OSError, ValueError):
        table = {}
    table[gpu_name()] = {"tuning": best, "ms_per_frame_set": {"default": round(base, 4), "tuned": round(tuned, 4)},
                         "search": record, "workload": f"{a.maps} independent maps (rooms 2-12 m, "
                         "320x240/640x480/1280x960, voxels 4-10 mm), one frame each per call"}
    with open(a.out, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    print(json.dumps({"gpu": gpu_name(), "tuning": best, "default_ms": round(base, 4), "tuned_ms": round(tuned, 4),
                      "seconds": round(time.time() - t0, 1)}))


if __name__ == "__main__":
    main()
