"""Throughput of the fusion + incremental-meshing path on B200.

Workload (one map per GPU): the whole 1000-frame random walk of the larger
synthetic room -- 640x480 uint16 depth + BGR8 frames of a seeded 8x8x3 m
room with 80 boxes/spheres, rendered along a seeded random walk (2 cm steps,
2 degree yaw jitter, 1.2 m height; fx=fy=525).  Fusion at 5 mm voxels, 10 mm
truncation, 4 m maximum camera distance, 8^3 bricks, FP32 storage;
incremental meshing every 10 frames.  One step = 10 addMap calls plus one
updateMeshes.  Every run fuses the whole walk (100 steps); `--steps K` of
them, spread evenly over the walk after the `--warmup W` first ones, are
timed, so the timed steps sample the map from small to full size whatever K
is.

Reported (one JSON line from rank 0):
  value      frames/s over all ranks, depth/BGR already in HBM (ff_add_map_u16_device)
  e2e        the same through the host API: ff_add_map_sequence_u16 (the
             reference's several-frames addMap) from page-locked host frames,
             ff_update_meshes, and the whole mesh copied back to the host every
             step; e2e_pageable: the same from pageable host frames;
             e2e_single_frame_calls: one ff_add_map_u16 per frame
  roofline   the dominant stage's algorithmic bytes / CUDA-event time vs the
             measured HBM copy bandwidth; roofline_fuse: the same for the
             voxel-update kernel
  cpu_baseline  the reference's FusionMipMapCPU (compiled from its sources)
             pinned to one host core over the same walk and the same timed
             steps, median of 3 runs, plus a row with its threaded meshing;
             sdf_err_vs_fp64: the walk's first 20 frames fused with FP32 and
             FP16 storage against the FP64 restatement (the checker)

`--impl reference` times the reference's CPU implementation instead: one map
per host core (all cores the box gives this process, bounded by host memory),
each pinned to its core and running the same walk, aggregated frames/s over
the same timed steps.

Multi-GPU (`torchrun --nproc-per-node N bench.py --gpus N`): every rank fuses
its own independent map (walk seed = rank); no data-path collective; weak
scaling; the timed region is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

FRAMES_PER_STEP = 10
WIDTH, HEIGHT = 640, 480
SCALING = 1.0 / 5000.0
MAXCAM = 4.0
VOXEL = 0.005
THRESHOLD = 0.01
METRIC = "depth frames/s fused+meshed (640x480, 5 mm)"
UNIT = "frames/s"
FALLBACK_HBM_GBS = 6650.0
_T0 = time.monotonic()


def log(msg: str) -> None:
    """Progress on stderr (the JSON line stays alone on stdout)."""
    print(f"[bench {time.monotonic() - _T0:7.1f} s] {msg}", file=sys.stderr, flush=True)
L2_FLUSH_BYTES = 256 << 20
WALK_FRAMES = 1000  # the random walk's length: every run fuses all of it
CPU_RUNS = 3        # the CPU baseline: median of this many pinned runs

# stage -> kernels it times (for the roofline record)
# the reference's brick pool: its 2 GB cap in bricks (treeandbrick.cpp:169-229)
REFERENCE_POOL_BRICKS = 271420

STAGE_KERNELS = {
    "grow": "k_shift_branches+k_shift_leaves+copies",
    "dedupe": "k_dedupe (projection + de-duplication)",
    "insert": "k_insert",
    "finalize": "k_finalize_bitmap",
    "fuse": "k_fuse",
    "mesh_cells": "k_keep_cells+k_gen_levels+k_cell_keys+argsort (k_sort_small or k_rs_*)+k_merge_cells/k_gather_cells",
    "mesh_count": "k_mesh_lattice<count>+k_mesh_corner<count>",
    "mesh_emit": "k_mesh_lattice<emit>+k_mesh_corner<emit>+k_copy_clean",
    "confidence": "k_cnn_features+k_conv x3 (learned weight)",
}


# stage -> the algorithmic bytes its roofline counts (per launch)
STAGE_BYTES = {
    "grow": "octree and leaf positions read and written",
    "dedupe": "W*H*2 B: the depth image read (voxel keys and flags it writes stay in L2)",
    "insert": "16 B per octree level probed per processed pixel (counted on the device)",
    "finalize": "8 B per new brick",
    "fuse": "14,336 B per queued brick per frame (512 voxels x (4 SDF + 4 weight + 6 colour) B, read and written; "
            "10,240 B with FP16 storage)",
    "mesh_cells": "44 B per cell read or written: the previous list read by the keep test, each new cell written "
                  "by the octree traversal and read by the merge, the kept cells read by the merge, the list written",
    "mesh_count": "SDF and weight (8 B, 4 B FP16) of every sample of the re-meshed cells",
    "mesh_emit": "14 B (10 B FP16) per sample read + 15 B per vertex + 12 B per face written",
    "confidence": "per pixel: depth in, features, two activations and the confidence written and read once",
}


def parse_args(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=97)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--storage", choices=["fp32", "fp16"], default=None,
                    help="voxel storage (default fp32; fp16 for the corridor workload)")
    ap.add_argument("--rcp", choices=["host", "exact"], default="host")
    ap.add_argument("--weight", choices=["plain", "learned"], default="plain",
                    help="learned: the trained per-pixel confidence network weights every frame")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workers", type=int, default=0, help="reference arm: maps in parallel (0 = all cores)")
    ap.add_argument("--workload", choices=["walk", "corridor"], default="walk",
                    help="corridor: the large-map workload (1280x960, FP16 storage, pool of --pool-gb)")
    ap.add_argument("--pool-gb", type=float, default=120.0, help="corridor: brick pool size in GB of HBM")
    ap.add_argument("--stride", type=int, default=0,
                    help="corridor: use every stride-th frame of the path (0: spread the frames over all of it)")
    ap.add_argument("--no-tuning", action="store_true",
                    help="batched workload: default launch shapes instead of the autotuner's table")
    ap.add_argument("--walk-frames", type=int, default=WALK_FRAMES,
                    help="frames of the walk to fuse (default: all 1000; a shorter prefix for profiling captures)")
    ap.add_argument("--batch-frames", type=int, default=0,
                    help="batched workload: frames per map (0: each map its own length, 200-2000)")
    ap.add_argument("--maps", type=int, default=0,
                    help="batched workload instead: this many independent maps of uneven size fused together "
                         "(ff_add_maps_u16_device), one frame of each per launch set")
    a = ap.parse_args(argv)
    if a.storage is None:
        a.storage = "fp16" if a.workload == "corridor" else "fp32"
    if a.warmup < 3:
        ap.error("--warmup must be at least 3")
    if a.steps < 1:
        ap.error("--steps must be at least 1")
    return a


def step_plan(a, frames: int | None = None):
    """(steps run, indices of the timed steps): every step of the walk runs;
    K timed steps are spread evenly over the steps after the W warm-up ones
    (a walk longer than 1000 frames only when W + K steps need it).  A
    profiling capture may run a prefix of the walk (--walk-frames)."""
    if frames is None:
        frames = getattr(a, "walk_frames", WALK_FRAMES) or WALK_FRAMES
    total = max(frames // FRAMES_PER_STEP, a.warmup + a.steps)
    span = total - a.warmup
    return total, [a.warmup + (i * span) // a.steps for i in range(a.steps)]


def n_frames_needed(a) -> int:
    return step_plan(a)[0] * FRAMES_PER_STEP


def make_sequence(seed: int, n_frames: int):
    from fastfusion_b200.scene import room_walk_sequence
    # the scene keeps its primitives clear of the whole trajectory, so the
    # trajectory length is fixed at 1000 frames unless more are needed
    return room_walk_sequence(seed, n_frames=max(1000, n_frames), width=WIDTH, height=HEIGHT)


def render_frames(seq, n_frames: int, device):
    """All frames as device tensors: depth int16 [F,H,W] (uint16 bits), bgr uint8 [F,H,W,3]."""
    import torch
    from fastfusion_b200.scene import render_torch
    depth = torch.empty((n_frames, HEIGHT, WIDTH), dtype=torch.int16, device=device)
    bgr = torch.empty((n_frames, HEIGHT, WIDTH, 3), dtype=torch.uint8, device=device)
    for k in range(n_frames):
        R, t = seq.poses[k]
        d, c = render_torch(seq.scene, R, t, WIDTH, HEIGHT, seq.K, seq.seed, k, device=device)
        depth[k].copy_(d)
        bgr[k].copy_(c)
    return depth, bgr


def workload_config(a, n_frames: int) -> dict:
    total, timed = step_plan(a)
    return {
        "workload": f"walk{n_frames}: {'the whole' if n_frames >= WALK_FRAMES else 'the first'} {n_frames} "
                    f"frames of the 1000-frame seeded random walk (640x480) in the 8x8x3 m room "
                    f"with 80 primitives (the larger synthetic configuration), voxel 5 mm, threshold 10 mm, maxcam "
                    f"4 m, 8^3 bricks, multi-resolution levels, updateMeshes every {FRAMES_PER_STEP} frames; "
                    f"{len(timed)} of its {total} steps timed, spread over the walk after {a.warmup} warm-up steps",
        "frames": n_frames,
        "timed_steps": timed,
        "frames_per_step": FRAMES_PER_STEP,
        "width": WIDTH,
        "height": HEIGHT,
        "voxel_m": VOXEL,
        "threshold_m": THRESHOLD,
        "maxcam_m": MAXCAM,
        "storage": a.storage,
        "rcp": a.rcp,
        "weight": getattr(a, "weight", "plain"),
        "seed": a.seed,
        "l2": "flushed between timed steps (256 MB write)",
    }


# -- clocks ---------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of the SM clock and throttle reasons (every 200 ms)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: str):
        self.path = tempfile.mktemp(prefix="ffclk_", suffix=".csv")
        self.f = open(self.path, "w")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", gpu_index, f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict | None:
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            self.p.wait()
        self.f.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "reasons": sorted(reasons)}


def measured_hbm_peak():
    p = os.path.join(HERE, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def read_traffic_table() -> dict:
    """DRAM traffic per algorithmic byte of each stage, from the committed ncu
    capture (lines `traffic <stage> <dram bytes / algorithmic byte> ratio`).
    A stage's traffic per launch is that ratio times its algorithmic bytes per
    launch measured here: the capture's traffic scaled to this launch size."""
    out = {}
    p = os.path.join(HERE, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return out
    with open(p) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 4 and parts[0] == "traffic" and parts[3] == "ratio":
                out[parts[1]] = float(parts[2])
    return out


# -- ranks -----------------------------------------------------------------------
def reduce_over_ranks(x: float, op: str, device=None) -> float:
    """Max or sum of a per-rank scalar over the process group (the value
    itself without one).  The timed region of a multi-GPU run is the max over
    ranks; the work done is the sum."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def copy_bandwidth(dev, nbytes: int = 64 << 20, reps: int = 5) -> dict:
    """Page-locked host <-> device copy bandwidth (GB/s): the best of a few
    64 MB copies each way, timed with CUDA events."""
    import torch
    host = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    devbuf = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    out = {}
    for name, dst, src in (("h2d_gbs", devbuf, host), ("d2h_gbs", host, devbuf)):
        best = None
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            dst.copy_(src, non_blocking=True)
            e1.record()
            e1.synchronize()
            ms = e0.elapsed_time(e1)
            best = ms if best is None else min(best, ms)
        out[name] = round(nbytes / (best / 1e3) / 1e9, 1)
    return out


def whole_job_rate(frames_this_rank: float, ms_this_rank: float, device=None):
    """(frames/s of the whole job, slowest rank's ms): every rank's frames
    over the max-over-ranks device time."""
    frames = reduce_over_ranks(frames_this_rank, "sum", device)
    ms = reduce_over_ranks(ms_this_rank, "max", device)
    return frames / (ms / 1e3), ms


# -- the B200 arm ------------------------------------------------------------------
def run_b200(a):
    import torch
    import torch.distributed as dist
    from fastfusion_b200 import fusion as ff

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != a.gpus:
        raise SystemExit(f"--gpus {a.gpus} but WORLD_SIZE={world}")
    if not torch.cuda.is_available():
        raise SystemExit("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    learned = None
    if a.weight == "learned":
        from fastfusion_b200.confidence import load_weights
        learned = load_weights()
    total, timed_idx = step_plan(a)
    timed_set = set(timed_idx)
    nf = total * FRAMES_PER_STEP
    seq = make_sequence(a.seed + rank, nf)
    log(f"rendering {nf} frames")
    depth, bgr = render_frames(seq, nf, dev)
    cams = [ff.CameraInfo(seq.K, *seq.poses[k]) for k in range(nf)]
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    torch.cuda.synchronize(dev)

    def new_map():
        m = ff.FusionMipMapCPU(0, 0, 0, VOXEL, THRESHOLD, 0, True, device=local, storage=a.storage, rcp=a.rcp)
        m.set_stream(stream.cuda_stream)
        if a.weight == "learned":
            m.set_confidence(*learned)
        return m

    def device_step(m, s):
        # the step's frames in one call (ff_add_map_sequence_u16_device)
        ks = range(s * FRAMES_PER_STEP, (s + 1) * FRAMES_PER_STEP)
        m.addMapSequenceDevice([depth[k].data_ptr() for k in ks], [bgr[k].data_ptr() for k in ks], WIDTH, HEIGHT,
                               [cams[k] for k in ks], SCALING, MAXCAM)
        m.updateMeshes()

    def device_step_single(m, s):
        # one call per frame (ff_add_map_u16_device)
        for k in range(s * FRAMES_PER_STEP, (s + 1) * FRAMES_PER_STEP):
            m.addMapDevice(depth[k].data_ptr(), bgr[k].data_ptr(), WIDTH, HEIGHT, cams[k], SCALING, MAXCAM)
        m.updateMeshes()

    launches = [0, 0]

    def timed(step_fn, m, on_timed_start=None):
        """The whole walk: W untimed warm-up steps, then every further step,
        of which the K timed ones are bracketed by CUDA events (L2 flushed
        before each); returns (device ms summed over the timed steps, wall s
        of the walk after the warm-up).  Own kernel launches of the timed
        steps are counted in `launches`."""
        for s in range(a.warmup):
            step_fn(m, s)
        if on_timed_start:
            on_timed_start(m)
        ev = []
        launches[0] = launches[1] = 0
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        w0 = time.perf_counter()
        for s in range(a.warmup, total):
            if s not in timed_set:
                step_fn(m, s)
                continue
            flush.fill_(s)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            own0, lib0 = ff.kernel_launches()
            e0.record(stream)
            step_fn(m, s)
            e1.record(stream)
            own1, lib1 = ff.kernel_launches()
            launches[0] += own1 - own0
            launches[1] += lib1 - lib0
            ev.append((e0, e1))
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - w0
        return sum(e0.elapsed_time(e1) for e0, e1 in ev), wall

    gpu_index = os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[local] if \
        os.environ.get("CUDA_VISIBLE_DEVICES") else str(local)
    clk = ClockSampler(gpu_index) if rank == 0 else None

    # 1. device-resident throughput
    log("device-resident walk (sequence call)")
    m = new_map()
    dev_ms, dev_wall = timed(device_step, m)
    gpu_launches, lib_calls = launches
    st = m.stats()
    m.close()
    del m
    # the same with one call per frame
    log("device-resident walk (one call per frame)")
    m = new_map()
    single_ms, _ = timed(device_step_single, m)
    m.close()
    del m

    # 2. per-stage profile of the walk after the warm-up (separate map; events per stage)
    log("stage profile")
    m = new_map()
    dirty, rounds, generated, top_kept = [], [], [], []

    def device_step_stats(mm, s):
        device_step(mm, s)
        st_ = mm.stats()
        rounds.append(st_["dedupe_rounds"])
        dirty.append(st_["mesh_cells_dirty"])
        generated.append(st_["mesh_cells_generated"] / max(st_["mesh_cells"], 1))
        top_kept.append(st_["mesh_top_kept"])

    for s_ in range(a.warmup):
        device_step(m, s_)
    m.profile(True)
    torch.cuda.synchronize(dev)
    p0 = time.perf_counter()
    for s_ in range(a.warmup, total):
        device_step_stats(m, s_)
    stages = m.profile_read()
    prof_wall_ms = 1e3 * (time.perf_counter() - p0)
    m.close()
    del m

    # 3. end to end through the host API: host frames in, whole mesh out, every step
    e2e = e2e_pageable = e2e_single = None
    rms = None
    if not a.no_e2e:
        last_mesh = {}
        # page-locked mesh buffer reserved before the timed region, like a
        # viewer would size it for its scene (it grows if the mesh outgrows it)
        mesh_buf = ff.MeshBuffer(4 << 20, 6 << 20)

        def host_run(hd, hb, per_frame=False):
            d2h = []

            def host_step(mm, s):
                ks = range(s * FRAMES_PER_STEP, (s + 1) * FRAMES_PER_STEP)
                if per_frame:
                    for k in ks:
                        mm.addMap(hd[k], cams[k], hb[k], SCALING, MAXCAM)
                else:
                    # the reference's several-frames addMap (host images)
                    mm.addMapSequence([hd[k] for k in ks], [cams[k] for k in ks], [hb[k] for k in ks], SCALING,
                                      MAXCAM)
                mm.updateMeshes()
                # the whole mesh to the host, the copy overlapping the next
                # step's frames (ff_get_mesh_async; every copy has finished
                # when the timed region's closing synchronisation returns)
                mesh = mm.getMeshInterleavedMarchingCubes(out=mesh_buf, wait=False)
                d2h.append(mesh.vertices.nbytes + mesh.colors.nbytes + mesh.faces.nbytes)
                last_mesh["m"] = mesh

            # The copies run on a second stream, overlapping the next step, so
            # per-step events on one stream cannot hold them: the whole walk
            # after the warm-up is timed as one span, from an event before its
            # first step to one recorded after the last mesh copy has landed.
            mm = new_map()
            for s_ in range(a.warmup):
                host_step(mm, s_)
            mm.mesh_wait()
            d2h.clear()
            torch.cuda.synchronize(dev)
            barrier()
            torch.cuda.synchronize(dev)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            own0, _ = ff.kernel_launches()
            e0.record(stream)
            for s_ in range(a.warmup, total):
                host_step(mm, s_)
            mm.mesh_wait()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            barrier()
            own1, _ = ff.kernel_launches()
            span_steps = total - a.warmup
            ms = e0.elapsed_time(e1)
            mm.close()
            rate, ms = whole_job_rate(span_steps * FRAMES_PER_STEP, ms, dev)
            return {"value": rate, "unit": UNIT,
                    "h2d_bytes_per_step": FRAMES_PER_STEP * (WIDTH * HEIGHT * 2 + WIDTH * HEIGHT * 3),
                    "d2h_bytes_per_step": int(np.mean(d2h)) if d2h else 0, "ms_per_step": ms / span_steps,
                    "steps": span_steps, "gpu_launches_per_step": round((own1 - own0) / span_steps, 1),
                    "api": "ff_add_map_u16 per frame" if per_frame else
                           "ff_add_map_sequence_u16 (the step's 10 host frames per call)",
                    "span": f"steps {a.warmup}..{total - 1} of the walk back to back (every step: 10 frames from "
                            "host memory, updateMeshes, the whole mesh copied to page-locked host memory on a "
                            "second stream); CUDA events around the span, the closing one after the last copy"}

        # page-locked host frames (ff_alloc_host-style pinned memory)
        log("end to end, page-locked host frames")
        h_depth = depth.cpu().pin_memory()
        h_bgr = bgr.cpu().pin_memory()
        e2e = host_run(h_depth.numpy().view(np.uint16), h_bgr.numpy())
        e2e["host_frames"] = "page-locked"
        log("end to end, page-locked host frames, one call per frame")
        e2e_single = host_run(h_depth.numpy().view(np.uint16), h_bgr.numpy(), per_frame=True)
        e2e_single["host_frames"] = "page-locked"
        if rank == 0 and "m" in last_mesh and len(last_mesh["m"].vertices):
            v = last_mesh["m"].vertices
            rng = np.random.default_rng(0)
            sel = rng.choice(len(v), size=min(len(v), 300000), replace=False)
            rms = float(np.sqrt(np.mean(seq.scene.sdf(v[sel].astype(np.float64)) ** 2)))
        del h_depth, h_bgr
        # pageable host frames, as a caller's cv::Mat images are
        log("end to end, pageable host frames")
        p_depth = depth.cpu().numpy().view(np.uint16).copy()
        p_bgr = bgr.cpu().numpy().copy()
        e2e_pageable = host_run(p_depth, p_bgr)
        e2e_pageable["host_frames"] = "pageable"
        del p_depth, p_bgr
        mesh_buf.close()
        # the copy bandwidth between page-locked host memory and the device on
        # this box: what the e2e step's copies cost at best
        pcie = copy_bandwidth(dev)
        for e in (e2e, e2e_single, e2e_pageable):
            e["copy_bound_ms_per_step"] = round(max(e["h2d_bytes_per_step"] / pcie["h2d_gbs"],
                                                    e["d2h_bytes_per_step"] / pcie["d2h_gbs"]) / 1e6, 3)
        e2e["pcie"] = pcie
    clocks = clk.stop() if clk else None

    value, dev_ms_max = whole_job_rate(a.steps * FRAMES_PER_STEP, dev_ms, dev)
    value_single, _ = whole_job_rate(a.steps * FRAMES_PER_STEP, single_ms, dev)

    peak, peak_kind = measured_hbm_peak()
    tt = read_traffic_table()

    def roofline_of(stage):
        ms_d, bytes_d, n_d = stages[stage]
        achieved = bytes_d / (ms_d / 1e3) / 1e9 if ms_d > 0 else 0.0
        traffic = round(tt[stage] * bytes_d / n_d) if (stage in tt and n_d) else None
        return {"bound": "hbm", "kernel": STAGE_KERNELS[stage], "stage": stage, "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "peak_source": f"{peak_kind} (copy bandwidth)",
                "algorithmic_bytes_per_launch": round(bytes_d / n_d) if n_d else 0, "launches": n_d,
                "avg_launch_us": round(1e3 * ms_d / n_d, 3) if n_d else 0, "traffic": traffic,
                "bytes_rule": STAGE_BYTES[stage]}

    dom = max(stages, key=lambda k: stages[k][0])
    roofline = roofline_of(dom)
    roofline_fuse = roofline_of("fuse")
    prof_ms = sum(v[0] for v in stages.values())
    stage_rec = {k: {"ms": round(v[0], 3), "share": round(v[0] / prof_ms, 4) if prof_ms else 0,
                     "GB/s": round(v[1] / (v[0] / 1e3) / 1e9, 1) if v[0] > 0 else 0, "launches": v[2],
                     "bytes_per_launch": round(v[1] / v[2]) if v[2] else 0,
                     "traffic_per_launch": round(tt[k] * v[1] / v[2]) if (k in tt and v[2]) else None}
                 for k, v in stages.items()}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(depth, bgr, seq, a)
        log("FP32/FP16 storage against the FP64 restatement")
        cpu["sdf_err_vs_fp64"] = precision_vs_fp64(depth, bgr, seq, local)
        log("done")

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(dev_ms_max / a.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if a.storage == "fp32" else "f16-storage/f32",
            "data": "synthetic: seeded room scene rendered to depth+BGR on the GPU (the TUM RGB-D sequences "
                    "the reference documents are not available offline)",
            "config": dict(workload_config(a, nf), parallelism=f"independent maps x{world}"),
            "api": "value: ff_add_map_sequence_u16_device (a step's 10 frames per call); "
                   "value_single_frame_calls: ff_add_map_u16_device per frame; e2e: ff_add_map_sequence_u16 (the "
                   "reference's several-frames addMap, host images); e2e_single_frame_calls: ff_add_map_u16 per "
                   "frame",
            "value_single_frame_calls": round(value_single, 2),
            "e2e": e2e, "e2e_pageable": e2e_pageable, "e2e_single_frame_calls": e2e_single,
            "roofline": roofline, "roofline_fuse": roofline_fuse,
            "cpu_baseline": cpu, "gpu_launches": gpu_launches,
            "library_calls": lib_calls, "clocks": clocks, "stages": stage_rec,
            "stage_profile": f"CUDA events per stage over steps {a.warmup}-{total - 1} of a separate run "
                             f"({round(prof_wall_ms)} ms wall)",
            "wall_s_walk": round(dev_wall, 3), "surface_rms_m": rms,
            "fused_bricks": {"frame_bricks": st["fused_frame_bricks"], "bricks_read_and_written": st["fused_bricks"],
                             "note": "the deferred update pass reads and writes each brick once per pass, "
                                     "whatever the number of its frames"},
            "map": {"leaves": st["leaves_used"], "leaves_max": st["leaves_max"], "n": st["n"],
                    "mesh_vertices": st["mesh_vertices"], "mesh_faces": st["mesh_faces"],
                    "mesh_cells": st["mesh_cells"], "grows": st["grows"], "meshing_ok": st["meshing_ok"],
                    "mesh_cells_dirty_mean": float(np.mean(dirty)) if dirty else None,
                    "mesh_cells_generated_frac_mean": round(float(np.mean(generated)), 4) if generated else None,
                    "mesh_updates_from_kept_top_levels": round(float(np.mean(top_kept)), 4) if top_kept else None,
                    "dedupe_rounds_mean": float(np.mean(rounds)) if rounds else None},
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


# -- CPU baseline (oracle side: the reference compiled from its sources) --------------
def _cpu_impl():
    from oracle import ref
    if ref.available():
        return "reference", ref
    return "port", None


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def _save_frames(depth, bgr):
    tmp = tempfile.mkdtemp(prefix="ffref_")
    dpath, bpath = os.path.join(tmp, "depth.npy"), os.path.join(tmp, "bgr.npy")
    np.save(dpath, depth.cpu().numpy().view(np.uint16))
    np.save(bpath, bgr.cpu().numpy())
    return tmp, dpath, bpath


def _drop_frames(tmp, dpath, bpath):
    for f in (dpath, bpath):
        os.unlink(f)
    os.rmdir(tmp)


def _ref_worker(args):
    """One map of the reference (or the restatement where the reference is
    not built) pinned to `cores`, running the whole walk: W warm-up steps,
    then every step, the timed ones measured with the wall clock.  Puts
    (index, seconds of the timed steps) on the queue."""
    (idx, cores, dpath, bpath, K, poses, warmup, total, timed, thread_meshing, barrier, q) = args
    import numpy as np  # noqa: F811
    if cores:
        os.sched_setaffinity(0, cores)
    from oracle import ref as refmod
    hd = np.load(dpath, mmap_mode="r")
    hb = np.load(bpath, mmap_mode="r")
    if refmod.available():
        m = refmod.RefFusion(VOXEL, THRESHOLD, True)
        if thread_meshing:
            m.set_thread_meshing(True)
        add = lambda k: m.add_map(np.asarray(hd[k]), np.asarray(hb[k]), K, *poses[k], SCALING, MAXCAM)
    else:
        from oracle.port import PortFusion
        m = PortFusion(update_mode=2)
        add = lambda k: m.add_map(np.asarray(hd[k]), np.asarray(hb[k]), K, *poses[k], SCALING, MAXCAM)

    # a step: 10 addMap, updateMeshes, and the mesh copied out
    # (getMeshInterleavedMarchingCubes returns the reference's mesh by value)
    def step(s):
        for k in range(s * FRAMES_PER_STEP, (s + 1) * FRAMES_PER_STEP):
            add(k)
        m.update_meshes()
        m.mesh()

    for s in range(warmup):
        step(s)
    timed = set(timed)
    if barrier is not None:
        barrier.wait()
    secs = 0.0
    for s in range(warmup, total):
        if s in timed:
            t0 = time.perf_counter()
            step(s)
            secs += time.perf_counter() - t0
        else:
            step(s)
    q.put((idx, secs))
    if thread_meshing:
        # the reference's destructor frees its mesh cells' meshes before it
        # joins a mesher thread that may still run (geometryfusion_mipmap_cpu.cpp
        # :754 before :966): leave the object to the process exit, after the
        # queue's feeder thread has handed the result over
        q.close()
        q.join_thread()
        os._exit(0)


def _run_workers(jobs, with_barrier: bool, limit_s: float = 900.0):
    """Run the reference workers; their timed seconds in job order, or None
    if a worker died or the whole set did not finish within limit_s."""
    import multiprocessing as mp
    import queue as queue_mod
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(len(jobs), timeout=limit_s) if with_barrier else None
    q = ctx.Queue()
    procs = [ctx.Process(target=_ref_worker, args=(j[:10] + (barrier, q),)) for j in jobs]
    for pr in procs:
        pr.start()
    out = []
    deadline = time.monotonic() + limit_s
    try:
        while len(out) < len(procs):
            left = deadline - time.monotonic()
            if left <= 0:
                raise queue_mod.Empty
            try:
                out.append(q.get(timeout=min(left, 5.0)))
            except queue_mod.Empty:
                # a worker that exited without a result will never send one
                if any(pr.exitcode not in (None, 0) for pr in procs):
                    raise
    except queue_mod.Empty:
        for pr in procs:
            if pr.is_alive():
                pr.kill()
        for pr in procs:
            pr.join(10)
        log(f"reference workers: {len(out)} of {len(procs)} finished "
            f"(exit codes {[pr.exitcode for pr in procs]})")
        return None
    for pr in procs:
        pr.join(30)
    return [t for _, t in sorted(out)]


def cpu_baseline(depth, bgr, seq, a) -> dict:
    """The reference on one pinned host core over the same walk and the same
    timed steps: CPU_RUNS runs at once, each on its own core, the median
    reported; plus one run with the reference's threaded meshing on two
    cores."""
    kind, _ = _cpu_impl()
    total, timed = step_plan(a)
    nf = total * FRAMES_PER_STEP
    tmp, dpath, bpath = _save_frames(depth, bgr)
    avail = sorted(os.sched_getaffinity(0))
    runs = min(CPU_RUNS, len(avail))
    jobs = [(i, {avail[i]}, dpath, bpath, seq.K, seq.poses[:nf], a.warmup, total, timed, False)
            for i in range(runs)]
    log(f"cpu baseline: {runs} runs of the reference on one core each")
    secs = _run_workers(jobs, with_barrier=False)
    threaded = None
    if secs and kind == "reference" and len(avail) >= 2:
        log("cpu baseline: the reference with threaded meshing")
        tsecs = _run_workers([(0, set(avail[:2]), dpath, bpath, seq.K, seq.poses[:nf], a.warmup, total, timed,
                               True)], with_barrier=False)
        threaded = None if not tsecs else {
            "value": round(a.steps * FRAMES_PER_STEP / tsecs[0], 3), "unit": UNIT, "cores": 2,
            "note": "setThreadMeshing(true): meshing on a second thread, updateMeshes returning false "
                    "while it runs (the mesh copied each step is the last finished one)"}
    _drop_frames(tmp, dpath, bpath)
    if not secs:
        return {"value": None, "unit": UNIT, "cores": 1, "kind": kind,
                "unavailable": "the reference runs did not finish within their time limit"}
    med = float(np.median(secs))
    return {"value": round(a.steps * FRAMES_PER_STEP / med, 3), "unit": UNIT, "cores": 1, "kind": kind,
            "runs": [round(a.steps * FRAMES_PER_STEP / t, 3) for t in secs], "statistic": f"median of {runs}",
            "cpu_model": cpu_model(), "host_cores": os.cpu_count(), "pinned": "one core per run (sched_setaffinity)",
            "sample": f"the whole walk ({nf} frames) on one core per run, {a.warmup} warm-up steps, the same "
                      f"{a.steps} timed steps (10 addMap + updateMeshes + mesh copy each); setThreadMeshing(false)",
            "threaded_meshing": threaded}


PRECISION_FRAMES = 20


def precision_vs_fp64(depth, bgr, seq, device, frames=PRECISION_FRAMES) -> dict:
    """Part of the host-side baseline leg: the walk's first frames fused by
    the FP64 restatement on the host (the checker) and by this library with
    FP32 and with FP16 storage (exact round-toward-zero reciprocals, so that
    only the storage and float arithmetic differ); SDF error over every voxel
    the FP64 fusion weighted, in metres."""
    from fastfusion_b200 import fusion as ff
    from oracle import port
    p64 = port.PortFusion(leaves_total=271420, branches_total=4793488, update_mode=3)
    maps = {s: ff.FusionMipMapCPU(0, 0, 0, VOXEL, THRESHOLD, 0, True, leaves_max=271420, branches_max=4793488,
                                  device=device, storage=s, rcp="exact") for s in ("fp32", "fp16")}
    for k in range(frames):
        hd = depth[k].cpu().numpy().view(np.uint16)
        hb = bgr[k].cpu().numpy()
        R, t = seq.poses[k]
        p64.add_map(hd, hb, seq.K, R, t, SCALING, MAXCAM)
        for m in maps.values():
            m.addMap(hd, ff.CameraInfo(seq.K, R, t), hb, SCALING, MAXCAM)
    d64, w64 = p64.bricks64()
    out = {"frames": frames, "reciprocal": "exact", "voxels": int((w64 > 0).sum())}
    for s, m in maps.items():
        d, _, _ = m.bricks()
        sel = w64 > 0
        err = np.abs(d.astype(np.float64)[sel] - d64[sel]) if d.shape == d64.shape else None
        out[s] = None if err is None else {"rms_m": float(np.sqrt(np.mean(err ** 2))),
                                           "p99_m": float(np.quantile(err, 0.99)), "max_m": float(err.max())}
        m.close()
    p64.close()
    return out


# -- the reference arm ------------------------------------------------------------
def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import torch
    kind, _ = _cpu_impl()
    total, timed = step_plan(a)
    nf = total * FRAMES_PER_STEP
    seq = make_sequence(a.seed, nf)
    device = "cuda" if torch.cuda.is_available() else "cpu"
    depth, bgr = render_frames(seq, nf, device)
    tmp, dpath, bpath = _save_frames(depth, bgr)
    del depth, bgr
    avail = sorted(os.sched_getaffinity(0))
    try:
        import psutil
        mem_maps = int(psutil.virtual_memory().available // (3 << 30))
    except ImportError:
        mem_maps = len(avail)
    workers = a.workers or max(1, min(len(avail), mem_maps))
    jobs = [(i, {avail[i % len(avail)]}, dpath, bpath, seq.K, seq.poses[:nf], a.warmup, total, timed, False)
            for i in range(workers)]
    secs = _run_workers(jobs, with_barrier=True)
    _drop_frames(tmp, dpath, bpath)
    if not secs:
        print(json.dumps({"impl": "reference",
                          "unavailable": "the reference's maps did not finish within their time limit"}), flush=True)
        return
    wall = max(secs)
    value = workers * a.steps * FRAMES_PER_STEP / wall
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(1e3 * wall / a.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: same frames as the B200 arm",
        "config": dict(workload_config(a, nf), parallelism=f"{workers} independent maps on {workers} host cores"),
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": workers, "kind": kind,
                         "cpu_model": cpu_model(),
                         "sample": f"{workers} maps in parallel, each pinned to its own core and running the whole "
                                   f"walk; the same {a.steps} timed steps after {a.warmup} warm-up steps"},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# -- the batched workload -------------------------------------------------------
def run_batch(a):
    """Independent maps of uneven size (rooms 2-12 m, 10-150 primitives,
    320x240 / 640x480 / 1280x960, voxels 4-10 mm, 200-2000 frames each):
    maps placed over the ranks by longest processing time first (frames x
    pixels); on each rank one frame of every map that still has frames per
    ff_add_maps_u16_device call, updateMeshes per map every 10 frames.  Every
    map fuses its whole sequence; K steps spread over the run are timed (CUDA
    events; the frames of a step are rendered on the GPU before its timer
    starts).  frames/s over all ranks' maps over the slowest rank's time."""
    import torch
    import torch.distributed as dist
    from fastfusion_b200 import fusion as ff
    from fastfusion_b200.scene import batch_sequences, render_torch
    from fastfusion_b200.shard import lpt_placement
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != a.gpus:
        raise SystemExit(f"--gpus {a.gpus} but WORLD_SIZE={world}")
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    fixed = a.batch_frames if a.batch_frames > 0 else None
    seqs_all = batch_sequences(a.maps, n_frames=fixed)
    lengths_all = [len(sq.poses) for sq, _ in seqs_all]
    costs = [n * sq.width * sq.height for n, (sq, _) in zip(lengths_all, seqs_all)]
    placement = lpt_placement(costs, world)
    mine = placement[rank]
    seqs = [seqs_all[i] for i in mine]
    lengths = [lengths_all[i] for i in mine]
    # one step plan for every rank: the longest map of the whole job
    total = max(-(-max(lengths_all) // FRAMES_PER_STEP), a.warmup + a.steps)
    span = total - a.warmup
    timed = set(a.warmup + (i * span) // a.steps for i in range(a.steps))
    stream = torch.cuda.current_stream(dev)
    maps = []
    for seq, voxel in seqs:
        m = ff.FusionMipMapCPU(0, 0, 0, voxel, 2 * voxel, 0, True, leaves_max=400000, branches_max=8000000,
                               storage=a.storage, rcp=a.rcp, device=local)
        m.set_stream(stream.cuda_stream)
        maps.append(m)
    from fastfusion_b200.autotune import DEFAULT, load_tuning
    tuning = {} if a.no_tuning else load_tuning()
    if tuning and maps:
        maps[0].set_tuning(**{**DEFAULT, **tuning})
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    # frames of one step, rendered before it (outside its timer)
    buf = [(torch.empty((FRAMES_PER_STEP, sq.height, sq.width), dtype=torch.int16, device=dev),
            torch.empty((FRAMES_PER_STEP, sq.height, sq.width, 3), dtype=torch.uint8, device=dev)) for sq, _ in seqs]
    render_s = [0.0]

    def render_step(s_):
        t0 = time.perf_counter()
        for (sq, _), (d, c), n in zip(seqs, buf, lengths):
            for j in range(FRAMES_PER_STEP):
                k = s_ * FRAMES_PER_STEP + j
                if k < n:
                    dk, ck = render_torch(sq.scene, *sq.poses[k], sq.width, sq.height, sq.K, sq.seed, k, device=dev)
                    d[j].copy_(dk)
                    c[j].copy_(ck)
        torch.cuda.synchronize(dev)
        render_s[0] += time.perf_counter() - t0

    frames_done = [0]

    def step(s_):
        for j in range(FRAMES_PER_STEP):
            k = s_ * FRAMES_PER_STEP + j
            act = [i for i, n in enumerate(lengths) if k < n]
            if not act:
                continue
            ff.add_maps_device([maps[i] for i in act], [buf[i][0][j].data_ptr() for i in act],
                               [buf[i][1][j].data_ptr() for i in act], [seqs[i][0].width for i in act],
                               [seqs[i][0].height for i in act],
                               [ff.CameraInfo(seqs[i][0].K, *seqs[i][0].poses[k]) for i in act], SCALING, MAXCAM)
            frames_done[0] += len(act)
        for i, m in enumerate(maps):
            if s_ * FRAMES_PER_STEP < lengths[i]:
                m.updateMeshes()

    def barrier():
        if world > 1:
            dist.barrier()

    for s_ in range(a.warmup):
        render_step(s_)
        step(s_)
    if maps:
        maps[0].profile(True)
    ev = []
    timed_frames = 0
    torch.cuda.synchronize(dev)
    barrier()
    for s_ in range(a.warmup, total):
        render_step(s_)
        if s_ not in timed:
            step(s_)
            continue
        flush.fill_(s_)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0 = frames_done[0]
        e0.record(stream)
        step(s_)
        e1.record(stream)
        timed_frames += frames_done[0] - f0
        ev.append((e0, e1))
    torch.cuda.synchronize(dev)
    barrier()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    value, ms_max = whole_job_rate(timed_frames, ms, dev)
    stages = maps[0].profile_read() if maps else {}
    peak, peak_kind = measured_hbm_peak()
    fms, fbytes, fl = stages.get("fuse", (0.0, 0.0, 0))
    fuse_gbs = fbytes / (fms / 1e3) / 1e9 if fms > 0 else 0.0
    if rank == 0:
        line = {
            "metric": METRIC.replace("(640x480, 5 mm)", "(batched maps)"), "value": round(value, 2),
            "unit": UNIT, "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": round(ms_max / a.steps, 4), "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32" if a.storage == "fp32" else "f16-storage/f32",
            "data": "synthetic: seeded rooms of uneven size rendered on the GPU",
            "config": {"workload": f"batch{len(seqs_all)}: independent maps, rooms 2-12 m, 10-150 primitives, "
                                   f"320x240/640x480/1280x960, voxels 4-10 mm, "
                                   f"{'%d frames each' % fixed if fixed else '200-2000 frames each'}, one frame "
                                   f"of every map per launch set, updateMeshes every {FRAMES_PER_STEP} frames; "
                                   f"{a.steps} of {total} steps timed",
                       "maps": len(seqs_all), "frames": lengths_all,
                       "widths": [sq.width for sq, _ in seqs_all],
                       "voxels_mm": [round(v * 1e3, 2) for _, v in seqs_all],
                       "placement": placement, "tuning": tuning or "defaults",
                       "l2": "flushed between timed steps (256 MB write)",
                       "parallelism": f"maps over {world} GPUs by longest processing time first"},
            "timed_frames_rank0": timed_frames, "render_s_rank0": round(render_s[0], 1),
            "fuse": {"GB/s": round(fuse_gbs, 1), "frac_of_hbm": round(fuse_gbs / peak, 4), "peak": peak,
                     "peak_source": peak_kind, "launches": fl,
                     "avg_launch_us": round(1e3 * fms / fl, 2) if fl else 0,
                     "bytes_per_launch": round(fbytes / fl) if fl else 0},
            "stages_lead_map": {k: {"ms": round(v[0], 3), "launches": v[2]} for k, v in stages.items()},
        }
        print(json.dumps(line), flush=True)
    for m in maps:
        m.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_corridor(a):
    """The large map: the 50 x 20 x 3 m corridor/office floor (400
    primitives), 1280x960 depth at fx = fy = 1050 along the seeded
    10,000-frame spline at 1.0-1.6 m, every --stride-th frame of it (so the
    path is covered end to end), FP16 storage, the brick pool sized to
    --pool-gb of HBM, updateMeshes every 10 frames; frames device-resident,
    CUDA events per step."""
    import torch
    import torch.distributed as dist
    from fastfusion_b200 import fusion as ff
    from fastfusion_b200.scene import corridor_sequence, render_torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != a.gpus:
        raise SystemExit(f"--gpus {a.gpus} but WORLD_SIZE={world}")
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    nf = (a.warmup + a.steps) * FRAMES_PER_STEP
    W, H = 1280, 960
    stride = a.stride if a.stride > 0 else max(1, 10000 // nf)
    seq = corridor_sequence(a.seed, n_frames=10000, width=W, height=H)
    idx = [min(k * stride, 9999) for k in range(nf)]
    # frames are rendered CHUNK steps at a time, outside the timed windows
    CHUNK = 50
    depth = torch.empty((CHUNK * FRAMES_PER_STEP, H, W), dtype=torch.int16, device=dev)
    bgr = torch.empty((CHUNK * FRAMES_PER_STEP, H, W, 3), dtype=torch.uint8, device=dev)
    render_s = [0.0]

    def render_chunk(s0):
        t0 = time.perf_counter()
        for i in range(s0 * FRAMES_PER_STEP, min((s0 + CHUNK) * FRAMES_PER_STEP, nf)):
            k = idx[i]
            d, c = render_torch(seq.scene, *seq.poses[k], W, H, seq.K, seq.seed, k, device=dev,
                                cull_m=MAXCAM + 1.0)
            depth[i - s0 * FRAMES_PER_STEP].copy_(d)
            bgr[i - s0 * FRAMES_PER_STEP].copy_(c)
        torch.cuda.synchronize(dev)
        render_s[0] += time.perf_counter() - t0

    cams = [ff.CameraInfo(seq.K, *seq.poses[k]) for k in idx]
    stream = torch.cuda.current_stream(dev)
    free0, total = torch.cuda.mem_get_info(dev)
    m = ff.FusionMipMapCPU(0, 0, 0, VOXEL, THRESHOLD, 0, True, storage=a.storage, rcp=a.rcp,
                           pool_bytes=int(a.pool_gb * 1e9), device=local)
    if world > 1:
        # one map over all GPUs: every rank is given every frame and holds the
        # whole octree; rank r updates the bricks and meshes the cells whose
        # keys hash to r, after a halo all-gather of the changed bricks
        m.set_shard(rank, world)
    halo_bytes = [0]
    free1, _ = torch.cuda.mem_get_info(dev)
    m.set_stream(stream.cuda_stream)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    leaves, ref_cap_step = [], None

    def step(s_, render=True):
        if render and s_ % CHUNK == 0:
            m.sync()  # the previous chunk's frames are no longer read
            render_chunk(s_)
        base = (s_ // CHUNK) * CHUNK * FRAMES_PER_STEP
        for i in range(s_ * FRAMES_PER_STEP, (s_ + 1) * FRAMES_PER_STEP):
            m.addMapDevice(depth[i - base].data_ptr(), bgr[i - base].data_ptr(), W, H, cams[i], SCALING, MAXCAM)
        if world > 1:
            from fastfusion_b200.shard import halo_exchange
            halo_bytes[0] += halo_exchange(m, dev)["bytes_sent"]
        m.updateMeshes()

    for s_ in range(a.warmup):
        step(s_)
    # Every PROFILE_EVERY-th step runs with the per-stage CUDA-event profile
    # on (its events and synchronisations would slow the step) and is not
    # timed; the others are timed with the profile off.
    PROFILE_EVERY = 10
    stage_sum = {}
    mc_steps = []  # (step, cell-list ms, cells) of the profiled steps
    ev, timed_i = [], []
    torch.cuda.synchronize(dev)
    for i in range(a.steps):
        if (a.warmup + i) % CHUNK == 0:
            m.sync()
            render_chunk(a.warmup + i)
        if i % PROFILE_EVERY == PROFILE_EVERY - 1:
            m.profile(True)
            step(a.warmup + i, render=False)
            p_ = m.profile_read()
            m.profile(False)
            for k_, v_ in p_.items():
                acc = stage_sum.setdefault(k_, [0.0, 0.0, 0])
                acc[0] += v_[0]
                acc[1] += v_[1]
                acc[2] += v_[2]
            mc_steps.append((i, p_["mesh_cells"][0], m.stats()["mesh_cells"]))
        else:
            flush.fill_(i)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step(a.warmup + i, render=False)
            e1.record(stream)
            ev.append((e0, e1))
            timed_i.append(i)
        st = m.stats()
        leaves.append(st["leaves_used"])
        if ref_cap_step is None and st["leaves_used"] > REFERENCE_POOL_BRICKS:
            ref_cap_step = a.warmup + i
    torch.cuda.synchronize(dev)
    ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    # the whole map's frames over the slowest part's device time
    ms_total = reduce_over_ranks(float(sum(ms)), "max", dev)
    leaves_all = int(m.stats()["leaves_used"])  # every part holds the whole leaf table
    stages = {k_: tuple(v_) for k_, v_ in stage_sum.items()}
    st = m.stats()
    peak, peak_kind = measured_hbm_peak()
    fms, fbytes, fl = stages.get("fuse", (0.0, 0.0, 0))
    fuse_gbs = fbytes / (fms / 1e3) / 1e9 if fms > 0 else 0.0
    q = max(1, len(ms) // 4)
    mq = max(1, len(mc_steps) // 4)
    mc_ms = [x[1] for x in mc_steps]
    line = {
        "metric": METRIC.replace("(640x480, 5 mm)", "(large map, 1280x960, 5 mm)"),
        "value": round(len(ms) * FRAMES_PER_STEP / (ms_total / 1e3), 2), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "timed_steps": len(ms),
        "profiled_steps": f"every {PROFILE_EVERY}th step ran with the stage profile on and is not timed",
        "warmup": a.warmup, "ms_per_step": round(ms_total / len(ms), 4),
        "ms_per_step_median": round(float(np.median(ms)), 3), "ms_per_step_max": round(float(np.max(ms)), 3),
        "ms_per_step_first_quarter": round(float(np.mean(ms[:q])), 3),
        "ms_per_step_last_quarter": round(float(np.mean(ms[-q:])), 3),
        # the cell list per update over the profiled steps: the median of each
        # quarter (a growth of the volume moves every cell and regenerates the
        # whole list: those few updates show in the maximum)
        "mesh_cells_ms_per_update_first_quarter": round(float(np.median(mc_ms[:mq])), 4) if mc_ms else None,
        "mesh_cells_ms_per_update_last_quarter": round(float(np.median(mc_ms[-mq:])), 4) if mc_ms else None,
        "mesh_cells_ms_per_update_max": round(float(np.max(mc_ms)), 3) if mc_ms else None,
        "mesh_cells_first_quarter": int(np.mean([x[2] for x in mc_steps[:mq]])) if mc_steps else None,
        "mesh_cells_last_quarter": int(np.mean([x[2] for x in mc_steps[-mq:]])) if mc_steps else None,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32" if a.storage == "fp32" else "f16-storage/f32",
        "data": "synthetic: seeded corridor/office floor rendered on the GPU (primitives beyond maxcam + 1 m "
                "culled per frame: no depth below maxcam changes)",
        "config": {"workload": f"corridor: 50x20x3 m floor, 400 primitives, 1280x960 fx=fy=1050, frames 0, "
                               f"{stride}, 2x{stride}, ... of a 10,000-frame spline at 1.0-1.6 m ({nf} frames), "
                               f"voxel 5 mm, threshold 10 mm, maxcam 4 m, updateMeshes every {FRAMES_PER_STEP} "
                               f"frames", "storage": a.storage, "pool_gb": a.pool_gb, "stride": stride,
                   "l2": "flushed between timed steps (256 MB write)",
                   "parallelism": f"one map, bricks sharded over {world} GPUs" if world > 1 else "one map"},
        "map": {"leaves": leaves_all, "leaves_rank0": st["leaves_used"], "leaves_max": st["leaves_max"], "n": st["n"],
                "grows": st["grows"],
                "mesh_vertices": st["mesh_vertices"], "mesh_faces": st["mesh_faces"], "mesh_cells": st["mesh_cells"],
                "meshing_ok": st["meshing_ok"], "pool_bytes_on_device": int(free0 - free1),
                "device_bytes_total": int(total)},
        "reference_pool": {"bricks": REFERENCE_POOL_BRICKS,
                           "exceeded_at_step": ref_cap_step,
                           "note": "the reference's brick pool (2 GB cap) holds 271,420 bricks; past this step "
                                   "it cannot complete the workload"},
        "fuse": {"GB/s": round(fuse_gbs, 1), "frac_of_hbm": round(fuse_gbs / peak, 4), "peak": peak,
                 "peak_source": peak_kind, "avg_launch_us": round(1e3 * fms / fl, 2) if fl else 0},
        "stages": {k: {"ms": round(v[0], 3), "launches": v[2]} for k, v in stages.items()},
        "render_s": round(render_s[0], 1),
        "halo_bytes_sent_rank0": halo_bytes[0],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    m.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def main(argv=None):
    a = parse_args(argv)
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "corridor":
        run_corridor(a)
    elif a.maps:
        run_batch(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
