"""Throughput of the fusion + incremental-meshing path on B200.

Workload (one map per GPU): 640x480 uint16 depth + BGR8 frames of a seeded
8x8x3 m room with 80 boxes/spheres, rendered along a seeded random walk
(2 cm steps, 2 degree yaw jitter, 1.2 m height; fx=fy=525).  Fusion at 5 mm
voxels, 10 mm truncation, 4 m maximum camera distance, 8^3 bricks, FP32
storage; incremental meshing every 10 frames.  One step = 10 addMap calls
plus one updateMeshes.  The default run (3 warm-up + 97 timed steps) covers
the 1000-frame walk.

Reported (one JSON line from rank 0):
  value      frames/s over all ranks, depth/BGR already in HBM (ff_add_map_u16_device)
  e2e        the same through the host API (ff_add_map_u16 from pinned host
             memory, ff_update_meshes, and the whole mesh copied back to the host
             every step)
  roofline   the dominant stage's algorithmic bytes / CUDA-event time vs the
             measured HBM copy bandwidth
  cpu_baseline  the reference's FusionMipMapCPU (compiled from its sources) on
             one host core over a bounded prefix of the same frames

`--impl reference` times the reference's CPU implementation instead: one map
per host core (all cores the box gives this process, bounded by host memory),
each running the same frames, aggregated frames/s.

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
L2_FLUSH_BYTES = 256 << 20
CPU_SAMPLE_SECONDS = 20.0

# stage -> kernels it times (for the roofline record)
# the reference's brick pool: its 2 GB cap in bricks (treeandbrick.cpp:169-229)
REFERENCE_POOL_BRICKS = 271420

STAGE_KERNELS = {
    "grow": "k_shift_branches+k_shift_leaves+copies",
    "dedupe": "k_dedupe (projection + de-duplication)",
    "insert": "k_insert",
    "finalize": "k_finalize_bitmap",
    "fuse": "k_fuse",
    "mesh_cells": "k_gen_level+k_cell_keys+radix sort+k_gather_cells",
    "mesh_count": "k_mesh_lattice<count>+k_mesh_corner<count>",
    "mesh_emit": "k_mesh_lattice<emit>+k_mesh_corner<emit>+k_copy_clean",
    "confidence": "k_cnn_features+k_conv x3 (learned weight)",
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


def n_frames_needed(a) -> int:
    return (a.warmup + a.steps) * FRAMES_PER_STEP


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
    return {
        "workload": f"walk{n_frames}: 8x8x3 m room, 80 primitives, {n_frames} frames 640x480 along a seeded "
                    f"random walk, voxel 5 mm, threshold 10 mm, maxcam 4 m, 8^3 bricks, updateMeshes every "
                    f"{FRAMES_PER_STEP} frames",
        "frames": n_frames,
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
    nf = n_frames_needed(a)
    seq = make_sequence(a.seed + rank, nf)
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
        for k in range(s * FRAMES_PER_STEP, (s + 1) * FRAMES_PER_STEP):
            m.addMapDevice(depth[k].data_ptr(), bgr[k].data_ptr(), WIDTH, HEIGHT, cams[k], SCALING, MAXCAM)
        m.updateMeshes()

    def timed(step_fn, m, on_timed_start=None):
        """W untimed steps, then K steps timed one by one with CUDA events
        (L2 flushed before each); returns (device ms summed, wall s)."""
        for s in range(a.warmup):
            step_fn(m, s)
        if on_timed_start:
            on_timed_start(m)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        w0 = time.perf_counter()
        for i in range(a.steps):
            flush.fill_(i)
            ev[i][0].record(stream)
            step_fn(m, a.warmup + i)
            ev[i][1].record(stream)
        torch.cuda.synchronize(dev)
        barrier()
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - w0
        return sum(e0.elapsed_time(e1) for e0, e1 in ev), wall

    gpu_index = os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[local] if \
        os.environ.get("CUDA_VISIBLE_DEVICES") else str(local)
    clk = ClockSampler(gpu_index) if rank == 0 else None

    # 1. device-resident throughput
    m = new_map()
    launches = {}

    def mark(mm):
        launches["own0"], launches["lib0"] = ff.kernel_launches()

    dirty, rounds = [], []

    def device_step_stats(mm, s):
        for k in range(s * FRAMES_PER_STEP, (s + 1) * FRAMES_PER_STEP):
            mm.addMapDevice(depth[k].data_ptr(), bgr[k].data_ptr(), WIDTH, HEIGHT, cams[k], SCALING, MAXCAM)
            rounds.append(mm.stats()["dedupe_rounds"])
        mm.updateMeshes()
        dirty.append(mm.stats()["mesh_cells_dirty"])

    dev_ms, dev_wall = timed(device_step, m, mark)
    own1, lib1 = ff.kernel_launches()
    gpu_launches, lib_calls = own1 - launches["own0"], lib1 - launches["lib0"]
    st = m.stats()
    m.close()
    del m

    # 2. per-stage profile of the same steps (separate map; events per stage)
    m = new_map()
    prof_ms, _ = timed(device_step_stats, m, lambda mm: mm.profile(True))
    stages = m.profile_read()
    m.close()
    del m

    # 3. end to end through the host API
    e2e = None
    rms = None
    if not a.no_e2e:
        h_depth = depth.cpu().pin_memory()
        h_bgr = bgr.cpu().pin_memory()
        hd = h_depth.numpy().view(np.uint16)
        hb = h_bgr.numpy()
        d2h = []
        last_mesh = {}
        # page-locked mesh buffer reserved before the timed region, like a
        # viewer would size it for its scene (it grows if the mesh outgrows it)
        mesh_buf = ff.MeshBuffer(4 << 20, 6 << 20)

        def host_step(mm, s):
            for k in range(s * FRAMES_PER_STEP, (s + 1) * FRAMES_PER_STEP):
                mm.addMap(hd[k], cams[k], hb[k], SCALING, MAXCAM)
            mm.updateMeshes()
            mesh = mm.getMeshInterleavedMarchingCubes(out=mesh_buf)
            d2h.append(mesh.vertices.nbytes + mesh.colors.nbytes + mesh.faces.nbytes)
            last_mesh["m"] = mesh

        m = new_map()
        e2e_ms, _ = timed(host_step, m, lambda mm: d2h.clear())
        m.close()
        del m
        e2e_value, e2e_ms = whole_job_rate(a.steps * FRAMES_PER_STEP, e2e_ms, dev)
        e2e = {"value": e2e_value, "unit": UNIT,
               "h2d_bytes_per_step": FRAMES_PER_STEP * (WIDTH * HEIGHT * 2 + WIDTH * HEIGHT * 3),
               "d2h_bytes_per_step": int(np.mean(d2h)) if d2h else 0,
               "ms_per_step": e2e_ms / a.steps}
        if rank == 0 and "m" in last_mesh and len(last_mesh["m"].vertices):
            v = last_mesh["m"].vertices
            rng = np.random.default_rng(0)
            sel = rng.choice(len(v), size=min(len(v), 300000), replace=False)
            rms = float(np.sqrt(np.mean(seq.scene.sdf(v[sel].astype(np.float64)) ** 2)))
        mesh_buf.close()
    clocks = clk.stop() if clk else None

    value, dev_ms_max = whole_job_rate(a.steps * FRAMES_PER_STEP, dev_ms, dev)

    # roofline of the dominant stage
    peak, peak_kind = measured_hbm_peak()
    dom = max(stages, key=lambda k: stages[k][0])
    ms_d, bytes_d, n_d = stages[dom]
    achieved = bytes_d / (ms_d / 1e3) / 1e9 if ms_d > 0 else 0.0
    traffic = None
    tt = read_traffic_table()
    if dom in tt and n_d:
        traffic = round(tt[dom] * bytes_d / n_d)
    roofline = {"bound": "hbm", "kernel": STAGE_KERNELS[dom], "stage": dom, "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "peak_source": f"{peak_kind} (copy bandwidth)",
                "algorithmic_bytes_per_launch": bytes_d / n_d if n_d else 0, "launches": n_d,
                "avg_launch_us": 1e3 * ms_d / n_d if n_d else 0, "traffic": traffic}
    stage_rec = {k: {"ms": round(v[0], 3), "share": round(v[0] / prof_ms, 4) if prof_ms else 0,
                     "GB/s": round(v[1] / (v[0] / 1e3) / 1e9, 1) if v[0] > 0 else 0, "launches": v[2],
                     "bytes_per_launch": round(v[1] / v[2]) if v[2] else 0,
                     "traffic_per_launch": round(tt[k] * v[1] / v[2]) if (k in tt and v[2]) else None}
                 for k, v in stages.items()}

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        cpu = cpu_baseline(depth, bgr, seq, a)

    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 2), "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(dev_ms_max / a.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if a.storage == "fp32" else "f16-storage/f32",
            "data": "synthetic: seeded room scene rendered to depth+BGR on the GPU (the TUM RGB-D sequences "
                    "the reference documents are not available offline)",
            "config": dict(workload_config(a, n_frames_needed(a)), parallelism=f"independent maps x{world}"),
            "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "gpu_launches": gpu_launches,
            "library_calls": lib_calls, "clocks": clocks, "stages": stage_rec,
            "wall_s_timed": round(dev_wall, 3), "surface_rms_m": rms,
            "map": {"leaves": st["leaves_used"], "leaves_max": st["leaves_max"], "n": st["n"],
                    "mesh_vertices": st["mesh_vertices"], "mesh_faces": st["mesh_faces"],
                    "mesh_cells": st["mesh_cells"], "grows": st["grows"], "meshing_ok": st["meshing_ok"],
                    "mesh_cells_dirty_mean": float(np.mean(dirty)) if dirty else None,
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


def cpu_baseline(depth, bgr, seq, a) -> dict:
    """The reference on one core over a bounded prefix of the same steps."""
    kind, ref = _cpu_impl()
    steps_max = a.warmup + a.steps
    hd = depth.cpu().numpy().view(np.uint16)
    hb = bgr.cpu().numpy()
    if kind == "reference":
        m = ref.RefFusion(VOXEL, THRESHOLD, True)
        add = lambda k: m.add_map(hd[k], hb[k], seq.K, *seq.poses[k], SCALING, MAXCAM)
        upd = m.update_meshes
    else:
        from oracle.port import PortFusion
        m = PortFusion(update_mode=2)
        add = lambda k: m.add_map(hd[k], hb[k], seq.K, *seq.poses[k], SCALING, MAXCAM)
        upd = m.update_meshes
    t0 = time.perf_counter()
    steps = 0
    while steps < steps_max and time.perf_counter() - t0 < CPU_SAMPLE_SECONDS:
        for k in range(steps * FRAMES_PER_STEP, (steps + 1) * FRAMES_PER_STEP):
            add(k)
        upd()
        m.mesh()
        steps += 1
    el = time.perf_counter() - t0
    if kind == "reference":
        m.close()
    return {"value": round(steps * FRAMES_PER_STEP / el, 3), "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"first {steps} steps ({steps * FRAMES_PER_STEP} frames, {steps} updateMeshes and mesh copies) of the "
                      f"same walk on one host core, {el:.1f} s"}


# -- the reference arm ------------------------------------------------------------
def _ref_worker(args):
    (idx, dpath, bpath, K, poses, warmup, steps, barrier, q) = args
    import numpy as np  # noqa: F811
    from oracle import ref as refmod
    hd = np.load(dpath, mmap_mode="r")
    hb = np.load(bpath, mmap_mode="r")
    if refmod.available():
        m = refmod.RefFusion(VOXEL, THRESHOLD, True)
        add = lambda k: m.add_map(np.asarray(hd[k]), np.asarray(hb[k]), K, *poses[k], SCALING, MAXCAM)
    else:
        from oracle.port import PortFusion
        m = PortFusion(update_mode=2)
        add = lambda k: m.add_map(np.asarray(hd[k]), np.asarray(hb[k]), K, *poses[k], SCALING, MAXCAM)
    # a step: 10 addMap, updateMeshes, and the mesh copied out
    # (getMeshInterleavedMarchingCubes returns the reference's mesh by value)
    for s in range(warmup):
        for k in range(s * FRAMES_PER_STEP, (s + 1) * FRAMES_PER_STEP):
            add(k)
        m.update_meshes()
        m.mesh()
    barrier.wait()
    t0 = time.perf_counter()
    for s in range(warmup, warmup + steps):
        for k in range(s * FRAMES_PER_STEP, (s + 1) * FRAMES_PER_STEP):
            add(k)
        m.update_meshes()
        m.mesh()
    q.put((idx, time.perf_counter() - t0))


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    import multiprocessing as mp
    import torch
    kind, _ = _cpu_impl()
    nf = n_frames_needed(a)
    seq = make_sequence(a.seed, nf)
    device = "cuda" if torch.cuda.is_available() else "cpu"
    depth, bgr = render_frames(seq, nf, device)
    tmp = tempfile.mkdtemp(prefix="ffref_")
    dpath, bpath = os.path.join(tmp, "depth.npy"), os.path.join(tmp, "bgr.npy")
    np.save(dpath, depth.cpu().numpy().view(np.uint16))
    np.save(bpath, bgr.cpu().numpy())
    del depth, bgr
    cores = len(os.sched_getaffinity(0))
    try:
        import psutil
        mem_maps = int(psutil.virtual_memory().available // (3 << 30))
    except ImportError:
        mem_maps = cores
    workers = a.workers or max(1, min(cores, mem_maps))
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(workers)
    q = ctx.Queue()
    procs = [ctx.Process(target=_ref_worker, args=((i, dpath, bpath, seq.K, seq.poses[:nf], a.warmup, a.steps,
                                                    barrier, q),)) for i in range(workers)]
    for p in procs:
        p.start()
    times = [q.get() for _ in procs]
    for p in procs:
        p.join()
    for f in (dpath, bpath):
        os.unlink(f)
    os.rmdir(tmp)
    wall = max(t for _, t in times)
    value = workers * a.steps * FRAMES_PER_STEP / wall
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(1e3 * wall / a.steps, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic: same frames as the B200 arm",
        "config": dict(workload_config(a, nf), parallelism=f"{workers} independent maps on {workers} host cores"),
        "cpu_baseline": {"value": round(value, 3), "unit": UNIT, "cores": workers, "kind": kind,
                         "sample": f"{workers} maps in parallel, each {a.steps} timed steps after {a.warmup} "
                                   f"warm-up steps of the walk"},
        "e2e": {"value": round(value, 3), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# -- the batched workload -------------------------------------------------------
def run_batch(a):
    """Independent maps of uneven size (rooms 2-12 m, 10-150 primitives,
    320x240 / 640x480 / 1280x960, voxels 4-10 mm), one frame of every map per
    ff_add_maps_u16_device call, updateMeshes per map every 10 frames; frames/s
    over all maps, device-resident inputs, CUDA events per step."""
    import torch
    from fastfusion_b200 import fusion as ff
    from fastfusion_b200.scene import batch_sequences, render_torch
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nf = n_frames_needed(a)
    seqs = batch_sequences(a.maps, n_frames=nf)
    frames = []
    for seq, _ in seqs:
        d = torch.empty((nf, seq.height, seq.width), dtype=torch.int16, device=dev)
        c = torch.empty((nf, seq.height, seq.width, 3), dtype=torch.uint8, device=dev)
        for k in range(nf):
            dk, ck = render_torch(seq.scene, *seq.poses[k], seq.width, seq.height, seq.K, seq.seed, k, device=dev)
            d[k].copy_(dk)
            c[k].copy_(ck)
        frames.append((d, c))
    cams = [[ff.CameraInfo(seq.K, *seq.poses[k]) for k in range(nf)] for seq, _ in seqs]
    stream = torch.cuda.current_stream(dev)
    maps = []
    for seq, voxel in seqs:
        m = ff.FusionMipMapCPU(0, 0, 0, voxel, 2 * voxel, 0, True, leaves_max=400000, branches_max=8000000,
                               storage=a.storage, rcp=a.rcp)
        m.set_stream(stream.cuda_stream)
        maps.append(m)
    widths = [seq.width for seq, _ in seqs]
    heights = [seq.height for seq, _ in seqs]
    # launch shapes chosen by the autotuner for this GPU (python -m fastfusion_b200.autotune), if any
    from fastfusion_b200.autotune import DEFAULT, load_tuning
    tuning = {} if a.no_tuning else load_tuning()
    if tuning:
        maps[0].set_tuning(**{**DEFAULT, **tuning})
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)

    def step(s_):
        for k in range(s_ * FRAMES_PER_STEP, (s_ + 1) * FRAMES_PER_STEP):
            ff.add_maps_device(maps, [f[0][k].data_ptr() for f in frames], [f[1][k].data_ptr() for f in frames],
                               widths, heights, [c[k] for c in cams], SCALING, MAXCAM)
        for m in maps:
            m.updateMeshes()

    for s_ in range(a.warmup):
        step(s_)
    maps[0].profile(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    torch.cuda.synchronize(dev)
    for i in range(a.steps):
        flush.fill_(i)
        ev[i][0].record(stream)
        step(a.warmup + i)
        ev[i][1].record(stream)
    torch.cuda.synchronize(dev)
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    stages = maps[0].profile_read()
    frames_total = a.steps * FRAMES_PER_STEP * len(maps)
    peak, peak_kind = measured_hbm_peak()
    fms, fbytes, fl = stages["fuse"]
    fuse_gbs = fbytes / (fms / 1e3) / 1e9 if fms > 0 else 0.0
    line = {
        "metric": METRIC.replace("(640x480, 5 mm)", "(batched maps)"), "value": round(frames_total / (ms / 1e3), 2),
        "unit": UNIT, "n_gpus": 1, "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32" if a.storage == "fp32" else "f16-storage/f32",
        "data": "synthetic: seeded rooms of uneven size rendered on the GPU",
        "config": {"workload": f"batch{len(maps)}: independent maps, rooms 2-12 m, 10-150 primitives, "
                               f"320x240/640x480/1280x960, voxels 4-10 mm, {nf} frames each, one frame of "
                               f"every map per launch set, updateMeshes every {FRAMES_PER_STEP} frames",
                   "maps": len(maps), "widths": widths, "voxels_mm": [round(v * 1e3, 2) for _, v in seqs],
                   "tuning": tuning or "defaults",
                   "l2": "flushed between timed steps (256 MB write)"},
        "fuse": {"GB/s": round(fuse_gbs, 1), "frac_of_hbm": round(fuse_gbs / peak, 4), "peak": peak,
                 "peak_source": peak_kind, "launches": fl, "avg_launch_us": round(1e3 * fms / fl, 2) if fl else 0,
                 "bytes_per_launch": round(fbytes / fl) if fl else 0},
        "stages_lead_map": {k: {"ms": round(v[0], 3), "launches": v[2]} for k, v in stages.items()},
    }
    print(json.dumps(line), flush=True)
    for m in maps:
        m.close()


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
    nf = n_frames_needed(a)
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
        # one map over all GPUs: rank r holds the bricks whose key hashes to r
        # (every rank is given every frame; no data-path collective)
        m.set_shard(rank, world)
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
        m.updateMeshes()

    for s_ in range(a.warmup):
        step(s_)
    m.profile(True)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    torch.cuda.synchronize(dev)
    for i in range(a.steps):
        if (a.warmup + i) % CHUNK == 0:
            m.sync()
            render_chunk(a.warmup + i)
        flush.fill_(i)
        ev[i][0].record(stream)
        step(a.warmup + i, render=False)
        ev[i][1].record(stream)
        st = m.stats()
        leaves.append(st["leaves_used"])
        if ref_cap_step is None and st["leaves_used"] > REFERENCE_POOL_BRICKS:
            ref_cap_step = a.warmup + i
    torch.cuda.synchronize(dev)
    ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    # the whole map's frames over the slowest part's device time
    ms_total = reduce_over_ranks(float(sum(ms)), "max", dev)
    leaves_all = int(reduce_over_ranks(float(m.stats()["leaves_used"]), "sum", dev))
    stages = m.profile_read()
    st = m.stats()
    peak, peak_kind = measured_hbm_peak()
    fms, fbytes, fl = stages["fuse"]
    fuse_gbs = fbytes / (fms / 1e3) / 1e9 if fms > 0 else 0.0
    q = max(1, len(ms) // 4)
    line = {
        "metric": METRIC.replace("(640x480, 5 mm)", "(large map, 1280x960, 5 mm)"),
        "value": round(a.steps * FRAMES_PER_STEP / (ms_total / 1e3), 2), "unit": UNIT, "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(ms_total / a.steps, 4),
        "ms_per_step_median": round(float(np.median(ms)), 3), "ms_per_step_max": round(float(np.max(ms)), 3),
        "ms_per_step_first_quarter": round(float(np.mean(ms[:q])), 3),
        "ms_per_step_last_quarter": round(float(np.mean(ms[-q:])), 3),
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
