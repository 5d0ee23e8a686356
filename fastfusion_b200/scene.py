"""Seeded synthetic RGB-D sequences with an analytic scene SDF.

The reference is exercised on TUM RGB-D sequences (640x480 uint16 depth at
5000 units/m, fx=fy=525, cx=319.5, cy=239.5; reference
src/onlinefusionviewer_main.cpp:234-237, README.md:60-70).  No dataset is
available offline, so this module ray-casts depth and colour frames of the
same shape from an analytic scene in FP64:

* a room (an axis-aligned box seen from the inside) holding seeded random
  axis-aligned boxes and spheres, each with one uint8 RGB albedo;
* per-pixel depth z along the optical axis, plus Gaussian noise with
  sigma = noise_k * z^2 metres and a fraction of random zero "holes";
* depth stored as round(z * 5000) in uint16 (0 where z >= 13.1 m), colour as
  BGR uint8, the reference's channel order (update_functions.cpp:1262-1290
  reads red from byte 2).

Poses are camera-to-world [R|t] with the OpenCV camera frame (x right, y
down, z forward), the convention of the reference's CameraInfo.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

DEPTH_UNITS_PER_M = 5000.0


@dataclasses.dataclass
class Scene:
    room: np.ndarray          # (3,) room extent in metres, room = [0, room]^3
    box_lo: np.ndarray        # (B, 3)
    box_hi: np.ndarray        # (B, 3)
    box_rgb: np.ndarray       # (B, 3) uint8 (R, G, B)
    sph_c: np.ndarray         # (S, 3)
    sph_r: np.ndarray         # (S,)
    sph_rgb: np.ndarray       # (S, 3) uint8
    wall_rgb: np.ndarray      # (6, 3) uint8: -x, +x, -y, +y, -z, +z walls

    def sdf(self, p: np.ndarray) -> np.ndarray:
        """Signed distance of points p (N,3) to the scene surfaces, positive in
        free space: min over the room walls (seen from inside) and the solids."""
        p = np.asarray(p, dtype=np.float64)
        d = np.min(np.concatenate([p, self.room[None, :] - p], axis=1), axis=1)
        for lo, hi in zip(self.box_lo, self.box_hi):
            c = 0.5 * (lo + hi)
            h = 0.5 * (hi - lo)
            q = np.abs(p - c) - h
            outside = np.linalg.norm(np.maximum(q, 0.0), axis=1)
            inside = np.minimum(np.max(q, axis=1), 0.0)
            d = np.minimum(d, outside + inside)
        for c, r in zip(self.sph_c, self.sph_r):
            d = np.minimum(d, np.linalg.norm(p - c, axis=1) - r)
        return d


def make_scene(seed: int, room=(4.0, 4.0, 3.0), n_prims: int = 20, size=(0.1, 0.8),
               keep_clear=None) -> Scene:
    """Room plus n_prims seeded boxes/spheres (p = 1/2 each), sizes U(size)."""
    rng = np.random.default_rng(seed)
    room = np.asarray(room, dtype=np.float64)
    box_lo, box_hi, box_rgb, sph_c, sph_r, sph_rgb = [], [], [], [], [], []
    tries = 0
    while len(box_lo) + len(sph_c) < n_prims and tries < 100 * max(n_prims, 1):
        tries += 1
        c = rng.uniform(0.0, 1.0, 3) * room
        rgb = rng.integers(0, 256, 3).astype(np.uint8)
        is_box = rng.uniform() < 0.5
        if is_box:
            ext = rng.uniform(size[0], size[1], 3)
            radius = float(np.linalg.norm(ext) / 2)
        else:
            radius = float(rng.uniform(size[0], size[1]) / 2)
        if keep_clear is not None and not keep_clear(c, radius + 0.15):
            continue
        if is_box:
            box_lo.append(c - ext / 2)
            box_hi.append(c + ext / 2)
            box_rgb.append(rgb)
        else:
            sph_c.append(c)
            sph_r.append(radius)
            sph_rgb.append(rgb)
    wall_rgb = rng.integers(40, 256, (6, 3)).astype(np.uint8)
    z3 = np.zeros((0, 3))
    return Scene(room=room,
                 box_lo=np.array(box_lo) if box_lo else z3, box_hi=np.array(box_hi) if box_hi else z3,
                 box_rgb=np.array(box_rgb, dtype=np.uint8).reshape(-1, 3),
                 sph_c=np.array(sph_c) if sph_c else z3, sph_r=np.array(sph_r, dtype=np.float64),
                 sph_rgb=np.array(sph_rgb, dtype=np.uint8).reshape(-1, 3), wall_rgb=wall_rgb)


def look_at(pos, target, up=(0.0, 0.0, 1.0)) -> np.ndarray:
    """Camera-to-world rotation (columns = camera x right, y down, z forward)."""
    pos = np.asarray(pos, dtype=np.float64)
    z = np.asarray(target, dtype=np.float64) - pos
    z /= np.linalg.norm(z)
    x = np.cross(z, np.asarray(up, dtype=np.float64))
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    return np.stack([x, y, z], axis=1)


def circle_trajectory(n_frames: int, centre=(2.0, 2.0), radius=1.5, height=1.2, target=(2.0, 2.0, 1.5)):
    """Pose k at angle 2*pi*k/n on a horizontal circle, looking at target."""
    poses = []
    for k in range(n_frames):
        a = 2.0 * math.pi * k / n_frames
        pos = np.array([centre[0] + radius * math.cos(a), centre[1] + radius * math.sin(a), height])
        poses.append((look_at(pos, target), pos))
    return poses


def random_walk_trajectory(n_frames: int, seed: int, room=(8.0, 8.0, 3.0), step=0.02, yaw_jitter_deg=2.0,
                           height=1.2, margin=0.8):
    """Seeded random walk at fixed height, bouncing off a margin to the walls."""
    rng = np.random.default_rng(seed + 7919)
    pos = np.array([room[0] / 2, room[1] / 2, height])
    yaw = rng.uniform(0, 2 * math.pi)
    poses = []
    for _ in range(n_frames):
        yaw += math.radians(rng.normal(0.0, yaw_jitter_deg))
        d = np.array([math.cos(yaw), math.sin(yaw), 0.0])
        nxt = pos + step * d
        if not (margin < nxt[0] < room[0] - margin and margin < nxt[1] < room[1] - margin):
            yaw += math.pi
            d = -d
            nxt = pos + step * d
        pos = nxt
        target = pos + d + np.array([0.0, 0.0, 0.1])
        poses.append((look_at(pos, target), pos.copy()))
    return poses


def _hit_box(o, d, lo, hi):
    with np.errstate(divide='ignore', invalid='ignore'):
        inv = 1.0 / d
        t1 = (lo[None, :] - o[None, :]) * inv
        t2 = (hi[None, :] - o[None, :]) * inv
    tn = np.nanmax(np.minimum(t1, t2), axis=1)
    tf = np.nanmin(np.maximum(t1, t2), axis=1)
    hit = (tn <= tf) & (tn > 1e-9)
    return np.where(hit, tn, np.inf)


def _hit_sphere(o, d, c, r):
    oc = o - c
    a = np.einsum('ij,ij->i', d, d)
    b = d @ oc
    cc = float(oc @ oc) - r * r
    disc = b * b - a * cc
    ok = disc >= 0
    sq = np.sqrt(np.where(ok, disc, 0.0))
    t = (-b - sq) / a
    return np.where(ok & (t > 1e-9), t, np.inf)


def render(scene: Scene, R: np.ndarray, t: np.ndarray, width: int, height: int, fx: float, fy: float,
           cx: float, cy: float, rng: np.random.Generator | None = None, noise_k: float = 0.0012,
           hole_frac: float = 0.02):
    """Ray-cast one frame.  Returns (depth uint16 [H,W], bgr uint8 [H,W,3], z_true float64 [H,W])."""
    xs = (np.arange(width, dtype=np.float64) - cx) / fx
    ys = (np.arange(height, dtype=np.float64) - cy) / fy
    dcam = np.stack(np.broadcast_arrays(xs[None, :], ys[:, None], np.ones((height, width))), axis=-1).reshape(-1, 3)
    d = dcam @ R.T          # ray direction in world, parametrised so that t == camera z
    o = np.asarray(t, dtype=np.float64)
    # room from the inside: exit distance
    with np.errstate(divide='ignore', invalid='ignore'):
        inv = 1.0 / d
        ta = (0.0 - o[None, :]) * inv
        tb = (scene.room[None, :] - o[None, :]) * inv
    texit = np.where(np.isfinite(ta), np.maximum(ta, tb), np.inf)
    axis = np.argmin(texit, axis=1)
    tbest = texit[np.arange(len(axis)), axis]
    side = (d[np.arange(len(axis)), axis] > 0).astype(np.int64)
    colour = scene.wall_rgb[2 * axis + side].astype(np.uint8)
    for lo, hi, rgb in zip(scene.box_lo, scene.box_hi, scene.box_rgb):
        th = _hit_box(o, d, lo, hi)
        closer = th < tbest
        tbest = np.where(closer, th, tbest)
        colour[closer] = rgb
    for c, r, rgb in zip(scene.sph_c, scene.sph_r, scene.sph_rgb):
        th = _hit_sphere(o, d, c, r)
        closer = th < tbest
        tbest = np.where(closer, th, tbest)
        colour[closer] = rgb
    z_true = tbest.reshape(height, width)
    z = z_true.copy()
    if rng is not None:
        if noise_k > 0:
            z = z + rng.normal(0.0, 1.0, z.shape) * noise_k * z * z
        if hole_frac > 0:
            z[rng.uniform(size=z.shape) < hole_frac] = 0.0
    z = np.where(np.isfinite(z) & (z > 0), z, 0.0)
    depth = np.round(z * DEPTH_UNITS_PER_M)
    depth[(z >= 13.1) | (depth > 65535)] = 0
    depth = depth.astype(np.uint16)
    bgr = colour[:, ::-1].reshape(height, width, 3).copy()
    return depth, bgr, z_true


@dataclasses.dataclass
class Sequence:
    scene: Scene
    K: np.ndarray             # fx, fy, cx, cy (float64)
    width: int
    height: int
    poses: list               # [(R (3,3), t (3,)), ...]
    seed: int
    noise_k: float = 0.0012
    hole_frac: float = 0.02

    def frame(self, k: int):
        rng = np.random.default_rng((self.seed, k))
        R, t = self.poses[k]
        fx, fy, cx, cy = self.K
        depth, bgr, _ = render(self.scene, R, t, self.width, self.height, fx, fy, cx, cy, rng,
                               self.noise_k, self.hole_frac)
        return depth, bgr, R, t

    def __len__(self):
        return len(self.poses)


def room_circle_sequence(seed: int = 0, n_frames: int = 100, width: int = 640, height: int = 480,
                         n_prims: int = 20, room=(4.0, 4.0, 3.0)) -> Sequence:
    """The plain-method workload: a 4x4x3 m room with 20 seeded primitives,
    frames on a circle of radius 1.5 m at 1.2 m height around the room centre
    looking at (2, 2, 1.5).  Intrinsics scale with the resolution from the
    640x480 values fx=fy=525, cx=319.5, cy=239.5."""
    s = width / 640.0
    K = np.array([525.0 * s, 525.0 * s, (width - 1) / 2.0, (height - 1) / 2.0])
    centre = (room[0] / 2, room[1] / 2)

    def clear(c, rad):
        dxy = math.hypot(c[0] - centre[0], c[1] - centre[1])
        return abs(dxy - 1.5) > rad or abs(c[2] - 1.2) > rad

    scene = make_scene(seed, room=room, n_prims=n_prims, keep_clear=clear)
    poses = circle_trajectory(n_frames, centre=centre, radius=1.5, height=1.2,
                              target=(centre[0], centre[1], 1.5))
    return Sequence(scene=scene, K=K, width=width, height=height, poses=poses, seed=seed)


def room_walk_sequence(seed: int = 0, n_frames: int = 1000, width: int = 640, height: int = 480,
                       n_prims: int = 80, room=(8.0, 8.0, 3.0)) -> Sequence:
    """The larger workload: an 8x8x3 m room with 80 primitives and a seeded
    random walk (2 cm steps, 2 degree yaw jitter) at 1.2 m height."""
    s = width / 640.0
    K = np.array([525.0 * s, 525.0 * s, (width - 1) / 2.0, (height - 1) / 2.0])
    poses = random_walk_trajectory(n_frames, seed, room=room)
    cams = np.array([p[1] for p in poses])

    def clear(c, rad):
        return np.min(np.linalg.norm(cams - c[None, :], axis=1)) > rad + 0.3

    scene = make_scene(seed, room=room, n_prims=n_prims, keep_clear=clear)
    return Sequence(scene=scene, K=K, width=width, height=height, poses=poses, seed=seed)


def corridor_scene(seed: int, size=(50.0, 20.0, 3.0), n_prims: int = 400, corridor=(9.0, 11.0),
                   office: float = 5.0, wall: float = 0.1, door: float = 1.2, prim_size=(0.1, 0.8)) -> Scene:
    """The large-map layout: a size[0] x size[1] x size[2] m floor with a
    corridor along x (y in `corridor`), offices of `office` m on both sides
    behind 0.1 m walls with a door each, and n_prims seeded boxes/spheres in
    the offices (none in the corridor the camera moves along)."""
    rng = np.random.default_rng(seed)
    L, Wd, Ht = size
    lo, hi = [], []
    for side in (0, 1):
        y0 = corridor[0] - wall if side == 0 else corridor[1]
        for i in range(int(round(L / office))):
            x0 = i * office
            mid = x0 + office / 2
            lo.append([x0, y0, 0.0])                       # corridor wall left of the door
            hi.append([mid - door / 2, y0 + wall, Ht])
            lo.append([mid + door / 2, y0, 0.0])           # and right of it
            hi.append([x0 + office, y0 + wall, Ht])
            if i > 0:                                      # wall between two offices
                ya, yb = (0.0, corridor[0] - wall) if side == 0 else (corridor[1] + wall, Wd)
                lo.append([x0 - wall / 2, ya, 0.0])
                hi.append([x0 + wall / 2, yb, Ht])
    wall_lo, wall_hi = np.array(lo), np.array(hi)
    wall_rgb_boxes = rng.integers(60, 230, (len(lo), 3)).astype(np.uint8)
    box_lo, box_hi, box_rgb, sph_c, sph_r, sph_rgb = [], [], [], [], [], []
    while len(box_lo) + len(sph_c) < n_prims:
        c = rng.uniform(0.0, 1.0, 3) * np.array([L, Wd, Ht])
        if corridor[0] - 0.6 < c[1] < corridor[1] + 0.6:
            continue
        rgb = rng.integers(0, 256, 3).astype(np.uint8)
        if rng.uniform() < 0.5:
            ext = rng.uniform(prim_size[0], prim_size[1], 3)
            box_lo.append(c - ext / 2)
            box_hi.append(c + ext / 2)
            box_rgb.append(rgb)
        else:
            sph_c.append(c)
            sph_r.append(float(rng.uniform(prim_size[0], prim_size[1]) / 2))
            sph_rgb.append(rgb)
    return Scene(room=np.array(size, dtype=np.float64),
                 box_lo=np.concatenate([wall_lo, np.array(box_lo).reshape(-1, 3)]),
                 box_hi=np.concatenate([wall_hi, np.array(box_hi).reshape(-1, 3)]),
                 box_rgb=np.concatenate([wall_rgb_boxes, np.array(box_rgb, dtype=np.uint8).reshape(-1, 3)]),
                 sph_c=np.array(sph_c).reshape(-1, 3), sph_r=np.array(sph_r, dtype=np.float64),
                 sph_rgb=np.array(sph_rgb, dtype=np.uint8).reshape(-1, 3),
                 wall_rgb=rng.integers(40, 256, (6, 3)).astype(np.uint8))


def _catmull_rom(p: np.ndarray, t: float) -> np.ndarray:
    """Point of the uniform Catmull-Rom spline through points p at t in [0, len(p) - 1]."""
    i = min(int(t), len(p) - 2)
    u = t - i
    p0, p1, p2, p3 = p[max(i - 1, 0)], p[i], p[i + 1], p[min(i + 2, len(p) - 1)]
    return 0.5 * ((2 * p1) + (-p0 + p2) * u + (2 * p0 - 5 * p1 + 4 * p2 - p3) * u * u +
                  (-p0 + 3 * p1 - 3 * p2 + p3) * u * u * u)


def spline_trajectory(n_frames: int, seed: int, x_range=(2.0, 48.0), y_mid: float = 10.0, y_jitter: float = 0.5,
                      height=(1.0, 1.6), knot_spacing: float = 4.0, yaw_amp_deg: float = 55.0,
                      yaw_period: int = 400):
    """Seeded spline along the corridor: knots every knot_spacing m in x with
    y jitter and heights U(height); the camera looks along the path, swinging
    its yaw by +-yaw_amp_deg (period yaw_period frames) into the offices."""
    rng = np.random.default_rng(seed + 104729)
    xs = np.arange(x_range[0], x_range[1] + 1e-9, knot_spacing)
    knots = np.stack([xs, y_mid + rng.uniform(-y_jitter, y_jitter, len(xs)),
                      rng.uniform(height[0], height[1], len(xs))], axis=1)
    poses = []
    for k in range(n_frames):
        t = (len(knots) - 1) * k / max(n_frames - 1, 1)
        pos = _catmull_rom(knots, t)
        ahead = _catmull_rom(knots, min(t + 0.05, len(knots) - 1.0)) - pos
        if np.linalg.norm(ahead[:2]) < 1e-9:
            ahead = np.array([1.0, 0.0, 0.0])
        yaw = math.atan2(ahead[1], ahead[0]) + math.radians(yaw_amp_deg) * math.sin(2 * math.pi * k / yaw_period)
        d = np.array([math.cos(yaw), math.sin(yaw), -0.1])
        poses.append((look_at(pos, pos + d), pos.copy()))
    return poses


def corridor_sequence(seed: int = 0, n_frames: int = 10000, width: int = 1280, height: int = 960,
                      n_prims: int = 400) -> Sequence:
    """The large-map workload: the 50 x 20 x 3 m corridor/office layout with
    400 primitives, frames along the seeded spline at 1.0-1.6 m; intrinsics
    fx = fy = 1050 at 1280 x 960 (scaled with the width)."""
    s = width / 1280.0
    K = np.array([1050.0 * s, 1050.0 * s, (width - 1) / 2.0, (height - 1) / 2.0])
    return Sequence(scene=corridor_scene(seed, n_prims=n_prims), K=K, width=width, height=height,
                    poses=spline_trajectory(n_frames, seed), seed=seed)


def render_torch(scene: Scene, R, t, width: int, height: int, K, seed: int, frame: int, device="cuda",
                 noise_k: float = 0.0012, hole_frac: float = 0.02, flying_frac: float = 0.0,
                 flying_m: float = 0.1, edge_m: float = 0.05, return_true: bool = False,
                 cull_m: float | None = None):
    """render() on a torch device in FP64 (same geometry and colour rules;
    noise and holes from a torch generator seeded by (seed, frame)).
    flying_frac: that fraction of the depth-edge pixels (a 4-neighbour more
    than edge_m away in true depth) is displaced by +-flying_m ("flying
    pixels"), drawn after the noise and the holes.
    cull_m: primitives farther than this from the camera are left out (a
    surface beyond it cannot hide a nearer one, so every depth below cull_m
    is unchanged; use maxcam + a margin).
    Returns (depth uint16 [H,W], bgr uint8 [H,W,3]) as device tensors, plus
    the true depth (float64 [H,W], metres) when return_true."""
    import torch
    dev = torch.device(device)
    f64 = torch.float64
    fx, fy, cx, cy = (float(v) for v in K)
    xs = (torch.arange(width, dtype=f64, device=dev) - cx) / fx
    ys = (torch.arange(height, dtype=f64, device=dev) - cy) / fy
    dcam = torch.stack(torch.broadcast_tensors(xs[None, :], ys[:, None], torch.ones(height, width, dtype=f64,
                                                                                   device=dev)), -1).reshape(-1, 3)
    Rt = torch.as_tensor(np.asarray(R), dtype=f64, device=dev)
    o = torch.as_tensor(np.asarray(t), dtype=f64, device=dev)
    d = dcam @ Rt.T
    room = torch.as_tensor(scene.room, dtype=f64, device=dev)
    inv = 1.0 / d
    ta = (0.0 - o[None, :]) * inv
    tb = (room[None, :] - o[None, :]) * inv
    texit = torch.where(torch.isfinite(ta), torch.maximum(ta, tb), torch.full_like(ta, float("inf")))
    tbest, axis = torch.min(texit, dim=1)
    side = (d.gather(1, axis[:, None])[:, 0] > 0).long()
    wall = torch.as_tensor(scene.wall_rgb, dtype=torch.uint8, device=dev)
    colour = wall[2 * axis + side]
    box_lo, box_hi, box_rgb = scene.box_lo, scene.box_hi, scene.box_rgb
    sph_c, sph_r, sph_rgb = scene.sph_c, scene.sph_r, scene.sph_rgb
    if cull_m is not None:
        on = np.asarray(t, dtype=np.float64).reshape(3)
        if len(box_lo):
            near = np.linalg.norm(np.maximum(np.maximum(box_lo - on, on - box_hi), 0.0), axis=1) < cull_m
            box_lo, box_hi, box_rgb = box_lo[near], box_hi[near], box_rgb[near]
        if len(sph_c):
            near = np.linalg.norm(sph_c - on, axis=1) - sph_r < cull_m
            sph_c, sph_r, sph_rgb = sph_c[near], sph_r[near], sph_rgb[near]
    if len(box_lo):
        lo = torch.as_tensor(box_lo, dtype=f64, device=dev)
        hi = torch.as_tensor(box_hi, dtype=f64, device=dev)
        rgb = torch.as_tensor(box_rgb, dtype=torch.uint8, device=dev)
        t1 = (lo[None] - o[None, None]) * inv[:, None]
        t2 = (hi[None] - o[None, None]) * inv[:, None]
        tn = torch.nan_to_num(torch.minimum(t1, t2), nan=-float("inf")).amax(-1)
        tf = torch.nan_to_num(torch.maximum(t1, t2), nan=float("inf")).amin(-1)
        th = torch.where((tn <= tf) & (tn > 1e-9), tn, torch.full_like(tn, float("inf")))
        tmin, idx = th.min(1)
        closer = tmin < tbest
        tbest = torch.where(closer, tmin, tbest)
        colour = torch.where(closer[:, None], rgb[idx], colour)
    if len(sph_c):
        c = torch.as_tensor(sph_c, dtype=f64, device=dev)
        r = torch.as_tensor(sph_r, dtype=f64, device=dev)
        rgb = torch.as_tensor(sph_rgb, dtype=torch.uint8, device=dev)
        oc = o[None] - c
        a = (d * d).sum(1)[:, None]
        b = d @ oc.T
        cc = (oc * oc).sum(1)[None] - r[None] ** 2
        disc = b * b - a * cc
        ok = disc >= 0
        th = (-b - torch.sqrt(torch.clamp(disc, min=0.0))) / a
        th = torch.where(ok & (th > 1e-9), th, torch.full_like(th, float("inf")))
        tmin, idx = th.min(1)
        closer = tmin < tbest
        tbest = torch.where(closer, tmin, tbest)
        colour = torch.where(closer[:, None], rgb[idx], colour)
    z = tbest.reshape(height, width)
    z_true = z
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed) * 1000003 + int(frame))
    if noise_k > 0:
        z = z + torch.randn(z.shape, generator=g, dtype=f64, device=dev) * noise_k * z * z
    if hole_frac > 0:
        z = torch.where(torch.rand(z.shape, generator=g, dtype=f64, device=dev) < hole_frac, torch.zeros_like(z), z)
    if flying_frac > 0:
        zt = torch.nan_to_num(z_true, posinf=1e3)
        pad = torch.nn.functional.pad(zt[None, None], (1, 1, 1, 1), mode="replicate")[0, 0]
        jump = torch.zeros_like(zt, dtype=torch.bool)
        for dy, dx in ((0, 1), (2, 1), (1, 0), (1, 2)):
            jump |= (pad[dy:dy + height, dx:dx + width] - zt).abs() > edge_m
        pick = torch.rand(z.shape, generator=g, dtype=f64, device=dev) < flying_frac
        sign = torch.where(torch.rand(z.shape, generator=g, dtype=f64, device=dev) < 0.5, -1.0, 1.0)
        z = torch.where(jump & pick & (z > 0), z + sign * flying_m, z)
    z = torch.where(torch.isfinite(z) & (z > 0), z, torch.zeros_like(z))
    depth = torch.round(z * DEPTH_UNITS_PER_M)
    depth = torch.where((z >= 13.1) | (depth > 65535), torch.zeros_like(depth), depth)
    depth = depth.to(torch.int32).to(torch.int16)  # bit pattern of the uint16 value
    bgr = colour.flip(-1).reshape(height, width, 3).contiguous()
    if return_true:
        return depth, bgr, z_true
    return depth, bgr


def batch_sequences(n_maps: int = 16, n_frames: int | None = 200, seed0: int = 100):
    """Independent maps of uneven size (the batched workload): per map i, seed
    seed0 + i draws room sides U(2, 12) m (3 m high), U{10..150} primitives,
    an image size from 320x240 / 640x480 / 1280x960, a voxel size U(4, 10) mm
    and a length U{200..2000} frames (used when n_frames is None; otherwise
    every map has n_frames); each map walks its own room.  Returns
    [(Sequence, voxel metres)]; len(Sequence.poses) is the map's length."""
    out = []
    sizes = [(320, 240), (640, 480), (1280, 960)]
    for i in range(n_maps):
        rng = np.random.default_rng(seed0 + i)
        room = (float(rng.uniform(2, 12)), float(rng.uniform(2, 12)), 3.0)
        prims = int(rng.integers(10, 151))
        w, h = sizes[int(rng.integers(0, 3))]
        voxel = float(rng.uniform(0.004, 0.010))
        length = int(rng.integers(200, 2001))
        if n_frames is not None:
            length = n_frames
        margin = min(0.8, 0.3 * min(room[0], room[1]))
        s = w / 640.0
        K = np.array([525.0 * s, 525.0 * s, (w - 1) / 2.0, (h - 1) / 2.0])
        poses = random_walk_trajectory(length, seed0 + i, room=room, margin=margin)
        cams = np.array([p[1] for p in poses])

        def clear(c, rad, cams=cams):
            return np.min(np.linalg.norm(cams - c[None, :], axis=1)) > rad + 0.3

        scene = make_scene(seed0 + i, room=room, n_prims=prims, keep_clear=clear)
        out.append((Sequence(scene=scene, K=K, width=w, height=h, poses=poses, seed=seed0 + i), voxel))
    return out
