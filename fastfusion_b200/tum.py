"""TUM RGB-D input: association files with poses, 16-bit depth and colour PNGs.

Mirrors the reference viewer's reader (src/onlinefusionviewer_main.cpp:
278-345): every non-empty line of an association file holds

    timestamp tx ty tz qx qy qz qw  timestamp depth.png  [timestamp rgb.png]

with paths relative to the file's directory.  Numbers are read as float
(the reference streams them into float variables), the rotation is the
quaternion's matrix (the reference builds it with Eigen's
Quaterniond(qw, qx, qy, qz).toRotationMatrix()), and with several
association files each trajectory starts at the last pose of the previous
one.  Depth PNGs are read unchanged (uint16, 5000 units per metre in the TUM
data), colour PNGs as BGR.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np

# the reference viewer's default intrinsics (onlinefusionviewer_main.cpp:234-237)
TUM_K = (525.0, 525.0, 319.5, 239.5)
TUM_SCALING = 1.0 / 5000.0


def quaternion_to_rotation(qw: float, qx: float, qy: float, qz: float) -> np.ndarray:
    """Rotation matrix of a unit quaternion (the standard formula, evaluated in
    double precision the way Eigen's toRotationMatrix arranges it)."""
    w, x, y, z = (float(v) for v in (qw, qx, qy, qz))
    tx, ty, tz = 2.0 * x, 2.0 * y, 2.0 * z
    twx, twy, twz = tx * w, ty * w, tz * w
    txx, txy, txz = tx * x, ty * x, tz * x
    tyy, tyz, tzz = ty * y, tz * y, tz * z
    return np.array([[1.0 - (tyy + tzz), txy - twz, txz + twy],
                     [txy + twz, 1.0 - (txx + tzz), tyz - twx],
                     [txz - twy, tyz + twx, 1.0 - (txx + tyy)]], dtype=np.float64)


@dataclasses.dataclass
class TumFrame:
    R: np.ndarray       # camera-to-world rotation (3x3 double)
    t: np.ndarray       # camera-to-world translation (3, double)
    depth_path: str
    rgb_path: str | None


def read_associations(paths, use_color: bool = True) -> list[TumFrame]:
    """Frames of one or more association files, chained like the reference."""
    if isinstance(paths, (str, os.PathLike)):
        paths = [paths]
    frames: list[TumFrame] = []
    start_R, start_t = np.eye(3), np.zeros(3)
    for path in paths:
        prefix = os.path.dirname(os.path.abspath(path))
        first = len(frames)
        with open(path) as f:
            for line in f:
                if not line.strip():
                    continue
                tok = line.split()
                vals = [float(np.float32(v)) for v in tok[:8]]
                t = np.array(vals[1:4], dtype=np.float64)
                qx, qy, qz, qw = vals[4:8]
                depth = os.path.join(prefix, tok[9])
                rgb = os.path.join(prefix, tok[11]) if use_color and len(tok) > 11 else None
                frames.append(TumFrame(quaternion_to_rotation(qw, qx, qy, qz), t, depth, rgb))
        # each trajectory is composed with the pose where the previous one ended
        for fr in frames[first:]:
            fr.R, fr.t = start_R @ fr.R, start_R @ fr.t + start_t
        if len(frames) > first:
            start_R, start_t = frames[-1].R, frames[-1].t
    return frames


def load_frame(frame: TumFrame):
    """(depth uint16 HxW, bgr uint8 HxWx3 or None) of one frame."""
    import cv2
    depth = cv2.imread(frame.depth_path, cv2.IMREAD_ANYDEPTH)
    if depth is None:
        raise FileNotFoundError(frame.depth_path)
    bgr = None
    if frame.rgb_path:
        bgr = cv2.imread(frame.rgb_path, cv2.IMREAD_COLOR)
        if bgr is None:
            raise FileNotFoundError(frame.rgb_path)
    return depth.astype(np.uint16, copy=False), bgr


def fuse_sequence(fusion, paths, K=TUM_K, scaling: float = TUM_SCALING, maxcam: float = 4.0,
                  mesh_every: int = 0, on_mesh=None):
    """Fuse a TUM sequence into a FusionMipMapCPU the way the reference viewer
    does: addMap per frame, updateMeshes every `mesh_every` frames (0: only at
    the end); `on_mesh(frame_index, mesh)` receives each mesh."""
    from fastfusion_b200.fusion import CameraInfo
    frames = read_associations(paths)
    for i, fr in enumerate(frames):
        depth, bgr = load_frame(fr)
        if bgr is None:
            bgr = np.zeros(depth.shape + (3,), np.uint8)
        fusion.addMap(depth, CameraInfo(K, fr.R, fr.t), bgr, scaling, maxcam)
        if mesh_every and (i + 1) % mesh_every == 0:
            fusion.updateMeshes()
            if on_mesh:
                on_mesh(i, fusion.getMeshInterleavedMarchingCubes())
    fusion.updateMeshes()
    if on_mesh:
        on_mesh(len(frames) - 1, fusion.getMeshInterleavedMarchingCubes())
    return len(frames)
