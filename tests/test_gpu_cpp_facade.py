"""The C++ drop-in, run: a viewer-style C++ program (tests/cpp/viewer_like.cpp)
written against the reference's FusionMipMapCPU interface and compiled
against this library's fastfusion_b200/FusionMipMapCPU.hpp, with the
reference's own CameraInfo and MeshInterleaved, fuses frames on the GPU
(addMap per frame, updateMeshes every 10th frame) and writes the mesh with the
reference's MeshInterleaved::writePLY.  Its addMap return values must equal
the restatement's (host RCPPS mode, the facade's default reciprocal) and its
PLY file must equal, byte for byte, the restatement's mesh written by the
reference-identical writer (fastfusion_b200.fusion.MeshInterleaved.writePLY,
pinned against the reference's in tests/test_ply.py).

The program is built with the oracle (`make -C oracle viewer`, part of
__graft_entry__.build()) where the reference's headers are present, and
travels with the repository."""
import os
import struct
import subprocess

import numpy as np
import pytest

from tests.helpers import MAXCAM, SCALING, circle_frames

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
VIEWER = os.path.join(ROOT, "oracle", "_ref", "viewer_like")


def _write_frames(path, K, frames, every):
    h, w = frames[0][0].shape
    with open(path, "wb") as f:
        f.write(struct.pack("<4i", len(frames), w, h, every))
        f.write(np.asarray(K, np.float64).tobytes())
        for depth, bgr, R, t in frames:
            f.write(np.ascontiguousarray(R, np.float64).tobytes())
            f.write(np.ascontiguousarray(t, np.float64).tobytes())
            f.write(np.ascontiguousarray(depth, np.uint16).tobytes())
            f.write(np.ascontiguousarray(bgr, np.uint8).tobytes())


@pytest.mark.skipif(not os.path.exists(VIEWER), reason="oracle/_ref/viewer_like not built (reference headers absent)")
def test_viewer_style_cpp_program_runs_on_the_gpu(lib_built, port_lib, tmp_path):
    from fastfusion_b200.fusion import MeshInterleaved
    K, frames = circle_frames(0, 20, 320, 240)
    fpath = str(tmp_path / "frames.bin")
    _write_frames(fpath, K, frames, 10)
    r = subprocess.run([VIEWER, fpath, str(tmp_path / "cpp")], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    queued = [int(x) for x in r.stdout.split()]
    p = port_lib.PortFusion(leaves_total=271420, branches_total=4793488, update_mode=2)
    want = []
    for k, (depth, bgr, R, t) in enumerate(frames):
        want.append(p.add_map(depth, bgr, K, R, t, SCALING, MAXCAM))
        if k % 10 == 9:
            p.update_meshes()
    assert queued == want
    _, _, xyz, rgb, faces = p.mesh()
    assert len(faces) > 1000
    MeshInterleaved(xyz, rgb, faces).writePLY(str(tmp_path / "oracle"), True)
    got = open(tmp_path / "cpp.ply", "rb").read()
    exp = open(tmp_path / "oracle.ply", "rb").read()
    assert len(got) == len(exp)
    assert got == exp
