"""TUM RGB-D reader (fastfusion_b200/tum.py): association files, quaternion
poses, PNG depth/colour, chained trajectories, and the viewer-style fusion
loop (driven here with a recording stand-in for the map)."""
import numpy as np
import pytest

cv2 = pytest.importorskip("cv2")


def _write_sequence(root, n, t0=0.0, seed=0):
    rng = np.random.default_rng(seed)
    lines, arrays, quats = [], [], []
    for k in range(n):
        depth = rng.integers(0, 20000, (48, 64), dtype=np.uint16)
        bgr = rng.integers(0, 256, (48, 64, 3), dtype=np.uint8)
        cv2.imwrite(str(root / f"depth_{k}.png"), depth)
        cv2.imwrite(str(root / f"rgb_{k}.png"), bgr)
        q = rng.normal(size=4)
        q /= np.linalg.norm(q)
        t = rng.normal(size=3)
        quats.append((q, t))
        arrays.append((depth, bgr))
        lines.append(f"{t0 + k:.6f} {t[0]:.6f} {t[1]:.6f} {t[2]:.6f} {q[0]:.6f} {q[1]:.6f} {q[2]:.6f} {q[3]:.6f} "
                     f"{t0 + k:.6f} depth_{k}.png {t0 + k:.6f} rgb_{k}.png")
    (root / "assoc.txt").write_text("\n".join(lines) + "\n\n")
    return arrays, quats


def test_read_associations_and_frames(tmp_path):
    from scipy.spatial.transform import Rotation
    from fastfusion_b200 import tum
    arrays, quats = _write_sequence(tmp_path, 3)
    frames = tum.read_associations(str(tmp_path / "assoc.txt"))
    assert len(frames) == 3
    for fr, (depth, bgr), (q, t) in zip(frames, arrays, quats):
        want = Rotation.from_quat(q).as_matrix()  # (x, y, z, w) order
        assert np.allclose(fr.R, want, atol=2e-6)
        assert np.allclose(fr.R @ fr.R.T, np.eye(3), atol=2e-6)
        assert np.allclose(fr.t, t, atol=1e-6)
        d, c = tum.load_frame(fr)
        assert d.dtype == np.uint16 and np.array_equal(d, depth)
        assert np.array_equal(c, bgr)


def test_chained_trajectories(tmp_path):
    from fastfusion_b200 import tum
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    _write_sequence(a, 2, seed=1)
    _write_sequence(b, 2, seed=2)
    one = tum.read_associations(str(a / "assoc.txt"))
    two = tum.read_associations(str(b / "assoc.txt"))
    both = tum.read_associations([str(a / "assoc.txt"), str(b / "assoc.txt")])
    assert len(both) == 4
    Rs, ts = one[-1].R, one[-1].t
    for fr, raw in zip(both[2:], two):
        assert np.allclose(fr.R, Rs @ raw.R)
        assert np.allclose(fr.t, Rs @ raw.t + ts)


def test_fuse_sequence_drives_the_map_like_the_viewer(tmp_path):
    from fastfusion_b200 import tum

    class Recorder:
        def __init__(self):
            self.calls = []

        def addMap(self, depth, cam, bgr, scaling, maxcam):
            self.calls.append(("add", depth.shape, bgr.shape, scaling, maxcam, tuple(cam.K)))
            return 1

        def updateMeshes(self):
            self.calls.append(("update",))
            return True

        def getMeshInterleavedMarchingCubes(self):
            return "mesh"

    _write_sequence(tmp_path, 4)
    rec, meshes = Recorder(), []
    n = tum.fuse_sequence(rec, str(tmp_path / "assoc.txt"), mesh_every=2, on_mesh=lambda i, m: meshes.append(i))
    assert n == 4
    kinds = [c[0] for c in rec.calls]
    assert kinds == ["add", "add", "update", "add", "add", "update", "update"]
    assert rec.calls[0][3] == pytest.approx(1 / 5000.0) and rec.calls[0][5] == tum.TUM_K
    assert meshes == [1, 3, 3]
